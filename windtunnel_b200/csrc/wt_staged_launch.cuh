// wt_staged_launch.cuh — host-side launcher of the staged step kernel.
#pragma once

#include <algorithm>

#include "wt_staged.cuh"

namespace wt {

// Persistent grid: as many CTAs as fit on the device at once (cached per
// device), never more than there are units.
template <class S, bool EXACT, class IDX>
void launch_staged_idx(const StepArgs<S>& args, cudaStream_t s) {
  using C = Staged<S>;
  StepArgs<S> a = args;   // units are x-segments of C::TX cells
  a.gx = (a.nx + C::TX - 1) / C::TX;
  a.units = (long long)a.gx * a.ny * a.nz;
  constexpr int kMaxDevices = 64;
  static int grid_of[kMaxDevices] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  int& grid = grid_of[dev % kMaxDevices];
  if (grid == 0) {
    cudaFuncSetAttribute(k_step_staged<S, EXACT, IDX>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_step_staged<S, EXACT, IDX>, C::THREADS,
                                                  C::SMEM);
    grid = std::max(1, sms * std::max(per, 1));
  }
  const long long g = std::min<long long>(grid, a.units);
  k_step_staged<S, EXACT, IDX><<<(unsigned)g, C::THREADS, C::SMEM, s>>>(a);
}

template <class S, bool EXACT>
void launch_staged(const StepArgs<S>& a, cudaStream_t s) {
  if (19 * a.n >= (1LL << 31)) launch_staged_idx<S, EXACT, long long>(a, s);
  else launch_staged_idx<S, EXACT, int>(a, s);
}

}  // namespace wt
