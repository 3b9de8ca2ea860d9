// wt_kernels_fast.cu — float32-arithmetic instantiations of the fused step
// (float32 and half-deviation storage), plus the force reduction. Built with
// the default multiply-add contraction.
#include "wt_internal.h"
#include "wt_pbb.cuh"
#include "wt_lean.cuh"
#include "wt_pair.cuh"

namespace wt {

void launch_step_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step<float, false, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step<float, false, int>, grid, dim3(STEP_BX), s, a);
}

void launch_step_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step<__half, false, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step<__half, false, int>, grid, dim3(STEP_BX), s, a);
}

void launch_lean_f32(const StepArgs<float>& a, dim3 grid, bool, cudaStream_t s) {
  launch_pdl(k_step_lean<float>, grid, dim3(STEP_BX), s, a);
}

void launch_lean_f16(const StepArgs<__half>& a, dim3 grid, bool, cudaStream_t s) {
  launch_pdl(k_step_lean<__half>, grid, dim3(STEP_BX), s, a);
}

template <class S>
inline dim3 pair_grid(int nx, int ny, int nz) {
  constexpr int seg = 2 * pair_bx<S>();   // cells per block
  return dim3((unsigned)((nx + seg - 1) / seg), (unsigned)ny, (unsigned)nz);
}

// Every step kernel (direct, lean, pair, partial bounce-back, adjoint)
// launches with programmatic dependent launch (launch_pdl): a step's blocks
// fill the slots the previous step's tail frees and start the moment it
// completes. Measured on B200: pair float32 +2.5% on 256x128x128, half
// storage +1-2%; the partial-bounce-back step on 128x64x64 +10%.
template <class S>
void launch_pair_pdl(void (*k)(StepArgs<S>), const StepArgs<S>& a, cudaStream_t s) {
  launch_pdl(k, pair_grid<S>(a.nx, a.ny, a.nz), dim3(pair_bx<S>()), s, a);
}

void launch_pair_f16(const StepArgs<__half>& a, dim3, bool, cudaStream_t s) {
  if (a.f16_sr) launch_pair_pdl<__half>(k_step_pair<__half, true>, a, s);
  else launch_pair_pdl<__half>(k_step_pair<__half, false>, a, s);
}

void launch_pair_f32(const StepArgs<float>& a, dim3, bool, cudaStream_t s) {
  launch_pair_pdl<float>(k_step_pair<float, false>, a, s);
}

// ---- partial bounce-back and adjoint (float32 arithmetic) -------------------------

void launch_pbb_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step_pbb<float, false, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step_pbb<float, false, int>, grid, dim3(STEP_BX), s, a);
}

void launch_pbb_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step_pbb<__half, false, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step_pbb<__half, false, int>, grid, dim3(STEP_BX), s, a);
}

void launch_adj_f32(const StepArgs<float>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s) {
  launch_adjoint<float, float>(a, Tn, Tc, ds, wJ, comp, s);
}

void launch_adj_f16(const StepArgs<__half>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s) {
  launch_adjoint<__half, float>(a, Tn, Tc, ds, wJ, comp, s);
}

// Marks the 32-cell segments that hold at least one near-wall cell.
__global__ void k_mark_segments(const uint8_t* __restrict__ flags, int nx, int ny, int nz,
                             uint8_t* __restrict__ mark) {
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (flags[i] & FLAG_NEAR) {
      const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
      mark[seg_of(x, y, z, nx, ny)] = 1;
    }
  }
}

void launch_mark_segments(const uint8_t* flags, int nx, int ny, int nz, uint8_t* mark,
                          cudaStream_t s) {
  k_mark_segments<<<148 * 16, 256, 0, s>>>(flags, nx, ny, nz, mark);
}

// One block per step; each thread sums a fixed strided subset of the warp
// partials, then a fixed-shape tree combines them. The order never depends
// on timing, so the force series is reproducible run to run.
constexpr int RED_T = 256;

__global__ void __launch_bounds__(RED_T) k_force_reduce(const double* __restrict__ part,
                                                        unsigned nblocks,
                                                        double* __restrict__ out) {
  __shared__ double sm[3][RED_T];
  const double* p = part + (size_t)blockIdx.x * nblocks * 3;
  double ax = 0, ay = 0, az = 0;
  for (unsigned b = threadIdx.x; b < nblocks; b += RED_T) {
    ax += p[3 * (size_t)b];
    ay += p[3 * (size_t)b + 1];
    az += p[3 * (size_t)b + 2];
  }
  sm[0][threadIdx.x] = ax;
  sm[1][threadIdx.x] = ay;
  sm[2][threadIdx.x] = az;
  __syncthreads();
  for (int w = RED_T / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sm[0][threadIdx.x] += sm[0][threadIdx.x + w];
      sm[1][threadIdx.x] += sm[1][threadIdx.x + w];
      sm[2][threadIdx.x] += sm[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[3 * (size_t)blockIdx.x] = sm[0][0];
    out[3 * (size_t)blockIdx.x + 1] = sm[1][0];
    out[3 * (size_t)blockIdx.x + 2] = sm[2][0];
  }
}

void launch_force_reduce(const double* part, unsigned nslots, int nsteps, double* out,
                         cudaStream_t s) {
  k_force_reduce<<<nsteps, RED_T, 0, s>>>(part, nslots, out);
}

cudaError_t configure_step_kernels() {
  // The pair kernels use no shared memory: the whole unified L1 / shared
  // array goes to L1 (measured on B200: +1.6% for half storage on
  // 256x128x128, +0.5% on 512x192x192, float32 unchanged).
  const void* fns[] = {(const void*)k_step_pair<__half, false>,
                       (const void*)k_step_pair<__half, true>,
                       (const void*)k_step_pair<float, false>};
  for (const void* f : fns) {
    const cudaError_t e =
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t preload_step_kernels() {
  cudaFuncAttributes fa;
  const void* fns[] = {
      (const void*)k_step<float, false, int>, (const void*)k_step<float, false, long long>,
      (const void*)k_step<__half, false, int>, (const void*)k_step<__half, false, long long>,
      (const void*)k_step_lean<float>, (const void*)k_step_lean<__half>,
      (const void*)k_step_pair<__half, false>, (const void*)k_step_pair<__half, true>,
      (const void*)k_step_pair<float, false>,
      (const void*)k_force_reduce};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
  }
  return preload_exact_step_kernels();
}

}  // namespace wt
