// wt_pipe.cuh — the fused step, software-pipelined along z.
//
// Same semantics and per-cell rules as k_step (wt_step.cuh). A thread owns
// cell x of row y for PIPE_K consecutive z planes. Before colliding the
// cell of plane z it issues the 19 pull loads and the occupancy byte of the
// cell of plane z+1, so every warp keeps a full set of HBM loads in flight
// through its arithmetic instead of alternating a load phase and a compute
// phase: the step is bound by memory latency x bytes in flight, and this
// raises the bytes in flight per resident warp to a full cell's worth at all
// times. Used for the float32 collision (float32 and half storage).
#pragma once

#include "wt_step.cuh"

namespace wt {

constexpr int PIPE_K = 8;   // z planes per thread

// Pull loads of cell i: plain gathers of the 19 directions (the special
// rules are applied after arrival by patch_special).
template <class S, class IDX>
__device__ __forceinline__ void pipe_load(const StepArgs<S>& a, long long i, S (&raw)[Q]) {
  const S* Fi = a.F + i;
#pragma unroll
  for (int q = 0; q < Q; q++) raw[q] = Fi[(IDX)a.src[q]];
}

template <class S, class IDX>
__global__ void __launch_bounds__(STEP_BX, 6) k_step_pipe(const __grid_constant__ StepArgs<S> a) {
  const int x = blockIdx.x * STEP_BX + threadIdx.x;
  const int y = blockIdx.y;
  const int zb = blockIdx.z * PIPE_K;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int ze = min(nz, zb + PIPE_K);
  const bool xcell = x < nx - 1;           // x = nx-1 is written by its left neighbour
  const bool xin = x >= 1 && x <= nx - 2;
  const bool yin = y >= 1 && y <= ny - 2;
  const bool ycell = y <= ny - 2;          // y = ny-1 is an equilibrium row

  // what a cell of this column needs from HBM before it can be categorised
  auto wants_pull = [&](int z) { return xin && yin && z >= 1 && z <= nz - 2; };
  auto wants_flag = [&](int z) { return xin && ycell && z >= 1 && z <= nz - 2; };

  S raw_next[Q];
  uint8_t fl_next = 0;
  {
    const long long i = (long long)x + (long long)nx * y + a.nxy * zb;
    if (wants_flag(zb)) fl_next = a.flags[i];
    if (wants_pull(zb)) pipe_load<S, IDX>(a, i, raw_next);
  }

#pragma unroll 1
  for (int z = zb; z < ze; z++) {
    const long long i = (long long)x + (long long)nx * y + a.nxy * z;
    S raw[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) raw[q] = raw_next[q];
    const uint8_t fl = fl_next;
    if (z + 1 < ze) {
      const long long in = i + a.nxy;
      if (wants_flag(z + 1)) fl_next = a.flags[in];
      if (wants_pull(z + 1)) pipe_load<S, IDX>(a, in, raw_next);
    }

    double Fx = 0, Fy = 0, Fz = 0;
    bool near_cell = false;
    if (xcell) {
      const bool dup = (x == nx - 2);
      int cat;
      if (x == 0 || z == 0 || z == nz - 1 || y == ny - 1) cat = CAT_EQ;
      else if (fl & FLAG_SOLID_MASK) cat = CAT_KEEP;
      else if (y == 0) cat = CAT_EQ;
      else cat = CAT_FLUID;
      S* Gi = a.G + i;
      if (cat == CAT_FLUID) {
        float f[Q];
#pragma unroll
        for (int q = 0; q < Q; q++) f[q] = Store<S>::load_f(raw[q]);
        near_cell = (fl & FLAG_NEAR) != 0;
        const bool shell = a.freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
        if (near_cell || shell) patch_special<S, float>(a, i, x, y, z, shell, f, Fx, Fy, Fz);
        S out[Q];
        collide_fast<S>(a, f, i, dup, near_cell, RegOut<S>{out});
#pragma unroll
        for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q]] = out[q];
        if (dup) {
#pragma unroll
          for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = out[q];
        }
      } else if (cat == CAT_EQ) {
#pragma unroll
        for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q]] = a.eq[q];
        if (dup) {
#pragma unroll
          for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = a.eq[q];
        }
        if (a.write_fields) {
          a.ux[i] = a.u0f; a.uy[i] = 0.0f; a.uz[i] = 0.0f; a.rho[i] = 1.0f;
          if (dup) { a.ux[i + 1] = a.u0f; a.uy[i + 1] = 0.0f; a.uz[i + 1] = 0.0f; a.rho[i + 1] = 1.0f; }
        }
      } else if (dup) {
        // outlet copy of a solid cell in column nx-2: its g is not written this step
#pragma unroll
        for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = Gi[(IDX)a.dst[q]];
        if (a.write_fields) {
          a.ux[i + 1] = a.ux[i]; a.uy[i + 1] = a.uy[i]; a.uz[i + 1] = a.uz[i]; a.rho[i + 1] = a.rho[i];
        }
      }
    }
    const int xw = blockIdx.x * STEP_BX + (threadIdx.x & ~31);
    warp_force_partial_w(Fx, Fy, Fz, near_cell, a, seg_of(xw, y, z, nx, ny));
  }
}

inline dim3 pipe_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nx + STEP_BX - 1) / STEP_BX), (unsigned)ny,
              (unsigned)((nz + PIPE_K - 1) / PIPE_K));
}

}  // namespace wt
