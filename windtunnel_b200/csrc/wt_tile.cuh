// wt_tile.cuh — the fused step with the block's rows staged in shared memory.
//
// Same semantics and per-cell arithmetic as the lean kernel (wt_lean.cuh):
// every cell is collided by collide_x2<S, float> in storage units from the
// same pulled values, so the two kernels store bit-identical populations.
// What differs is how the values move. A block owns 128 consecutive cells of
// one row. Its threads first copy, with 16-byte loads, the 19 source row
// segments the block pulls from (each segment one vector wider on either
// side for the x-shifted directions) into shared memory; each thread then
// reads its 19 pulled values there at compile-time offsets, collides, and
// writes its 19 results to a shared output tile, which the block finally
// writes to the population buffer with 16-byte stores. A cell's 38 global
// accesses, each with its own 64-bit address, become ~5 vector accesses per
// thread plus shared-memory accesses that need no address arithmetic.
//
// Cells outside the fluid keep their rules: inlet, floor, ceiling and end
// planes store the equilibrium; a solid cell keeps its stale populations
// (its tile column is filled from the write buffer, so the vector store
// writes them back unchanged); the outlet column takes column nx-2's output
// column after the step (no recomputation). Near-wall and free-slip cells
// patch their pulled values from global memory as the lean kernel does.
//
// Requirements (checked by the host): the float32 collision, stationary
// walls, nx a multiple of 8, buffers under 2^31 bytes.
//
// On B200 it ran 35-40% slower than the lean kernel (256x128x128: 22.2k
// against 37.6k MLUPS for float32, 28.5k against 44.3k for half storage):
// the barriers between the load, collide and store phases of a block cost
// more latency than the resident blocks hide. It is kept as a selectable
// alternative (WT_KERNEL_TILE).
#pragma once

#include "wt_lean.cuh"

namespace wt {

template <class S>
struct Tile {
  static constexpr int VEC = 16 / (int)sizeof(S);     // elements per 16-byte vector
  static constexpr int W = STEP_BX + 2 * VEC;         // staged segment: halo vector each side
  static constexpr int CH = W / VEC;                  // vectors per staged segment
  static constexpr int OCH = STEP_BX / VEC;           // vectors per output segment
};

// ex of direction q for a runtime q (the staging loop is not unrolled).
__device__ __forceinline__ int ex_rt(int q) {
  // directions 1,7,9,11,13: +1; 2,8,10,12,14: -1 (js/lbm.js:29-37)
  const unsigned plus = (1u << 1) | (1u << 7) | (1u << 9) | (1u << 11) | (1u << 13);
  const unsigned minus = (1u << 2) | (1u << 8) | (1u << 10) | (1u << 12) | (1u << 14);
  return ((plus >> q) & 1u) ? 1 : (((minus >> q) & 1u) ? -1 : 0);
}

template <class S>
__global__ void __launch_bounds__(STEP_BX, 8) k_step_tile(const __grid_constant__ StepArgs<S> a) {
  using T = X2<S>;
  using C = Tile<S>;
  constexpr float SC = T::SC;
  __shared__ __align__(16) S sin[Q][C::W];
  __shared__ __align__(16) S sout[Q][STEP_BX];
  const int t = threadIdx.x;
  const int x0 = blockIdx.x * STEP_BX;
  const int x = x0 + t;
  const int y = blockIdx.y, z = blockIdx.z;
  const int nx = a.nx;
  const long long row = (long long)nx * y + a.nxy * z;
  const bool edge_row = z == 0 || z == a.nz - 1 || y == a.ny - 1;
  const bool interior_row = !edge_row && y >= 1;

  // 1. stage the source segments: source positions [x0 - VEC, x0 + 128 + VEC)
  // of the row each direction pulls from, whole vectors inside [0, nx) only
  // (the positions a computed cell pulls, x-1 .. x+1 for 1 <= x <= nx-2,
  // always lie in them)
  if (interior_row) {
    const int lo = x0 - C::VEC;
    for (int c = t; c < Q * C::CH; c += STEP_BX) {
      const int q = c / C::CH, k = c - q * C::CH;
      const int s = lo + k * C::VEC;
      if (s < 0 || s > nx - C::VEC) continue;
      const long long e = row + s + a.src[q] + ex_rt(q);   // element of source position s
      *reinterpret_cast<uint4*>(&sin[q][k * C::VEC]) =
          *reinterpret_cast<const uint4*>(a.F + e);
    }
  }
  __syncthreads();

  // 2. collide into the output tile
  double Fx = 0, Fy = 0, Fz = 0;
  bool near_cell = false;
  const bool active = x < nx;
  const bool outlet = x == nx - 1;
  const long long i = x + row;
  int cat = CAT_NONE;
  uint8_t fl = 0;
  if (active && !outlet) {
    if (x == 0 || edge_row) {
      cat = CAT_EQ;
    } else {
      fl = a.flags[i];
      if (fl & FLAG_SOLID_MASK) cat = CAT_KEEP;
      else if (y == 0) cat = CAT_EQ;
      else cat = CAT_FLUID;
    }
  }
  if (cat == CAT_FLUID) {
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) f[q] = T::raw(sin[q][C::VEC + t - ex(q)]);
    const bool wall = (fl & FLAG_NEAR) != 0;
    const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
    if (wall || shell) patch_raw<S, 0>(a, i, x, y, z, wall, shell, f, Fx, Fy, Fz);
    near_cell = wall;
    float r, vx, vy, vz;
    collide_x2<S, float>(a, f, r, vx, vy, vz);
    if (!(r > 0.0f && r < 3.0e38f)) atomicOr(a.err, 1u);
    if (a.write_fields) {
      a.rho[i] = r * (1.0f / SC); a.ux[i] = vx; a.uy[i] = vy; a.uz[i] = vz;
    }
    bool stored = false;
    if constexpr (std::is_same<S, __half>::value) {
      if (a.f16_sr) {
        // the direct and lean kernels' per-cell, per-step random chain
        uint32_t h = ((uint32_t)i ^ (uint32_t)(i >> 32)) * 0x9E3779B1u ^ a.sr_seed;
        h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
#pragma unroll
        for (int k = 1; k < Q; k += 2) {
          h ^= h << 13; h ^= h >> 17; h ^= h << 5;
          const __half2 p = sr_half2(f[k], f[k + 1], h);
          sout[k][t] = __high2half(p);
          sout[k + 1][t] = __low2half(p);
        }
        h ^= h << 13; h ^= h >> 17; h ^= h << 5;
        sout[0][t] = __low2half(sr_half2(0.0f, f[0], h));
        stored = true;
      }
    }
    if (!stored) {
#pragma unroll
      for (int q = 0; q < Q; q++) sout[q][t] = T::to_s(f[q]);
    }
  } else if (cat == CAT_EQ) {
#pragma unroll
    for (int q = 0; q < Q; q++) sout[q][t] = a.eq[q];
    if (a.write_fields) {
      a.ux[i] = a.u0f; a.uy[i] = 0.0f; a.uz[i] = 0.0f; a.rho[i] = 1.0f;
    }
  } else if (cat == CAT_KEEP) {
    // a solid cell keeps what the write buffer holds (written back unchanged)
#pragma unroll
    for (int q = 0; q < Q; q++) sout[q][t] = a.G[a.dst[q] + i];
  }
  __syncthreads();
  if (outlet) {
    // js/lbm.js:504-511: the outlet takes column nx-2's values after the step
    // (in this block: nx is a multiple of 8, so nx-2 and nx-1 share a block)
#pragma unroll
    for (int q = 0; q < Q; q++) sout[q][t] = sout[q][t - 1];
    if (a.write_fields) {
      a.ux[i] = a.ux[i - 1]; a.uy[i] = a.uy[i - 1]; a.uz[i] = a.uz[i - 1]; a.rho[i] = a.rho[i - 1];
    }
  }
  __syncthreads();

  // 3. write the output tile with 16-byte stores (whole vectors inside [0, nx))
  for (int c = t; c < Q * C::OCH; c += STEP_BX) {
    const int q = c / C::OCH, k = c - q * C::OCH;
    const int s = x0 + k * C::VEC;
    if (s >= nx) continue;
    *reinterpret_cast<uint4*>(a.G + a.dst[q] + row + s) =
        *reinterpret_cast<const uint4*>(&sout[q][k * C::VEC]);
  }
  if (!near_cell) Fx = Fy = Fz = 0.0;
  constexpr double inv_sc = 1.0 / (double)SC;   // a power of two: exact
  warp_force_partial(Fx * inv_sc, Fy * inv_sc, Fz * inv_sc, near_cell, a);
}

}  // namespace wt
