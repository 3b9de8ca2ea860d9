// wt_lean.cuh — the fused step, one thread per cell, with lean addressing.
//
// Same semantics and per-cell rules as k_step (wt_step.cuh); the arithmetic
// is collide_x2 on one cell (scaled storage units, approximate reciprocal and
// square root, wt_x2.cuh). What differs is how the 38 population accesses of
// a cell are addressed: every thread forms one byte pointer to its cell in
// the read buffer and one in the write buffer, and each access adds a 32-bit
// byte offset that is the same for every thread of the launch (StepArgs
// srcb / dstb). A direction therefore costs one load or store plus at most
// one add, instead of a 64-bit multiply-add chain per access. Used when both
// population buffers span less than 2^31 bytes. The outlet column is computed
// by its own threads (a recomputation of column nx-2), so the common path has
// no second store per population. Half storage rounds to nearest or
// stochastically (StepArgs f16_sr), as the direct kernel does.
#pragma once

#include "wt_x2.cuh"

namespace wt {

// Byte offset added to a cell pointer: zero-extended for half storage,
// sign-extended for float32 (the two measured fastest on B200 for each form;
// the offsets are non-negative either way).
template <class S>
__device__ __forceinline__ long long lean_off(uint32_t b) {
  if constexpr (sizeof(S) == 4) return (long long)(int)b;
  else return (long long)b;
}

// Resident blocks per SM the register budget is set for: float32 storage
// fits 72 registers without spills at 7 (28 warps; +3% over 64 registers
// and 8 blocks on B200), half storage is issue-bound and runs best at 8
// (32 warps, 64 registers; 7 measured -4%).
template <class S>
constexpr int lean_min_blocks() { return sizeof(S) == 4 ? 7 : 8; }

template <class S>
__global__ void __launch_bounds__(STEP_BX, lean_min_blocks<S>())
    k_step_lean(const __grid_constant__ StepArgs<S> a) {
  pdl_enter();   // programmatic dependent launch (launch_pdl)
  using T = X2<S>;
  constexpr float SC = T::SC;
  const int x = blockIdx.x * STEP_BX + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  prefetch_ahead(a, (long long)(x - (int)(threadIdx.x & 31)) + (long long)a.nx * y + a.nxy * z);
  double Fx = 0, Fy = 0, Fz = 0;
  bool near_cell = false;
  if (x < a.nx) {
    // The outlet column x = nx-1 holds a copy of column nx-2 after the step
    // (js/lbm.js:504-511): its thread recomputes cell nx-2 and writes its own
    // cell, so no thread stores twice.
    const bool outlet = x == a.nx - 1;
    const int xs = outlet ? a.nx - 2 : x;
    const long long row = (long long)a.nx * y + a.nxy * z;
    const long long is = xs + row, id = x + row;
    // The pulls of every cell that can be fluid are issued before its flags
    // byte arrives (all their sources lie inside the lattice), so a cell
    // waits for one memory latency instead of two.
    const bool inner = xs >= 1 && y >= 1 && y <= a.ny - 2 && z >= 1 && z <= a.nz - 2;
    float f[Q];
    if (inner) {
      const char* Fb = reinterpret_cast<const char*>(a.F + is);
#pragma unroll
      for (int q = 0; q < Q; q++)
        f[q] = T::raw(*reinterpret_cast<const S*>(Fb + lean_off<S>(a.srcb[q])));
    }
    int cat;
    uint8_t fl = 0;
    if (xs == 0) {
      cat = CAT_EQ;
    } else {
      fl = a.flags[is];
      if (z == 0 || z == a.nz - 1 || y == a.ny - 1) cat = CAT_EQ;
      else if (fl & FLAG_SOLID_MASK) cat = CAT_KEEP;
      else if (y == 0) cat = CAT_EQ;
      else cat = CAT_FLUID;
    }
    char* Gb = reinterpret_cast<char*>(a.G + id);
    auto gs = [&](int q) -> S& { return *reinterpret_cast<S*>(Gb + lean_off<S>(a.dstb[q])); };
    if (cat == CAT_FLUID) {   // implies inner
      const bool wall = (fl & FLAG_NEAR) != 0;
      const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
      if (wall || shell) patch_raw<S, 0>(a, is, xs, y, z, wall, shell, f, Fx, Fy, Fz);
      near_cell = wall && !outlet;   // the copy's links are not counted twice
      float r, vx, vy, vz;
      collide_x2<S, float>(a, f, r, vx, vy, vz);
      if (!(r > 0.0f && r < 3.0e38f)) atomicOr(a.err, 1u);
      if (a.write_fields) {
        a.rho[id] = r * (1.0f / SC); a.ux[id] = vx; a.uy[id] = vy; a.uz[id] = vz;
      } else if (a.mov && near_cell) {
        a.rho[is] = r * (1.0f / SC);
      }
      bool stored = false;
      if constexpr (std::is_same<S, __half>::value) {
        if (a.f16_sr) {
          // stochastic rounding, pairs converted together with the direct
          // kernel's per-cell, per-step random chain (seeded by the computed
          // cell, so the outlet copy rounds as column nx-2 does)
          uint32_t h = ((uint32_t)is ^ (uint32_t)(is >> 32)) * 0x9E3779B1u ^ a.sr_seed;
          h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
#pragma unroll
          for (int k = 1; k < Q; k += 2) {
            h ^= h << 13; h ^= h >> 17; h ^= h << 5;
            const __half2 p = sr_half2(f[k], f[k + 1], h);
            gs(k) = __high2half(p);
            gs(k + 1) = __low2half(p);
          }
          h ^= h << 13; h ^= h >> 17; h ^= h << 5;
          gs(0) = __low2half(sr_half2(0.0f, f[0], h));
          stored = true;
        }
      }
      if (!stored) {
#pragma unroll
        for (int q = 0; q < Q; q++) gs(q) = T::to_s(f[q]);
      }
    } else if (cat == CAT_EQ) {
#pragma unroll
      for (int q = 0; q < Q; q++) gs(q) = a.eq[q];
      if (a.write_fields) {
        a.ux[id] = a.u0f; a.uy[id] = 0.0f; a.uz[id] = 0.0f; a.rho[id] = 1.0f;
      }
    } else if (outlet) {
      // copy of a solid cell in column nx-2: its g is not written this step
      const char* Gs = reinterpret_cast<const char*>(a.G + is);
#pragma unroll
      for (int q = 0; q < Q; q++) gs(q) = *reinterpret_cast<const S*>(Gs + lean_off<S>(a.dstb[q]));
      if (a.write_fields) {
        a.ux[id] = a.ux[is]; a.uy[id] = a.uy[is]; a.uz[id] = a.uz[is]; a.rho[id] = a.rho[is];
      }
    }
    if (!near_cell) Fx = Fy = Fz = 0.0;
  }
  constexpr double inv_sc = 1.0 / (double)SC;   // a power of two: exact
  warp_force_partial(Fx * inv_sc, Fy * inv_sc, Fz * inv_sc, near_cell, a);
}

}  // namespace wt
