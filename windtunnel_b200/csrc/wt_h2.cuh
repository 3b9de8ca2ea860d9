// wt_h2.cuh — the fused step for half storage, two cells per thread.
//
// Same semantics and per-cell arithmetic as the lean kernel (wt_lean.cuh):
// each cell is collided on its own by collide_x2<__half, float> in storage
// units, so the two kernels store bit-identical populations. What differs is
// the memory side. A thread owns the cell pair (x0, x0+1), x0 even, and
// holds its 19 pulled pairs as 19 packed half2 words: one 32-bit load per
// direction (the source pair of an x-shifted direction is assembled from its
// own word and the neighbouring lane's with one shuffle and one byte
// permute), and one 32-bit store per direction. A pair therefore costs 19
// loads and 19 stores instead of 38 + 38, with one address per access.
// Cell A is unpacked to floats, collided and rounded back into the low
// halves; then cell B from the high halves, by the same code (a loop over
// the two cells that is not unrolled, so the collision is one copy in the
// instruction cache). The launched form parks the packed words in the
// thread's column of shared memory meanwhile (64 registers); the register
// form needs 96. On B200 both ran slower than the lean kernel (39.7k and
// 37.8k against 44.3k MLUPS on 256x128x128): the kernel is kept as a
// selectable alternative (WT_KERNEL_PAIR).
//
// Requirements (checked by the host): half storage, the float32 collision,
// stationary walls, nx even, buffers under 2^31 bytes.
#pragma once

#include "wt_x2.cuh"

namespace wt {

constexpr int H2_BX = 64;   // threads per block: 128 cells of one row

// Source pair of direction q for the pair of this thread, as a packed word
// (low half: cell x0, high half: cell x0 + 1).
template <int q>
__device__ __forceinline__ uint32_t pull_word(const char* Fb, uint32_t srcb, int lane,
                                              bool active) {
  // aligned source pair (x0 - ex + ex, ...): the word at x0 of the source row
  const char* p = Fb + srcb + ex(q) * (int)sizeof(__half);
  uint32_t w = 0;
  if (active) w = *reinterpret_cast<const uint32_t*>(p);
  if constexpr (ex(q) == 0) {
    return w;
  } else if constexpr (ex(q) == 1) {
    // cell x0 pulls x0-1 (the previous pair's high half), x0+1 pulls x0
    uint32_t wp = __shfl_up_sync(0xffffffffu, w, 1);
    if (lane == 0 && active) wp = (uint32_t)*reinterpret_cast<const uint16_t*>(p - 2) << 16;
    return __byte_perm(wp, w, 0x5432);
  } else {
    // cell x0 pulls x0+1 (this word's high half), x0+1 pulls x0+2
    uint32_t wn = __shfl_down_sync(0xffffffffu, w, 1);
    if (lane == 31 && active) wn = (uint32_t)*reinterpret_cast<const uint16_t*>(p + 4);
    return __byte_perm(w, wn, 0x5432);
  }
}

// The half at bit offset sh (0: cell x0, 16: cell x0+1) of a packed word.
__device__ __forceinline__ float half_at(uint32_t w, int sh) {
  return __half2float(__ushort_as_half((unsigned short)(w >> sh)));
}
__device__ __forceinline__ uint32_t set_half(uint32_t w, int sh, __half h) {
  return (w & ~(0xffffu << sh)) | ((uint32_t)__half_as_ushort(h) << sh);
}

// Where a thread keeps its 19 packed words between the pulls and the stores:
// in registers (RegWords), or in its column of a shared-memory array
// (SmemWords), which frees 19 registers for the collision so that the
// kernel fits the 64 registers of 32 resident warps per SM.
struct RegWords {
  uint32_t w[Q];
  __device__ __forceinline__ uint32_t get(int q) const { return w[q]; }
  __device__ __forceinline__ void put(int q, uint32_t v) { w[q] = v; }
  __device__ __forceinline__ void put_half(int q, int sh, __half h) { w[q] = set_half(w[q], sh, h); }
};
struct SmemWords {
  uint32_t (*s)[H2_BX];   // [Q][H2_BX]: consecutive threads, consecutive words
  int t;
  __device__ __forceinline__ uint32_t get(int q) const { return s[q][t]; }
  __device__ __forceinline__ void put(int q, uint32_t v) { s[q][t] = v; }
  __device__ __forceinline__ void put_half(int q, int sh, __half h) {
    reinterpret_cast<__half*>(&s[q][t])[sh >> 4] = h;
  }
};

// Collide the cell at bit offset sh of the pair in place: the pulled values
// are unpacked, patched, collided and rounded back into the same halves;
// r, v the cell's density (storage units) and velocity. One copy of this
// code serves both cells (the caller loops over them without unrolling).
template <class W>
__device__ __forceinline__ void collide_half(const StepArgs<__half>& a, W& w, int sh,
                                             long long i, int x, int y, int z, bool wall,
                                             bool shell, double& Fx, double& Fy, double& Fz,
                                             float& r, float& vx, float& vy, float& vz) {
  float f[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) f[q] = half_at(w.get(q), sh);
  if (wall || shell) patch_raw<__half, 0>(a, i, x, y, z, wall, shell, f, Fx, Fy, Fz);
  collide_x2<__half, float>(a, f, r, vx, vy, vz);
  if (a.f16_sr) {
    // the direct and lean kernels' per-cell, per-step random chain
    uint32_t h = ((uint32_t)i ^ (uint32_t)(i >> 32)) * 0x9E3779B1u ^ a.sr_seed;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      h ^= h << 13; h ^= h >> 17; h ^= h << 5;
      const __half2 p = sr_half2(f[k], f[k + 1], h);
      w.put_half(k, sh, __high2half(p));
      w.put_half(k + 1, sh, __low2half(p));
    }
    h ^= h << 13; h ^= h >> 17; h ^= h << 5;
    w.put_half(0, sh, __low2half(sr_half2(0.0f, f[0], h)));
  } else {
#pragma unroll
    for (int q = 0; q < Q; q++) w.put_half(q, sh, __float2half_rn(f[q]));
  }
}

// SMEM: the packed words live in shared memory between the pulls and the
// stores (64 registers, 16 blocks per SM) instead of registers (96, 10).
template <bool SMEM>
__global__ void __launch_bounds__(H2_BX, SMEM ? 16 : 10)
    k_step_h2(const __grid_constant__ StepArgs<__half> a) {
  constexpr float SC = X2<__half>::SC;
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int x0 = 2 * (blockIdx.x * H2_BX + t);
  const int y = blockIdx.y, z = blockIdx.z;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long i0 = (long long)x0 + (long long)nx * y + a.nxy * z;
  prefetch_ahead(a, i0 - 2 * lane);
  const bool active = x0 < nx;
  double Fx = 0, Fy = 0, Fz = 0;
  bool near_any = false;
  char* Gb = reinterpret_cast<char*>(a.G + i0);
  auto gw = [&](int q) -> uint32_t& { return *reinterpret_cast<uint32_t*>(Gb + a.dstb[q]); };
  auto gh = [&](int q, int c) -> __half& {
    return *reinterpret_cast<__half*>(Gb + a.dstb[q] + c * (int)sizeof(__half));
  };

  if (z == 0 || z == nz - 1 || y == ny - 1) {
    // ceiling / end planes: the equilibrium for both cells (and the outlet's
    // copy of an equilibrium cell is the equilibrium)
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; q++) {
        const uint32_t e = (uint32_t)__half_as_ushort(a.eq[q]);
        gw(q) = e | (e << 16);
      }
      if (a.write_fields) {
        a.ux[i0] = a.u0f; a.uy[i0] = 0.0f; a.uz[i0] = 0.0f; a.rho[i0] = 1.0f;
        a.ux[i0 + 1] = a.u0f; a.uy[i0 + 1] = 0.0f; a.uz[i0 + 1] = 0.0f; a.rho[i0 + 1] = 1.0f;
      }
    }
    pair_force_partial(Fx, Fy, Fz, near_any, a, x0 & ~31, y, z);
    return;
  }

  // the pulled pairs of an interior row (every lane takes part in the
  // shuffles); the floor row pulls nothing
  __shared__ uint32_t sw[SMEM ? Q : 1][H2_BX];
  typename std::conditional<SMEM, SmemWords, RegWords>::type w;
  if constexpr (SMEM) {
    w.s = sw;
    w.t = t;
  }
  if (y >= 1) {
    const char* Fb = reinterpret_cast<const char*>(a.F + i0);
#define WT_PULL(q) w.put(q, pull_word<q>(Fb, a.srcb[q], lane, active));
    WT_PULL(0) WT_PULL(1) WT_PULL(2) WT_PULL(3) WT_PULL(4) WT_PULL(5) WT_PULL(6) WT_PULL(7)
    WT_PULL(8) WT_PULL(9) WT_PULL(10) WT_PULL(11) WT_PULL(12) WT_PULL(13) WT_PULL(14)
    WT_PULL(15) WT_PULL(16) WT_PULL(17) WT_PULL(18)
#undef WT_PULL
  } else {
#pragma unroll
    for (int q = 0; q < Q; q++) w.put(q, 0u);
  }
  if (active) {
    const uint16_t fl2 = *reinterpret_cast<const uint16_t*>(a.flags + i0);
    const uint8_t flA = (uint8_t)fl2, flB = (uint8_t)(fl2 >> 8);
    const bool outB = x0 + 1 == nx - 1;   // cell B is the outlet: a copy of cell A
    const int catA = cell_category(a, x0, y, flA);
    const int catB = outB ? CAT_NONE : cell_category(a, x0 + 1, y, flB);
    const bool shell = a.freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
#pragma unroll 1
    for (int c = 0; c < 2; c++) {
      const int cat = c ? catB : catA;
      const uint8_t fl = c ? flB : flA;
      const long long i = i0 + c;
      const int sh = 16 * c;
      if (cat == CAT_FLUID) {
        const bool wall = (fl & FLAG_NEAR) != 0;
        near_any = near_any || wall;
        float r, vx, vy, vz;
        collide_half(a, w, sh, i, x0 + c, y, z, wall, shell, Fx, Fy, Fz, r, vx, vy, vz);
        if (!(r > 0.0f && r < 3.0e38f)) atomicOr(a.err, 1u);
        if (a.write_fields) {
          a.rho[i] = r * (1.0f / SC); a.ux[i] = vx; a.uy[i] = vy; a.uz[i] = vz;
        }
      } else if (cat == CAT_EQ) {
#pragma unroll
        for (int q = 0; q < Q; q++) w.put_half(q, sh, a.eq[q]);
        if (a.write_fields) { a.ux[i] = a.u0f; a.uy[i] = 0.0f; a.uz[i] = 0.0f; a.rho[i] = 1.0f; }
      }
    }
    const long long iB = i0 + 1;
    if (outB) {
      // js/lbm.js:504-511: the outlet takes what column nx-2 holds after the
      // step (a solid cell there keeps its stale populations and fields)
      if (catA == CAT_KEEP) {
#pragma unroll
        for (int q = 0; q < Q; q++) w.put_half(q, 16, gh(q, 0));
      } else {
#pragma unroll
        for (int q = 0; q < Q; q++) {
          const uint32_t v = w.get(q);
          w.put(q, (v & 0xffffu) | (v << 16));
        }
      }
      if (a.write_fields) {
        a.ux[iB] = a.ux[i0]; a.uy[iB] = a.uy[i0]; a.uz[iB] = a.uz[i0]; a.rho[iB] = a.rho[i0];
      }
    }
    const bool storeA = catA != CAT_KEEP, storeB = catB != CAT_KEEP;
    if (storeA && storeB) {
#pragma unroll
      for (int q = 0; q < Q; q++) gw(q) = w.get(q);
    } else if (storeA) {
#pragma unroll
      for (int q = 0; q < Q; q++) gh(q, 0) = __ushort_as_half((unsigned short)(w.get(q) & 0xffffu));
    } else if (storeB) {
#pragma unroll
      for (int q = 0; q < Q; q++) gh(q, 1) = __ushort_as_half((unsigned short)(w.get(q) >> 16));
    }
  }
  constexpr double inv_sc = 1.0 / (double)SC;   // a power of two: exact
  pair_force_partial(Fx * inv_sc, Fy * inv_sc, Fz * inv_sc, near_any, a, x0 & ~31, y, z);
}

}  // namespace wt
