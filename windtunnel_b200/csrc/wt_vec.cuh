// wt_vec.cuh — the fused step with two cells per thread and vector loads.
//
// Same semantics as k_step (wt_step.cuh). Thread t of a block owns the two
// adjacent cells x0 = 2*(blockIdx.x*VEC_BX + t) and x0+1 of row (y, z) =
// (blockIdx.y, blockIdx.z). For every direction q it loads the aligned pair
// (x0, x0+1) of the source row (y - ey, z - ez) with one vector load
// (float2 / half2). Directions with ex = +1 need (x0-1, x0): the x0-1
// element is the previous lane's upper element, taken with a warp shuffle
// (lane 0 loads it); ex = -1 needs (x0+1, x0+2) with x0+2 from the next lane
// (lane 31 loads it). Address arithmetic and load / store instructions are
// thereby shared by two cells; the collision runs per cell in float32.
//
// Cells that are not plain fluid fall back to the per-cell rules of k_step:
// bounce-back / free-slip directions are patched from HBM (patch_special),
// inlet and edge rows store the equilibrium, solid cells keep their stale
// populations (scalar stores of the other cell of the pair), and the outlet
// column x = nx-1 receives column nx-2's values as the second half of its
// pair. Needs nx even; every row then starts on a pair boundary.
#pragma once

#include "wt_step.cuh"

namespace wt {

constexpr int VEC_BX = 64;   // threads per block: 128 cells of one row

template <class S>
struct Pair;
template <>
struct Pair<float> {
  using T = float2;
  __device__ __forceinline__ static float lo(T v) { return v.x; }
  __device__ __forceinline__ static float hi(T v) { return v.y; }
  __device__ __forceinline__ static T make(float a, float b) { return make_float2(a, b); }
};
template <>
struct Pair<__half> {
  using T = __half2;
  __device__ __forceinline__ static __half lo(T v) { return __low2half(v); }
  __device__ __forceinline__ static __half hi(T v) { return __high2half(v); }
  __device__ __forceinline__ static T make(__half a, __half b) { return __halves2half2(a, b); }
};

template <class S>
__device__ __forceinline__ S shfl_up1(S v) {
  if constexpr (sizeof(S) == 4) {
    return __shfl_up_sync(0xffffffffu, v, 1);
  } else {
    const unsigned short b = __shfl_up_sync(0xffffffffu, (unsigned)__half_as_ushort(v), 1);
    return __ushort_as_half(b);
  }
}
template <class S>
__device__ __forceinline__ S shfl_down1(S v) {
  if constexpr (sizeof(S) == 4) {
    return __shfl_down_sync(0xffffffffu, v, 1);
  } else {
    const unsigned short b = __shfl_down_sync(0xffffffffu, (unsigned)__half_as_ushort(v), 1);
    return __ushort_as_half(b);
  }
}

// Per-half-warp force partial: lanes 0-15 cover one 32-cell segment, lanes
// 16-31 the next. Every lane must call it.
template <class S>
__device__ __forceinline__ void pair_force_partial(double fx, double fy, double fz, bool near_any,
                                                   const StepArgs<S>& a, int xlane0, int y,
                                                   int z) {
  const unsigned m = __ballot_sync(0xffffffffu, near_any);
  if (!m) return;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o, 16);
    fy += __shfl_down_sync(0xffffffffu, fy, o, 16);
    fz += __shfl_down_sync(0xffffffffu, fz, o, 16);
  }
  const int lane = threadIdx.x & 31;
  const bool mine = (lane == 0 && (m & 0x0000ffffu)) || (lane == 16 && (m & 0xffff0000u));
  if (mine) {
    const int slot = a.wslot[seg_of(xlane0, y, z, a.nx, a.ny)];
    if (slot >= 0) {
      a.part[3 * (size_t)slot] = fx;
      a.part[3 * (size_t)slot + 1] = fy;
      a.part[3 * (size_t)slot + 2] = fz;
    } else {
      atomicOr(a.err, 2u);
    }
  }
}

// Per-cell category and collision into out[19]; returns false for a solid
// cell (its stale g must stay). `f` holds the plain pulled values.
template <class S>
__device__ __forceinline__ int cell_category(const StepArgs<S>& a, int x, int y, uint8_t fl) {
  if (x == 0) return CAT_EQ;
  if (fl & FLAG_SOLID_MASK) return CAT_KEEP;
  if (y == 0) return CAT_EQ;
  return CAT_FLUID;
}

template <class S, class IDX>
__global__ void __launch_bounds__(VEC_BX, 8) k_step_vec(const __grid_constant__ StepArgs<S> a) {
  using P = Pair<S>;
  using V = typename P::T;
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int x0 = 2 * (blockIdx.x * VEC_BX + t);
  const int y = blockIdx.y, z = blockIdx.z;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long i0 = (long long)x0 + (long long)nx * y + a.nxy * z;
  const bool active = x0 < nx;
  const bool edge_row = z == 0 || z == nz - 1 || y == ny - 1;
  const bool interior_row = !edge_row && y >= 1;
  double Fx = 0, Fy = 0, Fz = 0;
  bool near_any = false;

  if (!edge_row) {
    // occupancy of the pair (x0 == nx-2 .. nx-1 never needs nx-1's byte)
    uint8_t flA = 0, flB = 0;
    if (active) {
      flA = a.flags[i0];
      flB = a.flags[i0 + 1];
    }
    float fA[Q], fB[Q];
    if (interior_row) {
      // ---- vector pull of the 19 source rows (all lanes: shuffles need them) ----
      const S* Fi = a.F + i0;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        const IDX base = (IDX)a.src[q] + (IDX)ex(q);   // aligned pair of the source row
        V v;
        if (active) v = *reinterpret_cast<const V*>(Fi + base);
        else v = P::make(S(), S());
        S a0, a1;
        if (ex(q) == 0) {
          a0 = P::lo(v); a1 = P::hi(v);
        } else if (ex(q) == 1) {
          S prev = shfl_up1<S>(P::hi(v));
          if (lane == 0 && active) prev = Fi[base - 1];
          a0 = prev; a1 = P::lo(v);
        } else {
          S nxt = shfl_down1<S>(P::lo(v));
          if (lane == 31 && active) nxt = Fi[base + 2];
          a0 = P::hi(v); a1 = nxt;
        }
        fA[q] = Store<S>::load_f(a0);
        fB[q] = Store<S>::load_f(a1);
      }
    }
    if (active) {
      const int catA = cell_category(a, x0, y, flA);
      const int catB = (x0 + 1 == nx - 1) ? CAT_NONE : cell_category(a, x0 + 1, y, flB);
      const bool dupA = false;   // the pair (nx-2, nx-1) carries the outlet copy itself
      S oA[Q], oB[Q];
      const bool shell = a.freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
      if (catA == CAT_FLUID) {
        const bool nearA = (flA & FLAG_NEAR) != 0;
        near_any |= nearA;
        if (nearA || shell) patch_special<S, float>(a, i0, x0, y, z, shell, fA, Fx, Fy, Fz);
        collide_fast<S>(a, fA, i0, dupA, nearA, RegOut<S>{oA});
      } else if (catA == CAT_EQ) {
#pragma unroll
        for (int q = 0; q < Q; q++) oA[q] = a.eq[q];
        if (a.write_fields) { a.ux[i0] = a.u0f; a.uy[i0] = 0.0f; a.uz[i0] = 0.0f; a.rho[i0] = 1.0f; }
      }
      if (catB == CAT_FLUID) {
        const bool nearB = (flB & FLAG_NEAR) != 0;
        near_any |= nearB;
        if (nearB || shell) patch_special<S, float>(a, i0 + 1, x0 + 1, y, z, shell, fB, Fx, Fy, Fz);
        collide_fast<S>(a, fB, i0 + 1, false, nearB, RegOut<S>{oB});
      } else if (catB == CAT_EQ) {
#pragma unroll
        for (int q = 0; q < Q; q++) oB[q] = a.eq[q];
        if (a.write_fields) {
          a.ux[i0 + 1] = a.u0f; a.uy[i0 + 1] = 0.0f; a.uz[i0 + 1] = 0.0f; a.rho[i0 + 1] = 1.0f;
        }
      } else if (catB == CAT_NONE) {
        // x0+1 is the outlet: it takes whatever cell nx-2 (= x0) ends up holding
        if (catA == CAT_KEEP) {
          S* Gi = a.G + i0;
#pragma unroll
          for (int q = 0; q < Q; q++) oB[q] = Gi[(IDX)a.dst[q]];
          if (a.write_fields) {
            a.ux[i0 + 1] = a.ux[i0]; a.uy[i0 + 1] = a.uy[i0]; a.uz[i0 + 1] = a.uz[i0];
            a.rho[i0 + 1] = a.rho[i0];
          }
        } else {
#pragma unroll
          for (int q = 0; q < Q; q++) oB[q] = oA[q];
          if (a.write_fields) {
            a.ux[i0 + 1] = a.ux[i0]; a.uy[i0 + 1] = a.uy[i0]; a.uz[i0 + 1] = a.uz[i0];
            a.rho[i0 + 1] = a.rho[i0];
          }
        }
      }
      S* Gi = a.G + i0;
      const bool keepA = catA == CAT_KEEP, keepB = catB == CAT_KEEP;
      if (!keepA && !keepB) {
#pragma unroll
        for (int q = 0; q < Q; q++)
          *reinterpret_cast<V*>(Gi + (IDX)a.dst[q]) = P::make(oA[q], oB[q]);
      } else {
#pragma unroll
        for (int q = 0; q < Q; q++) {
          if (!keepA) Gi[(IDX)a.dst[q]] = oA[q];
          if (!keepB) Gi[(IDX)a.dst[q] + 1] = oB[q];
        }
      }
    }
  } else if (active) {
    // ceiling / end planes: equilibrium for both cells (the outlet's copy of an
    // equilibrium cell is the equilibrium)
    S* Gi = a.G + i0;
#pragma unroll
    for (int q = 0; q < Q; q++)
      *reinterpret_cast<V*>(Gi + (IDX)a.dst[q]) = P::make(a.eq[q], a.eq[q]);
    if (a.write_fields) {
      a.ux[i0] = a.u0f; a.uy[i0] = 0.0f; a.uz[i0] = 0.0f; a.rho[i0] = 1.0f;
      a.ux[i0 + 1] = a.u0f; a.uy[i0 + 1] = 0.0f; a.uz[i0 + 1] = 0.0f; a.rho[i0 + 1] = 1.0f;
    }
  }
  pair_force_partial(Fx, Fy, Fz, near_any, a, x0 & ~31, y, z);
}

inline dim3 vec_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nx + 2 * VEC_BX - 1) / (2 * VEC_BX)), (unsigned)ny, (unsigned)nz);
}

}  // namespace wt
