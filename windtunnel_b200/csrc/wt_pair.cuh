// wt_pair.cuh — the fused step, two adjacent cells per thread, both collided
// at once with sm_100's packed float32x2 instructions (half or float32
// storage; PairIO holds what differs between the two).
//
// Same semantics and per-cell rules as k_step (wt_step.cuh) and the lean
// kernel: js/lbm.js:303-466 (stepSlab) followed by js/lbm.js:473-512
// (_boundaries), the collision of collide_x2 (js/lbm.js:377-460
// re-associated over opposite pairs) in the storage's scaled units.
//
// Thread t of block b owns cells x0 = 2 (b*pair_bx + t) and x0 + 1 of row
// (y, z); nx is even, so every 32-bit word (x0, x0+1) of a population plane
// is aligned. What the layout of the work buys, per pair of cells:
//   * one aligned load of the pair per direction (the x-shifted directions:
//     half storage adds one 16-bit load of the neighbouring half at the same
//     address +-2 bytes and a byte permute, float32 storage loads the
//     straddling pair as two 4-byte words), one store of the pair (for half
//     storage after one conversion to a half pair);
//   * every floating-point operation of the collision issued once for both
//     cells (FADD2 / FMUL2 / FFMA2); only the five reciprocals / square roots
//     per cell stay scalar.
// Registers: the 19 loaded words stay packed (half pairs for half storage).
// A first pass converts them pair of directions by pair and accumulates the
// moments (density, momentum, the six second moments); the equilibrium and
// the Smagorinsky stress follow from those analytically (the D3Q19
// equilibrium's second moment is dr/3 + r u u). A second pass converts the
// words again and writes each output word as soon as it is formed. The
// momentum exchange of the re-gathered body links is reduced per 32-cell
// segment before the collision, so its float64 sums are not live across it.
//
// Boundary cells: the inlet cell x = 0 stores the equilibrium and the outlet
// cell x = nx-1 stores a copy of cell nx-2 (js/lbm.js:504-511); both sit in
// a pair whose other cell is computed, so the store of that pair selects its
// halves with one byte permute per word (the outlet half takes the computed
// half of cell nx-2, its own arithmetic is discarded). Near-wall and
// free-slip shell cells re-gather the affected halves of their words before
// the first pass; solid cells keep their stale populations (pairs holding
// one store only the other half). Rows of the edge planes and the floor row
// (whose cells are solid or equilibrium) take their own store-only paths.
// Conditions: half or float32 storage, float32 collision, stationary walls, nx even,
// both population buffers under 2^31 bytes (the lean kernel's 32-bit byte
// offsets, StepArgs srcb / dstb).
#pragma once

#include "wt_x2.cuh"

namespace wt {

// Threads per block (each block one x-segment of one row, two cells per
// thread) and the resident blocks per SM the register budget is set for, the
// fastest measured on B200 (launched with programmatic dependent launch):
// 128 threads for both storages; half storage 7 blocks (72 registers, 28
// warps; 80 registers at 24 warps lose 3%; 64-thread blocks 0.9% and 32-thread
// blocks 8% slower), float32 storage 6 blocks (80 registers, no spills, 24
// warps; 64-thread blocks 1.5% slower).
template <class S>
constexpr int pair_bx() { return 128; }
template <class S>
constexpr int pair_min_blocks() { return sizeof(S) == 2 ? 7 : 6; }

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  return __byte_perm(a, b, sel);
}

// half pair word (lo = cell x0, hi = cell x0+1) -> float pair (.x, .y)
__device__ __forceinline__ f2 h2f(uint32_t w) {
  __half2 h;
  memcpy(&h, &w, 4);
  return __half22float2(h);
}

// float pair -> half pair word, round to nearest
__device__ __forceinline__ uint32_t f2h(f2 v) {
  const __half2 h = __float22half2_rn(v);
  uint32_t w;
  memcpy(&w, &h, 4);
  return w;
}

// float pair -> half pair word, stochastic rounding with 32 random bits
__device__ __forceinline__ uint32_t f2h_sr(f2 v, uint32_t rbits) {
  const __half2 h = sr_half2(v.y, v.x, rbits);   // (hi <- .y, lo <- .x)
  uint32_t w;
  memcpy(&w, &h, 4);
  return w;
}

__device__ __forceinline__ uint32_t ld32(const char* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}
__device__ __forceinline__ uint32_t ld16(const char* p) {
  return *reinterpret_cast<const uint16_t*>(p);
}

// Byte-permute selector that writes the half v (low 16 bits) into half L of w.
__device__ __forceinline__ uint32_t put_half(uint32_t w, uint32_t v, int L) {
  return prmt(w, v, L ? 0x5410u : 0x3254u);
}

// Storage-specific pieces of the pair kernel. W is the pair (x0, x0+1) of
// one direction as it sits in memory, R one stored element.
template <class S>
struct PairIO;

template <>
struct PairIO<__half> {
  using W = uint32_t;
  using R = uint16_t;
  static constexpr float SC = (float)WT_F16_SCALE;
  // (x0, x0+1) at p; (x0-1, x0) from the half at p and the word at p+2;
  // (x0+1, x0+2) from the word at p-2 and the half at p+2
  __device__ __forceinline__ static W load0(const char* p) { return ld32(p); }
  __device__ __forceinline__ static W load_plus(const char* p) {
    return prmt(ld16(p), ld32(p + 2), 0x5410u);
  }
  __device__ __forceinline__ static W load_minus(const char* p) {
    return prmt(ld32(p - 2), ld16(p + 2), 0x5432u);
  }
  __device__ __forceinline__ static f2 to_f2(W w) { return h2f(w); }
  __device__ __forceinline__ static W pack(f2 g) { return f2h(g); }
  __device__ __forceinline__ static W pack_sr(f2 g, uint32_t r) { return f2h_sr(g, r); }
  __device__ __forceinline__ static W eq(const StepArgs<__half>& a, int q) { return a.eq2[q]; }
  __device__ __forceinline__ static W fix(W v, W e, bool inlet, bool outlet) {
    return prmt(v, e, inlet ? 0x3254u : (outlet ? 0x1010u : 0x3210u));
  }
  __device__ __forceinline__ static W put(W w, R v, int L) { return put_half(w, v, L); }
  __device__ __forceinline__ static R lane(W w, int L) { return (R)(L ? w >> 16 : w); }
  __device__ __forceinline__ static float raw(R v) {
    __half h;
    memcpy(&h, &v, 2);
    return __half2float(h);
  }
};

template <>
struct PairIO<float> {
  using W = float2;
  using R = float;
  static constexpr float SC = 1.0f;
  // (x0, x0+1) at p as one 8-byte load; the x-shifted pairs straddle two
  // aligned words and are two 4-byte loads at p and p+4
  __device__ __forceinline__ static W load0(const char* p) {
    return *reinterpret_cast<const float2*>(p);
  }
  __device__ __forceinline__ static W load_plus(const char* p) {
    return make_float2(*reinterpret_cast<const float*>(p), *reinterpret_cast<const float*>(p + 4));
  }
  __device__ __forceinline__ static W load_minus(const char* p) {
    return make_float2(*reinterpret_cast<const float*>(p), *reinterpret_cast<const float*>(p + 4));
  }
  __device__ __forceinline__ static f2 to_f2(W w) { return w; }
  __device__ __forceinline__ static W pack(f2 g) { return g; }
  __device__ __forceinline__ static W pack_sr(f2 g, uint32_t) { return g; }
  __device__ __forceinline__ static W eq(const StepArgs<float>& a, int q) {
    return make_float2(a.eq[q], a.eq[q]);
  }
  __device__ __forceinline__ static W fix(W v, W e, bool inlet, bool outlet) {
    return make_float2(inlet ? e.x : v.x, outlet ? v.x : v.y);
  }
  __device__ __forceinline__ static W put(W w, R v, int L) {
    return L ? make_float2(w.x, v) : make_float2(v, w.y);
  }
  __device__ __forceinline__ static R lane(W w, int L) { return L ? w.y : w.x; }
  __device__ __forceinline__ static float raw(R v) { return v; }
};

// Re-gather the bounce-back and free-slip directions of cell xL = x0 + L (raw
// half bits into half L of each word), js/lbm.js:334-368 for the bounce-back
// links (stationary walls). The momentum exchange of body links accumulates
// in float64 in raw units.
template <class S>
__device__ __forceinline__ void pair_patch(const StepArgs<S>& a, long long iL, int xL, int y,
                                           int z, bool near_cell, bool shell, int L,
                                           typename PairIO<S>::W (&w)[Q], double& Fx,
                                           double& Fy, double& Fz) {
  using IO = PairIO<S>;
  using R = typename IO::R;
  const unsigned long long m = near_cell ? a.nmask[iL] : 0ull;
  const unsigned sm = (unsigned)m, om = (unsigned)(m >> 32);
  const R* F = reinterpret_cast<const R*>(a.F);
#define WT_PAIR_PATCH(q)                                                                   \
  if ((sm >> (q)) & 1u) {                                                                  \
    const R v = F[opp(q) * a.n + iL];                                                      \
    if ((om >> (q)) & 1u) {                                                                \
      const float d = 2.0f * IO::raw(v);                                                   \
      Fx -= (double)(d * (float)ex(q));                                                    \
      Fy -= (double)(d * (float)ey(q));                                                    \
      Fz -= (double)(d * (float)ez(q));                                                    \
    }                                                                                      \
    w[q] = IO::put(w[q], v, L);                                                            \
  } else if (shell) {                                                                      \
    const int sy0 = y - ey(q), sz0 = z - ez(q);                                            \
    const bool ym = sy0 == 0 || sy0 == a.ny - 1, zm = sz0 == 0 || sz0 == a.nz - 1;         \
    if (ym || zm) {                                                                        \
      /* the mirrored direction, chosen among compile-time constants */                    \
      const int qq = ym ? (zm ? mirror_z(mirror_y(q)) : mirror_y(q)) : mirror_z(q);        \
      const long long src = (xL - ex(q)) + (long long)a.nx * (ym ? y : sy0) +              \
                            a.nxy * (zm ? z : sz0);                                        \
      w[q] = IO::put(w[q], F[qq * a.n + src], L);                                          \
    }                                                                                      \
  }
  WT_PAIR_PATCH(1) WT_PAIR_PATCH(2) WT_PAIR_PATCH(3) WT_PAIR_PATCH(4) WT_PAIR_PATCH(5)
  WT_PAIR_PATCH(6) WT_PAIR_PATCH(7) WT_PAIR_PATCH(8) WT_PAIR_PATCH(9) WT_PAIR_PATCH(10)
  WT_PAIR_PATCH(11) WT_PAIR_PATCH(12) WT_PAIR_PATCH(13) WT_PAIR_PATCH(14) WT_PAIR_PATCH(15)
  WT_PAIR_PATCH(16) WT_PAIR_PATCH(17) WT_PAIR_PATCH(18)
#undef WT_PAIR_PATCH
}

// Force partial of a pair-kernel warp: its 64 cells are two 32-cell
// segments (lanes 0-15 and 16-31). Each half-warp that holds a near-wall
// cell sums its doubles in a fixed order and its first lane stores them in
// the segment's slot. Every lane must call it.
template <class S>
__device__ __forceinline__ void pair_force_partial(double fx, double fy, double fz,
                                                   bool near_cell, const StepArgs<S>& a, int y,
                                                   int z) {
  const unsigned any = __ballot_sync(0xffffffffu, near_cell);
  if (any == 0u) return;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o, 16);
    fy += __shfl_down_sync(0xffffffffu, fy, o, 16);
    fz += __shfl_down_sync(0xffffffffu, fz, o, 16);
  }
  const int lane = threadIdx.x & 31;
  const unsigned half_bits = lane < 16 ? (any & 0xffffu) : (any >> 16);
  if ((lane & 15) == 0 && half_bits) {
    const int x = 2 * (blockIdx.x * pair_bx<S>() + (threadIdx.x & ~15));
    const int slot = a.wslot[seg_of(x, y, z, a.nx, a.ny)];
    if (slot >= 0) {
      a.part[3 * (size_t)slot] = fx;
      a.part[3 * (size_t)slot + 1] = fy;
      a.part[3 * (size_t)slot + 2] = fz;
    } else {
      atomicOr(a.err, 2u);   // slot table out of date: reported, never silently dropped
    }
  }
}

// Store of the pair's two cells in the store-only rows: the edge planes and
// the ceiling take the free-stream equilibrium, the floor row the
// equilibrium unless solid (js/lbm.js:488-503).
template <class S>
__device__ __forceinline__ void pair_edge_row(const StepArgs<S>& a, long long i0, int x0, int y,
                                              int z) {
  using IO = PairIO<S>;
  using W = typename IO::W;
  using R = typename IO::R;
  char* Gb = reinterpret_cast<char*>(a.G + i0);
  auto gw = [&](int q) -> W& { return *reinterpret_cast<W*>(Gb + a.dstb[q]); };
  auto gh = [&](int q, int L) -> R& {
    return *reinterpret_cast<R*>(Gb + a.dstb[q] + sizeof(R) * L);
  };
  if (z == 0 || z == a.nz - 1 || y == a.ny - 1) {
    // end planes and ceiling: the free-stream equilibrium (js/lbm.js:490-503)
#pragma unroll
    for (int q = 0; q < Q; q++) gw(q) = IO::eq(a, q);
    if (a.write_fields) {
      *reinterpret_cast<float2*>(a.ux + i0) = make_float2(a.u0f, a.u0f);
      *reinterpret_cast<float2*>(a.uy + i0) = make_float2(0.f, 0.f);
      *reinterpret_cast<float2*>(a.uz + i0) = make_float2(0.f, 0.f);
      *reinterpret_cast<float2*>(a.rho + i0) = make_float2(1.f, 1.f);
    }
  } else if (y == 0) {
    // floor row: equilibrium unless solid (js/lbm.js:492-494), the inlet
    // cell always (js/lbm.js:489 comes first); the outlet copies column
    // nx-2, which ends up as that column's choice
    const uint32_t fl = ld16(reinterpret_cast<const char*>(a.flags + i0));
    const bool outlet = x0 == a.nx - 2;
#pragma unroll
    for (int L = 0; L < 2; L++) {
      const uint32_t fb = (L == 0 && x0 == 0) ? 0u : (outlet ? fl : (fl >> (8 * L)));
      if (fb & FLAG_SOLID_MASK) {
        if (L == 1 && outlet) {
#pragma unroll
          for (int q = 0; q < Q; q++) gh(q, 1) = gh(q, 0);
          if (a.write_fields) {
            a.ux[i0 + 1] = a.ux[i0]; a.uy[i0 + 1] = a.uy[i0];
            a.uz[i0 + 1] = a.uz[i0]; a.rho[i0 + 1] = a.rho[i0];
          }
        }
        continue;
      }
#pragma unroll
      for (int q = 0; q < Q; q++) gh(q, L) = IO::lane(IO::eq(a, q), 0);
      if (a.write_fields) {
        a.ux[i0 + L] = a.u0f; a.uy[i0 + L] = 0.f; a.uz[i0 + L] = 0.f; a.rho[i0 + L] = 1.f;
      }
    }
  }
}

// The cells of a pair and what the step does with each.
struct PairCells {
  bool inlet, outlet, solid0, solid1, fluid0, fluid1, near0, near1;
};

__device__ __forceinline__ PairCells pair_cells(uint32_t fl, int x0, int nx) {
  PairCells c;
  c.inlet = x0 == 0;
  c.outlet = x0 == nx - 2;
  c.solid0 = (fl & FLAG_SOLID_MASK) != 0;
  // the outlet cell is a copy of cell nx-2 whatever its own code
  c.solid1 = !c.outlet && ((fl >> 8) & FLAG_SOLID_MASK) != 0;
  // cells whose collision is kept: cell 0 unless inlet or solid; cell 1
  // unless solid or the outlet copy
  c.fluid0 = !c.inlet && !c.solid0;
  c.fluid1 = !c.outlet && !c.solid1;
  c.near0 = c.fluid0 && (fl & FLAG_NEAR);
  c.near1 = c.fluid1 && ((fl >> 8) & FLAG_NEAR);
  return c;
}

// Collision of an interior pair whose 19 words are loaded and re-gathered,
// and the store of its outputs (and, on the last step, its fields).
template <class S, bool SR>
__device__ __forceinline__ void pair_collide_store(const StepArgs<S>& a,
                                                   const typename PairIO<S>::W (&w)[Q],
                                                   long long i0, const PairCells& cells) {
  using IO = PairIO<S>;
  using W = typename IO::W;
  using R = typename IO::R;
  constexpr float SC = IO::SC;
  const bool inlet = cells.inlet, outlet = cells.outlet, solid0 = cells.solid0,
             solid1 = cells.solid1, fluid0 = cells.fluid0, fluid1 = cells.fluid1;
  char* Gb = reinterpret_cast<char*>(a.G + i0);
  auto gw = [&](int q) -> W& { return *reinterpret_cast<W*>(Gb + a.dstb[q]); };
  auto gh = [&](int q, int L) -> R& {
    return *reinterpret_cast<R*>(Gb + a.dstb[q] + sizeof(R) * L);
  };
  // ---- pass 1: moments --------------------------------------------------
  f2 dr, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
  {
    const f2 f0 = IO::to_f2(w[0]);
    f2 fa = IO::to_f2(w[1]), fb = IO::to_f2(w[2]);
    f2 s = padd(fa, fb), d = psub(fa, fb);
    dr = padd(f0, s); jx = d; pxx = s;
    fa = IO::to_f2(w[3]); fb = IO::to_f2(w[4]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jy = d; pyy = s;
    fa = IO::to_f2(w[5]); fb = IO::to_f2(w[6]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jz = d; pzz = s;
    fa = IO::to_f2(w[7]); fb = IO::to_f2(w[8]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jx = padd(jx, d); jy = padd(jy, d); pxx = padd(pxx, s);
    pyy = padd(pyy, s); pxy = s;
    fa = IO::to_f2(w[9]); fb = IO::to_f2(w[10]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jx = padd(jx, d); jy = psub(jy, d); pxx = padd(pxx, s);
    pyy = padd(pyy, s); pxy = psub(pxy, s);
    fa = IO::to_f2(w[11]); fb = IO::to_f2(w[12]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jx = padd(jx, d); jz = padd(jz, d); pxx = padd(pxx, s);
    pzz = padd(pzz, s); pxz = s;
    fa = IO::to_f2(w[13]); fb = IO::to_f2(w[14]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jx = padd(jx, d); jz = psub(jz, d); pxx = padd(pxx, s);
    pzz = padd(pzz, s); pxz = psub(pxz, s);
    fa = IO::to_f2(w[15]); fb = IO::to_f2(w[16]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jy = padd(jy, d); jz = padd(jz, d); pyy = padd(pyy, s);
    pzz = padd(pzz, s); pyz = s;
    fa = IO::to_f2(w[17]); fb = IO::to_f2(w[18]); s = padd(fa, fb); d = psub(fa, fb);
    dr = padd(dr, s); jy = padd(jy, d); jz = psub(jz, d); pyy = padd(pyy, s);
    pzz = padd(pzz, s); pyz = psub(pyz, s);
  }
  // ---- macroscopic state, relaxation rates -------------------------------
  const f2 r = padd(pk(SC), dr);
  const f2 inv = prcp(r);
  const f2 vx = pmul(jx, inv), vy = pmul(jy, inv), vz = pmul(jz, inv);
  const f2 usq = pfma(vz, vz, pfma(vy, vy, pmul(vx, vx)));
  const f2 A = pfma(pmul(pk(-1.5f), r), usq, dr);   // dr - 1.5 r u^2 (raw)
  const bool ok0 = !fluid0 || (r.x > 0.0f && r.x < 3.0e38f);
  const bool ok1 = !fluid1 || (r.y > 0.0f && r.y < 3.0e38f);
  if (!(ok0 && ok1)) atomicOr(a.err, 1u);
  f2 om = pk(a.omega0f), omm = pk(a.omm0f);
  if (a.les) {
    // non-equilibrium second moments: P - (dr/3 + r u u), js/lbm.js:420-425
    const f2 rvx = pmul(r, vx), rvy = pmul(r, vy), rvz = pmul(r, vz);
    const f2 dr3 = pmul(pk(1.0f / 3.0f), dr);
    const f2 sxx = pfma(pmul(pk(-1.0f), rvx), vx, psub(pxx, dr3));
    const f2 syy = pfma(pmul(pk(-1.0f), rvy), vy, psub(pyy, dr3));
    const f2 szz = pfma(pmul(pk(-1.0f), rvz), vz, psub(pzz, dr3));
    const f2 sxy = pfma(pmul(pk(-1.0f), rvx), vy, pxy);
    const f2 sxz = pfma(pmul(pk(-1.0f), rvx), vz, pxz);
    const f2 syz = pfma(pmul(pk(-1.0f), rvy), vz, pyz);
    const f2 off = pfma(syz, syz, pfma(sxz, sxz, pmul(sxy, sxy)));
    const f2 q2 = pfma(sxx, sxx, pfma(syy, syy, pfma(szz, szz, padd(off, off))));
    // 18 sqrt(2) Cs^2 |Pi| / rho with |Pi| = sqrt(2 q2): 36 Cs^2 sqrt(q2) / r
    const f2 x = pmul(pmul(pk(0.5f * a.les_cf), psqrt(q2)), inv);
    const f2 te = pfma(pk(0.5f), psqrt(pfma(pk(a.tau0f), pk(a.tau0f), x)), pk(0.5f * a.tau0f));
    om = prcp(te);
    if (a.trt) {
      const f2 t5 = psub(te, pk(0.5f));
      omm = pmul(t5, prcp(pfma(pk(0.5f), t5, pk(a.lamf))));
    } else {
      omm = om;
    }
  }
  if (a.write_fields) {
    const f2 rho = pmul(r, pk(1.0f / SC));
    if (fluid0 && (fluid1 || outlet)) {
      const float2 u = outlet ? make_float2(vx.x, vx.x) : vx;
      const float2 v = outlet ? make_float2(vy.x, vy.x) : vy;
      const float2 ww = outlet ? make_float2(vz.x, vz.x) : vz;
      const float2 rr = outlet ? make_float2(rho.x, rho.x) : rho;
      *reinterpret_cast<float2*>(a.ux + i0) = u;
      *reinterpret_cast<float2*>(a.uy + i0) = v;
      *reinterpret_cast<float2*>(a.uz + i0) = ww;
      *reinterpret_cast<float2*>(a.rho + i0) = rr;
    } else {
      if (fluid0) {
        a.ux[i0] = vx.x; a.uy[i0] = vy.x; a.uz[i0] = vz.x; a.rho[i0] = rho.x;
      } else if (inlet) {
        a.ux[i0] = a.u0f; a.uy[i0] = 0.f; a.uz[i0] = 0.f; a.rho[i0] = 1.f;
      }
      if (fluid1) {
        a.ux[i0 + 1] = vx.y; a.uy[i0 + 1] = vy.y; a.uz[i0 + 1] = vz.y;
        a.rho[i0 + 1] = rho.y;
      } else if (outlet) {
        // copy of a solid cell nx-2: its fields as they stand
        a.ux[i0 + 1] = a.ux[i0]; a.uy[i0 + 1] = a.uy[i0];
        a.uz[i0 + 1] = a.uz[i0]; a.rho[i0 + 1] = a.rho[i0];
      }
    }
  }
  // ---- per-cell constants of the update ---------------------------------
  // g_a = P + M, g_b = P - M over the opposite pair (a, b) with
  //   P = (1 - om)/2 s + om w (A + 4.5 r c^2),  M = (1 - omm)/2 d + omm 3 w r c
  // (s = f_a + f_b, d = f_a - f_b, c = c_a . u); w = 1/18 face, 1/36 edge
  const f2 al = pfma(pk(-0.5f), om, pk(0.5f));
  const f2 be = pfma(pk(-0.5f), omm, pk(0.5f));
  const f2 omr = pmul(om, r), ommr = pmul(omm, r), omA = pmul(om, A);
  const f2 k45f = pmul(pk(0.25f), omr), k45e = pmul(pk(0.125f), omr);
  const f2 kaf = pmul(pk((float)(1.0 / 18)), omA), kae = pmul(pk((float)(1.0 / 36)), omA);
  const f2 k3f = pmul(pk((float)(1.0 / 6)), ommr), k3e = pmul(pk((float)(1.0 / 12)), ommr);
  // a solid cell keeps its stale populations, and so does the outlet copy
  // of a solid cell nx-2 until the copy below
  const bool keep0 = solid0 && !inlet, keep1 = solid1 || (outlet && solid0);
  const bool keep_any = keep0 || keep1;
  // stochastic rounding: a hash of (pair, step), then per output word its
  // product with a distinct odd constant (one multiply per word)
  uint32_t h = 0;
  if constexpr (SR) {
    h = ((uint32_t)i0 ^ (uint32_t)(i0 >> 32)) * 0x9E3779B1u ^ a.sr_seed;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
  }
  auto put = [&](int q, f2 g) {
    W v;
    if constexpr (SR) {
      v = IO::pack_sr(g, h * (0x9E3779B1u * (2u * (uint32_t)q + 1u)));
    } else {
      v = IO::pack(g);
    }
    // the inlet's low cell takes the equilibrium, the outlet's high cell
    // takes cell nx-2's value
    v = IO::fix(v, IO::eq(a, q), inlet, outlet);
    if (!keep_any) {
      gw(q) = v;
    } else {
      // a solid cell of the pair keeps its stale population
      if (!keep0) gh(q, 0) = IO::lane(v, 0);
      if (!keep1) gh(q, 1) = IO::lane(v, 1);
    }
  };
  // ---- pass 2: outputs ----------------------------------------------------
  {
    const f2 f0 = IO::to_f2(w[0]);
    put(0, pfma(pfma(pk(-1.0f), om, pk(1.0f)), f0, pmul(pk((float)(1.0 / 3)), omA)));
  }
#define WT_PAIR_OUT(qa, C, K45, KA, K3)                 \
  {                                                     \
const f2 fa = IO::to_f2(w[qa]), fb = IO::to_f2(w[qa + 1]);      \
const f2 s = padd(fa, fb), d = psub(fa, fb);        \
const f2 c = C;                                     \
const f2 X = pfma(pmul(c, c), K45, KA);             \
const f2 Y = pmul(K3, c);                           \
const f2 P = pfma(al, s, X), M = pfma(be, d, Y);    \
put(qa, padd(P, M));                                \
put(qa + 1, psub(P, M));                            \
  }
  WT_PAIR_OUT(1, vx, k45f, kaf, k3f)
  WT_PAIR_OUT(3, vy, k45f, kaf, k3f)
  WT_PAIR_OUT(5, vz, k45f, kaf, k3f)
  WT_PAIR_OUT(7, padd(vx, vy), k45e, kae, k3e)
  WT_PAIR_OUT(9, psub(vx, vy), k45e, kae, k3e)
  WT_PAIR_OUT(11, padd(vx, vz), k45e, kae, k3e)
  WT_PAIR_OUT(13, psub(vx, vz), k45e, kae, k3e)
  WT_PAIR_OUT(15, padd(vy, vz), k45e, kae, k3e)
  WT_PAIR_OUT(17, psub(vy, vz), k45e, kae, k3e)
#undef WT_PAIR_OUT
  if (outlet && solid0) {
    // copy of a solid cell nx-2, whose g this step does not write
#pragma unroll
    for (int q = 0; q < Q; q++) gh(q, 1) = gh(q, 0);
  }
}

template <class S, bool SR>
__global__ void __launch_bounds__(pair_bx<S>(), pair_min_blocks<S>())
    k_step_pair(const __grid_constant__ StepArgs<S> a) {
  using IO = PairIO<S>;
  using W = typename IO::W;
  constexpr float SC = IO::SC;
  pdl_enter();   // programmatic dependent launch (launch_pdl)
  const int x0 = 2 * (blockIdx.x * pair_bx<S>() + threadIdx.x);
  const int y = blockIdx.y, z = blockIdx.z;
  const long long i0 = (long long)x0 + (long long)a.nx * y + a.nxy * z;
  const bool active = x0 < a.nx;
  if (z == 0 || z == a.nz - 1 || y == a.ny - 1 || y == 0) {
    // rows that pull nothing; they hold no near-wall cell, so no force partial
    if (active) pair_edge_row<S>(a, i0, x0, y, z);
    return;
  }
  // interior row: pull every direction of both cells. The sources of the
  // pair (x0 - ex, x0 + 1 - ex) of row (y - ey, z - ez) lie inside the
  // buffer for every cell of an interior row.
  // L2 prefetch of the populations the warp a fixed distance ahead will
  // pull (StepArgs pf; set for half storage on lattices within twice the L2)
  prefetch_ahead(a, i0 - 2 * (long long)(threadIdx.x & 31));
  const char* Fb = reinterpret_cast<const char*>(a.F + i0);
  W w[Q];
  if (active) {
#define WT_PAIR_LOAD(q)                                                                  \
  {                                                                                      \
    const char* p = Fb + a.srcb[q];   /* byte address of the source of cell x0 */        \
    if constexpr (ex(q) == 0) w[q] = IO::load0(p);                                       \
    else if constexpr (ex(q) == 1) w[q] = IO::load_plus(p);                              \
    else w[q] = IO::load_minus(p);                                                       \
  }
    WT_PAIR_LOAD(0) WT_PAIR_LOAD(1) WT_PAIR_LOAD(2) WT_PAIR_LOAD(3) WT_PAIR_LOAD(4)
    WT_PAIR_LOAD(5) WT_PAIR_LOAD(6) WT_PAIR_LOAD(7) WT_PAIR_LOAD(8) WT_PAIR_LOAD(9)
    WT_PAIR_LOAD(10) WT_PAIR_LOAD(11) WT_PAIR_LOAD(12) WT_PAIR_LOAD(13) WT_PAIR_LOAD(14)
    WT_PAIR_LOAD(15) WT_PAIR_LOAD(16) WT_PAIR_LOAD(17) WT_PAIR_LOAD(18)
#undef WT_PAIR_LOAD
  }
  const uint32_t fl = active ? ld16(reinterpret_cast<const char*>(a.flags + i0)) : 0u;
  const PairCells c = pair_cells(fl, x0, a.nx);
  const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
  {
    // the momentum exchange of the re-gathered body links, summed per
    // 32-cell segment here, so that its doubles are not live across the
    // collision
    double Fx = 0, Fy = 0, Fz = 0;
    if (active && (c.near0 || (shell && c.fluid0)))
      pair_patch(a, i0, x0, y, z, c.near0, shell, 0, w, Fx, Fy, Fz);
    if (active && (c.near1 || (shell && c.fluid1)))
      pair_patch(a, i0 + 1, x0 + 1, y, z, c.near1, shell, 1, w, Fx, Fy, Fz);
    constexpr double inv_sc = 1.0 / (double)SC;   // a power of two: exact
    pair_force_partial(Fx * inv_sc, Fy * inv_sc, Fz * inv_sc, c.near0 || c.near1, a, y, z);
  }
  if (active) pair_collide_store<S, SR>(a, w, i0, c);
}

}  // namespace wt
