// wt_step.cuh — the fused D3Q19 step: pull-stream + halfway bounce-back +
// momentum exchange + moments + equilibrium + Smagorinsky + TRT collide +
// inlet / outlet / far-field boundaries, one launch per time step.
//
// Semantics follow one reference step, js/lbm.js:285-291: stepSlab over the
// interior (js/lbm.js:303-466) followed by _boundaries (js/lbm.js:473-512).
// The boundary pass is folded into the same launch by giving every cell a
// category that reproduces the reference's write order:
//   x == 0                         inlet: equilibrium (rho=1, u=(u0,0,0))
//   z == 0 | z == nz-1 | y == ny-1 end planes / ceiling: equilibrium
//   solid                          untouched (solid cells keep stale values)
//   y == 0 (not solid)             floor: equilibrium
//   otherwise                      fluid: collide and pull-stream
// and the outlet column x = nx-1 receives a copy of whatever column nx-2
// ends up holding; the thread of cell (nx-2, y, z) writes both cells, so the
// copy needs neither a second pass nor a second computation.
#pragma once

#include <type_traits>

#include "wt_common.cuh"

namespace wt {

// Load a stored deviation as the arithmetic type M.
template <class M, class S>
__device__ __forceinline__ M ld(S v) {
  if constexpr (std::is_same<M, double>::value) return Store<S>::load_d(v);
  else return Store<S>::load_f(v);
}

// Stochastic rounding of two floats to a half pair (hi <- a, lo <- b) with
// the random bits rbits (sm_100a cvt.rs).
__device__ __forceinline__ __half2 sr_half2(float a, float b, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
  return *reinterpret_cast<__half2*>(&d);
}

// Output writer of the collision: a register array of the step's outputs.
template <class S>
struct RegOut {
  S (&o)[Q];
  __device__ __forceinline__ void put(int q, S v) { o[q] = v; }
};

enum : int { CAT_NONE = 0, CAT_EQ = 1, CAT_KEEP = 2, CAT_FLUID = 3 };

// Sum three doubles over a warp that covers one 32-cell segment, in a fixed
// order, and store them in the segment's partial slot. Exactly the segments
// that hold a near-wall cell own a slot (the table is rebuilt by voxelize),
// and each of them is written every step -- zeros when none of its links
// touches the body -- so all-fluid warps write nothing and no block-wide
// barrier is needed. Every lane of the warp must call it; `near_cell` marks a
// computed near-wall cell.
template <class S>
__device__ __forceinline__ void warp_force_partial_w(double fx, double fy, double fz,
                                                     bool near_cell, const StepArgs<S>& a,
                                                     long long seg) {
  if (__any_sync(0xffffffffu, near_cell)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      fx += __shfl_down_sync(0xffffffffu, fx, o);
      fy += __shfl_down_sync(0xffffffffu, fy, o);
      fz += __shfl_down_sync(0xffffffffu, fz, o);
    }
    if ((threadIdx.x & 31) == 0) {
      const int slot = a.wslot[seg];
      if (slot >= 0) {
        a.part[3 * (size_t)slot] = fx;
        a.part[3 * (size_t)slot + 1] = fy;
        a.part[3 * (size_t)slot + 2] = fz;
      } else {
        atomicOr(a.err, 2u);   // slot table out of date: reported, never silently dropped
      }
    }
  }
}

// Warp partial of the direct kernel: its warps cover 32-cell segments.
template <class S>
__device__ __forceinline__ void warp_force_partial(double fx, double fy, double fz,
                                                   bool near_cell, const StepArgs<S>& a) {
  const int x0 = blockIdx.x * STEP_BX + (threadIdx.x & ~31);
  warp_force_partial_w(fx, fy, fz, near_cell, a, seg_of(x0, blockIdx.y, blockIdx.z, a.nx, a.ny));
}

// Bounce-back link q of cell i toward solid neighbour j (code s):
// js/lbm.js:339-359. Returns the pulled population and accumulates the
// momentum exchange of links into the body (SOLID_OBJ).
template <class S, class M, int q>
__device__ __forceinline__ M bounce_link(const StepArgs<S>& a, long long i, long long j, int s,
                                         M rho_prev, double& Fx, double& Fy, double& Fz) {
  const M fd = ld<M>(a.F[opp(q) * a.n + i]);
  M corr = 0;
  if (a.mov) {
    const M cu = (M)ex(q) * (M)a.uwx[j] + (M)ey(q) * (M)a.uwy[j] + (M)ez(q) * (M)a.uwz[j];
    if (cu != (M)0) corr = (M)6 * (M)wq(q) * rho_prev * cu;
  }
  if (s == WT_SOLID_OBJ) {
    const M d = (M)2 * fd + corr;
    Fx -= (double)(d * (M)ex(q));
    Fy -= (double)(d * (M)ey(q));
    Fz -= (double)(d * (M)ez(q));
  }
  return fd + corr;
}

// Overwrite, in f (already holding the plain pulled values), the directions
// whose source is solid (bounce-back) or lies on a free-slip side plane
// (mirror gather). The solid / body neighbours come from the cell's
// precomputed mask (one load); the loads below depend only on it and on the
// cell position, so they are all in flight at once.
template <class S, class M>
__device__ __forceinline__ void patch_special(const StepArgs<S>& a, long long i, int x, int y,
                                              int z, bool shell, M (&f)[Q], double& Fx,
                                              double& Fy, double& Fz) {
  const unsigned long long m = a.nmask[i];
  const unsigned sm = (unsigned)m, om = (unsigned)(m >> 32);
  const M rho_prev = (M)(a.mov && sm ? a.rho[i] : 1.0f);
#define WT_PATCH(q)                                                                         \
  if ((sm >> (q)) & 1u) {                                                                   \
    const long long j = i - (ex(q) + (long long)ey(q) * a.nx + (long long)ez(q) * a.nxy);   \
    f[q] = bounce_link<S, M, q>(a, i, j, ((om >> (q)) & 1u) ? WT_SOLID_OBJ : WT_SOLID_WALL, \
                                rho_prev, Fx, Fy, Fz);                                      \
  } else if (shell) {                                                                       \
    int sy = y - ey(q), sz = z - ez(q), qq = q;                                             \
    bool refl = false;                                                                      \
    if (sy == 0 || sy == a.ny - 1) { sy = y; qq = mirror_y(qq); refl = true; }              \
    if (sz == 0 || sz == a.nz - 1) { sz = z; qq = mirror_z(qq); refl = true; }              \
    if (refl)                                                                               \
      f[q] = ld<M>(a.F[qq * a.n + (x - ex(q)) + (long long)a.nx * sy + a.nxy * sz]);        \
  }
  WT_PATCH(1) WT_PATCH(2) WT_PATCH(3) WT_PATCH(4) WT_PATCH(5) WT_PATCH(6) WT_PATCH(7)
  WT_PATCH(8) WT_PATCH(9) WT_PATCH(10) WT_PATCH(11) WT_PATCH(12) WT_PATCH(13) WT_PATCH(14)
  WT_PATCH(15) WT_PATCH(16) WT_PATCH(17) WT_PATCH(18)
#undef WT_PATCH
}

// Hardware approximations (relative error ~2^-22) used by the float32
// collisions: one instruction each instead of a correctly rounded sequence.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Float32 collision, re-associated: opposite pairs are carried as half sums
// and half differences, so moments, the equilibrium, the stress tensor of the
// Smagorinsky model and the TRT update share their partial results. The
// mathematics is that of js/lbm.js:377-460; only the rounding differs.
template <class S, class Out>
__device__ __forceinline__ void collide_fast(const StepArgs<S>& a, const float (&f)[Q],
                                             long long i, bool dup, bool near_cell, Out out) {
  // opposite pairs (a, b) in the order of js/lbm.js:443-460
  const float s1 = f[1] + f[2], d1 = f[1] - f[2];
  const float s3 = f[3] + f[4], d3 = f[3] - f[4];
  const float s5 = f[5] + f[6], d5 = f[5] - f[6];
  const float s7 = f[7] + f[8], d7 = f[7] - f[8];
  const float s9 = f[9] + f[10], d9 = f[9] - f[10];
  const float s11 = f[11] + f[12], d11 = f[11] - f[12];
  const float s13 = f[13] + f[14], d13 = f[13] - f[14];
  const float s15 = f[15] + f[16], d15 = f[15] - f[16];
  const float s17 = f[17] + f[18], d17 = f[17] - f[18];
  const float dr = ((f[0] + s1) + (s3 + s5)) + ((s7 + s9) + (s11 + s13)) + (s15 + s17);
  const float r = 1.0f + dr;
  if (!(r > 0.0f && r < 3.0e38f)) atomicOr(a.err, 1u);
  // Half storage takes the one-instruction approximations (its step is
  // issue-bound); float32 keeps the correctly rounded forms, which measured
  // faster there (the approximations' register allocation spills at 64).
  constexpr bool APPROX = std::is_same<S, __half>::value;
  const float inv = APPROX ? rcp_approx(r) : __frcp_rn(r);
  const float vx = ((d1 + d7) + (d9 + d11) + d13) * inv;
  const float vy = ((d3 + d7) - d9 + (d15 + d17)) * inv;
  const float vz = ((d5 + d11) - d13 + (d15 - d17)) * inv;
  if (a.write_fields) {
    a.rho[i] = r; a.ux[i] = vx; a.uy[i] = vy; a.uz[i] = vz;
    if (dup) { a.rho[i + 1] = r; a.ux[i + 1] = vx; a.uy[i + 1] = vy; a.uz[i + 1] = vz; }
  } else if (a.mov && near_cell) {
    a.rho[i] = r;
  }
  const float A = dr - r * 1.5f * (vx * vx + vy * vy + vz * vz);
  const float r3 = 3.0f * r, r45 = 4.5f * r;
  constexpr float WF = (float)(1.0 / 18), WE = (float)(1.0 / 36), W0 = (float)(1.0 / 3);
  // per pair: symmetric equilibrium part es = w(A + 4.5 r cu^2) and
  // antisymmetric part ea = 3 w r cu; sp = (n_a + n_b)/2, sm = (n_a - n_b)/2
  const float c1 = vx, c3 = vy, c5 = vz, c7 = vx + vy, c9 = vx - vy, c11 = vx + vz,
              c13 = vx - vz, c15 = vy + vz, c17 = vy - vz;
  const float wAF = WF * A, wAE = WE * A, w45F = WF * r45, w45E = WE * r45, w3F = WF * r3,
              w3E = WE * r3;
#define WT_PAIR(k, C)                                                          \
  const float sp##k = fmaf(0.5f, s##k, -fmaf(w45##C * c##k, c##k, wA##C));   \
  const float sm##k = fmaf(0.5f, d##k, -w3##C * c##k);
  WT_PAIR(1, F) WT_PAIR(3, F) WT_PAIR(5, F) WT_PAIR(7, E) WT_PAIR(9, E) WT_PAIR(11, E)
  WT_PAIR(13, E) WT_PAIR(15, E) WT_PAIR(17, E)
#undef WT_PAIR
  float om = a.omega0f, omm = a.omm0f;
  if (a.les) {
    // Pi_ab = sum n_q c_qa c_qb from the pair half sums (n_a + n_b = 2 sp)
    const float sxx = (sp1 + sp7) + (sp9 + sp11) + sp13;
    const float syy = (sp3 + sp7) + (sp9 + sp15) + sp17;
    const float szz = (sp5 + sp11) + (sp13 + sp15) + sp17;
    const float sxy = sp7 - sp9, sxz = sp11 - sp13, syz = sp15 - sp17;
    const float qq = sxx * sxx + syy * syy + szz * szz + 2.0f * (sxy * sxy + sxz * sxz + syz * syz);
    // SQ18 * cs2 * |Pi| / r with |Pi| = 2 sqrt(2 qq): 72 cs2 sqrt(qq) / r
    const float tau0 = a.tau0f;
    const float te =
        APPROX ? 0.5f * (tau0 + sqrt_approx(fmaf(tau0, tau0, a.les_cf * sqrt_approx(qq) * inv)))
               : 0.5f * (tau0 + sqrtf(fmaf(tau0, tau0, a.les_cf * sqrtf(qq) * inv)));
    om = APPROX ? rcp_approx(te) : __frcp_rn(te);
    if (a.trt) {
      const float t5 = te - 0.5f;
      omm = __fdividef(t5, fmaf(0.5f, t5, a.lamf));
    } else {
      omm = om;
    }
  }
  const float e0 = W0 * A;
  const float g0 = fmaf(-om, f[0] - e0, f[0]);
#define WT_OUT(k, kb)                                                   \
  const float g##k = fmaf(-omm, sm##k, fmaf(-om, sp##k, f[k]));         \
  const float g##kb = fmaf(omm, sm##k, fmaf(-om, sp##k, f[kb]));
  WT_OUT(1, 2) WT_OUT(3, 4) WT_OUT(5, 6) WT_OUT(7, 8) WT_OUT(9, 10) WT_OUT(11, 12) WT_OUT(13, 14)
  WT_OUT(15, 16) WT_OUT(17, 18)
#undef WT_OUT
  if constexpr (std::is_same<S, __half>::value) {
    if (a.f16_sr) {
      // stochastic rounding to half: each opposite pair is converted together
      // with 32 random bits from a per-cell, per-step xorshift chain
      uint32_t h = ((uint32_t)i ^ (uint32_t)(i >> 32)) * 0x9E3779B1u ^ a.sr_seed;
      h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
      constexpr float SC = (float)WT_F16_SCALE;
#define WT_SR(k, kb)                                                               \
  {                                                                                \
    h ^= h << 13; h ^= h >> 17; h ^= h << 5;                                       \
    const __half2 p = sr_half2(g##k * SC, g##kb * SC, h);                          \
    out.put(k, __high2half(p));                                                    \
    out.put(kb, __low2half(p));                                                    \
  }
      WT_SR(1, 2) WT_SR(3, 4) WT_SR(5, 6) WT_SR(7, 8) WT_SR(9, 10) WT_SR(11, 12)
      WT_SR(13, 14) WT_SR(15, 16) WT_SR(17, 18)
#undef WT_SR
      h ^= h << 13; h ^= h >> 17; h ^= h << 5;
      out.put(0, __low2half(sr_half2(0.0f, g0 * SC, h)));
      return;
    }
  }
  out.put(0, Store<S>::from_f(g0));
#define WT_PUT(k, kb) out.put(k, Store<S>::from_f(g##k)); out.put(kb, Store<S>::from_f(g##kb));
  WT_PUT(1, 2) WT_PUT(3, 4) WT_PUT(5, 6) WT_PUT(7, 8) WT_PUT(9, 10) WT_PUT(11, 12) WT_PUT(13, 14)
  WT_PUT(15, 16) WT_PUT(17, 18)
#undef WT_PUT
}

// Float64 collision in the exact operation order of js/lbm.js:377-460. The
// translation unit that instantiates it is compiled with --fmad=false, so no
// multiply-add is contracted and every rounding matches the reference's
// IEEE double arithmetic; results are rounded to S only at the stores.
template <class S, class Out>
__device__ __forceinline__ void collide_exact(const StepArgs<S>& a, const double (&fq)[Q],
                                              long long i, bool dup, bool near_cell, Out out) {
  const double f0 = fq[0], f1 = fq[1], f2 = fq[2], f3 = fq[3], f4 = fq[4], f5 = fq[5],
               f6 = fq[6], f7 = fq[7], f8 = fq[8], f9 = fq[9], f10 = fq[10], f11 = fq[11],
               f12 = fq[12], f13 = fq[13], f14 = fq[14], f15 = fq[15], f16 = fq[16],
               f17 = fq[17], f18 = fq[18];
  const double dr = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8 + f9 + f10 + f11 + f12 + f13 +
                    f14 + f15 + f16 + f17 + f18;
  const double r = 1 + dr;
  if (!(r > 0.0 && r < 1.0e300)) atomicOr(a.err, 1u);
  const double inv = 1 / r;
  const double vx = (f1 - f2 + f7 - f8 + f9 - f10 + f11 - f12 + f13 - f14) * inv;
  const double vy = (f3 - f4 + f7 - f8 - f9 + f10 + f15 - f16 + f17 - f18) * inv;
  const double vz = (f5 - f6 + f11 - f12 - f13 + f14 + f15 - f16 - f17 + f18) * inv;
  if (a.write_fields) {
    const float rf = __double2float_rn(r), xf = __double2float_rn(vx),
                yf = __double2float_rn(vy), zf = __double2float_rn(vz);
    a.rho[i] = rf; a.ux[i] = xf; a.uy[i] = yf; a.uz[i] = zf;
    if (dup) { a.rho[i + 1] = rf; a.ux[i + 1] = xf; a.uy[i + 1] = yf; a.uz[i + 1] = zf; }
  } else if (a.mov && near_cell) {
    a.rho[i] = __double2float_rn(r);
  }
  const double A = dr - r * 1.5 * (vx * vx + vy * vy + vz * vz);
  const double r3 = 3 * r, r45 = 4.5 * r;
  const double ax = vx, ay = vy, az = vz;
  const double bxy = vx + vy, bxY = vx - vy;
  const double bxz = vx + vz, bxZ = vx - vz;
  const double byz = vy + vz, byZ = vy - vz;
  constexpr double W0 = 1.0 / 3, WF = 1.0 / 18, WE = 1.0 / 36;
  const double e0 = W0 * A;
  const double hx = r45 * ax * ax, hy = r45 * ay * ay, hz = r45 * az * az;
  const double e1 = WF * (A + r3 * ax + hx), e2 = WF * (A - r3 * ax + hx);
  const double e3 = WF * (A + r3 * ay + hy), e4 = WF * (A - r3 * ay + hy);
  const double e5 = WF * (A + r3 * az + hz), e6 = WF * (A - r3 * az + hz);
  const double h7 = r45 * bxy * bxy, h9 = r45 * bxY * bxY;
  const double h11 = r45 * bxz * bxz, h13 = r45 * bxZ * bxZ;
  const double h15 = r45 * byz * byz, h17 = r45 * byZ * byZ;
  const double e7 = WE * (A + r3 * bxy + h7), e8 = WE * (A - r3 * bxy + h7);
  const double e9 = WE * (A + r3 * bxY + h9), e10 = WE * (A - r3 * bxY + h9);
  const double e11 = WE * (A + r3 * bxz + h11), e12 = WE * (A - r3 * bxz + h11);
  const double e13 = WE * (A + r3 * bxZ + h13), e14 = WE * (A - r3 * bxZ + h13);
  const double e15 = WE * (A + r3 * byz + h15), e16 = WE * (A - r3 * byz + h15);
  const double e17 = WE * (A + r3 * byZ + h17), e18 = WE * (A - r3 * byZ + h17);
  const double n1 = f1 - e1, n2 = f2 - e2, n3 = f3 - e3, n4 = f4 - e4;
  const double n5 = f5 - e5, n6 = f6 - e6, n7 = f7 - e7, n8 = f8 - e8;
  const double n9 = f9 - e9, n10 = f10 - e10, n11 = f11 - e11, n12 = f12 - e12;
  const double n13 = f13 - e13, n14 = f14 - e14, n15 = f15 - e15, n16 = f16 - e16;
  const double n17 = f17 - e17, n18 = f18 - e18;
  const double tau0 = a.tau0;
  double om = a.omega0, tauEff = tau0;
  if (a.les) {
    const double pxx = n1 + n2 + n7 + n8 + n9 + n10 + n11 + n12 + n13 + n14;
    const double pyy = n3 + n4 + n7 + n8 + n9 + n10 + n15 + n16 + n17 + n18;
    const double pzz = n5 + n6 + n11 + n12 + n13 + n14 + n15 + n16 + n17 + n18;
    const double pxy = n7 + n8 - n9 - n10;
    const double pxz = n11 + n12 - n13 - n14;
    const double pyz = n15 + n16 - n17 - n18;
    const double mag = sqrt(2 * (pxx * pxx + pyy * pyy + pzz * pzz +
                                 2 * (pxy * pxy + pxz * pxz + pyz * pyz)));
    const double SQ18 = 18 * 1.4142135623730951;
    tauEff = 0.5 * (tau0 + sqrt(tau0 * tau0 + SQ18 * a.cs2 * mag * inv));
    om = 1 / tauEff;
  }
  const double omm = a.trt ? 1 / (0.5 + a.lam / (tauEff - 0.5)) : om;
  out.put(0, Store<S>::from_d(f0 - om * (f0 - e0)));
  double sp, sm;
#define WT_XOUT(A_, B_, NA, NB, FA, FB)                   \
  sp = 0.5 * (NA + NB); sm = 0.5 * (NA - NB);             \
  out.put(A_, Store<S>::from_d(FA - om * sp - omm * sm)); \
  out.put(B_, Store<S>::from_d(FB - om * sp + omm * sm));
  WT_XOUT(1, 2, n1, n2, f1, f2)
  WT_XOUT(3, 4, n3, n4, f3, f4)
  WT_XOUT(5, 6, n5, n6, f5, f6)
  WT_XOUT(7, 8, n7, n8, f7, f8)
  WT_XOUT(9, 10, n9, n10, f9, f10)
  WT_XOUT(11, 12, n11, n12, f11, f12)
  WT_XOUT(13, 14, n13, n14, f13, f14)
  WT_XOUT(15, 16, n15, n16, f15, f16)
  WT_XOUT(17, 18, n17, n18, f17, f18)
#undef WT_XOUT
}

// The float32 step is capped at 64 registers so that 8 blocks of 128 threads
// stay resident per SM: the step is bound by memory latency, and resident
// warps are what keep enough of the 19 load streams in flight. The float64
// (exact) step keeps 128 registers rather than spill.
constexpr int step_min_blocks(bool exact) { return exact ? 4 : 8; }

// IDX is the type of the per-direction offsets: int when 19*n fits in 31
// bits (every practical lattice), long long otherwise.
template <class S, bool EXACT, class IDX>
__global__ void __launch_bounds__(STEP_BX, step_min_blocks(EXACT)) k_step(const __grid_constant__ StepArgs<S> a) {
  using M = typename std::conditional<EXACT, double, float>::type;
  pdl_enter();   // programmatic dependent launch (launch_pdl)
  const int x = blockIdx.x * STEP_BX + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  const long long i = (long long)x + (long long)a.nx * y + a.nxy * z;
  double Fx = 0, Fy = 0, Fz = 0;
  bool near_cell = false;
  if (x < a.nx - 1) {
    int cat;
    uint8_t fl = 0;
    const bool dup = (x == a.nx - 2);   // this thread also writes the outlet cell x+1
    if (x == 0) {
      cat = CAT_EQ;
    } else {
      fl = a.flags[i];
      if (z == 0 || z == a.nz - 1 || y == a.ny - 1) cat = CAT_EQ;
      else if (fl & FLAG_SOLID_MASK) cat = CAT_KEEP;
      else if (y == 0) cat = CAT_EQ;
      else cat = CAT_FLUID;
    }
    S* Gi = a.G + i;
    if (cat == CAT_FLUID) {
      M f[Q];
      near_cell = (fl & FLAG_NEAR) != 0;
      const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
      const S* Fi = a.F + i;
#pragma unroll
      for (int q = 0; q < Q; q++) f[q] = ld<M>(Fi[(IDX)a.src[q]]);
      if (near_cell || shell) patch_special<S, M>(a, i, x, y, z, shell, f, Fx, Fy, Fz);
      S out[Q];
      if constexpr (EXACT) {
        collide_exact<S>(a, f, i, dup, near_cell, RegOut<S>{out});
      } else {
        collide_fast<S>(a, f, i, dup, near_cell, RegOut<S>{out});
      }
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
  warp_force_partial(Fx, Fy, Fz, near_cell, a);
}

}  // namespace wt
