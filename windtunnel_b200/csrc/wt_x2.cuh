// wt_x2.cuh — the float32 collision in the storage's scaled units, written
// once for a scalar float (one cell) and for a packed float2 (two cells in
// the .x and .y lanes of sm_100's add / sub / mul / fma .f32x2 instructions).
//
// The collision is that of collide_fast (opposite pairs carried as half sums
// and half differences, js/lbm.js:377-460 re-associated) evaluated in raw
// units: a half-storage lattice holds 4096 * (f - w), and the arithmetic is
// arranged so that this scale only enters through r~ = 4096 + sum(f~)
// (moments, equilibrium, stress and the TRT update are linear in f~, and the
// Smagorinsky term depends on |Pi|/rho, which the scale leaves unchanged), so
// loads and stores carry no scaling multiply. Reciprocals and square roots
// use the approximate hardware instructions (relative error ~2^-22).
// patch_raw re-gathers the bounce-back and free-slip directions of one cell
// in the same raw units.
#pragma once

#include "wt_step.cuh"

namespace wt {

// ---- packed float32 pairs: cell x0 in .x, cell x0+1 in .y --------------------------
using f2 = float2;
__device__ __forceinline__ f2 pk(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 padd(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 pmul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 pfma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 psub(f2 a, f2 b) {
  unsigned long long ra, rb, rd;
  memcpy(&ra, &a, 8);
  memcpy(&rb, &b, 8);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  f2 d;
  memcpy(&d, &rd, 8);
  return d;
}
__device__ __forceinline__ f2 prcp(f2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
__device__ __forceinline__ f2 psqrt(f2 a) { return make_float2(sqrt_approx(a.x), sqrt_approx(a.y)); }

// The same operations on one cell (a scalar float), so that the collision
// below also serves the one-cell-per-thread kernels.
template <class V>
__device__ __forceinline__ V splat(float a);
template <>
__device__ __forceinline__ f2 splat<f2>(float a) { return pk(a); }
template <>
__device__ __forceinline__ float splat<float>(float a) { return a; }
__device__ __forceinline__ float padd(float a, float b) { return a + b; }
__device__ __forceinline__ float psub(float a, float b) { return a - b; }
__device__ __forceinline__ float pmul(float a, float b) { return a * b; }
__device__ __forceinline__ float pfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float prcp(float a) { return rcp_approx(a); }
__device__ __forceinline__ float psqrt(float a) { return sqrt_approx(a); }

template <int C>
__device__ __forceinline__ float& lane_of(f2& v) {
  if constexpr (C == 0) return v.x;
  else return v.y;
}
template <int C>
__device__ __forceinline__ float& lane_of(float& v) {
  return v;
}

// Storage in scaled units: raw(v) is the stored number as a float (the
// deviation times SC), pack() rounds a pair of raw values to the storage.
template <class S>
struct X2;
template <>
struct X2<float> {
  using V = float2;
  static constexpr float SC = 1.0f;
  __device__ __forceinline__ static float raw(float v) { return v; }
  __device__ __forceinline__ static f2 unpack(V v) { return v; }
  __device__ __forceinline__ static V pack(f2 g) { return g; }
  __device__ __forceinline__ static float to_s(float v) { return v; }
};
template <>
struct X2<__half> {
  using V = __half2;
  static constexpr float SC = (float)WT_F16_SCALE;
  __device__ __forceinline__ static float raw(__half v) { return __half2float(v); }
  __device__ __forceinline__ static f2 unpack(V v) { return __half22float2(v); }
  __device__ __forceinline__ static V pack(f2 g) { return __float22half2_rn(g); }
  __device__ __forceinline__ static __half to_s(float v) { return __float2half_rn(v); }
};

// Bounce-back / free-slip re-gather of lane C's cell i, in raw units
// (js/lbm.js:334-368 for the bounce-back links; k_step's patch_special is
// the same rule in deviation units). The momentum exchange accumulates in
// raw units; the caller divides by SC.
template <class S, int C, class VV>
__device__ __forceinline__ void patch_raw(const StepArgs<S>& a, long long i, int x, int y, int z,
                                          bool near_cell, bool shell, VV (&f)[Q], double& Fx,
                                          double& Fy, double& Fz) {
  using T = X2<S>;
  const unsigned long long m = near_cell ? a.nmask[i] : 0ull;
  const unsigned sm = (unsigned)m, om = (unsigned)(m >> 32);
  const float rho_sc = (a.mov && sm ? a.rho[i] : 1.0f) * T::SC;
#define WT_PATCH_RAW(q)                                                                      \
  if ((sm >> (q)) & 1u) {                                                                    \
    const long long j = i - (ex(q) + (long long)ey(q) * a.nx + (long long)ez(q) * a.nxy);    \
    const float fd = T::raw(a.F[opp(q) * a.n + i]);                                          \
    float corr = 0.0f;                                                                       \
    if (a.mov) {                                                                             \
      const float cu = (float)ex(q) * a.uwx[j] + (float)ey(q) * a.uwy[j] +                   \
                       (float)ez(q) * a.uwz[j];                                              \
      if (cu != 0.0f) corr = 6.0f * (float)wq(q) * rho_sc * cu;                              \
    }                                                                                        \
    if ((om >> (q)) & 1u) {                                                                  \
      const float d = 2.0f * fd + corr;                                                      \
      Fx -= (double)(d * (float)ex(q));                                                      \
      Fy -= (double)(d * (float)ey(q));                                                      \
      Fz -= (double)(d * (float)ez(q));                                                      \
    }                                                                                        \
    lane_of<C>(f[q]) = fd + corr;                                                            \
  } else if (shell) {                                                                        \
    int sy = y - ey(q), sz = z - ez(q), qq = q;                                              \
    bool refl = false;                                                                       \
    if (sy == 0 || sy == a.ny - 1) { sy = y; qq = mirror_y(qq); refl = true; }               \
    if (sz == 0 || sz == a.nz - 1) { sz = z; qq = mirror_z(qq); refl = true; }               \
    if (refl)                                                                                \
      lane_of<C>(f[q]) =                                                                     \
          T::raw(a.F[qq * a.n + (x - ex(q)) + (long long)a.nx * sy + a.nxy * sz]);           \
  }
  WT_PATCH_RAW(1) WT_PATCH_RAW(2) WT_PATCH_RAW(3) WT_PATCH_RAW(4) WT_PATCH_RAW(5)
  WT_PATCH_RAW(6) WT_PATCH_RAW(7) WT_PATCH_RAW(8) WT_PATCH_RAW(9) WT_PATCH_RAW(10)
  WT_PATCH_RAW(11) WT_PATCH_RAW(12) WT_PATCH_RAW(13) WT_PATCH_RAW(14) WT_PATCH_RAW(15)
  WT_PATCH_RAW(16) WT_PATCH_RAW(17) WT_PATCH_RAW(18)
#undef WT_PATCH_RAW
}

// Packed collision of two cells in raw (scaled) units: f -> g, with the
// density r~ = SC * rho and the velocity of each lane. The mathematics is
// that of js/lbm.js:377-460 (collide_fast's re-association).
template <class S, class f2 = wt::f2>
__device__ __forceinline__ void collide_x2(const StepArgs<S>& a, f2 (&f)[Q], f2& r, f2& vx,
                                           f2& vy, f2& vz) {
  constexpr float SC = X2<S>::SC;
  auto pk = [](float v) { return splat<f2>(v); };
  const f2 s1 = padd(f[1], f[2]), d1 = psub(f[1], f[2]);
  const f2 s3 = padd(f[3], f[4]), d3 = psub(f[3], f[4]);
  const f2 s5 = padd(f[5], f[6]), d5 = psub(f[5], f[6]);
  const f2 s7 = padd(f[7], f[8]), d7 = psub(f[7], f[8]);
  const f2 s9 = padd(f[9], f[10]), d9 = psub(f[9], f[10]);
  const f2 s11 = padd(f[11], f[12]), d11 = psub(f[11], f[12]);
  const f2 s13 = padd(f[13], f[14]), d13 = psub(f[13], f[14]);
  const f2 s15 = padd(f[15], f[16]), d15 = psub(f[15], f[16]);
  const f2 s17 = padd(f[17], f[18]), d17 = psub(f[17], f[18]);
  const f2 dr = padd(padd(padd(f[0], s1), padd(s3, s5)),
                     padd(padd(padd(s7, s9), padd(s11, s13)), padd(s15, s17)));
  r = padd(pk(SC), dr);
  const f2 inv = prcp(r);
  const f2 jx = padd(padd(padd(d1, d7), padd(d9, d11)), d13);
  const f2 jy = padd(psub(padd(d3, d7), d9), padd(d15, d17));
  const f2 jz = padd(psub(padd(d5, d11), d13), psub(d15, d17));
  vx = pmul(jx, inv);
  vy = pmul(jy, inv);
  vz = pmul(jz, inv);
  const f2 usq = pfma(vz, vz, pfma(vy, vy, pmul(vx, vx)));
  const f2 A = pfma(pmul(pk(-1.5f), r), usq, dr);   // dr - 1.5 r u^2 (scaled)
  constexpr float WF = (float)(1.0 / 18), WE = (float)(1.0 / 36), W0 = (float)(1.0 / 3);
  const f2 nwAF = pmul(pk(-WF), A), nwAE = pmul(pk(-WE), A);
  const f2 nw45F = pmul(pk(-4.5f * WF), r), nw45E = pmul(pk(-4.5f * WE), r);
  const f2 nw3F = pmul(pk(-3.0f * WF), r), nw3E = pmul(pk(-3.0f * WE), r);
  const f2 c7 = padd(vx, vy), c9 = psub(vx, vy), c11 = padd(vx, vz), c13 = psub(vx, vz),
           c15 = padd(vy, vz), c17 = psub(vy, vz);
  const f2& c1 = vx;
  const f2& c3 = vy;
  const f2& c5 = vz;
  // sp = (n_a + n_b)/2 = s/2 - w(A + 4.5 r c^2); sm = (n_a - n_b)/2 = d/2 - 3 w r c
#define WT_PAIR2(k, C)                                                       \
  const f2 sp##k = pfma(pk(0.5f), s##k, pfma(pmul(nw45##C, c##k), c##k, nwA##C)); \
  const f2 sm##k = pfma(pk(0.5f), d##k, pmul(nw3##C, c##k));
  WT_PAIR2(1, F) WT_PAIR2(3, F) WT_PAIR2(5, F) WT_PAIR2(7, E) WT_PAIR2(9, E) WT_PAIR2(11, E)
  WT_PAIR2(13, E) WT_PAIR2(15, E) WT_PAIR2(17, E)
#undef WT_PAIR2
  f2 om = pk(a.omega0f), omm = pk(a.omm0f);
  if (a.les) {
    const f2 sxx = padd(padd(padd(sp1, sp7), padd(sp9, sp11)), sp13);
    const f2 syy = padd(padd(padd(sp3, sp7), padd(sp9, sp15)), sp17);
    const f2 szz = padd(padd(padd(sp5, sp11), padd(sp13, sp15)), sp17);
    const f2 sxy = psub(sp7, sp9), sxz = psub(sp11, sp13), syz = psub(sp15, sp17);
    const f2 off = pfma(syz, syz, pfma(sxz, sxz, pmul(sxy, sxy)));
    const f2 qq = pfma(sxx, sxx, pfma(syy, syy, pfma(szz, szz, padd(off, off))));
    // 72 cs2 sqrt(qq) / r: the scale of sqrt(qq~) and of r~ cancels
    const f2 x = pmul(pmul(pk(a.les_cf), psqrt(qq)), inv);
    const f2 te = pfma(pk(0.5f), psqrt(pfma(pk(a.tau0f), pk(a.tau0f), x)), pk(0.5f * a.tau0f));
    om = prcp(te);
    if (a.trt) {
      const f2 t5 = psub(te, pk(0.5f));
      omm = pmul(t5, prcp(pfma(pk(0.5f), t5, pk(a.lamf))));
    } else {
      omm = om;
    }
  }
  const f2 nom = pmul(pk(-1.0f), om);
  const f2 nomm = pmul(pk(-1.0f), omm);
  f[0] = pfma(nom, psub(f[0], pmul(pk(W0), A)), f[0]);
#define WT_OUT2(k, kb)                            \
  {                                               \
    const f2 base_a = pfma(nom, sp##k, f[k]);     \
    const f2 base_b = pfma(nom, sp##k, f[kb]);    \
    f[k] = pfma(nomm, sm##k, base_a);             \
    f[kb] = pfma(omm, sm##k, base_b);             \
  }
  WT_OUT2(1, 2) WT_OUT2(3, 4) WT_OUT2(5, 6) WT_OUT2(7, 8) WT_OUT2(9, 10) WT_OUT2(11, 12)
  WT_OUT2(13, 14) WT_OUT2(15, 16) WT_OUT2(17, 18)
#undef WT_OUT2
}

}  // namespace wt
