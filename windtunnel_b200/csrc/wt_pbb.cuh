// wt_pbb.cuh — partial bounce-back step and its discrete adjoint.
//
// Partial bounce-back (no counterpart in the reference): a fluid cell with
// solid fraction s in [0, 1] stores
//     g_q = (1 - s) gc_q + s f_opp(q)
// where f are its pulled populations and gc the collided ones, and adds
//     s * sum_q c_q (gc_q - f_opp(q))
// to the momentum-exchange force. s = 0 is the plain step; s = 1 reverses
// every population of the cell. The field lives on a box of cells
// (StepArgs::sfrac, float64, x fastest).
//
// k_step_pbb is k_step (wt_step.cuh) with the collision written as a plain
// per-direction sequence (cell_fw) so that the collided values can be blended
// before they are rounded to the storage type; its operation order is that of
// js/lbm.js:377-460, so with EXACT it reproduces the reference arithmetic
// bit for bit where s = 0.
//
// k_adjoint is one step of the discrete adjoint, run backwards in time over
// stored forward states. T^t[q][i] is dJ/d(value pulled by link q of cell i at
// step t). The adjoint of the population stored at location (q, j) after step
// t is the sum of T^{t+1} over the links that pull it at step t+1: the plain
// consumer j + c_q, the cell j itself when that neighbour is solid
// (bounce-back), and the mirrored consumer when that neighbour is a free-slip
// side plane; the outlet column x = nx-1 is a copy of column nx-2, so its
// adjoint is added to column nx-2's. Cells that do not pull (inlet, outlet,
// side planes, solids) write zero rows. Every adjoint step is therefore a
// pull-shaped pass like the forward step: per cell it gathers 19 adjoint
// values, recomputes the forward collision from the stored state, and writes
// the 19 adjoint values of its pulled links, accumulating dJ/ds on the box.
#pragma once

#include "wt_step.cuh"

namespace wt {

// Division and square root of the collision and its adjoint: IEEE in float64
// (the exact forms), the hardware approximations (relative error ~2^-22) in
// float32, where the fast forms already use them.
template <class T>
__device__ __forceinline__ T cdiv(T n, T d) {
  if constexpr (std::is_same<T, float>::value) return n * rcp_approx(d);
  else return n / d;
}
template <class T>
__device__ __forceinline__ T csqrt(T v) {
  if constexpr (std::is_same<T, float>::value) return sqrt_approx(v);
  else return sqrt(v);
}

// Forward collision of one cell and the intermediates its adjoint needs, in
// the operation order of js/lbm.js:377-460 (and of collide_exact).
template <class T>
struct CellFw {
  T f[Q], gc[Q], n[Q];
  T r, inv, jx, jy, jz, vx, vy, vz, usq, A, r3, r45;
  T pxx, pyy, pzz, pxy, pxz, pyz, mag, R, tauEff, om, omm;
};

// The float32 form of cell_fw: the same quantities re-associated over the
// nine opposite pairs (a, b), as the fast step collides: with s = f_a + f_b,
// d = f_a - f_b and cv = c_a . u, the pair's symmetric and antisymmetric
// non-equilibrium parts are sp = s/2 - w (A + 4.5 r cv^2) and
// sm = d/2 - 3 w r cv, n_a = sp + sm, n_b = sp - sm, and the stress sums are
// sums of 2 sp. No explicit equilibrium array.
template <class S>
__device__ __forceinline__ void cell_fw_pairs(const StepArgs<S>& a, CellFw<float>& c) {
  const float* f = c.f;
  float sp[Q], sm[Q];   // indexed by the pair's first direction (1, 3, ..., 17)
  float s[Q], d[Q];
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    s[k] = f[k] + f[k + 1];
    d[k] = f[k] - f[k + 1];
  }
  const float dr = ((f[0] + s[1]) + (s[3] + s[5])) +
                   (((s[7] + s[9]) + (s[11] + s[13])) + (s[15] + s[17]));
  const float r = 1.0f + dr;
  const float inv = cdiv(1.0f, r);
  const float jx = (((d[1] + d[7]) + (d[9] + d[11])) + d[13]);
  const float jy = (((d[3] + d[7]) - d[9]) + (d[15] + d[17]));
  const float jz = (((d[5] + d[11]) - d[13]) + (d[15] - d[17]));
  const float vx = jx * inv, vy = jy * inv, vz = jz * inv;
  const float usq = vx * vx + vy * vy + vz * vz;
  const float A = dr - r * 1.5f * usq;
  const float r3 = 3.0f * r, r45 = 4.5f * r;
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const float cv = (float)ex(k) * vx + (float)ey(k) * vy + (float)ez(k) * vz;
    const float w = (float)wq(k);
    sp[k] = 0.5f * s[k] - w * (A + r45 * cv * cv);
    sm[k] = 0.5f * d[k] - w * r3 * cv;
    c.n[k] = sp[k] + sm[k];
    c.n[k + 1] = sp[k] - sm[k];
  }
  c.n[0] = f[0] - (float)wq(0) * A;
  const float tau0 = (float)a.tau0;
  float om = cdiv(1.0f, tau0), tauEff = tau0;
  c.pxx = c.pyy = c.pzz = c.pxy = c.pxz = c.pyz = c.mag = c.R = 0.0f;
  if (a.les) {
    c.pxx = 2.0f * (((sp[1] + sp[7]) + (sp[9] + sp[11])) + sp[13]);
    c.pyy = 2.0f * (((sp[3] + sp[7]) + (sp[9] + sp[15])) + sp[17]);
    c.pzz = 2.0f * (((sp[5] + sp[11]) + (sp[13] + sp[15])) + sp[17]);
    c.pxy = 2.0f * (sp[7] - sp[9]);
    c.pxz = 2.0f * (sp[11] - sp[13]);
    c.pyz = 2.0f * (sp[15] - sp[17]);
    c.mag = csqrt(2.0f * (c.pxx * c.pxx + c.pyy * c.pyy + c.pzz * c.pzz +
                          2.0f * (c.pxy * c.pxy + c.pxz * c.pxz + c.pyz * c.pyz)));
    const float SQ18 = (float)(18 * 1.4142135623730951);
    c.R = csqrt(tau0 * tau0 + SQ18 * (float)a.cs2 * c.mag * inv);
    tauEff = 0.5f * (tau0 + c.R);
    om = cdiv(1.0f, tauEff);
  }
  const float omm = a.trt ? cdiv(1.0f, 0.5f + cdiv((float)a.lam, tauEff - 0.5f)) : om;
  c.gc[0] = f[0] - om * c.n[0];
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    c.gc[k] = f[k] - om * sp[k] - omm * sm[k];
    c.gc[k + 1] = f[k + 1] - om * sp[k] + omm * sm[k];
  }
  c.r = r; c.inv = inv; c.jx = jx; c.jy = jy; c.jz = jz; c.vx = vx; c.vy = vy; c.vz = vz;
  c.usq = usq; c.A = A; c.r3 = r3; c.r45 = r45; c.tauEff = tauEff; c.om = om; c.omm = omm;
}

template <class T, class S>
__device__ __forceinline__ void cell_fw(const StepArgs<S>& a, CellFw<T>& c) {
  if constexpr (std::is_same<T, float>::value) {
    cell_fw_pairs(a, c);
    return;
  }
  const T* f = c.f;
  const T dr = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] +
               f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  const T r = (T)1 + dr;
  const T inv = cdiv((T)1, r);
  const T jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  const T jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
  const T jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
  const T vx = jx * inv, vy = jy * inv, vz = jz * inv;
  const T usq = vx * vx + vy * vy + vz * vz;
  const T A = dr - r * (T)1.5 * usq;
  const T r3 = (T)3 * r, r45 = (T)4.5 * r;
  T e[Q];
  e[0] = (T)wq(0) * A;
#pragma unroll
  for (int q = 1; q < Q; q++) {
    const T cv = (T)ex(q) * vx + (T)ey(q) * vy + (T)ez(q) * vz;
    e[q] = (T)wq(q) * (A + r3 * cv + r45 * cv * cv);
  }
#pragma unroll
  for (int q = 0; q < Q; q++) c.n[q] = f[q] - e[q];
  const T* n = c.n;
  const T tau0 = (T)a.tau0;
  T om = cdiv((T)1, tau0), tauEff = tau0;
  c.pxx = c.pyy = c.pzz = c.pxy = c.pxz = c.pyz = c.mag = c.R = (T)0;
  if (a.les) {
    c.pxx = n[1] + n[2] + n[7] + n[8] + n[9] + n[10] + n[11] + n[12] + n[13] + n[14];
    c.pyy = n[3] + n[4] + n[7] + n[8] + n[9] + n[10] + n[15] + n[16] + n[17] + n[18];
    c.pzz = n[5] + n[6] + n[11] + n[12] + n[13] + n[14] + n[15] + n[16] + n[17] + n[18];
    c.pxy = n[7] + n[8] - n[9] - n[10];
    c.pxz = n[11] + n[12] - n[13] - n[14];
    c.pyz = n[15] + n[16] - n[17] - n[18];
    c.mag = csqrt((T)2 * (c.pxx * c.pxx + c.pyy * c.pyy + c.pzz * c.pzz +
                          (T)2 * (c.pxy * c.pxy + c.pxz * c.pxz + c.pyz * c.pyz)));
    const T SQ18 = (T)(18 * 1.4142135623730951);
    c.R = csqrt(tau0 * tau0 + SQ18 * (T)a.cs2 * c.mag * inv);
    tauEff = (T)0.5 * (tau0 + c.R);
    om = cdiv((T)1, tauEff);
  }
  const T omm = a.trt ? cdiv((T)1, (T)0.5 + cdiv((T)a.lam, tauEff - (T)0.5)) : om;
  c.gc[0] = f[0] - om * (f[0] - e[0]);
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const T sp = (T)0.5 * (n[k] + n[k + 1]), sm = (T)0.5 * (n[k] - n[k + 1]);
    c.gc[k] = f[k] - om * sp - omm * sm;
    c.gc[k + 1] = f[k + 1] - om * sp + omm * sm;
  }
  c.r = r; c.inv = inv; c.jx = jx; c.jy = jy; c.jz = jz; c.vx = vx; c.vy = vy; c.vz = vz;
  c.usq = usq; c.A = A; c.r3 = r3; c.r45 = r45; c.tauEff = tauEff; c.om = om; c.omm = omm;
}

// The float32 form of cell_vjp, over the nine opposite pairs: with
// P = nb_a + nb_b and D = nb_a - nb_b (the adjoints of the pair's
// symmetric and antisymmetric non-equilibrium parts), the stress terms add
// to P only, and the equilibrium's adjoint needs each pair once (c_b = -c_a).
template <class S>
__device__ __forceinline__ void cell_vjp_pairs(const StepArgs<S>& a, const CellFw<float>& c,
                                               const float (&ab)[Q], float (&fb)[Q]) {
  const float* n = c.n;
  float P[Q], D[Q];   // indexed by the pair's first direction (1, 3, ..., 17)
  float omb = -(ab[0] * n[0]);
  float ommb = 0.0f;
  const float nb0 = -(c.om * ab[0]);
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const float sp = 0.5f * (n[k] + n[k + 1]), sm = 0.5f * (n[k] - n[k + 1]);
    const float as = ab[k] + ab[k + 1], ad = ab[k] - ab[k + 1];
    omb -= as * sp;
    ommb -= ad * sm;
    P[k] = -(c.om * as);
    D[k] = -(c.omm * ad);
  }
  float invb = 0.0f;
  if (a.les) {
    float teb;
    if (a.trt) {
      const float tm = c.tauEff - 0.5f;
      teb = ommb * cdiv(c.omm * c.omm * (float)a.lam, tm * tm) - omb * (c.om * c.om);
    } else {
      teb = -(omb + ommb) * (c.om * c.om);
    }
    const float Rb = 0.5f * teb;
    const float Xb = cdiv(Rb, 2.0f * c.R);
    const float K = (float)(18 * 1.4142135623730951) * (float)a.cs2;
    const float magb = Xb * K * c.inv;
    invb += Xb * K * c.mag;
    const float Qb = c.mag > 0.0f ? cdiv(magb, c.mag) : 0.0f;
    const float pxxb = 4.0f * c.pxx * Qb, pyyb = 4.0f * c.pyy * Qb, pzzb = 4.0f * c.pzz * Qb;
    const float pxyb = 8.0f * c.pxy * Qb, pxzb = 8.0f * c.pxz * Qb, pyzb = 8.0f * c.pyz * Qb;
    P[1] += pxxb; P[3] += pyyb; P[5] += pzzb;
    P[7] += pxxb + pyyb + pxyb; P[9] += pxxb + pyyb - pxyb;
    P[11] += pxxb + pzzb + pxzb; P[13] += pxxb + pzzb - pxzb;
    P[15] += pyyb + pzzb + pyzb; P[17] += pyyb + pzzb - pyzb;
  }
  float Ab = (float)wq(0) * (-nb0), r3b = 0.0f, r45b = 0.0f, vxb = 0.0f, vyb = 0.0f, vzb = 0.0f;
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const float E = -P[k], Dm = -D[k], w = (float)wq(k);
    const float cv = (float)ex(k) * c.vx + (float)ey(k) * c.vy + (float)ez(k) * c.vz;
    Ab += w * E;
    r3b += w * cv * Dm;
    r45b += w * (cv * cv) * E;
    const float cvbd = w * (c.r3 * Dm + 2.0f * c.r45 * cv * E);
    vxb += (float)ex(k) * cvbd; vyb += (float)ey(k) * cvbd; vzb += (float)ez(k) * cvbd;
  }
  float drb = Ab;
  float rb = 3.0f * r3b + 4.5f * r45b - 1.5f * c.usq * Ab;
  const float usqb = -(c.r * 1.5f * Ab);
  vxb += 2.0f * c.vx * usqb; vyb += 2.0f * c.vy * usqb; vzb += 2.0f * c.vz * usqb;
  invb += vxb * c.jx + vyb * c.jy + vzb * c.jz;
  const float jxb = vxb * c.inv, jyb = vyb * c.inv, jzb = vzb * c.inv;
  rb -= c.inv * c.inv * invb;
  drb += rb;
  fb[0] += ab[0] + nb0 + drb;
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const float cj = (float)ex(k) * jxb + (float)ey(k) * jyb + (float)ez(k) * jzb;
    fb[k] += ab[k] + 0.5f * (P[k] + D[k]) + (drb + cj);
    fb[k + 1] += ab[k + 1] + 0.5f * (P[k] - D[k]) + (drb - cj);
  }
}

// fb += (d gc / d f)^T a for the collision of cell_fw.
template <class T, class S>
__device__ __forceinline__ void cell_vjp(const StepArgs<S>& a, const CellFw<T>& c, const T (&ab)[Q],
                                         T (&fb)[Q]) {
  if constexpr (std::is_same<T, float>::value) {
    cell_vjp_pairs(a, c, ab, fb);
    return;
  }
  const T* n = c.n;
  T nb[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) fb[q] += ab[q];
  T omb = -(ab[0] * n[0]);
  T ommb = (T)0;
  nb[0] = -(c.om * ab[0]);
#pragma unroll
  for (int k = 1; k < Q; k += 2) {
    const T sp = (T)0.5 * (n[k] + n[k + 1]), sm = (T)0.5 * (n[k] - n[k + 1]);
    const T as = ab[k] + ab[k + 1], ad = ab[k] - ab[k + 1];
    omb -= as * sp;
    ommb -= ad * sm;
    const T spb = -(c.om * as), smb = -(c.omm * ad);
    nb[k] = (T)0.5 * (spb + smb);
    nb[k + 1] = (T)0.5 * (spb - smb);
  }
  T invb = (T)0;
  if (a.les) {
    T teb;
    if (a.trt) {
      const T tm = c.tauEff - (T)0.5;
      teb = ommb * cdiv(c.omm * c.omm * (T)a.lam, tm * tm) - omb * (c.om * c.om);
    } else {
      teb = -(omb + ommb) * (c.om * c.om);
    }
    const T Rb = (T)0.5 * teb;
    const T Xb = cdiv(Rb, (T)2 * c.R);
    const T K = (T)(18 * 1.4142135623730951) * (T)a.cs2;
    const T magb = Xb * K * c.inv;
    invb += Xb * K * c.mag;
    const T Qb = c.mag > (T)0 ? cdiv(magb, c.mag) : (T)0;
    const T pxxb = (T)2 * c.pxx * Qb, pyyb = (T)2 * c.pyy * Qb, pzzb = (T)2 * c.pzz * Qb;
    const T pxyb = (T)4 * c.pxy * Qb, pxzb = (T)4 * c.pxz * Qb, pyzb = (T)4 * c.pyz * Qb;
    nb[1] += pxxb; nb[2] += pxxb;
    nb[3] += pyyb; nb[4] += pyyb;
    nb[5] += pzzb; nb[6] += pzzb;
    nb[7] += pxxb + pyyb + pxyb; nb[8] += pxxb + pyyb + pxyb;
    nb[9] += pxxb + pyyb - pxyb; nb[10] += pxxb + pyyb - pxyb;
    nb[11] += pxxb + pzzb + pxzb; nb[12] += pxxb + pzzb + pxzb;
    nb[13] += pxxb + pzzb - pxzb; nb[14] += pxxb + pzzb - pxzb;
    nb[15] += pyyb + pzzb + pyzb; nb[16] += pyyb + pzzb + pyzb;
    nb[17] += pyyb + pzzb - pyzb; nb[18] += pyyb + pzzb - pyzb;
  }
  T Ab = (T)0, r3b = (T)0, r45b = (T)0, vxb = (T)0, vyb = (T)0, vzb = (T)0;
#pragma unroll
  for (int q = 0; q < Q; q++) {
    fb[q] += nb[q];
    const T eb = -nb[q];
    Ab += (T)wq(q) * eb;
    if (q > 0) {
      const T cv = (T)ex(q) * c.vx + (T)ey(q) * c.vy + (T)ez(q) * c.vz;
      const T web = (T)wq(q) * eb;
      r3b += web * cv;
      r45b += web * (cv * cv);
      const T cvb = web * (c.r3 + (T)2 * c.r45 * cv);
      vxb += (T)ex(q) * cvb; vyb += (T)ey(q) * cvb; vzb += (T)ez(q) * cvb;
    }
  }
  T drb = Ab;
  T rb = (T)3 * r3b + (T)4.5 * r45b - (T)1.5 * c.usq * Ab;
  const T usqb = -(c.r * (T)1.5 * Ab);
  vxb += (T)2 * c.vx * usqb; vyb += (T)2 * c.vy * usqb; vzb += (T)2 * c.vz * usqb;
  invb += vxb * c.jx + vyb * c.jy + vzb * c.jz;
  const T jxb = vxb * c.inv, jyb = vyb * c.inv, jzb = vzb * c.inv;
  rb -= c.inv * c.inv * invb;
  drb += rb;
#pragma unroll
  for (int q = 0; q < Q; q++)
    fb[q] += drb + ((T)ex(q) * jxb + (T)ey(q) * jyb + (T)ez(q) * jzb);
}

// Solid fraction of cell (x, y, z); 0 outside the box.
template <class S>
__device__ __forceinline__ double sfrac_at(const StepArgs<S>& a, int x, int y, int z) {
  if (!a.sfrac) return 0.0;
  if (x < a.sb[0] || x >= a.sb[3] || y < a.sb[1] || y >= a.sb[4] || z < a.sb[2] || z >= a.sb[5])
    return 0.0;
  return a.sfrac[(x - a.sb[0]) + (long long)(a.sb[3] - a.sb[0]) *
                                     ((y - a.sb[1]) + (long long)(a.sb[4] - a.sb[1]) * (z - a.sb[2]))];
}

template <class T, class S>
__device__ __forceinline__ S to_store(T v) {
  if constexpr (std::is_same<T, double>::value) return Store<S>::from_d(v);
  else return Store<S>::from_f(v);
}

// The fused step with partial bounce-back: k_step's categories and boundary
// rules, the collision of cell_fw, then the blend and its force.
template <class S, bool EXACT, class IDX>
__global__ void __launch_bounds__(STEP_BX) k_step_pbb(const __grid_constant__ StepArgs<S> a) {
  using M = typename std::conditional<EXACT, double, float>::type;
  pdl_enter();
  const int x = blockIdx.x * STEP_BX + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  const long long i = (long long)x + (long long)a.nx * y + a.nxy * z;
  double Fx = 0, Fy = 0, Fz = 0;
  // Every 32-cell segment that touches the box owns a force slot and must
  // write it every step (zeros where nothing is exchanged): cells of the box
  // take part in the warp's partial whatever their category.
  bool near_cell = x < a.nx && x >= a.sb[0] && x < a.sb[3] && y >= a.sb[1] && y < a.sb[4] &&
                   z >= a.sb[2] && z < a.sb[5];
  if (x < a.nx - 1) {
    int cat;
    uint8_t fl = 0;
    const bool dup = (x == a.nx - 2);
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
      CellFw<M> c;
      const bool wall = (fl & FLAG_NEAR) != 0;
      near_cell = near_cell || wall;
      const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
      const S* Fi = a.F + i;
#pragma unroll
      for (int q = 0; q < Q; q++) c.f[q] = ld<M>(Fi[(IDX)a.src[q]]);
      if (wall || shell) patch_special<S, M>(a, i, x, y, z, shell, c.f, Fx, Fy, Fz);
      cell_fw<M>(a, c);
      if (!(c.r > (M)0 && c.r < (M)1.0e30)) atomicOr(a.err, 1u);
      if (a.write_fields) {
        const float rf = (float)c.r, xf = (float)c.vx, yf = (float)c.vy, zf = (float)c.vz;
        a.rho[i] = rf; a.ux[i] = xf; a.uy[i] = yf; a.uz[i] = zf;
        if (dup) { a.rho[i + 1] = rf; a.ux[i + 1] = xf; a.uy[i + 1] = yf; a.uz[i + 1] = zf; }
      } else if (a.mov && wall) {
        a.rho[i] = (float)c.r;
      }
      const double s = sfrac_at(a, x, y, z);
      S out[Q];
      if (s != 0.0) {
        const M sm = (M)s;
        M px = (M)0, py = (M)0, pz = (M)0;
#pragma unroll
        for (int q = 0; q < Q; q++) {
          const M fo = c.f[opp(q)];
          const M d = c.gc[q] - fo;
          px += (M)ex(q) * d; py += (M)ey(q) * d; pz += (M)ez(q) * d;
          out[q] = to_store<M, S>(((M)1 - sm) * c.gc[q] + sm * fo);
        }
        Fx += (double)(sm * px); Fy += (double)(sm * py); Fz += (double)(sm * pz);
      } else {
#pragma unroll
        for (int q = 0; q < Q; q++) out[q] = to_store<M, S>(c.gc[q]);
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
#pragma unroll
      for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = Gi[(IDX)a.dst[q]];
      if (a.write_fields) {
        a.ux[i + 1] = a.ux[i]; a.uy[i + 1] = a.uy[i]; a.uz[i + 1] = a.uz[i]; a.rho[i + 1] = a.rho[i];
      }
    }
  }
  warp_force_partial(Fx, Fy, Fz, near_cell, a);
}

// ---- adjoint ------------------------------------------------------------------------

template <class T>
struct AdjArgs {
  const T* Tn;     // adjoint of the next step: per consumer link, T[q*n + i]
  T* Tc;           // this step's
  double* ds;      // dJ/ds accumulated on the solid-fraction box
  double wJ;       // weight of this step's force in J
  int comp;        // force component of J
  long long gat[Q];   // element offset from cell i to its link-q consumer: q*n + ex + nx ey + nxy ez
  uint32_t gatb[Q];   // gat[q] * sizeof(T) (non-negative), when every offset fits in 31 bits
  uint32_t rowb[Q];   // q*n * sizeof(T), likewise
};

// The free-slip term of the adjoint of the population stored at (q, location
// lx,ly,lz): when the location's link-q consumer lies on a side plane y or z,
// the cell mirrored back into the interior pulls it through the mirrored link.
template <class T, class S>
__device__ __forceinline__ T adj_mirror(const StepArgs<S>& a, const T* Tn, int q, int lx, int ly,
                                        int lz) {
  const int px = lx + ex(q), py = ly + ey(q), pz = lz + ez(q);
  const bool ym = py == 0 || py == a.ny - 1, zm = pz == 0 || pz == a.nz - 1;
  if (!(ym || zm) || px < 0 || px >= a.nx) return (T)0;
  const int sy = ym ? py : ly, sz = zm ? pz : lz;
  if (a.flags[lx + (long long)a.nx * sy + a.nxy * sz] & FLAG_SOLID_MASK) return (T)0;
  const int cy = ym ? ly : py, cz = zm ? lz : pz;
  int qq = q;
  if (ym) qq = mirror_y(qq);
  if (zm) qq = mirror_z(qq);
  return Tn[(long long)qq * a.n + px + (long long)a.nx * cy + a.nxy * cz];
}

// The free-slip terms of a shell cell's gathered adjoint of link q: the
// mirrors of its own consumer and, at x = nx-2, those of the outlet column's
// copy of the cell.
template <class T, class S>
__device__ __forceinline__ T adj_shell(const StepArgs<S>& a, const T* Tn, int q, int x, int y,
                                       int z) {
  T v = adj_mirror<T>(a, Tn, q, x, y, z);
  if (x == a.nx - 2) v += adj_mirror<T>(a, Tn, q, x + 1, y, z);
  return v;
}

// One adjoint step, one thread per cell. A computed cell recomputes its
// forward collision from the stored state, gathers the adjoints of the 19
// populations it stored (the consumers of its links in the next step), runs
// the collision's vector-Jacobian product and writes the adjoints of the 19
// values it pulled; cells of the solid-fraction box also accumulate dJ/ds.
// NB: offsets in bytes (every buffer spans < 2^31 bytes) instead of 64-bit
// element indices.
// Resident blocks per SM the register budget is set for, the fastest measured
// on B200: float32 adjoints of a half-storage state 5 (96 registers; 4
// measured 7% slower), of a float32 state 4 (128 registers, no spills; 3%
// faster than 5); float64 adjoints 3 (168 registers).
template <class S, class T>
constexpr int adj_min_blocks() { return sizeof(T) == 8 ? 3 : (sizeof(S) == 4 ? 4 : 5); }

template <class S, class T, bool NB>
__global__ void __launch_bounds__(STEP_BX, adj_min_blocks<S, T>()) k_adjoint(const __grid_constant__ StepArgs<S> a,
                                                         const __grid_constant__ AdjArgs<T> j) {
  pdl_enter();
  const int x = blockIdx.x * STEP_BX + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  const long long i = (long long)x + (long long)a.nx * y + a.nxy * z;
  if (x >= a.nx) return;
  const bool inner = x >= 1 && x <= a.nx - 2 && y >= 1 && y <= a.ny - 2 && z >= 1 &&
                     z <= a.nz - 2;
  T* Tci = j.Tc + i;
  const T* Tni = j.Tn + i;
  const S* Fi = a.F + i;
  auto trow = [&](T* p, int q) -> T& {
    if constexpr (NB) return *reinterpret_cast<T*>(reinterpret_cast<char*>(p) + j.rowb[q]);
    else return p[a.dst[q]];
  };
  if (!inner) {
#pragma unroll
    for (int q = 0; q < Q; q++) trow(Tci, q) = (T)0;
    return;
  }
  auto tn_row = [&](int q) -> T {
    if constexpr (NB) return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(Tni) + j.rowb[q]);
    else return Tni[a.dst[q]];
  };
  auto tn_gat = [&](int q) -> T {
    if constexpr (NB) return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(Tni) + j.gatb[q]);
    else return Tni[j.gat[q]];
  };
  auto tn_gat1 = [&](int q) -> T {   // the consumer of cell i+1's link q
    if constexpr (NB) return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(Tni + 1) + j.gatb[q]);
    else return Tni[j.gat[q] + 1];
  };
  auto f_pull = [&](int q) -> T {
    if constexpr (NB) return (T)ld<T>(*reinterpret_cast<const S*>(reinterpret_cast<const char*>(Fi) + a.srcb[q]));
    else return (T)ld<T>(Fi[a.src[q]]);
  };
  auto f_own = [&](int q) -> T {
    if constexpr (NB) return (T)ld<T>(*reinterpret_cast<const S*>(reinterpret_cast<const char*>(Fi) + a.dstb[q]));
    else return (T)ld<T>(Fi[a.dst[q]]);
  };
  // The free-slip mirror terms of shell cells go first, while few values are
  // live, into this thread's column of shared memory.
  __shared__ T mir[Q][STEP_BX];
  const bool shell = a.freeslip && (y == 1 || y == a.ny - 2 || z == 1 || z == a.nz - 2);
  if (shell) {
#pragma unroll
    for (int q = 0; q < Q; q++) mir[q][threadIdx.x] = adj_shell<T>(a, j.Tn, q, x, y, z);
  }
  // Gathered adjoints of the stored populations (plain consumers) and the
  // pulled populations, issued before the cell's flags byte arrives: every
  // source of an inner cell lies inside the lattice.
  T g[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) g[q] = tn_gat(q);
  CellFw<T> c;
  if (!shell) {
#pragma unroll
    for (int q = 0; q < Q; q++) c.f[q] = f_pull(q);
  } else {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      int sy = y - ey(q), sz = z - ez(q), qq = q;
      if (sy == 0 || sy == a.ny - 1) { sy = y; qq = mirror_y(qq); }
      if (sz == 0 || sz == a.nz - 1) { sz = z; qq = mirror_z(qq); }
      c.f[q] = (T)ld<T>(a.F[qq * a.n + (x - ex(q)) + (long long)a.nx * sy + a.nxy * sz]);
    }
  }
  const uint8_t fl = a.flags[i];
  if (fl & FLAG_SOLID_MASK) {   // solids do not pull
#pragma unroll
    for (int q = 0; q < Q; q++) trow(Tci, q) = (T)0;
    return;
  }
  const unsigned long long m = (fl & FLAG_NEAR) ? a.nmask[i] : 0ull;
  const unsigned sm = (unsigned)m, om = (unsigned)(m >> 32);
  // the rest of the gathered adjoints: the cell itself where the link's
  // neighbour is solid (it bounces the value), at x = nx-2 the consumer of
  // the outlet column's copy (x+1 + c_q, inside the lattice when c_q has no
  // +x component), the free-slip mirrors
  if (sm) {
#pragma unroll
    for (int q = 0; q < Q; q++)
      if ((sm >> opp(q)) & 1u) g[q] += tn_row(opp(q));
  }
  if (x == a.nx - 2) {
#pragma unroll
    for (int q = 0; q < Q; q++)
      if (ex(q) <= 0) g[q] += tn_gat1(q);
  }
  if (shell) {
#pragma unroll
    for (int q = 0; q < Q; q++) g[q] += mir[q][threadIdx.x];
  }
  // stationary walls: a solid neighbour's link takes the cell's own opposite
  // population
  if (sm) {
#pragma unroll
    for (int q = 0; q < Q; q++)
      if ((sm >> q) & 1u) c.f[q] = f_own(opp(q));
  }
  cell_fw<T>(a, c);
  const T wJ = (T)j.wJ;
  // partial bounce-back: g = (1-s) gc + s f_opp, force s sum_q c_q (gc_q - f_opp(q))
  T st = (T)0;
  if (a.sfrac && x >= a.sb[0] && x < a.sb[3] && y >= a.sb[1] && y < a.sb[4] && z >= a.sb[2] &&
      z < a.sb[5]) {
    st = (T)sfrac_at(a, x, y, z);
    // dJ/ds = sum_q g_q (f_opp(q) - gc_q) + wJ sum_q c_q (gc_q - f_opp(q))
    T g1 = (T)0, g2 = (T)0;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const T cc = (T)(j.comp == 0 ? ex(q) : (j.comp == 1 ? ey(q) : ez(q)));
      const T d = c.f[opp(q)] - c.gc[q];
      g1 += g[q] * d;
      g2 -= cc * d;
    }
    j.ds[(x - a.sb[0]) + (long long)(a.sb[3] - a.sb[0]) *
                             ((y - a.sb[1]) + (long long)(a.sb[4] - a.sb[1]) * (z - a.sb[2]))] +=
        (double)(g1 + wJ * g2);
  }
  // adjoints of the collided values (ab) and, through the blend and the
  // force, of the pulled ones (fb); s = 0 leaves ab = g, fb = 0
  T ab[Q], fb[Q];
  if (st != (T)0) {
    const T ws = wJ * st, s1 = (T)1 - st;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const T cc = (T)(j.comp == 0 ? ex(q) : (j.comp == 1 ? ey(q) : ez(q)));
      ab[q] = s1 * g[q] + ws * cc;
      fb[q] = st * g[opp(q)] + ws * cc;
    }
  } else {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      ab[q] = g[q];
      fb[q] = (T)0;
    }
  }
  if (om) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const T cc = (T)(j.comp == 0 ? ex(q) : (j.comp == 1 ? ey(q) : ez(q)));
      if ((om >> q) & 1u) fb[q] -= (T)2 * wJ * cc;   // momentum exchange of a body link
    }
  }
  cell_vjp<T>(a, c, ab, fb);
#pragma unroll
  for (int q = 0; q < Q; q++) trow(Tci, q) = fb[q];
}

// Launch one adjoint step (both kernels' offset forms are instantiated by the
// translation unit that calls this).
template <class S, class T>
inline void launch_adjoint(const StepArgs<S>& a, const T* Tn, T* Tc, double* ds, double wJ,
                           int comp, cudaStream_t s) {
  AdjArgs<T> j{};
  j.Tn = Tn; j.Tc = Tc; j.ds = ds; j.wJ = wJ; j.comp = comp;
  const size_t wide_elem = sizeof(S) > sizeof(T) ? sizeof(S) : sizeof(T);
  const bool nb = 19 * a.n * (long long)wide_elem < (1LL << 31);
  for (int q = 0; q < Q; q++) {
    j.gat[q] = q * a.n + ex(q) + (long long)a.nx * ey(q) + a.nxy * ez(q);
    j.gatb[q] = nb ? (uint32_t)(j.gat[q] * (long long)sizeof(T)) : 0u;
    j.rowb[q] = nb ? (uint32_t)(q * a.n * (long long)sizeof(T)) : 0u;
  }
  const dim3 grid = step_grid(a.nx, a.ny, a.nz);
  if (nb) launch_pdl(k_adjoint<S, T, true>, grid, dim3(STEP_BX), s, a, j);
  else launch_pdl(k_adjoint<S, T, false>, grid, dim3(STEP_BX), s, a, j);
}

}  // namespace wt
