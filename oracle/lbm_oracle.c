/*
 * lbm_oracle.c — CPU oracle of windtunnel's D3Q19 step (js/lbm.js).
 *
 * TEST INFRASTRUCTURE. Only the tests, the smoke check and the CPU-baseline
 * leg of the benchmark load this library, and only as the checker; the
 * product (libwt.so) never links or calls it.
 *
 * It restates js/lbm.js:28-512 and the voxel-backed occupancy lookup of
 * js/shapes.js:365-388 in C: float64 arithmetic in the reference's operation
 * order, a rounding to the storage type at every store, no FMA contraction
 * (built with -ffp-contract=off, no -ffast-math). Two instantiations:
 *   or32_*  float32 storage = the reference's Float32Array solver,
 *   or64_*  float64 storage = the FP64 oracle.
 * Pinned against the reference itself: tests/golden holds states produced
 * by running the unmodified js/lbm.js and js/shapes.js (see
 * tests/golden/make_golden.py) and tests/test_oracle_golden.py checks this
 * code against them bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/wt.h"

#define OR_Q 19
#define OR_FLUID 0
#define OR_SOLID_OBJ 1
#define OR_SOLID_WALL 2
#define OR_SQRT2 1.4142135623730951

/* js/lbm.js:29-37: direction set, opposites and weights. */
static const int OR_EX[OR_Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int OR_EY[OR_Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int OR_EZ[OR_Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OR_OPP[OR_Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const double OR_W[OR_Q] = {
    1.0 / 3,  1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18,
    1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
    1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
/* Mirror images of each direction in y and in z (free-slip option). */
static const int OR_MY[OR_Q] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
static const int OR_MZ[OR_Q] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};

/* ECMAScript ToInt32 (the `| 0` of js/shapes.js:379 and js/lbm.js:521). */
static int32_t or_toint32(double v) {
  if (!isfinite(v)) return 0;
  if (v > -2147483649.0 && v < 2147483648.0) return (int32_t)v;
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}

/* splitmix64, draw k of stream `seed`; uniform in [0,1) with 53 bits. */
static double or_uniform(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

double or_uniform_draw(uint64_t seed, uint64_t k) { return or_uniform(seed, k); }
int32_t or_toint32_export(double v) { return or_toint32(v); }

/* js/lbm.js:106-111 defaults. */
void or_default_params(wt_params* p) {
  memset(p, 0, sizeof(*p));
  p->u0 = 0.06;
  p->tau = 0.5035;
  p->les = 1;
  p->csm = 0.14;
  p->trt = 1;
  p->lambda = 1.0 / 4;
  p->moving_walls = 0;
  p->side_bc = 0;
  p->math = 1;
  p->f16_rounding = 1;
}

static int or_clamp_int(double v) {
  if (v > 2147483647.0) return 2147483647;
  if (v < -2147483647.0) return -2147483647;
  return (int)v;
}

/* js/lbm.js:216-218: inclusive scan range {x0,x1,y0,y1,z0,z1}. */
void or_voxel_range(int nx, int ny, int nz, const double box[6], int rg[6]) {
  const double x0 = fmax(1, floor(box[0])), x1 = fmin(nx - 2, ceil(box[3]));
  const double y0 = fmax(1, floor(box[1])), y1 = fmin(ny - 2, ceil(box[4]));
  const double z0 = fmax(1, floor(box[2])), z1 = fmin(nz - 2, ceil(box[5]));
  rg[0] = or_clamp_int(x0); rg[1] = or_clamp_int(x1);
  rg[2] = or_clamp_int(y0); rg[3] = or_clamp_int(y1);
  rg[4] = or_clamp_int(z0); rg[5] = or_clamp_int(z1);
}

/* js/shapes.js:365-388: the voxel-backed Body.makeTest() closure, evaluated
 * at the cell centres of the voxelize scan range of `box` (js/lbm.js:225-229).
 * Writes one byte per range cell, x fastest; returns the number written. */
long or_lookup_mask(const uint8_t* grid, int gnx, int gny, int gnz, const double gmin[3],
                    double gi, const double M[9], const double P[3], double scale, int nx, int ny,
                    int nz, const double box[6], uint8_t* out) {
  int rg[6];
  or_voxel_range(nx, ny, nz, box, rg);
  const double inv = 1 / scale;
  const double gx0 = gmin[0], gy0 = gmin[1], gz0 = gmin[2];
  long m = 0;
  for (int z = rg[4]; z <= rg[5]; z++) {
    for (int y = rg[2]; y <= rg[3]; y++) {
      for (int x = rg[0]; x <= rg[1]; x++, m++) {
        const double X = x + 0.5, Y = y + 0.5, Z = z + 0.5;
        const double dx = X - P[0], dy = Y - P[1], dz = Z - P[2];
        const double lx = (M[0] * dx + M[3] * dy + M[6] * dz) * inv;
        const double ly = (M[1] * dx + M[4] * dy + M[7] * dz) * inv;
        const double lz = (M[2] * dx + M[5] * dy + M[8] * dz) * inv;
        uint8_t hit = 0;
        const int32_t a = or_toint32((lx - gx0) * gi);
        if (a >= 0 && a < gnx) {
          const int32_t b = or_toint32((ly - gy0) * gi);
          if (b >= 0 && b < gny) {
            const int32_t c = or_toint32((lz - gz0) * gi);
            if (c >= 0 && c < gnz) hit = grid[a + (long)gnx * (b + (long)gny * c)] != 0;
          }
        }
        out[m] = hit;
      }
    }
  }
  return m;
}

static int or_cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* ---- partial bounce-back and its discrete adjoint (no reference counterpart) ----
 *
 * Forward, per computed fluid cell with solid fraction s:
 *   g_q = (1 - s) gc_q + s f_opp(q),  F += s sum_q c_q (gc_q - f_opp(q)),
 * gc the collided populations and f the pulled ones. The objective is
 * J = mean over the last `window` steps of force component `comp`.
 *
 * The adjoint runs backwards in time over the stored forward states. T^t[q][i]
 * holds dJ/d(pulled value of link q at cell i, step t); the adjoint of the
 * population stored at location (q, j) after step t is the sum of T^{t+1} over
 * the links that pull it at step t+1 (or_adj_gather below), so every adjoint
 * step is a pull like the forward step. Quantities of the forward collision
 * are recomputed per cell from the stored pre-step state, in the operation
 * order of js/lbm.js:377-460. */
typedef struct {
  double f[OR_Q], gc[OR_Q], n[OR_Q];
  double dr, r, inv, jx, jy, jz, vx, vy, vz, usq, A, r3, r45;
  double pxx, pyy, pzz, pxy, pxz, pyz, mag, R, tauEff, om, omm;
} or_cellfw;

/* Forward collision of one cell from its pulled populations f (already in
 * c->f), js/lbm.js:377-460, keeping the intermediates. */
static void or_collide_fw(const wt_params* p, or_cellfw* c) {
  const double* f = c->f;
  const double W0 = 1.0 / 3, WF = 1.0 / 18, WE = 1.0 / 36;
  const double dr = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] +
                    f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
  const double r = 1 + dr;
  const double inv = 1 / r;
  const double jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
  const double jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
  const double jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
  const double vx = jx * inv, vy = jy * inv, vz = jz * inv;
  const double usq = vx * vx + vy * vy + vz * vz;
  const double A = dr - r * 1.5 * usq;
  const double r3 = 3 * r, r45 = 4.5 * r;
  double e[OR_Q];
  e[0] = W0 * A;
  for (int q = 1; q < OR_Q; q++) {
    const double cv = OR_EX[q] * vx + OR_EY[q] * vy + OR_EZ[q] * vz;
    e[q] = OR_W[q] * (A + r3 * cv + r45 * cv * cv);
  }
  (void)WF; (void)WE;
  for (int q = 0; q < OR_Q; q++) c->n[q] = f[q] - e[q];
  const double* n = c->n;
  const double tau0 = p->tau;
  double om = 1 / tau0, tauEff = tau0;
  c->pxx = c->pyy = c->pzz = c->pxy = c->pxz = c->pyz = c->mag = c->R = 0;
  if (p->les) {
    c->pxx = n[1] + n[2] + n[7] + n[8] + n[9] + n[10] + n[11] + n[12] + n[13] + n[14];
    c->pyy = n[3] + n[4] + n[7] + n[8] + n[9] + n[10] + n[15] + n[16] + n[17] + n[18];
    c->pzz = n[5] + n[6] + n[11] + n[12] + n[13] + n[14] + n[15] + n[16] + n[17] + n[18];
    c->pxy = n[7] + n[8] - n[9] - n[10];
    c->pxz = n[11] + n[12] - n[13] - n[14];
    c->pyz = n[15] + n[16] - n[17] - n[18];
    c->mag = sqrt(2 * (c->pxx * c->pxx + c->pyy * c->pyy + c->pzz * c->pzz +
                       2 * (c->pxy * c->pxy + c->pxz * c->pxz + c->pyz * c->pyz)));
    const double SQ18 = 18 * OR_SQRT2;
    c->R = sqrt(tau0 * tau0 + SQ18 * (p->csm * p->csm) * c->mag * inv);
    tauEff = 0.5 * (tau0 + c->R);
    om = 1 / tauEff;
  }
  const double omm = p->trt ? 1 / (0.5 + p->lambda / (tauEff - 0.5)) : om;
  c->gc[0] = f[0] - om * (f[0] - e[0]);
  for (int a = 1; a < OR_Q; a += 2) {
    const double sp = 0.5 * (n[a] + n[a + 1]), sm = 0.5 * (n[a] - n[a + 1]);
    c->gc[a] = f[a] - om * sp - omm * sm;
    c->gc[a + 1] = f[a + 1] - om * sp + omm * sm;
  }
  c->dr = dr; c->r = r; c->inv = inv; c->jx = jx; c->jy = jy; c->jz = jz;
  c->vx = vx; c->vy = vy; c->vz = vz; c->usq = usq; c->A = A; c->r3 = r3; c->r45 = r45;
  c->tauEff = tauEff; c->om = om; c->omm = omm;
}

/* Vector-Jacobian product of or_collide_fw: fb += (d gc / d f)^T a. */
static void or_collide_vjp(const wt_params* p, const or_cellfw* c, const double a[OR_Q],
                           double fb[OR_Q]) {
  const double* n = c->n;
  double nb[OR_Q];
  for (int q = 0; q < OR_Q; q++) fb[q] += a[q];
  double omb = -(a[0] * n[0]);
  double ommb = 0;
  nb[0] = -(c->om * a[0]);
  for (int k = 1; k < OR_Q; k += 2) {
    const double sp = 0.5 * (n[k] + n[k + 1]), sm = 0.5 * (n[k] - n[k + 1]);
    const double as = a[k] + a[k + 1], ad = a[k] - a[k + 1];
    omb -= as * sp;
    ommb -= ad * sm;
    const double spb = -(c->om * as), smb = -(c->omm * ad);
    nb[k] = 0.5 * (spb + smb);
    nb[k + 1] = 0.5 * (spb - smb);
  }
  double invb = 0;
  if (p->les) {
    double teb;
    if (p->trt) {
      const double tm = c->tauEff - 0.5;
      teb = ommb * (c->omm * c->omm * p->lambda / (tm * tm)) - omb * (c->om * c->om);
    } else {
      teb = -(omb + ommb) * (c->om * c->om);
    }
    const double Rb = 0.5 * teb;
    const double Xb = Rb / (2 * c->R);
    const double K = 18 * OR_SQRT2 * (p->csm * p->csm);
    const double magb = Xb * K * c->inv;
    invb += Xb * K * c->mag;
    const double Qb = c->mag > 0 ? magb / c->mag : 0;
    const double pxxb = 2 * c->pxx * Qb, pyyb = 2 * c->pyy * Qb, pzzb = 2 * c->pzz * Qb;
    const double pxyb = 4 * c->pxy * Qb, pxzb = 4 * c->pxz * Qb, pyzb = 4 * c->pyz * Qb;
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
  /* n = f - e */
  double Ab = 0, r3b = 0, r45b = 0, vxb = 0, vyb = 0, vzb = 0;
  for (int q = 0; q < OR_Q; q++) {
    fb[q] += nb[q];
    const double eb = -nb[q];
    Ab += OR_W[q] * eb;
    if (q > 0) {
      const double cv = OR_EX[q] * c->vx + OR_EY[q] * c->vy + OR_EZ[q] * c->vz;
      const double web = OR_W[q] * eb;
      r3b += web * cv;
      r45b += web * (cv * cv);
      const double cvb = web * (c->r3 + 2 * c->r45 * cv);
      vxb += OR_EX[q] * cvb; vyb += OR_EY[q] * cvb; vzb += OR_EZ[q] * cvb;
    }
  }
  /* A = dr - r * 1.5 * usq */
  double drb = Ab;
  double rb = 3 * r3b + 4.5 * r45b - 1.5 * c->usq * Ab;
  const double usqb = -(c->r * 1.5 * Ab);
  vxb += 2 * c->vx * usqb; vyb += 2 * c->vy * usqb; vzb += 2 * c->vz * usqb;
  /* v = j * inv */
  invb += vxb * c->jx + vyb * c->jy + vzb * c->jz;
  const double jxb = vxb * c->inv, jyb = vyb * c->inv, jzb = vzb * c->inv;
  /* inv = 1 / r, r = 1 + dr */
  rb -= c->inv * c->inv * invb;
  drb += rb;
  for (int q = 0; q < OR_Q; q++)
    fb[q] += drb + (OR_EX[q] * jxb + OR_EY[q] * jyb + OR_EZ[q] * jzb);
}

#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)

#define STORE float
#define OR_PFX or32_
#include "lbm_oracle_impl.h"
#undef OR_PFX
#undef STORE

#define STORE double
#define OR_PFX or64_
#include "lbm_oracle_impl.h"
#undef OR_PFX
#undef STORE
