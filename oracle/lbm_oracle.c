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

/* ---- Voxel.build, js/voxel.js:32-232 ------------------------------------------
 * Triangle soup (float32, 9 per triangle, body space) -> body-space occupancy
 * grid: surface shell rasterisation OR'd with a 2-of-3 vote of ray-parity
 * fills along x, y and z. float64 arithmetic in the reference's operation
 * order (JavaScript numbers). */
typedef struct {
  int nx, ny, nz, tris;
  double cell, inv, min[3], ext[3], centre[3], bbox[6];
  long solid;
  double openness;
} or_voxel_info;

/* js/voxel.js:32-42 and :48-71: bounds, cell size, padded dims, min corner.
 * Returns 0, -1 (no triangles), -2 (degenerate), -3 (grid too large). */
int or_voxel_dims(const float* P, long ntri, int res, or_voxel_info* vi) {
  if (res <= 0) res = 96;
  if (ntri <= 0) return -1;
  double x0 = INFINITY, y0 = INFINITY, z0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY, z1 = -INFINITY;
  for (long i = 0; i < 9 * ntri; i += 3) {
    const double x = P[i], y = P[i + 1], z = P[i + 2];
    if (x < x0) x0 = x;
    if (x > x1) x1 = x;
    if (y < y0) y0 = y;
    if (y > y1) y1 = y;
    if (z < z0) z0 = z;
    if (z > z1) z1 = z;
  }
  const double sx = x1 - x0, sy = y1 - y0, sz = z1 - z0;
  const double span = fmax(fmax(sx, sy), sz);
  if (!(span > 0)) return -2;
  const double cell = span / res;
  const int PAD = 2;
  const double dx = fmax(3, ceil(sx / cell) + 2 * PAD), dy = fmax(3, ceil(sy / cell) + 2 * PAD),
               dz = fmax(3, ceil(sz / cell) + 2 * PAD);
  if (dx * dy * dz > 40e6) return -3;
  vi->nx = (int)dx; vi->ny = (int)dy; vi->nz = (int)dz;
  vi->tris = (int)ntri;
  vi->cell = cell;
  vi->inv = 1 / cell;
  vi->min[0] = x0 - (vi->nx * cell - sx) * 0.5;
  vi->min[1] = y0 - (vi->ny * cell - sy) * 0.5;
  vi->min[2] = z0 - (vi->nz * cell - sz) * 0.5;
  vi->ext[0] = sx * 0.5; vi->ext[1] = sy * 0.5; vi->ext[2] = sz * 0.5;
  vi->centre[0] = (x0 + x1) * 0.5; vi->centre[1] = (y0 + y1) * 0.5; vi->centre[2] = (z0 + z1) * 0.5;
  vi->bbox[0] = x0; vi->bbox[1] = y0; vi->bbox[2] = z0;
  vi->bbox[3] = x1; vi->bbox[4] = y1; vi->bbox[5] = z1;
  vi->solid = 0;
  vi->openness = 0;
  return 0;
}

static int or_cmp_double(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return (x > y) - (x < y);
}

/* js/voxel.js:105-137: mark every cell the surface passes through. */
static void or_raster_surface(const float* P, long ntri, uint8_t* shell, const or_voxel_info* vi) {
  const int nx = vi->nx, ny = vi->ny, nz = vi->nz;
  const double inv = 1 / vi->cell;
  for (long t = 0; t < ntri; t++) {
    const float* o = P + 9 * t;
    const double ax = o[0], ay = o[1], az = o[2], bx = o[3], by = o[4], bz = o[5];
    const double cx = o[6], cy = o[7], cz = o[8];
    const double e1 = fmax(fmax(fabs(bx - ax), fabs(by - ay)), fabs(bz - az));
    const double e2 = fmax(fmax(fabs(cx - ax), fabs(cy - ay)), fabs(cz - az));
    double n1 = ceil(e1 * inv * 2) + 1, n2 = ceil(e2 * inv * 2) + 1;
    if (n1 * n2 > 4096) {
      const double k = sqrt(4096 / (n1 * n2));
      n1 = fmax(2, (double)or_toint32(n1 * k));
      n2 = fmax(2, (double)or_toint32(n2 * k));
    }
    for (double i = 0; i <= n1; i++) {
      const double u = i / n1;
      const double jmax = ceil((1 - u) * n2);
      for (double j = 0; j <= jmax; j++) {
        const double v = fmin(j / n2, 1 - u);
        const double x = ax + (bx - ax) * u + (cx - ax) * v;
        const double y = ay + (by - ay) * u + (cy - ay) * v;
        const double z = az + (bz - az) * u + (cz - az) * v;
        const int32_t gx = or_toint32((x - vi->min[0]) * inv);
        const int32_t gy = or_toint32((y - vi->min[1]) * inv);
        const int32_t gz = or_toint32((z - vi->min[2]) * inv);
        if (gx < 0 || gy < 0 || gz < 0 || gx >= nx || gy >= ny || gz >= nz) continue;
        shell[gx + (long)nx * (gy + (long)ny * gz)] = 1;
      }
    }
  }
}

/* js/voxel.js:144-232: ray parity along `axis`, one ray per column. */
static int or_parity_fill(const float* P, long ntri, uint8_t* votes, const or_voxel_info* vi,
                          int axis) {
  const int dim[3] = {vi->nx, vi->ny, vi->nz};
  const int A = axis, B = (axis + 1) % 3, C = (axis + 2) % 3;
  const int nA = dim[A], nB = dim[B], nC = dim[C];
  const double cell = vi->cell;
  const double minA = vi->min[A], minB = vi->min[B], minC = vi->min[C];
  const double spanB = nB * cell, spanC = nC * cell;
  const int nbB = nB < 48 ? nB : 48, nbC = nC < 48 ? nC : 48;
  const double kB = nbB / spanB, kC = nbC / spanC;
  const int nb = nbB * nbC;
  int* count = (int*)calloc((size_t)nb + 1, sizeof(int));
  int* lo = (int*)malloc(sizeof(int) * 2 * (size_t)ntri);
  int* hi = (int*)malloc(sizeof(int) * 2 * (size_t)ntri);
  double* hits = (double*)malloc(sizeof(double) * 512);
  if (!count || !lo || !hi || !hits) { free(count); free(lo); free(hi); free(hits); return -1; }
  for (long t = 0; t < ntri; t++) {
    const float* o = P + 9 * t;
    const double b0 = o[B], b1 = o[3 + B], b2 = o[6 + B];
    const double c0 = o[C], c1 = o[3 + C], c2 = o[6 + C];
    double bl = floor((fmin(fmin(b0, b1), b2) - minB) * kB);
    double bh = floor((fmax(fmax(b0, b1), b2) - minB) * kB);
    double cl = floor((fmin(fmin(c0, c1), c2) - minC) * kC);
    double ch = floor((fmax(fmax(c0, c1), c2) - minC) * kC);
    bl = bl < 0 ? 0 : bl; bh = bh >= nbB ? nbB - 1 : bh;
    cl = cl < 0 ? 0 : cl; ch = ch >= nbC ? nbC - 1 : ch;
    lo[2 * t] = (int)bl; hi[2 * t] = (int)bh; lo[2 * t + 1] = (int)cl; hi[2 * t + 1] = (int)ch;
    if (bl > bh || cl > ch) continue;
    for (int cc = (int)cl; cc <= (int)ch; cc++)
      for (int bb = (int)bl; bb <= (int)bh; bb++) count[bb + nbB * cc + 1]++;
  }
  for (int i = 0; i < nb; i++) count[i + 1] += count[i];
  int* items = (int*)malloc(sizeof(int) * ((size_t)count[nb] + 1));
  int* cursor = (int*)malloc(sizeof(int) * (size_t)nb);
  if (!items || !cursor) { free(count); free(lo); free(hi); free(hits); free(items); free(cursor); return -1; }
  memcpy(cursor, count, sizeof(int) * (size_t)nb);
  for (long t = 0; t < ntri; t++) {
    const int bl = lo[2 * t], bh = hi[2 * t], cl = lo[2 * t + 1], ch = hi[2 * t + 1];
    if (bl > bh || cl > ch) continue;
    for (int cc = cl; cc <= ch; cc++)
      for (int bb = bl; bb <= bh; bb++) items[cursor[bb + nbB * cc]++] = (int)t;
  }
  const long strideA = A == 0 ? 1 : (A == 1 ? dim[0] : (long)dim[0] * dim[1]);
  const long strideB = B == 0 ? 1 : (B == 1 ? dim[0] : (long)dim[0] * dim[1]);
  const long strideC = C == 0 ? 1 : (C == 1 ? dim[0] : (long)dim[0] * dim[1]);
  for (int ic = 0; ic < nC; ic++) {
    const double pc = minC + (ic + 0.5003719) * cell;
    const int bc = (int)fmin(nbC - 1, fmax(0, floor((pc - minC) * kC)));
    for (int ib = 0; ib < nB; ib++) {
      const double pb = minB + (ib + 0.4996281) * cell;
      const int bb = (int)fmin(nbB - 1, fmax(0, floor((pb - minB) * kB)));
      const int s = count[bb + nbB * bc], e = count[bb + nbB * bc + 1];
      if (s == e) continue;
      int nh = 0;
      for (int k = s; k < e && nh < 512; k++) {
        const float* o = P + 9 * (long)items[k];
        const double b0 = o[B], c0 = o[C], b1 = o[3 + B], c1 = o[3 + C], b2 = o[6 + B], c2 = o[6 + C];
        const double d = (c1 - c2) * (b0 - b2) + (b2 - b1) * (c0 - c2);
        if (d == 0) continue;
        const double id = 1 / d;
        const double l0 = ((c1 - c2) * (pb - b2) + (b2 - b1) * (pc - c2)) * id;
        if (l0 < 0 || l0 > 1) continue;
        const double l1 = ((c2 - c0) * (pb - b2) + (b0 - b2) * (pc - c2)) * id;
        if (l1 < 0 || l1 > 1) continue;
        const double l2 = 1 - l0 - l1;
        if (l2 < 0 || l2 > 1) continue;
        hits[nh++] = l0 * (double)o[A] + l1 * (double)o[3 + A] + l2 * (double)o[6 + A];
      }
      if (nh < 2) continue;
      qsort(hits, (size_t)nh, sizeof(double), or_cmp_double);
      const long colBase = ib * strideB + ic * strideC;
      for (int k = 0; k + 1 < nh; k += 2) {
        double i0 = ceil((hits[k] - minA) / cell - 0.5);
        double i1 = floor((hits[k + 1] - minA) / cell - 0.5);
        if (i0 < 0) i0 = 0;
        if (i1 >= nA) i1 = nA - 1;
        for (double ia = i0; ia <= i1; ia++) votes[colBase + (long)ia * strideA]++;
      }
    }
  }
  free(count); free(lo); free(hi); free(hits); free(items); free(cursor);
  return 0;
}

/* js/voxel.js:48-102: the grid (x fastest, nx*ny*nz bytes) and its stats. */
int or_voxel_build(const float* P, long ntri, int res, uint8_t* grid, or_voxel_info* vi) {
  int rc = or_voxel_dims(P, ntri, res, vi);
  if (rc) return rc;
  const long n = (long)vi->nx * vi->ny * vi->nz;
  uint8_t* votes = (uint8_t*)calloc((size_t)n, 1);
  uint8_t* shell = (uint8_t*)calloc((size_t)n, 1);
  if (!votes || !shell) { free(votes); free(shell); return -4; }
  or_raster_surface(P, ntri, shell, vi);
  for (int axis = 0; axis < 3; axis++) {
    if (or_parity_fill(P, ntri, votes, vi, axis)) { free(votes); free(shell); return -4; }
  }
  long solid = 0, disagree = 0;
  for (long i = 0; i < n; i++) {
    const int v = votes[i];
    const int inside = v >= 2 || shell[i] == 1;
    if (inside) solid++;
    if (v == 1 || v == 2) disagree++;
    grid[i] = inside ? 1 : 0;
  }
  vi->solid = solid;
  vi->openness = solid ? (double)disagree / solid : 0;
  free(votes); free(shell);
  return 0;
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
