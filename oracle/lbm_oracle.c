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
