/*
 * lbm_oracle_impl.h — body of the CPU oracle, included twice by
 * lbm_oracle.c with STORE = float (the reference's Float32Array storage)
 * and STORE = double (the FP64 oracle). TEST INFRASTRUCTURE ONLY: the
 * product never links or calls this code.
 *
 * Every function restates js/lbm.js (file:line given per function) with
 * float64 arithmetic in the reference's operation order and a rounding to
 * STORE at every array store. Compiled with -ffp-contract=off and without
 * -ffast-math, it reproduces the JavaScript engine's IEEE double results.
 */

#define OR_T STORE
#define OR_FN(name) OR_CAT(OR_PFX, name)

typedef struct {
  int nx, ny, nz;
  long n;
  int parity;
  OR_T *bufA, *bufB;
  uint8_t *solid, *near_;
  float *ux, *uy, *uz, *rho;
  float *uwx, *uwy, *uwz;
  long off[OR_Q];
  long src[OR_Q];
  wt_params p;
  double force[3];
  int frontal, planform, solid_cells, ride_height, ground;
  long steps;
  /* partial bounce-back: solid fraction on the half-open box sbox (x0,y0,z0,x1,y1,z1) */
  double* sfrac;
  int sbox[6];
} OR_FN(lbm);

void OR_FN(destroy)(OR_FN(lbm) * L);

static inline OR_T* OR_FN(cur_f)(OR_FN(lbm) * L) { return L->parity ? L->bufB : L->bufA; }
static inline OR_T* OR_FN(cur_g)(OR_FN(lbm) * L) { return L->parity ? L->bufA : L->bufB; }

/* js/lbm.js:155-162 (_writeEq). */
static void OR_FN(write_eq)(OR_FN(lbm) * L, OR_T* arr, long i, double r, double vx, double vy,
                            double vz) {
  const long n = L->n;
  const double usq = 1.5 * (vx * vx + vy * vy + vz * vz);
  for (int q = 0; q < OR_Q; q++) {
    const double cu = 3 * ((double)OR_EX[q] * vx + (double)OR_EY[q] * vy + (double)OR_EZ[q] * vz);
    arr[q * n + i] = (OR_T)(OR_W[q] * ((r - 1) + r * (cu + 0.5 * cu * cu - usq)));
  }
}

/* js/lbm.js:164-174 (reset). */
int OR_FN(reset)(OR_FN(lbm) * L) {
  OR_T* f = OR_FN(cur_f)(L);
  OR_T* g = OR_FN(cur_g)(L);
  for (long i = 0; i < L->n; i++) {
    const double v = L->solid[i] ? 0 : L->p.u0;
    OR_FN(write_eq)(L, f, i, 1, v, 0, 0);
    OR_FN(write_eq)(L, g, i, 1, v, 0, 0);
    L->ux[i] = (float)v; L->uy[i] = 0; L->uz[i] = 0; L->rho[i] = 1;
  }
  L->steps = 0;
  L->force[0] = L->force[1] = L->force[2] = 0;
  return 0;
}

/* reset() plus seeded velocity noise on non-solid cells (wt_init_eq_noise). */
int OR_FN(init_eq_noise)(OR_FN(lbm) * L, uint64_t seed, double amp) {
  OR_T* f = OR_FN(cur_f)(L);
  OR_T* g = OR_FN(cur_g)(L);
  for (long i = 0; i < L->n; i++) {
    double vx, vy, vz;
    if (L->solid[i]) {
      vx = 0; vy = 0; vz = 0;
    } else {
      vx = L->p.u0 + amp * (2 * or_uniform(seed, 3 * (uint64_t)i) - 1);
      vy = amp * (2 * or_uniform(seed, 3 * (uint64_t)i + 1) - 1);
      vz = amp * (2 * or_uniform(seed, 3 * (uint64_t)i + 2) - 1);
    }
    OR_FN(write_eq)(L, f, i, 1, vx, vy, vz);
    OR_FN(write_eq)(L, g, i, 1, vx, vy, vz);
    L->ux[i] = (float)vx; L->uy[i] = (float)vy; L->uz[i] = (float)vz; L->rho[i] = 1;
  }
  L->steps = 0;
  L->force[0] = L->force[1] = L->force[2] = 0;
  return 0;
}

/* js/lbm.js:176-180 (_seedCell). */
static void OR_FN(seed_cell)(OR_FN(lbm) * L, long i) {
  OR_FN(write_eq)(L, OR_FN(cur_f)(L), i, 1, L->p.u0, 0, 0);
  OR_FN(write_eq)(L, OR_FN(cur_g)(L), i, 1, L->p.u0, 0, 0);
  L->ux[i] = (float)L->p.u0; L->uy[i] = 0; L->uz[i] = 0; L->rho[i] = 1;
}

OR_FN(lbm) * OR_FN(create)(int nx, int ny, int nz) {
  if (nx < 3 || ny < 3 || nz < 3) return NULL;
  OR_FN(lbm)* L = (OR_FN(lbm)*)calloc(1, sizeof(OR_FN(lbm)));
  if (!L) return NULL;
  L->nx = nx; L->ny = ny; L->nz = nz;
  L->n = (long)nx * ny * nz;
  const long n = L->n;
  L->bufA = (OR_T*)calloc((size_t)n * OR_Q, sizeof(OR_T));
  L->bufB = (OR_T*)calloc((size_t)n * OR_Q, sizeof(OR_T));
  L->solid = (uint8_t*)calloc((size_t)n, 1);
  L->near_ = (uint8_t*)calloc((size_t)n, 1);
  L->ux = (float*)calloc((size_t)n, sizeof(float));
  L->uy = (float*)calloc((size_t)n, sizeof(float));
  L->uz = (float*)calloc((size_t)n, sizeof(float));
  L->rho = (float*)calloc((size_t)n, sizeof(float));
  L->uwx = (float*)calloc((size_t)n, sizeof(float));
  L->uwy = (float*)calloc((size_t)n, sizeof(float));
  L->uwz = (float*)calloc((size_t)n, sizeof(float));
  if (!L->bufA || !L->bufB || !L->solid || !L->near_ || !L->ux || !L->uy || !L->uz || !L->rho ||
      !L->uwx || !L->uwy || !L->uwz) {
    OR_FN(destroy)(L);
    return NULL;
  }
  /* js/lbm.js:97-104: off[q] = cell offset of c_q; src[q] = q*n - off[q]. */
  for (int q = 0; q < OR_Q; q++) {
    L->off[q] = OR_EX[q] + (long)nx * (OR_EY[q] + (long)ny * OR_EZ[q]);
    L->src[q] = q * n - L->off[q];
  }
  or_default_params(&L->p);
  L->frontal = 1;
  L->planform = 0; /* the reference leaves planformArea undefined until voxelize */
  OR_FN(reset)(L);
  return L;
}

void OR_FN(destroy)(OR_FN(lbm) * L) {
  if (!L) return;
  free(L->bufA); free(L->bufB); free(L->solid); free(L->near_);
  free(L->ux); free(L->uy); free(L->uz); free(L->rho);
  free(L->uwx); free(L->uwy); free(L->uwz);
  free(L->sfrac);
  free(L);
}

void OR_FN(set_params)(OR_FN(lbm) * L, const wt_params* p) { L->p = *p; }
void OR_FN(get_params)(OR_FN(lbm) * L, wt_params* p) { *p = L->p; }

/* js/lbm.js:268-282 (_rebuildNear). */
static void OR_FN(rebuild_near)(OR_FN(lbm) * L) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  memset(L->near_, 0, (size_t)L->n);
  for (int z = 1; z < nz - 1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      long i = 1 + (long)nx * (y + (long)ny * z);
      for (int x = 1; x < nx - 1; x++, i++) {
        if (L->solid[i]) continue;
        for (int q = 1; q < OR_Q; q++) {
          if (L->solid[i - L->off[q]]) { L->near_[i] = 1; break; }
        }
      }
    }
  }
}

/* js/lbm.js:191-266 (voxelize), with the inside() closure pre-evaluated by
 * the host over the scan range. */
int OR_FN(voxelize_mask)(OR_FN(lbm) * L, const double box[6], const uint8_t* inside,
                          size_t inside_len, const uint8_t* wall_set, const double* wall_vel,
                          int ground, double road_vel) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long n = L->n;
  int rg[6];
  or_voxel_range(nx, ny, nz, box, rg);
  const int x0 = rg[0], x1 = rg[1], y0 = rg[2], y1 = rg[3], z0 = rg[4], z1 = rg[5];
  const long ex = x1 >= x0 ? x1 - x0 + 1 : 0, ey = y1 >= y0 ? y1 - y0 + 1 : 0,
             ez = z1 >= z0 ? z1 - z0 + 1 : 0;
  if ((size_t)(ex * ey * ez) != inside_len) return -1;

  L->ground = ground ? 1 : 0;
  L->p.moving_walls = 0;
  for (long i = 0; i < n; i++) {
    if (L->solid[i] == OR_SOLID_OBJ) {
      L->solid[i] = OR_FLUID;
      OR_FN(seed_cell)(L, i);
      L->uwx[i] = L->uwy[i] = L->uwz[i] = 0;
    }
  }
  const uint8_t gy = ground ? OR_SOLID_WALL : OR_FLUID;
  const double rv = road_vel;
  if (rv != 0) L->p.moving_walls = 1;
  for (int z = 0; z < nz; z++) {
    for (int x = 0; x < nx; x++) {
      const long i = x + (long)nx * ny * z;
      if (L->solid[i] != gy) {
        L->solid[i] = gy;
        if (gy == OR_FLUID) OR_FN(seed_cell)(L, i);
      }
      L->uwx[i] = gy == OR_SOLID_WALL ? (float)rv : 0;
      L->uwy[i] = L->uwz[i] = 0;
    }
  }
  uint8_t* col = (uint8_t*)calloc((size_t)ny * nz, 1);
  uint8_t* plan = (uint8_t*)calloc((size_t)nx * nz, 1);
  int* low = (int*)malloc(sizeof(int) * (size_t)nx * nz);
  if (!col || !plan || !low) { free(col); free(plan); free(low); return -2; }
  for (long k = 0; k < (long)nx * nz; k++) low[k] = 32767;
  int cells = 0;
  long m = 0;
  OR_T* f = OR_FN(cur_f)(L);
  for (int z = z0; z <= z1; z++) {
    for (int y = y0; y <= y1; y++) {
      long i = x0 + (long)nx * (y + (long)ny * z);
      for (int x = x0; x <= x1; x++, i++, m++) {
        if (inside[m]) {
          L->solid[i] = OR_SOLID_OBJ;
          OR_FN(write_eq)(L, f, i, 1, 0, 0, 0);
          L->ux[i] = L->uy[i] = L->uz[i] = 0; L->rho[i] = 1;
          L->uwx[i] = L->uwy[i] = L->uwz[i] = 0;
          if (wall_set && wall_set[m]) {
            L->uwx[i] = (float)wall_vel[3 * m];
            L->uwy[i] = (float)wall_vel[3 * m + 1];
            L->uwz[i] = (float)wall_vel[3 * m + 2];
            L->p.moving_walls = 1;
          }
          col[y + (long)ny * z] = 1;
          const long pk = x + (long)nx * z;
          plan[pk] = 1;
          if (y < low[pk]) low[pk] = y;
          cells++;
        }
      }
    }
  }
  int a = 0;
  for (long k = 0; k < (long)ny * nz; k++) a += col[k];
  L->frontal = a > 1 ? a : 1;
  int pa = 0;
  for (long k = 0; k < (long)nx * nz; k++) pa += plan[k];
  L->planform = pa > 1 ? pa : 1;
  L->solid_cells = cells;
  int* gaps = (int*)malloc(sizeof(int) * ((size_t)nx * nz + 1));
  int ng = 0;
  for (long k = 0; k < (long)nx * nz; k++) {
    if (plan[k] && low[k] < 32767) {
      const int g = low[k] - 1;
      if (g > 0) gaps[ng++] = g;
    }
  }
  qsort(gaps, (size_t)ng, sizeof(int), or_cmp_int);
  L->ride_height = ng ? gaps[ng >> 1] : 0;
  free(gaps); free(col); free(plan); free(low);
  OR_FN(rebuild_near)(L);
  return 0;
}

/* Solid fraction of cell (x,y,z): 0 outside the partial bounce-back box. */
static inline double OR_FN(sfrac_at)(const OR_FN(lbm) * L, int x, int y, int z) {
  if (!L->sfrac) return 0;
  const int* b = L->sbox;
  if (x < b[0] || x >= b[3] || y < b[1] || y >= b[4] || z < b[2] || z >= b[5]) return 0;
  return L->sfrac[(x - b[0]) + (long)(b[3] - b[0]) * ((y - b[1]) + (long)(b[4] - b[1]) * (z - b[2]))];
}

/* Set the partial bounce-back field: s holds one value per cell of the
 * half-open box, x fastest; box == NULL clears it. */
int OR_FN(set_solid_fraction)(OR_FN(lbm) * L, const int box[6], const double* sv) {
  free(L->sfrac);
  L->sfrac = NULL;
  if (!box) return 0;
  const long m = (long)(box[3] - box[0]) * (box[4] - box[1]) * (box[5] - box[2]);
  if (box[0] < 0 || box[1] < 0 || box[2] < 0 || box[3] > L->nx || box[4] > L->ny ||
      box[5] > L->nz || m <= 0)
    return -1;
  L->sfrac = (double*)malloc(sizeof(double) * (size_t)m);
  if (!L->sfrac) return -2;
  memcpy(L->sfrac, sv, sizeof(double) * (size_t)m);
  memcpy(L->sbox, box, sizeof(int) * 6);
  return 0;
}

/* Free-slip gather (no reference counterpart; WT_SIDE_FREESLIP): the
 * population q arriving at cell (x,y,z) from a source on a side plane is the
 * mirrored population leaving the reflected source, which stays in the
 * cell's own y (resp. z) layer. */
static inline double OR_FN(gather_fs)(OR_FN(lbm) * L, const OR_T* F, int q, int x, int y, int z) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  int sx = x - OR_EX[q], sy = y - OR_EY[q], sz = z - OR_EZ[q];
  int qq = q;
  if (sy == 0 || sy == ny - 1) { sy = y; qq = OR_MY[qq]; }
  if (sz == 0 || sz == nz - 1) { sz = z; qq = OR_MZ[qq]; }
  return (double)F[(long)qq * L->n + sx + (long)nx * (sy + (long)ny * sz)];
}

/* js/lbm.js:303-466 (stepSlab): collide + pull-stream the z-slab [z0,z1). */
static void OR_FN(step_slab)(OR_FN(lbm) * L, int z0, int z1, double sf[3]) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long nn = L->n;
  const OR_T* F = OR_FN(cur_f)(L);
  OR_T* G = OR_FN(cur_g)(L);
  const uint8_t* solid = L->solid;
  const uint8_t* near_ = L->near_;
  const long* off = L->off;
  const long* src = L->src;
  float *ux = L->ux, *uy = L->uy, *uz = L->uz, *rho = L->rho;
  const float *uwx = L->uwx, *uwy = L->uwy, *uwz = L->uwz;
  const int mov = L->p.moving_walls;
  const double tau0 = L->p.tau;
  const int les = L->p.les;
  const double cs2 = L->p.csm * L->p.csm;
  const double omega0 = 1 / tau0;
  const int trt = L->p.trt;
  const double lam = L->p.lambda;
  const int freeslip = L->p.side_bc == 1;
  const double W0 = 1.0 / 3, WF = 1.0 / 18, WE = 1.0 / 36;
  const double SQ18 = 18 * OR_SQRT2;

  double Fx = 0, Fy = 0, Fz = 0;
  double fq[OR_Q];

  for (int z = z0; z < z1; z++) {
    for (int y = 1; y < ny - 1; y++) {
      long i = 1 + (long)nx * (y + (long)ny * z);
      const int shell = freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
      for (int x = 1; x < nx - 1; x++, i++) {
        if (solid[i]) continue;
        double f0, f1, f2, f3, f4, f5, f6, f7, f8, f9, f10, f11, f12, f13, f14, f15, f16, f17,
            f18;
        if (near_[i] || shell) {
          for (int q = 0; q < OR_Q; q++) {
            const long j = i - off[q];
            const uint8_t s = solid[j];
            if (s) {
              const double fd = (double)F[(long)OR_OPP[q] * nn + i];
              double corr = 0;
              if (mov) {
                const double cu = (double)OR_EX[q] * (double)uwx[j] +
                                  (double)OR_EY[q] * (double)uwy[j] +
                                  (double)OR_EZ[q] * (double)uwz[j];
                if (cu != 0) corr = 6 * OR_W[q] * (double)rho[i] * cu;
              }
              fq[q] = fd + corr;
              if (s == OR_SOLID_OBJ) {
                const double d = 2 * fd + corr;
                Fx -= d * OR_EX[q]; Fy -= d * OR_EY[q]; Fz -= d * OR_EZ[q];
              }
            } else if (shell) {
              fq[q] = OR_FN(gather_fs)(L, F, q, x, y, z);
            } else {
              fq[q] = (double)F[src[q] + i];
            }
          }
          f0 = fq[0]; f1 = fq[1]; f2 = fq[2]; f3 = fq[3]; f4 = fq[4]; f5 = fq[5]; f6 = fq[6];
          f7 = fq[7]; f8 = fq[8]; f9 = fq[9]; f10 = fq[10]; f11 = fq[11]; f12 = fq[12];
          f13 = fq[13]; f14 = fq[14]; f15 = fq[15]; f16 = fq[16]; f17 = fq[17]; f18 = fq[18];
        } else {
          f0 = F[src[0] + i]; f1 = F[src[1] + i]; f2 = F[src[2] + i]; f3 = F[src[3] + i];
          f4 = F[src[4] + i]; f5 = F[src[5] + i]; f6 = F[src[6] + i]; f7 = F[src[7] + i];
          f8 = F[src[8] + i]; f9 = F[src[9] + i]; f10 = F[src[10] + i]; f11 = F[src[11] + i];
          f12 = F[src[12] + i]; f13 = F[src[13] + i]; f14 = F[src[14] + i];
          f15 = F[src[15] + i]; f16 = F[src[16] + i]; f17 = F[src[17] + i];
          f18 = F[src[18] + i];
        }

        /* moments, js/lbm.js:377-385 */
        const double dr = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8 + f9 + f10 + f11 + f12 +
                          f13 + f14 + f15 + f16 + f17 + f18;
        const double r = 1 + dr;
        const double inv = 1 / r;
        const double vx = (f1 - f2 + f7 - f8 + f9 - f10 + f11 - f12 + f13 - f14) * inv;
        const double vy = (f3 - f4 + f7 - f8 - f9 + f10 + f15 - f16 + f17 - f18) * inv;
        const double vz = (f5 - f6 + f11 - f12 - f13 + f14 + f15 - f16 - f17 + f18) * inv;
        rho[i] = (float)r; ux[i] = (float)vx; uy[i] = (float)vy; uz[i] = (float)vz;

        /* equilibrium deviation, js/lbm.js:387-408 */
        const double A = dr - r * 1.5 * (vx * vx + vy * vy + vz * vz);
        const double r3 = 3 * r, r45 = 4.5 * r;
        const double ax = vx, ay = vy, az = vz;
        const double bxy = vx + vy, bxY = vx - vy;
        const double bxz = vx + vz, bxZ = vx - vz;
        const double byz = vy + vz, byZ = vy - vz;
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

        /* non-equilibrium parts, js/lbm.js:410-415 */
        const double n1 = f1 - e1, n2 = f2 - e2, n3 = f3 - e3, n4 = f4 - e4;
        const double n5 = f5 - e5, n6 = f6 - e6, n7 = f7 - e7, n8 = f8 - e8;
        const double n9 = f9 - e9, n10 = f10 - e10, n11 = f11 - e11, n12 = f12 - e12;
        const double n13 = f13 - e13, n14 = f14 - e14, n15 = f15 - e15, n16 = f16 - e16;
        const double n17 = f17 - e17, n18 = f18 - e18;

        /* relaxation rates, js/lbm.js:417-438 */
        double om = omega0, tauEff = tau0;
        if (les) {
          const double pxx = n1 + n2 + n7 + n8 + n9 + n10 + n11 + n12 + n13 + n14;
          const double pyy = n3 + n4 + n7 + n8 + n9 + n10 + n15 + n16 + n17 + n18;
          const double pzz = n5 + n6 + n11 + n12 + n13 + n14 + n15 + n16 + n17 + n18;
          const double pxy = n7 + n8 - n9 - n10;
          const double pxz = n11 + n12 - n13 - n14;
          const double pyz = n15 + n16 - n17 - n18;
          const double mag = sqrt(2 * (pxx * pxx + pyy * pyy + pzz * pzz +
                                       2 * (pxy * pxy + pxz * pxz + pyz * pyz)));
          tauEff = 0.5 * (tau0 + sqrt(tau0 * tau0 + SQ18 * cs2 * mag * inv));
          om = 1 / tauEff;
        }
        const double omm = trt ? 1 / (0.5 + lam / (tauEff - 0.5)) : om;

        /* collision in opposite pairs, js/lbm.js:440-460 */
        double gc[OR_Q];
        gc[0] = f0 - om * (f0 - e0);
        double sp, sm;
        sp = 0.5 * (n1 + n2); sm = 0.5 * (n1 - n2);
        gc[1] = f1 - om * sp - omm * sm; gc[2] = f2 - om * sp + omm * sm;
        sp = 0.5 * (n3 + n4); sm = 0.5 * (n3 - n4);
        gc[3] = f3 - om * sp - omm * sm; gc[4] = f4 - om * sp + omm * sm;
        sp = 0.5 * (n5 + n6); sm = 0.5 * (n5 - n6);
        gc[5] = f5 - om * sp - omm * sm; gc[6] = f6 - om * sp + omm * sm;
        sp = 0.5 * (n7 + n8); sm = 0.5 * (n7 - n8);
        gc[7] = f7 - om * sp - omm * sm; gc[8] = f8 - om * sp + omm * sm;
        sp = 0.5 * (n9 + n10); sm = 0.5 * (n9 - n10);
        gc[9] = f9 - om * sp - omm * sm; gc[10] = f10 - om * sp + omm * sm;
        sp = 0.5 * (n11 + n12); sm = 0.5 * (n11 - n12);
        gc[11] = f11 - om * sp - omm * sm; gc[12] = f12 - om * sp + omm * sm;
        sp = 0.5 * (n13 + n14); sm = 0.5 * (n13 - n14);
        gc[13] = f13 - om * sp - omm * sm; gc[14] = f14 - om * sp + omm * sm;
        sp = 0.5 * (n15 + n16); sm = 0.5 * (n15 - n16);
        gc[15] = f15 - om * sp - omm * sm; gc[16] = f16 - om * sp + omm * sm;
        sp = 0.5 * (n17 + n18); sm = 0.5 * (n17 - n18);
        gc[17] = f17 - om * sp - omm * sm; gc[18] = f18 - om * sp + omm * sm;
        const double sfr = OR_FN(sfrac_at)(L, x, y, z);
        if (sfr != 0) {
          /* partial bounce-back (no reference counterpart): g = (1-s) gc + s f_opp,
           * force += s * sum_q c_q (gc_q - f_opp(q)) */
          const double fl[OR_Q] = {f0, f1, f2, f3, f4, f5, f6, f7, f8, f9,
                                   f10, f11, f12, f13, f14, f15, f16, f17, f18};
          double px = 0, py = 0, pz = 0;
          for (int q = 0; q < OR_Q; q++) {
            const double fo = fl[OR_OPP[q]];
            const double d = gc[q] - fo;
            px += OR_EX[q] * d; py += OR_EY[q] * d; pz += OR_EZ[q] * d;
            G[q * nn + i] = (OR_T)((1 - sfr) * gc[q] + sfr * fo);
          }
          Fx += sfr * px; Fy += sfr * py; Fz += sfr * pz;
        } else {
          for (int q = 0; q < OR_Q; q++) G[q * nn + i] = (OR_T)gc[q];
        }
      }
    }
  }
  sf[0] = Fx; sf[1] = Fy; sf[2] = Fz;
}

/* js/lbm.js:473-512 (_boundaries) over z in [a,b), claiming the end planes
 * when endLo / endHi. */
static void OR_FN(boundaries)(OR_FN(lbm) * L, int a, int b, int endLo, int endHi) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long n = L->n;
  OR_T* g = OR_FN(cur_g)(L);
  const double u0 = L->p.u0;
  float *ux = L->ux, *uy = L->uy, *uz = L->uz, *rho = L->rho;
#define OR_SETEQ(idx)                                 \
  do {                                                \
    const long i_ = (idx);                            \
    OR_FN(write_eq)(L, g, i_, 1, u0, 0, 0);           \
    ux[i_] = (float)u0; uy[i_] = 0; uz[i_] = 0; rho[i_] = 1; \
  } while (0)
  for (int z = a; z < b; z++) {
    for (int y = 0; y < ny; y++) OR_SETEQ((long)nx * (y + (long)ny * z));
    for (int x = 0; x < nx; x++) {
      OR_SETEQ(x + (long)nx * ((ny - 1) + (long)ny * z));
      const long i0 = x + (long)nx * ny * z;
      if (!L->solid[i0]) OR_SETEQ(i0);
    }
  }
  if (endLo || endHi) {
    for (int y = 0; y < ny; y++) {
      for (int x = 0; x < nx; x++) {
        if (endLo) OR_SETEQ(x + (long)nx * y);
        if (endHi) OR_SETEQ(x + (long)nx * (y + (long)ny * (nz - 1)));
      }
    }
  }
#undef OR_SETEQ
  const int xo = nx - 1;
  for (int z = a; z < b; z++) {
    for (int y = 0; y < ny; y++) {
      const long i = xo + (long)nx * (y + (long)ny * z), j = i - 1;
      for (int q = 0; q < OR_Q; q++) g[q * n + i] = g[q * n + j];
      ux[i] = ux[j]; uy[i] = uy[j]; uz[i] = uz[j]; rho[i] = rho[j];
    }
  }
}

/* js/lbm.js:285-291 (step), repeated nsteps times. nthreads > 1 runs the
 * js/pool.js + js/lbmWorker.js decomposition instead: interior z split into
 * nthreads slabs (js/lbmWorker.js:177-182), each running stepSlab and its
 * share of _boundaries, one barrier per step, per-step force = the sum of
 * the slab partials in worker order (js/pool.js:108-118). */
int OR_FN(step)(OR_FN(lbm) * L, int nsteps, double* forces, int nthreads) {
  if (nsteps < 0) return -1;
  if (nthreads <= 1) {
    for (int s = 0; s < nsteps; s++) {
      double sf[3];
      OR_FN(step_slab)(L, 1, L->nz - 1, sf);
      OR_FN(boundaries)(L, 0, L->nz, 1, 1);
      L->parity ^= 1;
      L->force[0] = sf[0]; L->force[1] = sf[1]; L->force[2] = sf[2];
      L->steps++;
      if (forces) { forces[3 * s] = sf[0]; forces[3 * s + 1] = sf[1]; forces[3 * s + 2] = sf[2]; }
    }
    return 0;
  }
  const int W = nthreads;
  double* part = (double*)calloc((size_t)W * 3, sizeof(double));
  if (!part) return -2;
  for (int s = 0; s < nsteps; s++) {
#ifdef _OPENMP
#pragma omp parallel num_threads(W)
#endif
    {
#ifdef _OPENMP
      const int id = omp_get_thread_num();
      const int nw = omp_get_num_threads();
#else
      const int id = 0, nw = 1;
#endif
      const int lo = 1, hi = L->nz - 1, span = hi - lo;
      const int z0 = lo + (int)((long)span * id / nw);
      const int z1 = lo + (int)((long)span * (id + 1) / nw);
      const int bz0 = id == 0 ? 0 : z0;
      const int bz1 = id == nw - 1 ? L->nz : z1;
      double sf[3];
      OR_FN(step_slab)(L, z0, z1, sf);
      OR_FN(boundaries)(L, bz0, bz1, id == 0, id == nw - 1);
      part[3 * id] = sf[0]; part[3 * id + 1] = sf[1]; part[3 * id + 2] = sf[2];
      if (id == 0 && nw != W) {
        for (int k = nw; k < W; k++) part[3 * k] = part[3 * k + 1] = part[3 * k + 2] = 0;
      }
    }
    double fx = 0, fy = 0, fz = 0;
    for (int w = 0; w < W; w++) { fx += part[3 * w]; fy += part[3 * w + 1]; fz += part[3 * w + 2]; }
    L->parity ^= 1;
    L->steps++;
    L->force[0] = fx; L->force[1] = fy; L->force[2] = fz;
    if (forces) { forces[3 * s] = fx; forces[3 * s + 1] = fy; forces[3 * s + 2] = fz; }
  }
  free(part);
  return 0;
}

/* A bounded sample of one step for timing: stepSlab + _boundaries over the
 * interior z-range [z0,z1) only, split over nthreads slabs like the pool,
 * without flipping the buffers. Returns the cells updated. */
long OR_FN(step_sample)(OR_FN(lbm) * L, int z0, int z1, int nthreads) {
  if (z0 < 1) z0 = 1;
  if (z1 > L->nz - 1) z1 = L->nz - 1;
  if (z1 <= z0) return 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
#endif
  {
#ifdef _OPENMP
    const int id = omp_get_thread_num();
    const int nw = omp_get_num_threads();
#else
    const int id = 0, nw = 1;
#endif
    const int span = z1 - z0;
    const int a = z0 + (int)((long)span * id / nw);
    const int b = z0 + (int)((long)span * (id + 1) / nw);
    double sf[3];
    if (b > a) {
      OR_FN(step_slab)(L, a, b, sf);
      OR_FN(boundaries)(L, a, b, 0, 0);
    }
  }
  return (long)L->nx * L->ny * (z1 - z0);
}

/* Accessors (the LBM fields, js/lbm.js:74-125). */
void OR_FN(get_force)(OR_FN(lbm) * L, double out[3]) {
  out[0] = L->force[0]; out[1] = L->force[1]; out[2] = L->force[2];
}
void OR_FN(get_fields)(OR_FN(lbm) * L, float* ux, float* uy, float* uz, float* rho) {
  const size_t b = sizeof(float) * (size_t)L->n;
  if (ux) memcpy(ux, L->ux, b);
  if (uy) memcpy(uy, L->uy, b);
  if (uz) memcpy(uz, L->uz, b);
  if (rho) memcpy(rho, L->rho, b);
}
void OR_FN(get_solid)(OR_FN(lbm) * L, uint8_t* out) { memcpy(out, L->solid, (size_t)L->n); }
void OR_FN(get_near)(OR_FN(lbm) * L, uint8_t* out) { memcpy(out, L->near_, (size_t)L->n); }
/* which: 0 = f (current), 1 = g. Converted to double. */
void OR_FN(get_pop)(OR_FN(lbm) * L, int which, double* out) {
  const OR_T* b = which ? OR_FN(cur_g)(L) : OR_FN(cur_f)(L);
  for (long k = 0; k < L->n * OR_Q; k++) out[k] = (double)b[k];
}
void OR_FN(get_pop_raw)(OR_FN(lbm) * L, int which, OR_T* out) {
  memcpy(out, which ? OR_FN(cur_g)(L) : OR_FN(cur_f)(L), sizeof(OR_T) * (size_t)L->n * OR_Q);
}
void OR_FN(set_pop_raw)(OR_FN(lbm) * L, int which, const OR_T* in) {
  memcpy(which ? OR_FN(cur_g)(L) : OR_FN(cur_f)(L), in, sizeof(OR_T) * (size_t)L->n * OR_Q);
}
void OR_FN(get_body_stats)(OR_FN(lbm) * L, wt_body_stats* s) {
  s->frontal_area = L->frontal;
  s->planform_area = L->planform;
  s->solid_cells = L->solid_cells;
  s->ride_height = L->ride_height;
  s->ground = L->ground;
  s->moving_walls = L->p.moving_walls;
}
long OR_FN(get_steps)(OR_FN(lbm) * L) { return L->steps; }
int OR_FN(get_parity)(OR_FN(lbm) * L) { return L->parity; }

/* js/lbm.js:515-539 (sample). */
void OR_FN(sample)(OR_FN(lbm) * L, double x, double y, double z, double out[3]) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  if (x < 0.5 || y < 0.5 || z < 0.5 || x > nx - 1.5 || y > ny - 1.5 || z > nz - 1.5) {
    out[0] = L->p.u0; out[1] = 0; out[2] = 0;
    return;
  }
  const double xf = x - 0.5, yf = y - 0.5, zf = z - 0.5;
  const int x0 = or_toint32(xf), y0 = or_toint32(yf), z0 = or_toint32(zf);
  const double tx = xf - x0, ty = yf - y0, tz = zf - z0;
  double vx = 0, vy = 0, vz = 0;
  for (int k = 0; k < 2; k++) {
    const double wz = k ? tz : 1 - tz;
    for (int j = 0; j < 2; j++) {
      const double wy = (j ? ty : 1 - ty) * wz;
      const long base = (long)nx * ((y0 + j) + (long)ny * (z0 + k));
      const long ia = x0 + base, ib = ia + 1;
      const double wa = (1 - tx) * wy, wb = tx * wy;
      vx += (double)L->ux[ia] * wa + (double)L->ux[ib] * wb;
      vy += (double)L->uy[ia] * wa + (double)L->uy[ib] * wb;
      vz += (double)L->uz[ia] * wa + (double)L->uz[ib] * wb;
    }
  }
  out[0] = vx; out[1] = vy; out[2] = vz;
}

/* js/lbm.js:541-545 (isSolid). */
int OR_FN(is_solid)(OR_FN(lbm) * L, double x, double y, double z) {
  const int xi = or_toint32(x), yi = or_toint32(y), zi = or_toint32(z);
  if (xi < 0 || yi < 0 || zi < 0 || xi >= L->nx || yi >= L->ny || zi >= L->nz) return 0;
  return L->solid[xi + (long)L->nx * (yi + (long)L->ny * zi)] != 0;
}


/* ---- partial bounce-back adjoint (no reference counterpart) ---------------- */

static inline int OR_FN(computed)(const OR_FN(lbm) * L, int x, int y, int z) {
  return x >= 1 && x <= L->nx - 2 && y >= 1 && y <= L->ny - 2 && z >= 1 && z <= L->nz - 2 &&
         !L->solid[x + (long)L->nx * (y + (long)L->ny * z)];
}

/* Pulled populations of computed cell (x,y,z) from state F, with the
 * bounce-back and free-slip rules of step_slab (stationary walls). Sets bit q
 * of *obj for every link q that bounces off the body (SOLID_OBJ). */
static void OR_FN(adj_pull)(OR_FN(lbm) * L, const OR_T* F, int x, int y, int z, double f[OR_Q],
                            unsigned* obj) {
  const long nn = L->n;
  const long i = x + (long)L->nx * (y + (long)L->ny * z);
  const int shell = L->p.side_bc == 1 &&
                    (y == 1 || y == L->ny - 2 || z == 1 || z == L->nz - 2);
  *obj = 0;
  for (int q = 0; q < OR_Q; q++) {
    const long j = i - L->off[q];
    const uint8_t s = L->solid[j];
    if (s) {
      f[q] = (double)F[(long)OR_OPP[q] * nn + i];
      if (s == OR_SOLID_OBJ) *obj |= 1u << q;
    } else if (shell) {
      f[q] = OR_FN(gather_fs)(L, F, q, x, y, z);
    } else {
      f[q] = (double)F[L->src[q] + i];
    }
  }
}

/* Adjoint of the population stored at (q, location (x,y,z)) after a step:
 * the sum of Tn over the links that pull it in the next step -- the plain
 * consumer (x,y,z)+c_q, the location's own cell when that neighbour is solid
 * (bounce-back), and the mirrored consumer when that neighbour is a free-slip
 * side plane. Tn rows of cells that are not computed hold zeros. */
static double OR_FN(adj_gather)(const OR_FN(lbm) * L, const double* Tn, int q, int x, int y, int z,
                                int loc_computed) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long nn = L->n;
  const int px = x + OR_EX[q], py = y + OR_EY[q], pz = z + OR_EZ[q];
  double v = 0;
  if (px >= 0 && px < nx) v = Tn[(long)q * nn + px + (long)nx * (py + (long)ny * pz)];
  if (loc_computed && L->solid[px + (long)nx * (py + (long)ny * pz)])
    v += Tn[(long)OR_OPP[q] * nn + x + (long)nx * (y + (long)ny * z)];
  if (L->p.side_bc == 1) {
    const int ym = py == 0 || py == ny - 1, zm = pz == 0 || pz == nz - 1;
    if (ym || zm) {
      const int sy = ym ? py : y, sz = zm ? pz : z;
      if (!L->solid[x + (long)nx * (sy + (long)ny * sz)] && px >= 0 && px < nx) {
        const int cy = ym ? y : py, cz = zm ? z : pz;
        int qq = q;
        if (ym) qq = OR_MY[qq];
        if (zm) qq = OR_MZ[qq];
        v += Tn[(long)qq * nn + px + (long)nx * (cy + (long)ny * cz)];
      }
    }
  }
  return v;
}

/* One adjoint step: Tc from Tn over the pre-step state F, with force weight
 * wJ on component comp; accumulates dJ/ds into ds (box cells). */
static void OR_FN(adj_step)(OR_FN(lbm) * L, const OR_T* F, const double* Tn, double* Tc, double wJ,
                            int comp, double* ds) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  const long nn = L->n;
  const int* CC = comp == 0 ? OR_EX : (comp == 1 ? OR_EY : OR_EZ);
  for (int z = 0; z < nz; z++) {
    for (int y = 0; y < ny; y++) {
      for (int x = 0; x < nx; x++) {
        const long i = x + (long)nx * (y + (long)ny * z);
        if (!OR_FN(computed)(L, x, y, z)) {
          for (int q = 0; q < OR_Q; q++) Tc[q * nn + i] = 0;
          continue;
        }
        double gb[OR_Q];
        for (int q = 0; q < OR_Q; q++) {
          gb[q] = OR_FN(adj_gather)(L, Tn, q, x, y, z, 1);
          if (x == nx - 2) gb[q] += OR_FN(adj_gather)(L, Tn, q, x + 1, y, z, 0);  /* outlet copy */
        }
        or_cellfw c;
        unsigned obj;
        OR_FN(adj_pull)(L, F, x, y, z, c.f, &obj);
        or_collide_fw(&L->p, &c);
        const double s = OR_FN(sfrac_at)(L, x, y, z);
        double a[OR_Q], fb[OR_Q];
        for (int q = 0; q < OR_Q; q++) {
          a[q] = (1 - s) * gb[q] + wJ * s * CC[q];
          fb[q] = s * gb[OR_OPP[q]] + wJ * s * CC[q];
          if ((obj >> q) & 1u) fb[q] -= 2 * wJ * CC[q];
        }
        if (L->sfrac) {
          const int* b = L->sbox;
          if (x >= b[0] && x < b[3] && y >= b[1] && y < b[4] && z >= b[2] && z < b[5]) {
            /* dJ/ds = sum_q gb_q (f_opp(q) - gc_q) + wJ sum_q c_q (gc_q - f_opp(q)) */
            double g1 = 0, g2 = 0;
            for (int q = 0; q < OR_Q; q++) {
              const double d = c.f[OR_OPP[q]] - c.gc[q];
              g1 += gb[q] * d;
              g2 -= CC[q] * d;
            }
            ds[(x - b[0]) + (long)(b[3] - b[0]) * ((y - b[1]) + (long)(b[4] - b[1]) * (z - b[2]))] +=
                g1 + wJ * g2;
          }
        }
        or_collide_vjp(&L->p, &c, a, fb);
        for (int q = 0; q < OR_Q; q++) Tc[q * nn + i] = fb[q];
      }
    }
  }
}

/* J = mean of force component comp over the last `window` of nsteps steps
 * from the current state, and dJ/ds on the solid-fraction box (dJds, box
 * cells, x fastest). Runs the forward (the lattice ends nsteps later, as
 * after step()) keeping every state, then the adjoint backwards. Stationary
 * walls only. Returns 0, or <0 on bad arguments / allocation failure. */
int OR_FN(adjoint)(OR_FN(lbm) * L, int nsteps, int window, int comp, double* J, double* dJds) {
  if (nsteps < 1 || window < 1 || window > nsteps || comp < 0 || comp > 2 || !L->sfrac) return -1;
  if (L->p.moving_walls) return -1;
  const long nn = L->n;
  const size_t pop = (size_t)nn * OR_Q;
  OR_T* states = (OR_T*)malloc(sizeof(OR_T) * pop * (size_t)nsteps);
  double* forces = (double*)malloc(sizeof(double) * 3 * (size_t)nsteps);
  double* Tn = (double*)calloc(pop, sizeof(double));
  double* Tc = (double*)calloc(pop, sizeof(double));
  if (!states || !forces || !Tn || !Tc) {
    free(states); free(forces); free(Tn); free(Tc);
    return -2;
  }
  for (int t = 0; t < nsteps; t++) {
    memcpy(states + pop * (size_t)t, OR_FN(cur_f)(L), sizeof(OR_T) * pop);
    OR_FN(step)(L, 1, forces + 3 * (size_t)t, 1);
  }
  double acc = 0;
  for (int t = nsteps - window; t < nsteps; t++) acc += forces[3 * (size_t)t + comp];
  *J = acc / window;
  const int* b = L->sbox;
  const long m = (long)(b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]);
  for (long k = 0; k < m; k++) dJds[k] = 0;
  const double w = 1.0 / window;
  for (int t = nsteps - 1; t >= 0; t--) {
    const double wJ = t >= nsteps - window ? w : 0;
    OR_FN(adj_step)(L, states + pop * (size_t)t, Tn, Tc, wJ, comp, dJds);
    double* tmp = Tn; Tn = Tc; Tc = tmp;
  }
  free(states); free(forces); free(Tn); free(Tc);
  return 0;
}

#undef OR_T
#undef OR_FN
