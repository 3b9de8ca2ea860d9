// wt_kernels_exact.cu — every kernel whose float64 results must match the
// reference's IEEE double arithmetic bit for bit: the exact-order step, the
// equilibrium initialisers, the voxelize passes with the body-space lookup,
// and the trilinear sampler. This translation unit is compiled with
// --fmad=false so that no multiply-add is contracted; divisions and square
// roots are the IEEE round-to-nearest ones.
#include <math.h>

#include "wt_internal.h"
#include "wt_pbb.cuh"

namespace wt {

void launch_step_f32_exact(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step<float, true, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step<float, true, int>, grid, dim3(STEP_BX), s, a);
}

void launch_step_f64_exact(const StepArgs<double>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step<double, true, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step<double, true, int>, grid, dim3(STEP_BX), s, a);
}

void launch_pbb_f32_exact(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step_pbb<float, true, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step_pbb<float, true, int>, grid, dim3(STEP_BX), s, a);
}

void launch_pbb_f64_exact(const StepArgs<double>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) launch_pdl(k_step_pbb<double, true, long long>, grid, dim3(STEP_BX), s, a);
  else launch_pdl(k_step_pbb<double, true, int>, grid, dim3(STEP_BX), s, a);
}

void launch_adj_f32x(const StepArgs<float>& a, const double* Tn, double* Tc, double* ds,
                     double wJ, int comp, cudaStream_t s) {
  launch_adjoint<float, double>(a, Tn, Tc, ds, wJ, comp, s);
}

void launch_adj_f64(const StepArgs<double>& a, const double* Tn, double* Tc, double* ds,
                    double wJ, int comp, cudaStream_t s) {
  launch_adjoint<double, double>(a, Tn, Tc, ds, wJ, comp, s);
}

cudaError_t preload_exact_step_kernels() {
  cudaFuncAttributes fa;
  const void* fns[] = {(const void*)k_step<float, true, int>, (const void*)k_step<float, true, long long>,
                       (const void*)k_step<double, true, int>,
                       (const void*)k_step<double, true, long long>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// ---- helpers -----------------------------------------------------------------

// ECMAScript ToInt32: truncation toward zero, then wrap modulo 2^32.
__device__ __forceinline__ int js_toint32(double v) {
  if (v > -2147483649.0 && v < 2147483648.0) return (int)v;  // trunc
  if (!isfinite(v)) return 0;
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int)(unsigned)m;
}

// splitmix64 draw k of stream `seed`, as a uniform double in [0,1).
__device__ __forceinline__ double uniform_draw(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// js/lbm.js:155-162 (_writeEq): deviation equilibrium into arr at cell i.
template <class S>
__device__ __forceinline__ void write_eq(S* arr, long long n, long long i, double r, double vx,
                                         double vy, double vz) {
  const double usq = 1.5 * (vx * vx + vy * vy + vz * vz);
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const double cu = 3 * ((double)ex(q) * vx + (double)ey(q) * vy + (double)ez(q) * vz);
    arr[q * n + i] = Store<S>::from_d(wq(q) * ((r - 1) + r * (cu + 0.5 * cu * cu - usq)));
  }
}

struct Fields {
  float* ux;
  float* uy;
  float* uz;
  float* rho;
};

__device__ __forceinline__ long long gtid() {
  return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

constexpr int AUX_T = 256;

inline unsigned aux_blocks(long long count) {
  long long b = (count + AUX_T - 1) / AUX_T;
  if (b > 148LL * 64) b = 148LL * 64;
  return (unsigned)(b < 1 ? 1 : b);
}

// ---- reset / seeded initial state (js/lbm.js:164-174) -------------------------------
template <class S>
__global__ void k_init(S* f, S* g, const uint8_t* flags, Fields fl, long long n, double u0,
                       int mode, uint64_t seed, double amp) {
  for (long long i = gtid(); i < n; i += gstride()) {
    double vx = 0, vy = 0, vz = 0;
    if (!(flags[i] & FLAG_SOLID_MASK)) {
      if (mode == 0) {
        vx = u0;
      } else {
        vx = u0 + amp * (2 * uniform_draw(seed, 3 * (uint64_t)i) - 1);
        vy = amp * (2 * uniform_draw(seed, 3 * (uint64_t)i + 1) - 1);
        vz = amp * (2 * uniform_draw(seed, 3 * (uint64_t)i + 2) - 1);
      }
    }
    write_eq(f, n, i, 1, vx, vy, vz);
    write_eq(g, n, i, 1, vx, vy, vz);
    fl.ux[i] = __double2float_rn(vx);
    fl.uy[i] = __double2float_rn(vy);
    fl.uz[i] = __double2float_rn(vz);
    fl.rho[i] = 1.0f;
  }
}

// ---- voxelize (js/lbm.js:191-266) ----------------------------------------------------
struct Walls {
  float* uwx;
  float* uwy;
  float* uwz;
};

// js/lbm.js:176-180 (_seedCell).
template <class S>
__device__ __forceinline__ void seed_cell(S* f, S* g, Fields fl, long long n, long long i,
                                          double u0) {
  write_eq(f, n, i, 1, u0, 0, 0);
  write_eq(g, n, i, 1, u0, 0, 0);
  fl.ux[i] = __double2float_rn(u0);
  fl.uy[i] = 0.0f;
  fl.uz[i] = 0.0f;
  fl.rho[i] = 1.0f;
}

// js/lbm.js:197-202: the previous body's cells back to fluid at u0.
template <class S>
__global__ void k_clear_obj(S* f, S* g, uint8_t* flags, Fields fl, Walls w, long long n,
                            double u0) {
  for (long long i = gtid(); i < n; i += gstride()) {
    if ((flags[i] & FLAG_SOLID_MASK) == WT_SOLID_OBJ) {
      flags[i] = WT_FLUID;
      seed_cell(f, g, fl, n, i, u0);
      w.uwx[i] = 0.0f; w.uwy[i] = 0.0f; w.uwz[i] = 0.0f;
    }
  }
}

// js/lbm.js:204-214: the road row y = 0.
template <class S>
__global__ void k_floor(S* f, S* g, uint8_t* flags, Fields fl, Walls w, int nx, int ny, int nz,
                        long long n, double u0, int gy, double rv) {
  const long long cnt = (long long)nx * nz;
  for (long long k = gtid(); k < cnt; k += gstride()) {
    const int x = (int)(k % nx), z = (int)(k / nx);
    const long long i = x + (long long)nx * ny * z;
    if ((flags[i] & FLAG_SOLID_MASK) != gy) {
      flags[i] = (uint8_t)((flags[i] & ~FLAG_SOLID_MASK) | gy);
      if (gy == WT_FLUID) seed_cell(f, g, fl, n, i, u0);
    }
    w.uwx[i] = gy == WT_SOLID_WALL ? __double2float_rn(rv) : 0.0f;
    w.uwy[i] = 0.0f;
    w.uwz[i] = 0.0f;
  }
}

struct BoxStats {
  uint8_t* col;
  uint8_t* plan;
  int* low;
  int* counters;
};

// The voxel-backed Body.makeTest() closure, js/shapes.js:369-388.
struct GridLookup {
  const uint8_t* grid;
  int gnx, gny, gnz;
  double gx0, gy0, gz0, gi;
  double M[9];
  double P[3];
  double inv;
};

__device__ __forceinline__ bool grid_inside(const GridLookup& L, double X, double Y, double Z) {
  const double dx = X - L.P[0], dy = Y - L.P[1], dz = Z - L.P[2];
  const double lx = (L.M[0] * dx + L.M[3] * dy + L.M[6] * dz) * L.inv;
  const double ly = (L.M[1] * dx + L.M[4] * dy + L.M[7] * dz) * L.inv;
  const double lz = (L.M[2] * dx + L.M[5] * dy + L.M[8] * dz) * L.inv;
  const int a = js_toint32((lx - L.gx0) * L.gi);
  if (a < 0 || a >= L.gnx) return false;
  const int b = js_toint32((ly - L.gy0) * L.gi);
  if (b < 0 || b >= L.gny) return false;
  const int c = js_toint32((lz - L.gz0) * L.gi);
  if (c < 0 || c >= L.gnz) return false;
  return L.grid[a + (long long)L.gnx * (b + (long long)L.gny * c)] != 0;
}

// js/lbm.js:225-246: mark the body inside the scan range and gather the
// frontal / planform / lowest-cell projections. FROM_GRID evaluates the
// lookup on the device; otherwise `mask` holds the host's inside() results.
template <class S, bool FROM_GRID>
__global__ void k_box(S* f, uint8_t* flags, Fields fl, Walls w, BoxStats st, int nx, int ny,
                      long long n, int x0, int y0, int z0, int ex_, int ey_, int ez_,
                      const uint8_t* mask, const uint8_t* wall_set, const double* wall_vel,
                      GridLookup L) {
  const long long cnt = (long long)ex_ * ey_ * ez_;
  for (long long m = gtid(); m < cnt; m += gstride()) {
    const int x = x0 + (int)(m % ex_);
    const int y = y0 + (int)((m / ex_) % ey_);
    const int z = z0 + (int)(m / ((long long)ex_ * ey_));
    bool hit;
    if constexpr (FROM_GRID) {
      hit = grid_inside(L, x + 0.5, y + 0.5, z + 0.5);
    } else {
      hit = mask[m] != 0;
    }
    if (!hit) continue;
    const long long i = x + (long long)nx * (y + (long long)ny * z);
    flags[i] = (uint8_t)((flags[i] & ~FLAG_SOLID_MASK) | WT_SOLID_OBJ);
    write_eq(f, n, i, 1, 0, 0, 0);
    fl.ux[i] = 0.0f; fl.uy[i] = 0.0f; fl.uz[i] = 0.0f; fl.rho[i] = 1.0f;
    w.uwx[i] = 0.0f; w.uwy[i] = 0.0f; w.uwz[i] = 0.0f;
    if (!FROM_GRID && wall_set && wall_set[m]) {
      w.uwx[i] = __double2float_rn(wall_vel[3 * m]);
      w.uwy[i] = __double2float_rn(wall_vel[3 * m + 1]);
      w.uwz[i] = __double2float_rn(wall_vel[3 * m + 2]);
      st.counters[1] = 1;
    }
    st.col[y + (long long)ny * z] = 1;
    const long long pk = x + (long long)nx * z;
    st.plan[pk] = 1;
    atomicMin(&st.low[pk], y);
    atomicAdd(&st.counters[0], 1);
  }
}

// js/lbm.js:268-282 (_rebuildNear): interior fluid cells with any solid
// neighbour (object or wall) along the 18 moving directions.
// Also records, per near-wall cell, which of its 18 neighbours are solid
// (bits 0-18) and which of those belong to the body (bits 32-50), so the step
// can apply every bounce-back link of a cell after a single 8-byte load.
__global__ void k_near(uint8_t* flags, unsigned long long* nmask, int nx, int ny, int nz,
                       long long n) {
  const long long nxy = (long long)nx * ny;
  for (long long i = gtid(); i < n; i += gstride()) {
    const int x = (int)(i % nx);
    const int y = (int)((i / nx) % ny);
    const int z = (int)(i / nxy);
    const uint8_t v = flags[i];
    unsigned long long m = 0;
    if (x >= 1 && x < nx - 1 && y >= 1 && y < ny - 1 && z >= 1 && z < nz - 1 &&
        !(v & FLAG_SOLID_MASK)) {
#pragma unroll
      for (int q = 1; q < Q; q++) {
        const long long j = i - (ex(q) + (long long)ey(q) * nx + (long long)ez(q) * nxy);
        const int sj = flags[j] & FLAG_SOLID_MASK;
        if (sj) m |= 1ULL << q;
        if (sj == WT_SOLID_OBJ) m |= 1ULL << (32 + q);
      }
    }
    nmask[i] = m;
    const uint8_t nv = (uint8_t)((v & FLAG_SOLID_MASK) | (m ? FLAG_NEAR : 0));
    if (nv != v) flags[i] = nv;
  }
}

// ---- population format conversion ----------------------------------------------------
template <class S, class D>
__global__ void k_convert(const S* src, D* dst, long long count) {
  for (long long k = gtid(); k < count; k += gstride()) {
    dst[k] = (D)Store<S>::load_d(src[k]);
  }
}

template <class D, class S>
__global__ void k_convert_in(const D* src, S* dst, long long count) {
  for (long long k = gtid(); k < count; k += gstride()) {
    dst[k] = Store<S>::from_d((double)src[k]);
  }
}

// ---- js/lbm.js:515-539 (sample) ------------------------------------------------------
__global__ void k_sample(const float* ux, const float* uy, const float* uz, int nx, int ny,
                         int nz, double u0, const double* xyz, int npts, double* out) {
  for (long long p = gtid(); p < npts; p += gstride()) {
    const double x = xyz[3 * p], y = xyz[3 * p + 1], z = xyz[3 * p + 2];
    if (x < 0.5 || y < 0.5 || z < 0.5 || x > nx - 1.5 || y > ny - 1.5 || z > nz - 1.5) {
      out[3 * p] = u0; out[3 * p + 1] = 0; out[3 * p + 2] = 0;
      continue;
    }
    const double xf = x - 0.5, yf = y - 0.5, zf = z - 0.5;
    const int x0 = js_toint32(xf), y0 = js_toint32(yf), z0 = js_toint32(zf);
    const double tx = xf - x0, ty = yf - y0, tz = zf - z0;
    double vx = 0, vy = 0, vz = 0;
    for (int k = 0; k < 2; k++) {
      const double wz = k ? tz : 1 - tz;
      for (int j = 0; j < 2; j++) {
        const double wy = (j ? ty : 1 - ty) * wz;
        const long long base = (long long)nx * ((y0 + j) + (long long)ny * (z0 + k));
        const long long ia = x0 + base, ib = ia + 1;
        const double wa = (1 - tx) * wy, wb = tx * wy;
        vx += (double)ux[ia] * wa + (double)ux[ib] * wb;
        vy += (double)uy[ia] * wa + (double)uy[ib] * wb;
        vz += (double)uz[ia] * wa + (double)uz[ib] * wb;
      }
    }
    out[3 * p] = vx; out[3 * p + 1] = vy; out[3 * p + 2] = vz;
  }
}

// ---- launchers -----------------------------------------------------------------------
static Fields fields_of(wt_lattice* h) { return Fields{h->ux, h->uy, h->uz, h->rho}; }
static Walls walls_of(wt_lattice* h) { return Walls{h->uwx, h->uwy, h->uwz}; }

template <class S>
static S* cur_f(wt_lattice* h) { return (S*)h->buf[h->parity]; }
template <class S>
static S* cur_g(wt_lattice* h) { return (S*)h->buf[h->parity ^ 1]; }

#define WT_DISPATCH(h, CALL)                               \
  switch ((h)->storage) {                                  \
    case WT_STORE_F32: { using S = float; CALL; } break;   \
    case WT_STORE_F16DEV: { using S = __half; CALL; } break; \
    default: { using S = double; CALL; } break;            \
  }

void launch_init(wt_lattice* h, int mode, uint64_t seed, double amp) {
  WT_DISPATCH(h, (k_init<S><<<aux_blocks(h->n), AUX_T, 0, h->stream>>>(
                     cur_f<S>(h), cur_g<S>(h), h->flags, fields_of(h), h->n, h->p.u0, mode, seed,
                     amp)));
  h->launches++;
}

void launch_clear_obj(wt_lattice* h) {
  WT_DISPATCH(h, (k_clear_obj<S><<<aux_blocks(h->n), AUX_T, 0, h->stream>>>(
                     cur_f<S>(h), cur_g<S>(h), h->flags, fields_of(h), walls_of(h), h->n,
                     h->p.u0)));
  h->launches++;
}

void launch_floor(wt_lattice* h, int ground, double road_vel) {
  const int gy = ground ? WT_SOLID_WALL : WT_FLUID;
  WT_DISPATCH(h, (k_floor<S><<<aux_blocks((long long)h->nx * h->nz), AUX_T, 0, h->stream>>>(
                     cur_f<S>(h), cur_g<S>(h), h->flags, fields_of(h), walls_of(h), h->nx, h->ny,
                     h->nz, h->n, h->p.u0, gy, road_vel)));
  h->launches++;
}

void launch_box_mask(wt_lattice* h, const int rg[6], const uint8_t* mask_dev,
                     const uint8_t* wall_set_dev, const double* wall_vel_dev) {
  const int ex_ = rg[1] - rg[0] + 1, ey_ = rg[3] - rg[2] + 1, ez_ = rg[5] - rg[4] + 1;
  if (ex_ <= 0 || ey_ <= 0 || ez_ <= 0) return;
  BoxStats st{h->col, h->plan, h->low, h->counters};
  GridLookup L{};
  WT_DISPATCH(h, (k_box<S, false><<<aux_blocks((long long)ex_ * ey_ * ez_), AUX_T, 0,
                                     h->stream>>>(cur_f<S>(h), h->flags, fields_of(h),
                                                  walls_of(h), st, h->nx, h->ny, h->n, rg[0],
                                                  rg[2], rg[4], ex_, ey_, ez_, mask_dev,
                                                  wall_set_dev, wall_vel_dev, L)));
  h->launches++;
}

void launch_box_grid(wt_lattice* h, const int rg[6], const uint8_t* grid_dev, int gnx, int gny,
                     int gnz, const double gmin[3], double ginv, const double M[9],
                     const double P[3], double scale) {
  const int ex_ = rg[1] - rg[0] + 1, ey_ = rg[3] - rg[2] + 1, ez_ = rg[5] - rg[4] + 1;
  if (ex_ <= 0 || ey_ <= 0 || ez_ <= 0) return;
  BoxStats st{h->col, h->plan, h->low, h->counters};
  GridLookup L{};
  L.grid = grid_dev;
  L.gnx = gnx; L.gny = gny; L.gnz = gnz;
  L.gx0 = gmin[0]; L.gy0 = gmin[1]; L.gz0 = gmin[2]; L.gi = ginv;
  for (int k = 0; k < 9; k++) L.M[k] = M[k];
  for (int k = 0; k < 3; k++) L.P[k] = P[k];
  L.inv = 1 / scale;  // js/shapes.js:366: inv = 1 / this.scale (host double division)
  WT_DISPATCH(h, (k_box<S, true><<<aux_blocks((long long)ex_ * ey_ * ez_), AUX_T, 0,
                                    h->stream>>>(cur_f<S>(h), h->flags, fields_of(h), walls_of(h),
                                                 st, h->nx, h->ny, h->n, rg[0], rg[2], rg[4], ex_,
                                                 ey_, ez_, nullptr, nullptr, nullptr, L)));
  h->launches++;
}

void launch_near(wt_lattice* h) {
  k_near<<<aux_blocks(h->n), AUX_T, 0, h->stream>>>(h->flags, h->nmask, h->nx, h->ny, h->nz,
                                                     h->n);
  h->launches++;
}

void launch_convert(const void* src, int storage, void* dst, int dtype, long long count,
                    cudaStream_t s) {
  const unsigned b = aux_blocks(count);
  if (storage == WT_STORE_F32) {
    if (dtype == WT_STORE_F64) k_convert<float, double><<<b, AUX_T, 0, s>>>((const float*)src, (double*)dst, count);
    else k_convert<float, float><<<b, AUX_T, 0, s>>>((const float*)src, (float*)dst, count);
  } else if (storage == WT_STORE_F16DEV) {
    if (dtype == WT_STORE_F64) k_convert<__half, double><<<b, AUX_T, 0, s>>>((const __half*)src, (double*)dst, count);
    else k_convert<__half, float><<<b, AUX_T, 0, s>>>((const __half*)src, (float*)dst, count);
  } else {
    if (dtype == WT_STORE_F64) k_convert<double, double><<<b, AUX_T, 0, s>>>((const double*)src, (double*)dst, count);
    else k_convert<double, float><<<b, AUX_T, 0, s>>>((const double*)src, (float*)dst, count);
  }
}

void launch_convert_in(const void* src, int dtype, void* dst, int storage, long long count,
                       cudaStream_t s) {
  const unsigned b = aux_blocks(count);
  if (storage == WT_STORE_F32) {
    if (dtype == WT_STORE_F64) k_convert_in<double, float><<<b, AUX_T, 0, s>>>((const double*)src, (float*)dst, count);
    else k_convert_in<float, float><<<b, AUX_T, 0, s>>>((const float*)src, (float*)dst, count);
  } else if (storage == WT_STORE_F16DEV) {
    if (dtype == WT_STORE_F64) k_convert_in<double, __half><<<b, AUX_T, 0, s>>>((const double*)src, (__half*)dst, count);
    else k_convert_in<float, __half><<<b, AUX_T, 0, s>>>((const float*)src, (__half*)dst, count);
  } else {
    if (dtype == WT_STORE_F64) k_convert_in<double, double><<<b, AUX_T, 0, s>>>((const double*)src, (double*)dst, count);
    else k_convert_in<float, double><<<b, AUX_T, 0, s>>>((const float*)src, (double*)dst, count);
  }
}

void launch_sample(wt_lattice* h, const double* xyz_dev, int npts, double* out_dev) {
  k_sample<<<aux_blocks(npts), AUX_T, 0, h->stream>>>(h->ux, h->uy, h->uz, h->nx, h->ny, h->nz,
                                                       h->p.u0, xyz_dev, npts, out_dev);
  h->launches++;
}

void eq_u0_table(double u0, double out[19]) {
  const double r = 1, vx = u0, vy = 0, vz = 0;
  const double usq = 1.5 * (vx * vx + vy * vy + vz * vz);
  for (int q = 0; q < Q; q++) {
    const double cu = 3 * ((double)ex(q) * vx + (double)ey(q) * vy + (double)ez(q) * vz);
    out[q] = wq(q) * ((r - 1) + r * (cu + 0.5 * cu * cu - usq));
  }
}

}  // namespace wt
