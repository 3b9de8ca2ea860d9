// wt_view.cu — the arithmetic behind the reference's flow visualisation, on
// the device, writing plain buffers (no graphics API: the caller draws).
//
//   k_slice    the scalar of one lattice plane that js/main.js:925-968 colours:
//              |u| / u0, the pressure coefficient of the 5-point averaged
//              density, or the in-plane vorticity / u0; NaN on solid cells
//   k_advect   one smoke-particle step of js/main.js:691-709: trilinear
//              velocity (js/lbm.js:515-539), x += u k, the expiry test of
//              the domain margins and solid cells (js/lbm.js:541-545), and
//              |u| / u0 for the particle's colour
//
// Compiled without multiply-add contraction, in float64 like the reference.
#include <math.h>

#include <cmath>

#include "wt_internal.h"

namespace {

// ECMAScript ToInt32 of a double (js `x | 0`).
__device__ __forceinline__ int32_t view_toint32(double v) {
  if (!isfinite(v)) return 0;
  if (v > -2147483649.0 && v < 2147483648.0) return (int32_t)v;
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}

struct ViewFields {
  const float *ux, *uy, *uz, *rho;
  const uint8_t* flags;
  int nx, ny, nz;
  double u0;
};

// js/lbm.js:515-539: trilinear velocity at cell-centred coordinates,
// (u0, 0, 0) outside the half-cell margin.
__device__ void sample_vel(const ViewFields& f, double x, double y, double z, double v[3]) {
  if (x < 0.5 || y < 0.5 || z < 0.5 || x > f.nx - 1.5 || y > f.ny - 1.5 || z > f.nz - 1.5) {
    v[0] = f.u0; v[1] = 0; v[2] = 0;
    return;
  }
  const double xf = x - 0.5, yf = y - 0.5, zf = z - 0.5;
  const int x0 = view_toint32(xf), y0 = view_toint32(yf), z0 = view_toint32(zf);
  const double tx = xf - x0, ty = yf - y0, tz = zf - z0;
  double vx = 0, vy = 0, vz = 0;
  for (int k = 0; k < 2; k++) {
    const double wz = k ? tz : 1 - tz;
    for (int j = 0; j < 2; j++) {
      const double wy = (j ? ty : 1 - ty) * wz;
      const long long base = (long long)f.nx * ((y0 + j) + (long long)f.ny * (z0 + k));
      const long long ia = x0 + base, ib = ia + 1;
      const double wa = (1 - tx) * wy, wb = tx * wy;
      vx += (double)f.ux[ia] * wa + (double)f.ux[ib] * wb;
      vy += (double)f.uy[ia] * wa + (double)f.uy[ib] * wb;
      vz += (double)f.uz[ia] * wa + (double)f.uz[ib] * wb;
    }
  }
  v[0] = vx; v[1] = vy; v[2] = vz;
}

// js/lbm.js:541-545
__device__ bool is_solid_at(const ViewFields& f, double x, double y, double z) {
  const int xi = view_toint32(x), yi = view_toint32(y), zi = view_toint32(z);
  if (xi < 0 || yi < 0 || zi < 0 || xi >= f.nx || yi >= f.ny || zi >= f.nz) return false;
  return (f.flags[xi + (long long)f.nx * (yi + (long long)f.ny * zi)] & wt::FLAG_SOLID_MASK) != 0;
}

__global__ void k_slice(ViewFields f, int plane, int k, int field, float* out) {
  const int nx = f.nx, h = plane == 0 ? f.ny : f.nz;
  const long long cells = (long long)nx * h;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cells;
       c += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(c % nx), b = (int)(c / nx);
    auto at = [&](int aa, int bb) -> long long {
      return plane == 0 ? aa + (long long)nx * (bb + (long long)f.ny * k)
                        : aa + (long long)nx * (k + (long long)f.ny * bb);
    };
    const long long i = at(a, b);
    if (f.flags[i] & wt::FLAG_SOLID_MASK) {
      out[c] = __int_as_float(0x7fc00000);   // NaN marks a solid cell
      continue;
    }
    const long long ip = a < nx - 1 ? at(a + 1, b) : i, im = a > 0 ? at(a - 1, b) : i;
    const long long jp = b < h - 1 ? at(a, b + 1) : i, jm = b > 0 ? at(a, b - 1) : i;
    double t;
    if (field == 0) {
      const double x = f.ux[i], y = f.uy[i], z = f.uz[i];
      t = sqrt(x * x + y * y + z * z) / f.u0;
    } else if (field == 1) {
      const double r = ((double)f.rho[i] * 2 + (double)f.rho[ip] + (double)f.rho[im] +
                        (double)f.rho[jp] + (double)f.rho[jm]) / 6;
      t = ((r - 1) / 3) / (0.5 * f.u0 * f.u0);
    } else {
      double w;
      if (plane == 0)
        w = ((double)f.uy[ip] - (double)f.uy[im]) * 0.5 - ((double)f.ux[jp] - (double)f.ux[jm]) * 0.5;
      else
        w = ((double)f.ux[jp] - (double)f.ux[jm]) * 0.5 - ((double)f.uz[ip] - (double)f.uz[im]) * 0.5;
      t = w / f.u0;
    }
    out[c] = (float)t;
  }
}

__global__ void k_advect(ViewFields f, double* xyz, int n, double kstep, uint8_t* expired,
                         float* speed) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    double x = xyz[3 * p], y = xyz[3 * p + 1], z = xyz[3 * p + 2];
    double v[3];
    sample_vel(f, x, y, z, v);
    x += v[0] * kstep;
    y += v[1] * kstep;
    z += v[2] * kstep;
    const bool out = x > f.nx - 2 || x < 0.5 || y < 0.8 || y > f.ny - 1.2 || z < 0.8 ||
                     z > f.nz - 1.2 || is_solid_at(f, x, y, z);
    xyz[3 * p] = x; xyz[3 * p + 1] = y; xyz[3 * p + 2] = z;
    if (expired) expired[p] = out ? 1 : 0;
    if (speed) speed[p] = (float)(sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / f.u0);
  }
}

ViewFields view_of(const wt_lattice* h) {
  return ViewFields{h->ux, h->uy, h->uz, h->rho, h->flags, h->nx, h->ny, h->nz, h->p.u0};
}

int view_fail(wt_lattice* h, int code, const char* msg) {
  h->err = msg;
  return code;
}

}  // namespace

extern "C" {

int wt_slice(wt_lattice* h, int plane, int k, int field, float* out, size_t len) {
  if (!h) return WT_ERR_ARG;
  if (plane != 0 && plane != 1) return view_fail(h, WT_ERR_ARG, "plane must be 0 (xy) or 1 (xz)");
  if (field < 0 || field > 2) return view_fail(h, WT_ERR_ARG, "field must be 0, 1 or 2");
  const int depth = plane == 0 ? h->nz : h->ny;
  if (k < 0 || k >= depth) return view_fail(h, WT_ERR_ARG, "plane index out of range");
  const size_t cells = (size_t)h->nx * (plane == 0 ? h->ny : h->nz);
  if (!out || len != cells) return view_fail(h, WT_ERR_ARG, "out must hold nx * (ny or nz) floats");
  float* d = nullptr;
  if (cudaMalloc(&d, sizeof(float) * cells) != cudaSuccess)
    return view_fail(h, WT_ERR_OOM, "slice buffer");
  k_slice<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(view_of(h), plane, k, field, d);
  h->launches++;
  cudaError_t e = cudaMemcpyAsync(out, d, sizeof(float) * cells, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return view_fail(h, WT_ERR_CUDA, "slice failed");
  return WT_OK;
}

int wt_advect(wt_lattice* h, double* xyz, int n, double kstep, uint8_t* expired, float* speed) {
  if (!h) return WT_ERR_ARG;
  if (n < 0 || (n > 0 && !xyz) || !std::isfinite(kstep))
    return view_fail(h, WT_ERR_ARG, "bad particles or step");
  if (n == 0) return WT_OK;
  unsigned char* d = nullptr;
  const size_t bytes = sizeof(double) * 3 * (size_t)n + (size_t)n + sizeof(float) * (size_t)n + 16;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return view_fail(h, WT_ERR_OOM, "particle buffer");
  double* dxyz = (double*)d;
  float* dsp = (float*)(d + sizeof(double) * 3 * (size_t)n);
  uint8_t* dexp = (uint8_t*)(dsp + n);
  cudaError_t e = cudaMemcpyAsync(dxyz, xyz, sizeof(double) * 3 * (size_t)n,
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    k_advect<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(view_of(h), dxyz, n, kstep, dexp,
                                                               dsp);
    h->launches++;
    e = cudaMemcpyAsync(xyz, dxyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost,
                        h->stream);
  }
  if (e == cudaSuccess && expired)
    e = cudaMemcpyAsync(expired, dexp, (size_t)n, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && speed)
    e = cudaMemcpyAsync(speed, dsp, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return view_fail(h, WT_ERR_CUDA, "advect failed");
  return WT_OK;
}

}  // extern "C"
