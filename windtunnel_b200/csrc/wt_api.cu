// wt_api.cu — the extern "C" entry points of libwt.so (include/wt.h):
// handle lifetime, parameters, voxelize, the batched step and the getters.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "wt_internal.h"

namespace {

thread_local std::string g_create_error;

constexpr int kChunk = 32;         // steps whose force partials are reduced together
constexpr uint32_t kStateMagic = 0x57545354u;  // "WTST"

int fail(wt_lattice* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(wt_lattice* h, cudaError_t e, const char* what) {
  return fail(h, WT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define WT_CUDA(h, call)                                      \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call);  \
  } while (0)

size_t elem_size(int storage) {
  return storage == WT_STORE_F32 ? 4 : (storage == WT_STORE_F16DEV ? 2 : 8);
}

// ECMAScript ToInt32 on the host (the `| 0` of js/lbm.js:542).
int js_toint32(double v) {
  if (!std::isfinite(v)) return 0;
  if (v > -2147483649.0 && v < 2147483648.0) return (int)v;
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int)(uint32_t)m;
}

int clamp_int(double v) {
  if (v > 2147483647.0) return 2147483647;
  if (v < -2147483647.0) return -2147483647;
  return (int)v;
}

void voxel_range(int nx, int ny, int nz, const double box[6], int rg[6]) {
  rg[0] = clamp_int(fmax(1, floor(box[0])));
  rg[1] = clamp_int(fmin(nx - 2, ceil(box[3])));
  rg[2] = clamp_int(fmax(1, floor(box[1])));
  rg[3] = clamp_int(fmin(ny - 2, ceil(box[4])));
  rg[4] = clamp_int(fmax(1, floor(box[2])));
  rg[5] = clamp_int(fmin(nz - 2, ceil(box[5])));
}

long long range_cells(const int rg[6]) {
  const long long ex = rg[1] >= rg[0] ? rg[1] - rg[0] + 1 : 0;
  const long long ey = rg[3] >= rg[2] ? rg[3] - rg[2] + 1 : 0;
  const long long ez = rg[5] >= rg[4] ? rg[5] - rg[4] + 1 : 0;
  return ex * ey * ez;
}

void free_all(wt_lattice* h) {
  void* dev[] = {h->buf[0], h->buf[1], h->flags, h->nmask, h->ux, h->uy, h->uz, h->rho, h->uwx, h->uwy,
                 h->uwz, h->part, h->wslot, h->forces_dev, h->err_dev, h->col, h->plan, h->low,
                 h->counters};
  for (void* p : dev)
    if (p) cudaFree(p);
  if (h->forces_host) cudaFreeHost(h->forces_host);
  if (h->err_host) cudaFreeHost(h->err_host);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->adj_pool) cudaFree(h->adj_pool);
  h->adj_pool = nullptr;
}

int check_params(const wt_params* p) {
  if (!std::isfinite(p->u0) || !std::isfinite(p->tau) || !(p->tau > 0.5)) return WT_ERR_ARG;
  if (!std::isfinite(p->csm) || !std::isfinite(p->lambda)) return WT_ERR_ARG;
  if (p->trt && !(p->lambda > 0)) return WT_ERR_ARG;
  if (p->side_bc != WT_SIDE_EQ && p->side_bc != WT_SIDE_FREESLIP) return WT_ERR_ARG;
  if (p->math != WT_MATH_FAST && p->math != WT_MATH_EXACT) return WT_ERR_ARG;
  if (p->kernel != WT_KERNEL_AUTO && p->kernel != WT_KERNEL_DIRECT && p->kernel != WT_KERNEL_LEAN &&
      p->kernel != WT_KERNEL_PAIR)
    return WT_ERR_ARG;
  if (p->f16_rounding != WT_ROUND_NEAREST && p->f16_rounding != WT_ROUND_STOCHASTIC)
    return WT_ERR_ARG;
  if (p->reserved != 0) return WT_ERR_ARG;
  return WT_OK;
}

int grow_forces(wt_lattice* h, int nsteps) {
  if (nsteps <= h->forces_cap) return WT_OK;
  int cap = std::max(nsteps, 2 * h->forces_cap);
  if (h->forces_dev) cudaFree(h->forces_dev);
  if (h->forces_host) cudaFreeHost(h->forces_host);
  h->forces_dev = nullptr;
  h->forces_host = nullptr;
  h->forces_cap = 0;
  if (cudaMalloc(&h->forces_dev, sizeof(double) * 3 * (size_t)cap) != cudaSuccess)
    return fail(h, WT_ERR_OOM, "cannot allocate the device force series");
  if (cudaMallocHost(&h->forces_host, sizeof(double) * 3 * (size_t)cap) != cudaSuccess)
    return fail(h, WT_ERR_OOM, "cannot allocate the pinned force series");
  h->forces_cap = cap;
  return WT_OK;
}

template <class S>
S to_store(double v);
template <>
float to_store<float>(double v) { return (float)v; }
template <>
double to_store<double>(double v) { return v; }
template <>
__half to_store<__half>(double v) { return __double2half(v * WT_F16_SCALE); }

template <class S>
wt::StepArgs<S> make_args(wt_lattice* h) {
  wt::StepArgs<S> a{};
  a.flags = h->flags;
  a.nmask = h->nmask;
  a.ux = h->ux; a.uy = h->uy; a.uz = h->uz; a.rho = h->rho;
  a.uwx = h->uwx; a.uwy = h->uwy; a.uwz = h->uwz;
  a.wslot = h->wslot;
  a.err = h->err_dev;
  a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
  a.n = h->n;
  a.nxy = (long long)h->nx * h->ny;
  const bool narrow = 19 * h->n * (long long)sizeof(S) < (1LL << 31);
  for (int q = 0; q < 19; q++) {
    const long long off = wt::ex(q) + (long long)h->nx * wt::ey(q) + a.nxy * wt::ez(q);
    a.src[q] = q * h->n - off;
    a.dst[q] = q * h->n;
    a.srcb[q] = narrow ? (uint32_t)(a.src[q] * (long long)sizeof(S)) : 0u;
    a.dstb[q] = narrow ? (uint32_t)(a.dst[q] * (long long)sizeof(S)) : 0u;
  }
  const wt_params& p = h->p;
  a.tau0 = p.tau;
  a.omega0 = 1 / p.tau;
  a.cs2 = p.csm * p.csm;
  a.lam = p.lambda;
  a.tau0f = (float)p.tau;
  a.omega0f = (float)(1 / p.tau);
  a.omm0f = (float)(p.trt ? 1 / (0.5 + p.lambda / (p.tau - 0.5)) : 1 / p.tau);
  a.les_cf = (float)(72 * a.cs2);   // 18*sqrt(2)*cs2*|Pi| with |Pi| = 2*sqrt(2*qq)
  a.lamf = (float)p.lambda;
  a.u0f = (float)p.u0;
  a.les = p.les ? 1 : 0;
  a.trt = p.trt ? 1 : 0;
  a.mov = p.moving_walls ? 1 : 0;
  a.freeslip = p.side_bc == WT_SIDE_FREESLIP ? 1 : 0;
  a.f16_sr = p.f16_rounding == WT_ROUND_STOCHASTIC ? 1 : 0;
  double eq[19];
  wt::eq_u0_table(p.u0, eq);
  for (int q = 0; q < 19; q++) {
    a.eq[q] = to_store<S>(eq[q]);
    if constexpr (sizeof(S) == 2) {
      uint16_t b;
      memcpy(&b, &a.eq[q], 2);
      a.eq2[q] = (uint32_t)b | ((uint32_t)b << 16);
    }
  }
  a.sfrac = h->sfrac;
  for (int k = 0; k < 6; k++) a.sb[k] = h->sbox[k];
  a.pf = h->pf;   // read by the lean kernel only
  return a;
}

enum class Path { Direct, Lean, Pbb, Pair };

template <class S>
using StepLaunch = void (*)(const wt::StepArgs<S>&, dim3, bool, cudaStream_t);

// nsteps steps of one kernel: the force partials of up to `chunk` steps go to
// `part` (one block of slots per step) and are reduced into forces_dev once
// per chunk; error bits go to `err`.
template <class S>
void run_steps(wt_lattice* h, int nsteps, StepLaunch<S> launch, double* part, double* forces_dev,
               unsigned* err, int chunk_max) {
  wt::StepArgs<S> a = make_args<S>(h);
  a.err = err;
  const dim3 grid = wt::step_grid(h->nx, h->ny, h->nz);
  const bool wide = 19 * h->n >= (1LL << 31);
  const size_t stride = 3 * (size_t)h->nslots;
  for (int done = 0; done < nsteps;) {
    const int chunk = std::min(chunk_max, nsteps - done);
    for (int s = 0; s < chunk; s++) {
      a.F = (const S*)h->buf[h->parity];
      a.G = (S*)h->buf[h->parity ^ 1];
      a.part = part + (size_t)s * stride;
      a.write_fields = (done + s == nsteps - 1) ? 1 : 0;
      a.sr_seed = (unsigned)((uint64_t)(h->steps + done + s) * 0x9E3779B97F4A7C15ULL >> 32);
      launch(a, grid, wide, h->stream);
      h->launches++;
      h->parity ^= 1;
    }
    wt::launch_force_reduce(part, (unsigned)h->nslots, chunk, forces_dev + 3 * (size_t)done,
                            h->stream);
    h->launches++;
    done += chunk;
  }
}

bool lean_ok(const wt_lattice* h);
bool pair_ok(const wt_lattice* h);

// The kernel WT_KERNEL_AUTO runs, the fastest measured on B200 for the form
// (256x128x128 channel, 1000-step calls): the pair kernel where it can run
// (float32 storage 40.3k MLUPS against 37.9k for the lean kernel; half
// storage 55.2k against 44.4k), the lean kernel for an odd nx, the direct
// kernel otherwise (exact collision, float64, moving walls, buffers of 2^31
// bytes or more).
Path auto_path(const wt_lattice* h) {
  if (pair_ok(h)) return Path::Pair;
  if (lean_ok(h)) return Path::Lean;
  return Path::Direct;
}

// True when the lean-addressing kernel can run.
// Moving walls are excluded: their correction reads the previous step's
// density, which the thread of cell nx-2 rewrites while the outlet thread
// recomputes that cell.
bool lean_ok(const wt_lattice* h) {
  const bool exact = h->p.math == WT_MATH_EXACT || h->storage == WT_STORE_F64;
  return !exact && !h->p.moving_walls && 19 * h->n * (long long)h->elem < (1LL << 31);
}

// True when the pair kernel can run: the lean kernel's conditions (float32
// collision, so half or float32 storage) and an even nx (aligned pairs of
// cells).
bool pair_ok(const wt_lattice* h) { return lean_ok(h) && h->nx % 2 == 0; }

int select_path(wt_lattice* h, Path* out);
void dispatch_steps(wt_lattice* h, int nsteps, Path path, double* part, double* forces_dev,
                    unsigned* err, int chunk);
int check_err_word(wt_lattice* h, unsigned word);

// Assign a force-partial slot to every 32-cell segment that holds a
// near-wall cell (js/lbm.js:334-359 only accumulates there) and size the
// partial buffer.
int rebuild_slots(wt_lattice* h) {
  uint8_t* mark = nullptr;
  if (cudaMalloc(&mark, (size_t)h->nsegs) != cudaSuccess)
    return fail(h, WT_ERR_OOM, "cannot allocate the warp marks");
  std::vector<uint8_t> hm((size_t)h->nsegs);
  cudaError_t e = cudaMemsetAsync(mark, 0, (size_t)h->nsegs, h->stream);
  if (e == cudaSuccess) {
    wt::launch_mark_segments(h->flags, h->nx, h->ny, h->nz, mark, h->stream);
    h->launches++;
    e = cudaMemcpyAsync(hm.data(), mark, hm.size(), cudaMemcpyDeviceToHost, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(mark);
  if (e != cudaSuccess) return cuda_fail(h, e, "rebuild_slots");
  if (h->sfrac) {
    // every segment that touches the partial bounce-back box carries a force partial
    const int* b = h->sbox;
    const int nseg = (h->nx + 31) / 32;
    for (int z = b[2]; z < b[5]; z++)
      for (int y = b[1]; y < b[4]; y++)
        for (int sx = b[0] / 32; sx <= (b[3] - 1) / 32; sx++)
          hm[((size_t)z * h->ny + y) * nseg + sx] = 1;
  }
  std::vector<int> slot(hm.size());
  int n = 0;
  for (size_t w = 0; w < hm.size(); w++) slot[w] = hm[w] ? n++ : -1;
  if (n > h->part_cap || !h->part) {
    if (h->part) cudaFree(h->part);
    h->part = nullptr;
    h->part_cap = 0;
    const int cap = std::max(n, 1);
    if (cudaMalloc(&h->part, sizeof(double) * 3 * (size_t)cap * kChunk) != cudaSuccess)
      return fail(h, WT_ERR_OOM, "cannot allocate the force partials");
    h->part_cap = cap;
  }
  e = cudaMemcpyAsync(h->wslot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice,
                      h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "rebuild_slots upload");
  h->nslots = n;
  return WT_OK;
}

}  // namespace

extern "C" {

void wt_default_params(wt_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->u0 = 0.06;
  p->tau = 0.5035;
  p->les = 1;
  p->trt = 1;
  p->csm = 0.14;
  p->lambda = 1.0 / 4;
  p->moving_walls = 0;
  p->side_bc = WT_SIDE_EQ;
  p->math = WT_MATH_FAST;
  p->kernel = WT_KERNEL_AUTO;
  p->f16_rounding = WT_ROUND_NEAREST;
}

const char* wt_last_error(const wt_lattice* h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

int wt_create(int nx, int ny, int nz, int storage, wt_lattice** out) {
  g_create_error.clear();
  if (!out) { g_create_error = "out is NULL"; return WT_ERR_ARG; }
  *out = nullptr;
  if (nx < 3 || ny < 3 || nz < 3) {
    g_create_error = "lattice dims must be at least 3 in every direction";
    return WT_ERR_ARG;
  }
  if (ny > 65535 || nz > 65535) {
    g_create_error = "ny and nz must not exceed 65535";
    return WT_ERR_ARG;
  }
  if (storage != WT_STORE_F32 && storage != WT_STORE_F16DEV && storage != WT_STORE_F64) {
    g_create_error = "unknown storage format";
    return WT_ERR_ARG;
  }
  const long long n = (long long)nx * ny * nz;
  if (n > (1LL << 40) / 19) {
    g_create_error = "lattice too large";
    return WT_ERR_ARG;
  }
  wt_lattice* h = new wt_lattice();
  h->nx = nx; h->ny = ny; h->nz = nz; h->n = n; h->storage = storage;
  h->elem = elem_size(storage);
  wt_default_params(&h->p);
  h->stats.frontal_area = 1;
  cudaGetDevice(&h->device);
  {
    // The lean and pair kernels can prefetch into L2 the populations of the
    // warp this many cells further on in launch order: a third of the cells
    // the lean kernel's resident blocks (8 per SM) cover. Measured on B200 it
    // pays only for half storage on lattices whose population buffer fits in
    // twice the L2 (256x128x128: lean +7% over none, flat from 0.15 to 0.65 of
    // the resident cells; pair +3%); it cost the lean kernel 8% for float32
    // storage on the same lattice and 19% for half storage on 512x192x192,
    // whatever the distance, so it is off there. WT_PREFETCH_CELLS overrides it
    // (0: off).
    int sms = 0, l2 = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->device);
    const int gx = (nx + wt::STEP_BX - 1) / wt::STEP_BX;
    const bool small = (double)n * 19 * elem_size(storage) <= 2.0 * (double)l2;
    h->pf = storage == WT_STORE_F16DEV && small ? (long long)sms * 8 * nx / gx / 3 : 0;
    if (const char* e = getenv("WT_PREFETCH_CELLS")) h->pf = std::max(0LL, atoll(e));
  }
  h->nsegs = (long long)((nx + 31) / 32) * ny * nz;
  const size_t pop = (size_t)n * 19 * h->elem;
  if (const cudaError_t e = wt::configure_step_kernels(); e != cudaSuccess) {
    cudaGetLastError();
    delete h;
    g_create_error = std::string("setting the step kernels' attributes failed: ") +
                     cudaGetErrorString(e);
    return WT_ERR_CUDA;
  }
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&h->buf[0], pop) == cudaSuccess;
  ok = ok && cudaMalloc(&h->buf[1], pop) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->flags, (size_t)n) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->nmask, sizeof(unsigned long long) * (size_t)n) == cudaSuccess;
  float** fl[] = {&h->ux, &h->uy, &h->uz, &h->rho, &h->uwx, &h->uwy, &h->uwz};
  for (float** p : fl) ok = ok && cudaMalloc((void**)p, sizeof(float) * (size_t)n) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->wslot, sizeof(int) * (size_t)h->nsegs) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->err_dev, sizeof(unsigned)) == cudaSuccess;
  ok = ok && cudaMallocHost((void**)&h->err_host, sizeof(unsigned)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->col, (size_t)ny * nz) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->plan, (size_t)nx * nz) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->low, sizeof(int) * (size_t)nx * nz) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&h->counters, sizeof(int) * 2) == cudaSuccess;
  ok = ok && grow_forces(h, 64) == WT_OK;
  if (!ok) {
    cudaGetLastError();
    free_all(h);
    delete h;
    g_create_error = "device allocation failed for a " + std::to_string(nx) + "x" +
                     std::to_string(ny) + "x" + std::to_string(nz) + " lattice";
    return WT_ERR_OOM;
  }
  cudaMemsetAsync(h->flags, 0, (size_t)n, h->stream);
  cudaMemsetAsync(h->nmask, 0, sizeof(unsigned long long) * (size_t)n, h->stream);
  for (float* p : {h->uwx, h->uwy, h->uwz}) cudaMemsetAsync(p, 0, sizeof(float) * n, h->stream);
  wt::launch_init(h, 0, 0, 0);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess && rebuild_slots(h) != WT_OK) e = cudaErrorMemoryAllocation;
  if (e != cudaSuccess) {
    g_create_error = std::string("initialisation failed: ") + cudaGetErrorString(e);
    free_all(h);
    delete h;
    return WT_ERR_CUDA;
  }
  *out = h;
  return WT_OK;
}

int wt_destroy(wt_lattice* h) {
  if (!h) return WT_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return WT_OK;
}

int wt_get_dims(const wt_lattice* h, int* nx, int* ny, int* nz, int* storage) {
  if (!h) return WT_ERR_ARG;
  if (nx) *nx = h->nx;
  if (ny) *ny = h->ny;
  if (nz) *nz = h->nz;
  if (storage) *storage = h->storage;
  return WT_OK;
}

int wt_set_params(wt_lattice* h, const wt_params* p) {
  if (!h) return WT_ERR_ARG;
  if (!p) return fail(h, WT_ERR_ARG, "params is NULL");
  const int c = check_params(p);
  if (c != WT_OK)
    return fail(h, c, "invalid parameters (need finite u0/csm/lambda, tau > 0.5, lambda > 0 "
                      "with trt, known side_bc, math and kernel)");
  if (h->storage == WT_STORE_F16DEV && p->math == WT_MATH_EXACT)
    return fail(h, WT_ERR_UNSUPPORTED, "half storage runs the float32 collision only");
  h->p = *p;
  return WT_OK;
}

int wt_get_params(const wt_lattice* h, wt_params* p) {
  if (!h || !p) return WT_ERR_ARG;
  *p = h->p;
  return WT_OK;
}

int wt_reset(wt_lattice* h) {
  if (!h) return WT_ERR_ARG;
  wt::launch_init(h, 0, 0, 0);
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  WT_CUDA(h, cudaGetLastError());
  h->steps = 0;
  h->force[0] = h->force[1] = h->force[2] = 0;
  return WT_OK;
}

int wt_init_eq_noise(wt_lattice* h, uint64_t seed, double amp) {
  if (!h) return WT_ERR_ARG;
  if (!std::isfinite(amp)) return fail(h, WT_ERR_ARG, "amp must be finite");
  wt::launch_init(h, 1, seed, amp);
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  WT_CUDA(h, cudaGetLastError());
  h->steps = 0;
  h->force[0] = h->force[1] = h->force[2] = 0;
  return WT_OK;
}

int wt_voxel_range(const wt_lattice* h, const double box[6], int range[6]) {
  if (!h || !box || !range) return WT_ERR_ARG;
  voxel_range(h->nx, h->ny, h->nz, box, range);
  return WT_OK;
}

namespace {

// Shared tail of both voxelize forms: statistics and near flags.
int voxelize_finish(wt_lattice* h, int ground, double road_vel) {
  std::vector<uint8_t> col((size_t)h->ny * h->nz), plan((size_t)h->nx * h->nz);
  std::vector<int> low((size_t)h->nx * h->nz);
  int counters[2] = {0, 0};
  WT_CUDA(h, cudaMemcpyAsync(col.data(), h->col, col.size(), cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(plan.data(), h->plan, plan.size(), cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(low.data(), h->low, sizeof(int) * low.size(), cudaMemcpyDeviceToHost,
                             h->stream));
  WT_CUDA(h, cudaMemcpyAsync(counters, h->counters, sizeof(counters), cudaMemcpyDeviceToHost,
                             h->stream));
  wt::launch_near(h);
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  WT_CUDA(h, cudaGetLastError());
  // js/lbm.js:247-264
  long long a = 0, pa = 0;
  for (uint8_t v : col) a += v;
  for (uint8_t v : plan) pa += v;
  std::vector<int> gaps;
  for (size_t k = 0; k < plan.size(); k++) {
    if (plan[k] && low[k] < 32767) {
      const int g = low[k] - 1;
      if (g > 0) gaps.push_back(g);
    }
  }
  std::sort(gaps.begin(), gaps.end());
  h->stats.frontal_area = (int)std::max<long long>(1, a);
  h->stats.planform_area = (int)std::max<long long>(1, pa);
  h->stats.solid_cells = counters[0];
  h->stats.ride_height = gaps.empty() ? 0 : gaps[gaps.size() >> 1];
  h->stats.ground = ground ? 1 : 0;
  h->p.moving_walls = (road_vel != 0 || counters[1]) ? 1 : 0;
  h->stats.moving_walls = h->p.moving_walls;
  return rebuild_slots(h);
}

int voxelize_start(wt_lattice* h, int ground, double road_vel) {
  wt::launch_clear_obj(h);
  wt::launch_floor(h, ground, road_vel);
  std::vector<int> low((size_t)h->nx * h->nz, 32767);
  WT_CUDA(h, cudaMemsetAsync(h->col, 0, (size_t)h->ny * h->nz, h->stream));
  WT_CUDA(h, cudaMemsetAsync(h->plan, 0, (size_t)h->nx * h->nz, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(h->low, low.data(), sizeof(int) * low.size(), cudaMemcpyHostToDevice,
                             h->stream));
  WT_CUDA(h, cudaMemsetAsync(h->counters, 0, sizeof(int) * 2, h->stream));
  // the host vector must outlive the async copy
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  return WT_OK;
}

}  // namespace

int wt_voxelize_mask(wt_lattice* h, const double box[6], const uint8_t* inside, size_t inside_len,
                     const uint8_t* wall_set, const double* wall_vel, int ground, double road_vel) {
  if (!h) return WT_ERR_ARG;
  if (!box) return fail(h, WT_ERR_ARG, "box is NULL");
  if (!std::isfinite(road_vel)) return fail(h, WT_ERR_ARG, "road_vel must be finite");
  int rg[6];
  voxel_range(h->nx, h->ny, h->nz, box, rg);
  const long long cells = range_cells(rg);
  if ((long long)inside_len != cells)
    return fail(h, WT_ERR_ARG, "inside has " + std::to_string(inside_len) +
                                   " entries; the scan range of box holds " +
                                   std::to_string(cells));
  if (cells > 0 && !inside) return fail(h, WT_ERR_ARG, "inside is NULL");
  if (wall_set && !wall_vel) return fail(h, WT_ERR_ARG, "wall_set given without wall_vel");
  int c = voxelize_start(h, ground, road_vel);
  if (c != WT_OK) return c;
  if (cells > 0) {
    uint8_t* mask_dev = nullptr;
    uint8_t* ws_dev = nullptr;
    double* wv_dev = nullptr;
    cudaError_t e = cudaMalloc(&mask_dev, (size_t)cells);
    if (e == cudaSuccess && wall_set) e = cudaMalloc(&ws_dev, (size_t)cells);
    if (e == cudaSuccess && wall_set) e = cudaMalloc(&wv_dev, sizeof(double) * 3 * (size_t)cells);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(mask_dev, inside, (size_t)cells, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && wall_set)
      e = cudaMemcpyAsync(ws_dev, wall_set, (size_t)cells, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && wall_set)
      e = cudaMemcpyAsync(wv_dev, wall_vel, sizeof(double) * 3 * (size_t)cells,
                          cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) wt::launch_box_mask(h, rg, mask_dev, ws_dev, wv_dev);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (mask_dev) cudaFree(mask_dev);
    if (ws_dev) cudaFree(ws_dev);
    if (wv_dev) cudaFree(wv_dev);
    if (e != cudaSuccess) return cuda_fail(h, e, "voxelize");
  }
  return voxelize_finish(h, ground, road_vel);
}

int wt_voxelize_grid(wt_lattice* h, const uint8_t* grid, int gnx, int gny, int gnz,
                     const double gmin[3], double ginv, const double M[9], const double P[3],
                     double scale, const double box[6], int ground, double road_vel) {
  if (!h) return WT_ERR_ARG;
  if (!grid || !gmin || !M || !P || !box) return fail(h, WT_ERR_ARG, "NULL argument");
  if (gnx < 1 || gny < 1 || gnz < 1) return fail(h, WT_ERR_ARG, "grid dims must be positive");
  if (!std::isfinite(road_vel)) return fail(h, WT_ERR_ARG, "road_vel must be finite");
  int rg[6];
  voxel_range(h->nx, h->ny, h->nz, box, rg);
  const long long cells = range_cells(rg);
  int c = voxelize_start(h, ground, road_vel);
  if (c != WT_OK) return c;
  if (cells > 0) {
    const size_t gbytes = (size_t)gnx * gny * gnz;
    uint8_t* grid_dev = nullptr;
    cudaError_t e = cudaMalloc(&grid_dev, gbytes);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(grid_dev, grid, gbytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      wt::launch_box_grid(h, rg, grid_dev, gnx, gny, gnz, gmin, ginv, M, P, scale);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (grid_dev) cudaFree(grid_dev);
    if (e != cudaSuccess) return cuda_fail(h, e, "voxelize_grid");
  }
  return voxelize_finish(h, ground, road_vel);
}

int wt_get_body_stats(const wt_lattice* h, wt_body_stats* out) {
  if (!h || !out) return WT_ERR_ARG;
  *out = h->stats;
  out->moving_walls = h->p.moving_walls;
  return WT_OK;
}

int wt_step(wt_lattice* h, int nsteps, double* forces) {
  if (!h) return WT_ERR_ARG;
  if (nsteps < 0) return fail(h, WT_ERR_ARG, "nsteps must be >= 0");
  if (nsteps == 0) return WT_OK;
  int c = grow_forces(h, nsteps);
  if (c != WT_OK) return c;
  WT_CUDA(h, cudaMemsetAsync(h->err_dev, 0, sizeof(unsigned), h->stream));
  Path path = Path::Direct;
  c = select_path(h, &path);
  if (c != WT_OK) return c;
  dispatch_steps(h, nsteps, path, h->part, h->forces_dev, h->err_dev, kChunk);
  WT_CUDA(h, cudaGetLastError());
  WT_CUDA(h, cudaMemcpyAsync(h->forces_host, h->forces_dev, sizeof(double) * 3 * (size_t)nsteps,
                             cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(h->err_host, h->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  h->steps += nsteps;
  const double* last = h->forces_host + 3 * (size_t)(nsteps - 1);
  h->force[0] = last[0]; h->force[1] = last[1]; h->force[2] = last[2];
  if (forces) memcpy(forces, h->forces_host, sizeof(double) * 3 * (size_t)nsteps);
  return check_err_word(h, *h->err_host);
}

}  // extern "C"

namespace {

// The kernel a wt_step call runs, from the handle's parameters.
int select_path(wt_lattice* h, Path* out) {
  if (h->sfrac) {
    if (h->p.kernel != WT_KERNEL_AUTO && h->p.kernel != WT_KERNEL_DIRECT)
      return fail(h, WT_ERR_UNSUPPORTED,
                  "a lattice with a solid-fraction field runs the direct kernel only");
    *out = Path::Pbb;
    return WT_OK;
  }
  Path path = Path::Direct;
  switch (h->p.kernel) {
    case WT_KERNEL_LEAN:
      if (!lean_ok(h))
        return fail(h, WT_ERR_UNSUPPORTED,
                    "the lean kernel needs the float32 collision, buffers under 2 GiB "
                    "and stationary walls");
      path = Path::Lean;
      break;
    case WT_KERNEL_PAIR:
      if (!pair_ok(h))
        return fail(h, WT_ERR_UNSUPPORTED,
                    "the pair kernel needs the float32 collision, an even nx, buffers "
                    "under 2 GiB and stationary walls");
      path = Path::Pair;
      break;
    case WT_KERNEL_AUTO:
      path = auto_path(h);
      break;
    default:
      break;
  }
  *out = path;
  return WT_OK;
}

template <class S>
StepLaunch<S> pick(Path path, StepLaunch<S> direct, StepLaunch<S> lean, StepLaunch<S> pbb,
                   StepLaunch<S> pair = nullptr) {
  switch (path) {
    case Path::Lean: return lean;
    case Path::Pbb: return pbb;
    case Path::Pair: return pair ? pair : direct;
    default: return direct;
  }
}

// Run nsteps steps of the chosen kernel; per-step forces land in forces_dev.
void dispatch_steps(wt_lattice* h, int nsteps, Path path, double* part, double* forces_dev,
                    unsigned* err, int chunk) {
  const bool exact = h->p.math == WT_MATH_EXACT || h->storage == WT_STORE_F64;
  switch (h->storage) {
    case WT_STORE_F32:
      if (exact)
        run_steps<float>(h, nsteps,
                         pick<float>(path, wt::launch_step_f32_exact, wt::launch_step_f32_exact,
                                     wt::launch_pbb_f32_exact),
                         part, forces_dev, err, chunk);
      else
        run_steps<float>(h, nsteps,
                         pick<float>(path, wt::launch_step_f32_fast, wt::launch_lean_f32,
                                     wt::launch_pbb_f32_fast, wt::launch_pair_f32),
                         part, forces_dev, err, chunk);
      break;
    case WT_STORE_F16DEV:
      run_steps<__half>(h, nsteps,
                        pick<__half>(path, wt::launch_step_f16_fast, wt::launch_lean_f16,
                                     wt::launch_pbb_f16_fast, wt::launch_pair_f16),
                        part, forces_dev, err, chunk);
      break;
    default:
      run_steps<double>(h, nsteps,
                        pick<double>(path, wt::launch_step_f64_exact, wt::launch_step_f64_exact,
                                     wt::launch_pbb_f64_exact),
                        part, forces_dev, err, chunk);
      break;
  }
}

// Status of an error word the steps left: bit 1 (a near-wall warp without a
// force slot) and bit 0 (a non-finite or non-positive density).
int check_err_word(wt_lattice* h, unsigned word) {
  if (word & 2u)
    return fail(h, WT_ERR_STATE, "a near-wall warp had no force slot (occupancy changed "
                                 "without voxelize)");
  if (word & 1u)
    return fail(h, WT_ERR_DIVERGED, "a step produced a non-finite or non-positive density");
  return WT_OK;
}

}  // namespace

extern "C" {

int wt_get_force(const wt_lattice* h, double out[3]) {
  if (!h || !out) return WT_ERR_ARG;
  out[0] = h->force[0]; out[1] = h->force[1]; out[2] = h->force[2];
  return WT_OK;
}

int wt_get_steps(const wt_lattice* h, int64_t* steps, int* parity) {
  if (!h) return WT_ERR_ARG;
  if (steps) *steps = h->steps;
  if (parity) *parity = h->parity;
  return WT_OK;
}

int wt_get_fields(wt_lattice* h, float* ux, float* uy, float* uz, float* rho) {
  if (!h) return WT_ERR_ARG;
  const size_t b = sizeof(float) * (size_t)h->n;
  if (ux) WT_CUDA(h, cudaMemcpyAsync(ux, h->ux, b, cudaMemcpyDeviceToHost, h->stream));
  if (uy) WT_CUDA(h, cudaMemcpyAsync(uy, h->uy, b, cudaMemcpyDeviceToHost, h->stream));
  if (uz) WT_CUDA(h, cudaMemcpyAsync(uz, h->uz, b, cudaMemcpyDeviceToHost, h->stream));
  if (rho) WT_CUDA(h, cudaMemcpyAsync(rho, h->rho, b, cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_get_solid(wt_lattice* h, uint8_t* out) {
  if (!h || !out) return WT_ERR_ARG;
  std::vector<uint8_t> fl((size_t)h->n);
  WT_CUDA(h, cudaMemcpyAsync(fl.data(), h->flags, fl.size(), cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < fl.size(); i++) out[i] = fl[i] & wt::FLAG_SOLID_MASK;
  return WT_OK;
}

int wt_get_near(wt_lattice* h, uint8_t* out) {
  if (!h || !out) return WT_ERR_ARG;
  std::vector<uint8_t> fl((size_t)h->n);
  WT_CUDA(h, cudaMemcpyAsync(fl.data(), h->flags, fl.size(), cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < fl.size(); i++) out[i] = (fl[i] & wt::FLAG_NEAR) ? 1 : 0;
  return WT_OK;
}

int wt_get_populations(wt_lattice* h, int which, int dtype, void* out, size_t bytes) {
  if (!h) return WT_ERR_ARG;
  if (!out) return fail(h, WT_ERR_ARG, "out is NULL");
  if (which != WT_BUF_F && which != WT_BUF_G) return fail(h, WT_ERR_ARG, "which must be F or G");
  const bool raw = dtype == h->storage;
  if (!raw && dtype != WT_STORE_F32 && dtype != WT_STORE_F64)
    return fail(h, WT_ERR_ARG, "dtype must be F32, F64 or the handle's storage");
  const long long count = 19LL * h->n;
  const size_t want = (size_t)count * elem_size(dtype);
  if (bytes != want)
    return fail(h, WT_ERR_ARG, "bytes must be " + std::to_string(want));
  const void* src = h->buf[h->parity ^ (which == WT_BUF_G ? 1 : 0)];
  if (raw) {
    WT_CUDA(h, cudaMemcpyAsync(out, src, want, cudaMemcpyDeviceToHost, h->stream));
    WT_CUDA(h, cudaStreamSynchronize(h->stream));
    return WT_OK;
  }
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, want) != cudaSuccess) return fail(h, WT_ERR_OOM, "conversion buffer");
  wt::launch_convert(src, h->storage, tmp, dtype, count, h->stream);
  h->launches++;
  cudaError_t e = cudaMemcpyAsync(out, tmp, want, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "get_populations");
  return WT_OK;
}

int wt_set_populations(wt_lattice* h, int which, int dtype, const void* in, size_t bytes) {
  if (!h) return WT_ERR_ARG;
  if (!in) return fail(h, WT_ERR_ARG, "in is NULL");
  if (which != WT_BUF_F && which != WT_BUF_G) return fail(h, WT_ERR_ARG, "which must be F or G");
  const bool raw = dtype == h->storage;
  if (!raw && dtype != WT_STORE_F32 && dtype != WT_STORE_F64)
    return fail(h, WT_ERR_ARG, "dtype must be F32, F64 or the handle's storage");
  const long long count = 19LL * h->n;
  const size_t want = (size_t)count * elem_size(dtype);
  if (bytes != want)
    return fail(h, WT_ERR_ARG, "bytes must be " + std::to_string(want));
  void* dst = h->buf[h->parity ^ (which == WT_BUF_G ? 1 : 0)];
  if (raw) {
    WT_CUDA(h, cudaMemcpyAsync(dst, in, want, cudaMemcpyHostToDevice, h->stream));
    WT_CUDA(h, cudaStreamSynchronize(h->stream));
    return WT_OK;
  }
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, want) != cudaSuccess) return fail(h, WT_ERR_OOM, "conversion buffer");
  cudaError_t e = cudaMemcpyAsync(tmp, in, want, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    wt::launch_convert_in(tmp, dtype, dst, h->storage, count, h->stream);
    h->launches++;
    e = cudaStreamSynchronize(h->stream);
  }
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "set_populations");
  return WT_OK;
}

namespace {
struct StateHeader {
  uint32_t magic;
  int32_t nx, ny, nz, storage, parity;
  int64_t steps;
  double force[3];
  wt_params params;
  wt_body_stats stats;
};

size_t state_bytes(const wt_lattice* h) {
  return sizeof(StateHeader) + 2 * (size_t)h->n * 19 * h->elem + (size_t)h->n +
         7 * sizeof(float) * (size_t)h->n;
}
}  // namespace

int wt_state_size(const wt_lattice* h, size_t* bytes) {
  if (!h || !bytes) return WT_ERR_ARG;
  *bytes = state_bytes(h);
  return WT_OK;
}

int wt_get_state(wt_lattice* h, void* out, size_t bytes) {
  if (!h || !out) return WT_ERR_ARG;
  if (bytes != state_bytes(h)) return fail(h, WT_ERR_ARG, "state buffer has the wrong size");
  StateHeader hd{};
  hd.magic = kStateMagic;
  hd.nx = h->nx; hd.ny = h->ny; hd.nz = h->nz; hd.storage = h->storage; hd.parity = h->parity;
  hd.steps = h->steps;
  memcpy(hd.force, h->force, sizeof(hd.force));
  hd.params = h->p;
  hd.stats = h->stats;
  char* o = (char*)out;
  memcpy(o, &hd, sizeof(hd));
  o += sizeof(hd);
  const size_t pop = (size_t)h->n * 19 * h->elem, fb = sizeof(float) * (size_t)h->n;
  WT_CUDA(h, cudaMemcpyAsync(o, h->buf[0], pop, cudaMemcpyDeviceToHost, h->stream)); o += pop;
  WT_CUDA(h, cudaMemcpyAsync(o, h->buf[1], pop, cudaMemcpyDeviceToHost, h->stream)); o += pop;
  WT_CUDA(h, cudaMemcpyAsync(o, h->flags, (size_t)h->n, cudaMemcpyDeviceToHost, h->stream));
  o += h->n;
  for (float* p : {h->ux, h->uy, h->uz, h->rho, h->uwx, h->uwy, h->uwz}) {
    WT_CUDA(h, cudaMemcpyAsync(o, p, fb, cudaMemcpyDeviceToHost, h->stream));
    o += fb;
  }
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  return WT_OK;
}

int wt_set_state(wt_lattice* h, const void* in, size_t bytes) {
  if (!h || !in) return WT_ERR_ARG;
  if (bytes != state_bytes(h)) return fail(h, WT_ERR_ARG, "state buffer has the wrong size");
  StateHeader hd;
  memcpy(&hd, in, sizeof(hd));
  if (hd.magic != kStateMagic || hd.nx != h->nx || hd.ny != h->ny || hd.nz != h->nz ||
      hd.storage != h->storage)
    return fail(h, WT_ERR_ARG, "state was taken from a different lattice");
  if (check_params(&hd.params) != WT_OK) return fail(h, WT_ERR_ARG, "state holds invalid params");
  const char* o = (const char*)in + sizeof(hd);
  const size_t pop = (size_t)h->n * 19 * h->elem, fb = sizeof(float) * (size_t)h->n;
  WT_CUDA(h, cudaMemcpyAsync(h->buf[0], o, pop, cudaMemcpyHostToDevice, h->stream)); o += pop;
  WT_CUDA(h, cudaMemcpyAsync(h->buf[1], o, pop, cudaMemcpyHostToDevice, h->stream)); o += pop;
  WT_CUDA(h, cudaMemcpyAsync(h->flags, o, (size_t)h->n, cudaMemcpyHostToDevice, h->stream));
  o += h->n;
  for (float* p : {h->ux, h->uy, h->uz, h->rho, h->uwx, h->uwy, h->uwz}) {
    WT_CUDA(h, cudaMemcpyAsync(p, o, fb, cudaMemcpyHostToDevice, h->stream));
    o += fb;
  }
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  h->parity = hd.parity & 1;
  h->steps = hd.steps;
  memcpy(h->force, hd.force, sizeof(hd.force));
  h->p = hd.params;
  h->stats = hd.stats;
  wt::launch_near(h);   // near flags and neighbour masks follow from the restored occupancy
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  return rebuild_slots(h);
}

int wt_sample(wt_lattice* h, const double* xyz, int npts, double* out) {
  if (!h) return WT_ERR_ARG;
  if (npts < 0 || (npts > 0 && (!xyz || !out))) return fail(h, WT_ERR_ARG, "bad points");
  if (npts == 0) return WT_OK;
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * 6 * (size_t)npts) != cudaSuccess)
    return fail(h, WT_ERR_OOM, "sample buffer");
  cudaError_t e = cudaMemcpyAsync(d, xyz, sizeof(double) * 3 * (size_t)npts,
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    wt::launch_sample(h, d, npts, d + 3 * (size_t)npts);
    e = cudaMemcpyAsync(out, d + 3 * (size_t)npts, sizeof(double) * 3 * (size_t)npts,
                        cudaMemcpyDeviceToHost, h->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(h, e, "sample");
  return WT_OK;
}

int wt_is_solid(wt_lattice* h, double x, double y, double z, int* out) {
  if (!h || !out) return WT_ERR_ARG;
  const int xi = js_toint32(x), yi = js_toint32(y), zi = js_toint32(z);
  if (xi < 0 || yi < 0 || zi < 0 || xi >= h->nx || yi >= h->ny || zi >= h->nz) {
    *out = 0;
    return WT_OK;
  }
  uint8_t v = 0;
  const long long i = xi + (long long)h->nx * (yi + (long long)h->ny * zi);
  WT_CUDA(h, cudaMemcpyAsync(&v, h->flags + i, 1, cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  *out = (v & wt::FLAG_SOLID_MASK) != 0;
  return WT_OK;
}

int wt_get_stream(const wt_lattice* h, void** stream) {
  if (!h || !stream) return WT_ERR_ARG;
  *stream = (void*)h->stream;
  return WT_OK;
}

int wt_get_launch_count(const wt_lattice* h, int64_t* count) {
  if (!h || !count) return WT_ERR_ARG;
  *count = h->launches;
  return WT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Partial bounce-back field and the discrete adjoint of the step.

extern "C" int wt_set_solid_fraction(wt_lattice* h, const int box[6], const double* s) {
  if (!h) return WT_ERR_ARG;
  if (h->sfrac) {
    cudaFree(h->sfrac);
    h->sfrac = nullptr;
  }
  for (int k = 0; k < 6; k++) h->sbox[k] = 0;
  if (!box) return rebuild_slots(h);
  const int x0 = box[0], y0 = box[1], z0 = box[2], x1 = box[3], y1 = box[4], z1 = box[5];
  if (!s || x0 < 0 || y0 < 0 || z0 < 0 || x1 > h->nx || y1 > h->ny || z1 > h->nz || x1 <= x0 ||
      y1 <= y0 || z1 <= z0)
    return fail(h, WT_ERR_ARG, "solid-fraction box must be non-empty and inside the lattice, "
                               "with values");
  const size_t m = (size_t)(x1 - x0) * (y1 - y0) * (z1 - z0);
  for (size_t k = 0; k < m; k++)
    if (!std::isfinite(s[k]) || s[k] < 0.0 || s[k] > 1.0)
      return fail(h, WT_ERR_ARG, "solid fractions must lie in [0, 1]");
  if (cudaMalloc((void**)&h->sfrac, sizeof(double) * m) != cudaSuccess) {
    h->sfrac = nullptr;
    return fail(h, WT_ERR_OOM, "cannot allocate the solid-fraction field");
  }
  WT_CUDA(h, cudaMemcpy(h->sfrac, s, sizeof(double) * m, cudaMemcpyHostToDevice));
  for (int k = 0; k < 6; k++) h->sbox[k] = box[k];
  return rebuild_slots(h);
}

namespace {

// Device buffers of one adjoint run, released on every exit path.
// The adjoint's device memory (checkpoints, interval store, two adjoint
// buffers, dJ/ds, the force series) as one block carved in order. A run with
// cfg.keep leaves the block in the lattice for the next run that fits in it
// (an optimisation loop then pays for cudaMalloc / cudaFree once); a run
// without it frees any kept block when it ends, on every return path.
struct AdjBlock {
  wt_lattice* h;
  bool keep;
  size_t off = 0;
  unsigned char* base = nullptr;
  static size_t up(size_t n) { return (n + 255) & ~(size_t)255; }
  // one block of `total` bytes: the kept one if it is large enough
  bool acquire(size_t total) {
    if (h->adj_pool && h->adj_pool_bytes >= total) {
      base = (unsigned char*)h->adj_pool;
      return true;
    }
    release();
    void* p = nullptr;
    if (cudaMalloc(&p, total) != cudaSuccess) return false;
    h->adj_pool = p;
    h->adj_pool_bytes = total;
    base = (unsigned char*)p;
    return true;
  }
  void* carve(size_t n) {
    void* p = base + off;
    off += up(n);
    return p;
  }
  void release() {
    if (h->adj_pool) {
      cudaStreamSynchronize(h->stream);
      cudaFree(h->adj_pool);
    }
    h->adj_pool = nullptr;
    h->adj_pool_bytes = 0;
  }
  ~AdjBlock() {
    if (!keep) release();
  }
};

template <class S, class T, class LA, class LP>
int adjoint_run(wt_lattice* h, const wt_adj_cfg& cfg, int C, double* dJds, wt_adj_stats* st,
                LA launch_adj, LP launch_pbb) {
  const int N = cfg.nsteps, W = cfg.window;
  const size_t pop = (size_t)h->n * 19 * sizeof(S);
  const size_t tsz = (size_t)h->n * 19 * sizeof(T);
  const int ncp = (N + C - 1) / C;
  const int* b = h->sbox;
  const size_t nbox = (size_t)(b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]);
  AdjBlock mem{h, cfg.keep != 0};
  const size_t pel = pop / sizeof(S);                // elements of one state
  // checkpoints S^{kC} of every interval but the last, whose states the
  // forward sweep writes straight into an interval store (C + 1 states).
  // With two stores the recomputation of interval k-1 runs on a second
  // stream while the adjoint steps of interval k run on the lattice's
  // stream; one store (when two do not fit) runs them in turn.
  const size_t sz_cps = ncp > 1 ? pop * (size_t)(ncp - 1) : 0, sz_seg = pop * (size_t)(C + 1);
  const size_t sz_ds = sizeof(double) * nbox, sz_f = sizeof(double) * 3 * (size_t)N;
  auto total_for = [&](int stores) {
    return AdjBlock::up(sz_cps) + stores * AdjBlock::up(sz_seg) + 2 * AdjBlock::up(tsz) +
           AdjBlock::up(sz_ds) + AdjBlock::up(sz_f);
  };
  int ns = ncp > 1 ? 2 : 1;
  size_t total = total_for(ns);
  if (!mem.acquire(total) && ns == 2) {
    cudaGetLastError();
    ns = 1;
    total = total_for(ns);
    if (!mem.acquire(total))
      return fail(h, WT_ERR_OOM, "cannot allocate the adjoint's checkpoints (" +
                                     std::to_string(total >> 20) + " MiB)");
  } else if (!mem.base) {
    return fail(h, WT_ERR_OOM, "cannot allocate the adjoint's checkpoints (" +
                                   std::to_string(total >> 20) + " MiB)");
  }
  cudaGetLastError();
  S* cps = ncp > 1 ? (S*)mem.carve(sz_cps) : nullptr;
  S* seg[2] = {(S*)mem.carve(sz_seg), ns == 2 ? (S*)mem.carve(sz_seg) : nullptr};
  if (ns == 1) seg[1] = seg[0];
  T* Tbuf[2] = {(T*)mem.carve(tsz), (T*)mem.carve(tsz)};
  double* ds = (double*)mem.carve(sz_ds);
  double* fdev = (double*)mem.carve(sz_f);
  if (ncp > 1 && !h->aux)
    WT_CUDA(h, cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking));
  // the sweep timers and the per-interval completion events of the two
  // backward streams, destroyed on every return path
  struct Events {
    std::vector<cudaEvent_t> e;
    cudaError_t make(size_t n, unsigned flags) {
      for (size_t k = 0; k < n; k++) {
        cudaEvent_t x = nullptr;
        const cudaError_t r = cudaEventCreateWithFlags(&x, flags);
        if (r != cudaSuccess) return r;
        e.push_back(x);
      }
      return cudaSuccess;
    }
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev, rec_done, adj_done;
  WT_CUDA(h, ev.make(3, cudaEventDefault));
  WT_CUDA(h, rec_done.make((size_t)ncp, cudaEventDisableTiming));
  WT_CUDA(h, adj_done.make((size_t)ncp, cudaEventDisableTiming));
  cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];
  WT_CUDA(h, cudaMemsetAsync(h->err_dev, 0, sizeof(unsigned), h->stream));
  const dim3 grid = wt::step_grid(h->nx, h->ny, h->nz);
  const bool wide = 19 * h->n >= (1LL << 31);
  WT_CUDA(h, cudaEventRecord(e0, h->stream));
  // forward sweep: a checkpoint every C steps, the force series for J
  for (int k = 0; k + 1 < ncp; k++) {
    WT_CUDA(h, cudaMemcpyAsync(cps + (size_t)k * pel, h->buf[h->parity], pop,
                               cudaMemcpyDeviceToDevice, h->stream));
    dispatch_steps(h, C, Path::Pbb, h->part, fdev + 3 * (size_t)k * C, h->err_dev, kChunk);
  }
  const int tl = (ncp - 1) * C, nl = N - tl;   // the last interval
  S* last = seg[(ncp - 1) & 1];
  {
    WT_CUDA(h, cudaMemcpyAsync(last, h->buf[h->parity], pop, cudaMemcpyDeviceToDevice,
                               h->stream));
    wt::StepArgs<S> fa = make_args<S>(h);
    const size_t stride = 3 * (size_t)h->nslots;
    for (int done = 0; done < nl;) {
      const int chunk = std::min(kChunk, nl - done);
      for (int s = 0; s < chunk; s++) {
        fa.F = last + (size_t)(done + s) * pel;
        fa.G = last + (size_t)(done + s + 1) * pel;
        fa.part = h->part + (size_t)s * stride;
        fa.write_fields = (done + s == nl - 1) ? 1 : 0;
        launch_pbb(fa, grid, wide, h->stream);
        h->launches++;
      }
      wt::launch_force_reduce(h->part, (unsigned)h->nslots, chunk,
                              fdev + 3 * ((size_t)tl + done), h->stream);
      h->launches++;
      done += chunk;
    }
    WT_CUDA(h, cudaMemcpyAsync(h->buf[h->parity], last + (size_t)nl * pel, pop,
                               cudaMemcpyDeviceToDevice, h->stream));
  }
  WT_CUDA(h, cudaEventRecord(e1, h->stream));
  // backward sweep, interval by interval from the last: the adjoint steps of
  // interval k (last to first) on the lattice's stream, and meanwhile on the
  // second stream the recomputation of interval k-1's states from its
  // checkpoint into the other store. A recomputation waits for the adjoint
  // steps that last read its store; adjoint steps wait for their states.
  WT_CUDA(h, cudaMemsetAsync(Tbuf[0], 0, tsz, h->stream));
  WT_CUDA(h, cudaMemsetAsync(ds, 0, sizeof(double) * nbox, h->stream));
  int cur = 0;   // Tbuf[cur] holds T^{t+1}
  wt::StepArgs<S> a = make_args<S>(h), r = make_args<S>(h);
  a.write_fields = r.write_fields = 0;
  a.part = r.part = h->part;   // force partials of recomputed steps are not reduced
  auto adjoint_steps = [&](int k) {
    const int t0 = k * C, n = std::min(C, N - t0);
    S* sk = seg[k & 1];
    for (int t = t0 + n - 1; t >= t0; t--) {
      a.F = sk + (size_t)(t - t0) * pel;
      const double wJ = t >= N - W ? 1.0 / W : 0.0;
      launch_adj(a, Tbuf[cur], Tbuf[cur ^ 1], ds, wJ, cfg.component, h->stream);
      h->launches++;
      cur ^= 1;
    }
  };
  adjoint_steps(ncp - 1);
  WT_CUDA(h, cudaEventRecord(adj_done.e[ncp - 1], h->stream));
  for (int k = ncp - 2; k >= 0; k--) {
    // recompute interval k into seg[k & 1] on the second stream
    const int reuse = k + ns;   // the interval whose adjoint steps last read that store
    WT_CUDA(h, cudaStreamWaitEvent(h->aux, reuse < ncp ? adj_done.e[reuse] : e1, 0));
    S* sk = seg[k & 1];
    WT_CUDA(h, cudaMemcpyAsync(sk, cps + (size_t)k * pel, pop, cudaMemcpyDeviceToDevice,
                               h->aux));
    for (int j = 0; j + 1 < C; j++) {
      r.F = sk + (size_t)j * pel;
      r.G = sk + (size_t)(j + 1) * pel;
      launch_pbb(r, grid, wide, h->aux);
      h->launches++;
    }
    WT_CUDA(h, cudaEventRecord(rec_done.e[k], h->aux));
    // its adjoint steps on the lattice's stream
    WT_CUDA(h, cudaStreamWaitEvent(h->stream, rec_done.e[k], 0));
    adjoint_steps(k);
    WT_CUDA(h, cudaEventRecord(adj_done.e[k], h->stream));
  }
  WT_CUDA(h, cudaEventRecord(e2, h->stream));
  WT_CUDA(h, cudaGetLastError());
  std::vector<double> fh(3 * (size_t)N);
  WT_CUDA(h, cudaMemcpyAsync(fh.data(), fdev, sizeof(double) * fh.size(), cudaMemcpyDeviceToHost,
                             h->stream));
  WT_CUDA(h, cudaMemcpyAsync(dJds, ds, sizeof(double) * nbox, cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(h->err_host, h->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  float fwd_ms = 0, bwd_ms = 0;
  cudaEventElapsedTime(&fwd_ms, e0, e1);
  cudaEventElapsedTime(&bwd_ms, e1, e2);
  double J = 0;
  for (int t = N - W; t < N; t++) J += fh[3 * (size_t)t + cfg.component];
  J /= W;
  h->steps += N;
  h->force[0] = fh[3 * (size_t)(N - 1)];
  h->force[1] = fh[3 * (size_t)(N - 1) + 1];
  h->force[2] = fh[3 * (size_t)(N - 1) + 2];
  if (st) {
    st->J = J;
    st->forward_ms = fwd_ms;
    st->backward_ms = bwd_ms;
    st->device_bytes = (int64_t)total;
    st->checkpoints = ncp;
    st->segment = C;
  }
  return check_err_word(h, *h->err_host);
}

}  // namespace

extern "C" int wt_adjoint(wt_lattice* h, const wt_adj_cfg* cfg, double* dJds, wt_adj_stats* st) {
  if (!h) return WT_ERR_ARG;
  if (!cfg || !dJds) return fail(h, WT_ERR_ARG, "cfg and dJds are required");
  if (!h->sfrac) return fail(h, WT_ERR_STATE, "set a solid-fraction field first");
  if (cfg->nsteps < 1 || cfg->window < 1 || cfg->window > cfg->nsteps || cfg->component < 0 ||
      cfg->component > 2 || cfg->checkpoint < 0 || cfg->reserved[0] || cfg->reserved[1] ||
      cfg->reserved[2])
    return fail(h, WT_ERR_ARG, "need nsteps >= 1, 1 <= window <= nsteps, component 0..2, "
                               "checkpoint >= 0, reserved fields 0");
  if (h->p.moving_walls)
    return fail(h, WT_ERR_UNSUPPORTED, "the adjoint supports stationary walls only");
  if (h->p.kernel != WT_KERNEL_AUTO && h->p.kernel != WT_KERNEL_DIRECT)
    return fail(h, WT_ERR_UNSUPPORTED, "the adjoint runs the direct kernel");
  int C = cfg->checkpoint;
  if (C == 0) {
    // every state when they fit in three quarters of the free memory (no
    // recomputation), else segments of about sqrt(nsteps) steps
    size_t freeb = 0, total = 0;
    WT_CUDA(h, cudaMemGetInfo(&freeb, &total));
    const size_t pop = (size_t)h->n * 19 * h->elem;
    if ((double)pop * (cfg->nsteps + 3) <= 0.75 * (double)freeb) C = cfg->nsteps;
    else C = std::max(1, (int)std::ceil(std::sqrt((double)cfg->nsteps)));
  }
  C = std::min(C, cfg->nsteps);
  int c = grow_forces(h, 1);
  if (c != WT_OK) return c;
  const bool exact = h->p.math == WT_MATH_EXACT || h->storage == WT_STORE_F64;
  switch (h->storage) {
    case WT_STORE_F32:
      if (exact) return adjoint_run<float, double>(h, *cfg, C, dJds, st, wt::launch_adj_f32x,
                                                   wt::launch_pbb_f32_exact);
      return adjoint_run<float, float>(h, *cfg, C, dJds, st, wt::launch_adj_f32,
                                       wt::launch_pbb_f32_fast);
    case WT_STORE_F16DEV:
      return adjoint_run<__half, float>(h, *cfg, C, dJds, st, wt::launch_adj_f16,
                                        wt::launch_pbb_f16_fast);
    default:
      return adjoint_run<double, double>(h, *cfg, C, dJds, st, wt::launch_adj_f64,
                                         wt::launch_pbb_f64_exact);
  }
}

// ---------------------------------------------------------------------------
// wt_step_noalloc: the step for callers that must not allocate device memory
// while they run, such as a host whose own memory pool has already claimed
// the device's memory, or a host stepping inside a frame loop that must not
// stall (cudaMalloc / cudaFree may synchronise the whole device). wt_step
// may grow its force series buffers (cudaMalloc / cudaMallocHost); this entry
// point instead keeps the force partials, the per-step forces and the error
// word in one fixed device array declared below, whose address is looked up
// with cudaGetSymbolAddress on every call (a lookup allocates nothing once
// the module is loaded, and stays right after a device reset).
namespace {

constexpr int kNaSlots = 16384;     // force-partial slots (32-cell segments next to a wall)
constexpr int kNaChunk = 8;         // steps whose partials are reduced together
constexpr int kNaMaxSteps = 4096;   // steps per call
constexpr size_t kNaPartBytes = sizeof(double) * 3 * (size_t)kNaSlots * kNaChunk;   // 3 MiB
constexpr size_t kNaForceBytes = sizeof(double) * 3 * (size_t)kNaMaxSteps;          // 96 KiB
constexpr size_t kNaErrOffset = kNaPartBytes + kNaForceBytes;
constexpr size_t kNaBytes = kNaErrOffset + 256;   // error word and padding

// The scratch: partials | forces | error word.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Device address of the scratch on the current device. The first lookup on a
// device may load the module's device code, so it must not happen while a
// stream is being captured.
int noalloc_scratch(wt_lattice* h, unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaGetSymbolAddress(noalloc scratch)");
  *out = (unsigned char*)p;
  return WT_OK;
}

}  // namespace

extern "C" int wt_step_noalloc(wt_lattice* h, int nsteps, double* forces) {
  if (!h) return WT_ERR_ARG;
  if (nsteps < 0 || nsteps > kNaMaxSteps)
    return fail(h, WT_ERR_ARG, "wt_step_noalloc: nsteps must be in 0.." +
                                   std::to_string(kNaMaxSteps));
  if (h->nslots > kNaSlots)
    return fail(h, WT_ERR_UNSUPPORTED,
                "wt_step_noalloc: the body has " + std::to_string(h->nslots) +
                    " wall segments, more than the " + std::to_string(kNaSlots) +
                    " its fixed scratch holds; use wt_step");
  if (h->sfrac)
    return fail(h, WT_ERR_UNSUPPORTED, "wt_step_noalloc does not run partial bounce-back");
  int dev = -1;
  WT_CUDA(h, cudaGetDevice(&dev));
  if (dev != h->device)
    return fail(h, WT_ERR_STATE, "wt_step_noalloc: make the lattice's device current first");
  Path path = Path::Direct;
  int c = select_path(h, &path);   // the kernel wt_step runs for these parameters
  if (c != WT_OK) return c;
  unsigned char* base = nullptr;
  c = noalloc_scratch(h, &base);
  if (c != WT_OK) return c;
  if (nsteps == 0) {
    // set-up call: load every kernel a later call can launch, so that none
    // is loaded (which can need device memory) inside a later call
    WT_CUDA(h, wt::preload_step_kernels());
    return WT_OK;
  }
  double* part = (double*)base;
  double* fdev = (double*)(base + kNaPartBytes);
  unsigned* err = (unsigned*)(base + kNaErrOffset);
  // Only the error word must start at zero: every used partial slot and
  // every force entry is written before it is read.
  WT_CUDA(h, cudaMemsetAsync(err, 0, sizeof(unsigned), h->stream));
  dispatch_steps(h, nsteps, path, part, fdev, err, kNaChunk);
  WT_CUDA(h, cudaGetLastError());
  double last[3] = {0, 0, 0};
  unsigned errw = 0;
  if (forces)
    WT_CUDA(h, cudaMemcpyAsync(forces, fdev, sizeof(double) * 3 * (size_t)nsteps,
                               cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(last, fdev + 3 * (size_t)(nsteps - 1), sizeof(last),
                             cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaMemcpyAsync(&errw, err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  WT_CUDA(h, cudaStreamSynchronize(h->stream));
  h->steps += nsteps;
  h->force[0] = last[0]; h->force[1] = last[1]; h->force[2] = last[2];
  return check_err_word(h, errw);
}
