// wt_voxel.cu — Voxel.build (js/voxel.js:32-232) on the GPU.
//
// A triangle soup (float32, nine numbers per triangle, body space) becomes the
// body-space occupancy grid the device lookup (wt_voxelize_grid) samples: the
// cells the surface passes through (a sampled rasterisation of every
// triangle) OR'd with a two-of-three vote of ray-parity fills along x, y and
// z. This translation unit is compiled without multiply-add contraction and
// every step is float64 in the reference's operation order, so the grid is
// the reference's bit for bit.
//
// Kernels, per build:
//   k_vox_shell      one warp per triangle; lanes stride over the triangle's
//                    (u, v) sample rows and mark the shell cells
//   k_vox_ranges     per triangle its bucket rectangle in the plane normal to
//                    the ray axis (48 x 48 buckets at most, js/voxel.js:151-171)
//   k_vox_bucket     one warp per bucket walks the triangles in index order,
//                    32 at a time, counting (pass 0) or listing (pass 1) its
//                    members with ballot ranks, so each bucket lists its
//                    triangles in the reference's order; an exclusive scan of
//                    the counts runs in between (k_vox_scan)
//   k_vox_rays       one thread per ray (column): gathers the crossings of its
//                    bucket's triangles (at most 512, as the reference), sorts
//                    them, and adds a vote to the cells between alternate pairs
//   k_vox_combine    grid = (votes >= 2) | shell, with the solid and
//                    disagreeing-cell counts
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "wt_internal.h"

namespace {

constexpr int kBuckets = 48;
constexpr int kMaxHits = 512;
constexpr double kMaxSamples = 4096.0;

struct VoxGeom {
  int nx, ny, nz;
  double cell, inv;
  double min[3];
};

// ECMAScript ToInt32 of a finite or infinite double (js `x | 0`).
__device__ __forceinline__ int32_t to_int32(double v) {
  if (!isfinite(v)) return 0;
  if (v > -2147483649.0 && v < 2147483648.0) return (int32_t)v;
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}

__global__ void k_vox_shell(const float* __restrict__ P, long long ntri, VoxGeom g,
                            uint8_t* __restrict__ shell) {
  const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntri) return;
  const float* o = P + 9 * t;
  const double ax = o[0], ay = o[1], az = o[2], bx = o[3], by = o[4], bz = o[5];
  const double cx = o[6], cy = o[7], cz = o[8];
  const double inv = 1 / g.cell;
  const double e1 = fmax(fmax(fabs(bx - ax), fabs(by - ay)), fabs(bz - az));
  const double e2 = fmax(fmax(fabs(cx - ax), fabs(cy - ay)), fabs(cz - az));
  double n1 = ceil(e1 * inv * 2) + 1, n2 = ceil(e2 * inv * 2) + 1;
  if (n1 * n2 > kMaxSamples) {
    const double k = sqrt(kMaxSamples / (n1 * n2));
    n1 = fmax(2.0, (double)to_int32(n1 * k));
    n2 = fmax(2.0, (double)to_int32(n2 * k));
  }
  for (double i = lane; i <= n1; i += 32) {
    const double u = i / n1;
    const double jmax = ceil((1 - u) * n2);
    for (double j = 0; j <= jmax; j++) {
      const double v = fmin(j / n2, 1 - u);
      const double x = ax + (bx - ax) * u + (cx - ax) * v;
      const double y = ay + (by - ay) * u + (cy - ay) * v;
      const double z = az + (bz - az) * u + (cz - az) * v;
      const int32_t gx = to_int32((x - g.min[0]) * inv);
      const int32_t gy = to_int32((y - g.min[1]) * inv);
      const int32_t gz = to_int32((z - g.min[2]) * inv);
      if (gx < 0 || gy < 0 || gz < 0 || gx >= g.nx || gy >= g.ny || gz >= g.nz) continue;
      shell[gx + (long long)g.nx * (gy + (long long)g.ny * gz)] = 1;
    }
  }
}

struct AxisGeom {
  int A, B, C, nA, nB, nC, nbB, nbC;
  double minA, minB, minC, kB, kC, cell;
  long long strideA, strideB, strideC;
};

__global__ void k_vox_ranges(const float* __restrict__ P, long long ntri, AxisGeom x,
                             int4* __restrict__ rect) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ntri;
       t += (long long)gridDim.x * blockDim.x) {
    const float* o = P + 9 * t;
    const double b0 = o[x.B], b1 = o[3 + x.B], b2 = o[6 + x.B];
    const double c0 = o[x.C], c1 = o[3 + x.C], c2 = o[6 + x.C];
    double bl = floor((fmin(fmin(b0, b1), b2) - x.minB) * x.kB);
    double bh = floor((fmax(fmax(b0, b1), b2) - x.minB) * x.kB);
    double cl = floor((fmin(fmin(c0, c1), c2) - x.minC) * x.kC);
    double ch = floor((fmax(fmax(c0, c1), c2) - x.minC) * x.kC);
    bl = bl < 0 ? 0 : bl;
    bh = bh >= x.nbB ? x.nbB - 1 : bh;
    cl = cl < 0 ? 0 : cl;
    ch = ch >= x.nbC ? x.nbC - 1 : ch;
    // an empty rectangle (the triangle lies outside the buckets) is stored as one
    rect[t] = (bl > bh || cl > ch) ? make_int4(1, 0, 1, 0)
                                   : make_int4((int)bl, (int)bh, (int)cl, (int)ch);
  }
}

// pass 0: count[b] = members of bucket b; pass 1: items[start[b] ...] in
// triangle order. One warp per bucket: the lanes test 32 consecutive
// triangles at a time and a ballot gives each member its rank, so the list
// keeps the reference's order.
__global__ void k_vox_bucket(const int4* __restrict__ rect, long long ntri, int nbB, int nb,
                             int pass, int* __restrict__ count, const int* __restrict__ start,
                             int* __restrict__ items) {
  const int b = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (b >= nb) return;   // whole warps leave together
  const int bb = b % nbB, cc = b / nbB;
  int k = pass ? start[b] : 0;
  for (long long t0 = 0; t0 < ntri; t0 += 32) {
    const long long t = t0 + lane;
    bool hit = false;
    if (t < ntri) {
      const int4 r = rect[t];
      hit = bb >= r.x && bb <= r.y && cc >= r.z && cc <= r.w;
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (pass && hit) items[k + __popc(m & ((1u << lane) - 1u))] = (int)t;
    k += __popc(m);
  }
  if (!pass && lane == 0) count[b] = k;
}

// Exclusive scan of nb counts (one block; nb <= 48*48).
__global__ void k_vox_scan(const int* __restrict__ count, int nb, int* __restrict__ start) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int acc = 0;
    for (int b = 0; b < nb; b++) {
      start[b] = acc;
      acc += count[b];
    }
    start[nb] = acc;
  }
}

__global__ void k_vox_rays(const float* __restrict__ P, const int* __restrict__ start,
                           const int* __restrict__ items, AxisGeom x, uint8_t* __restrict__ votes,
                           double* __restrict__ scratch) {
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= (long long)x.nB * x.nC) return;
  const int ib = (int)(col % x.nB), ic = (int)(col / x.nB);
  const double pc = x.minC + (ic + 0.5003719) * x.cell;
  const int bc = (int)fmin((double)(x.nbC - 1), fmax(0.0, floor((pc - x.minC) * x.kC)));
  const double pb = x.minB + (ib + 0.4996281) * x.cell;
  const int bb = (int)fmin((double)(x.nbB - 1), fmax(0.0, floor((pb - x.minB) * x.kB)));
  const int s = start[bb + x.nbB * bc], e = start[bb + x.nbB * bc + 1];
  if (s == e) return;
  double* hits = scratch + col * kMaxHits;
  int nh = 0;
  for (int k = s; k < e && nh < kMaxHits; k++) {
    const float* o = P + 9 * (long long)items[k];
    const double b0 = o[x.B], c0 = o[x.C], b1 = o[3 + x.B], c1 = o[3 + x.C];
    const double b2 = o[6 + x.B], c2 = o[6 + x.C];
    const double d = (c1 - c2) * (b0 - b2) + (b2 - b1) * (c0 - c2);
    if (d == 0) continue;
    const double id = 1 / d;
    const double l0 = ((c1 - c2) * (pb - b2) + (b2 - b1) * (pc - c2)) * id;
    if (l0 < 0 || l0 > 1) continue;
    const double l1 = ((c2 - c0) * (pb - b2) + (b0 - b2) * (pc - c2)) * id;
    if (l1 < 0 || l1 > 1) continue;
    const double l2 = 1 - l0 - l1;
    if (l2 < 0 || l2 > 1) continue;
    hits[nh++] = l0 * (double)o[x.A] + l1 * (double)o[3 + x.A] + l2 * (double)o[6 + x.A];
  }
  if (nh < 2) return;
  for (int a = 1; a < nh; a++) {   // insertion sort: a ray crosses few triangles
    const double v = hits[a];
    int b = a - 1;
    while (b >= 0 && hits[b] > v) {
      hits[b + 1] = hits[b];
      b--;
    }
    hits[b + 1] = v;
  }
  const long long colBase = ib * x.strideB + ic * x.strideC;
  for (int k = 0; k + 1 < nh; k += 2) {
    double i0 = ceil((hits[k] - x.minA) / x.cell - 0.5);
    double i1 = floor((hits[k + 1] - x.minA) / x.cell - 0.5);
    if (i0 < 0) i0 = 0;
    if (i1 >= x.nA) i1 = x.nA - 1;
    for (double ia = i0; ia <= i1; ia++) votes[colBase + (long long)ia * x.strideA]++;
  }
}

__global__ void k_vox_combine(const uint8_t* __restrict__ votes, const uint8_t* __restrict__ shell,
                              long long n, uint8_t* __restrict__ grid,
                              unsigned long long* __restrict__ counts) {
  unsigned long long solid = 0, disagree = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = votes[i];
    const bool inside = v >= 2 || shell[i] == 1;
    solid += inside;
    disagree += (v == 1 || v == 2);
    grid[i] = inside ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    solid += __shfl_down_sync(0xffffffffu, solid, o);
    disagree += __shfl_down_sync(0xffffffffu, disagree, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counts[0], solid);
    atomicAdd(&counts[1], disagree);
  }
}

thread_local std::string g_vox_error;

int vox_fail(int code, const std::string& msg) {
  g_vox_error = msg;
  return code;
}

// Device buffers of one build, released on every exit path.
struct VoxBuffers {
  std::vector<void*> ptrs;
  void* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n ? n : 1) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return p;
  }
  ~VoxBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
};

}  // namespace

extern "C" {

const char* wt_voxel_last_error(void) { return g_vox_error.c_str(); }

int wt_voxel_dims(const float* tris, int64_t ntri, int res, wt_voxel_info* info) {
  g_vox_error.clear();
  if (!info || (ntri > 0 && !tris)) return vox_fail(WT_ERR_ARG, "tris and info are required");
  if (res <= 0) res = 96;
  if (ntri <= 0) return vox_fail(WT_ERR_ARG, "Mesh has no triangles.");
  // js/voxel.js:32-42 (bounds) and :48-71
  double x0 = INFINITY, y0 = INFINITY, z0 = INFINITY;
  double x1 = -INFINITY, y1 = -INFINITY, z1 = -INFINITY;
  for (int64_t i = 0; i < 9 * ntri; i += 3) {
    const double x = tris[i], y = tris[i + 1], z = tris[i + 2];
    if (x < x0) x0 = x;
    if (x > x1) x1 = x;
    if (y < y0) y0 = y;
    if (y > y1) y1 = y;
    if (z < z0) z0 = z;
    if (z > z1) z1 = z;
  }
  const double sx = x1 - x0, sy = y1 - y0, sz = z1 - z0;
  const double span = fmax(fmax(sx, sy), sz);
  if (!(span > 0)) return vox_fail(WT_ERR_ARG, "Mesh is degenerate (zero size).");
  const double cell = span / res;
  const double dx = fmax(3, ceil(sx / cell) + 4), dy = fmax(3, ceil(sy / cell) + 4),
               dz = fmax(3, ceil(sz / cell) + 4);
  if (dx * dy * dz > 40e6)
    return vox_fail(WT_ERR_ARG, "Voxel grid too large; lower the resolution.");
  memset(info, 0, sizeof(*info));
  info->nx = (int32_t)dx;
  info->ny = (int32_t)dy;
  info->nz = (int32_t)dz;
  info->tris = ntri;
  info->cell = cell;
  info->inv = 1 / cell;
  info->min[0] = x0 - (info->nx * cell - sx) * 0.5;
  info->min[1] = y0 - (info->ny * cell - sy) * 0.5;
  info->min[2] = z0 - (info->nz * cell - sz) * 0.5;
  info->ext[0] = sx * 0.5; info->ext[1] = sy * 0.5; info->ext[2] = sz * 0.5;
  info->centre[0] = (x0 + x1) * 0.5; info->centre[1] = (y0 + y1) * 0.5;
  info->centre[2] = (z0 + z1) * 0.5;
  info->bbox[0] = x0; info->bbox[1] = y0; info->bbox[2] = z0;
  info->bbox[3] = x1; info->bbox[4] = y1; info->bbox[5] = z1;
  return WT_OK;
}

int wt_voxel_build(const float* tris, int64_t ntri, int res, uint8_t* grid, size_t grid_len,
                   wt_voxel_info* info) {
  int c = wt_voxel_dims(tris, ntri, res, info);
  if (c != WT_OK) return c;
  const long long n = (long long)info->nx * info->ny * info->nz;
  if (!grid || grid_len != (size_t)n)
    return vox_fail(WT_ERR_ARG, "grid must hold nx*ny*nz = " + std::to_string(n) + " bytes");
  VoxBuffers mem;
  float* P = (float*)mem.get(sizeof(float) * 9 * (size_t)ntri);
  uint8_t* shell = (uint8_t*)mem.get((size_t)n);
  uint8_t* votes = (uint8_t*)mem.get((size_t)n);
  uint8_t* gdev = (uint8_t*)mem.get((size_t)n);
  int4* rect = (int4*)mem.get(sizeof(int4) * (size_t)ntri);
  unsigned long long* counts = (unsigned long long*)mem.get(2 * sizeof(unsigned long long));
  const int dim[3] = {info->nx, info->ny, info->nz};
  long long maxcols = 0;
  for (int A = 0; A < 3; A++) {
    const long long cols = (long long)dim[(A + 1) % 3] * dim[(A + 2) % 3];
    maxcols = cols > maxcols ? cols : maxcols;
  }
  double* scratch = (double*)mem.get(sizeof(double) * kMaxHits * (size_t)maxcols);
  int* bcount = (int*)mem.get(sizeof(int) * kBuckets * kBuckets);
  int* bstart = (int*)mem.get(sizeof(int) * (kBuckets * kBuckets + 1));
  if (!P || !shell || !votes || !gdev || !rect || !counts || !scratch || !bcount || !bstart)
    return vox_fail(WT_ERR_OOM, "cannot allocate the voxel build's device buffers");
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    return vox_fail(WT_ERR_CUDA, "cannot create a stream");
  auto done = [&](int code, const std::string& msg) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return code == WT_OK ? code : vox_fail(code, msg);
  };
  cudaMemcpyAsync(P, tris, sizeof(float) * 9 * (size_t)ntri, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(shell, 0, (size_t)n, s);
  cudaMemsetAsync(votes, 0, (size_t)n, s);
  cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s);
  VoxGeom g{info->nx, info->ny, info->nz, info->cell, info->inv,
            {info->min[0], info->min[1], info->min[2]}};
  k_vox_shell<<<(unsigned)((ntri * 32 + 255) / 256), 256, 0, s>>>(P, ntri, g, shell);
  for (int A = 0; A < 3; A++) {
    AxisGeom x;
    x.A = A; x.B = (A + 1) % 3; x.C = (A + 2) % 3;
    x.nA = dim[x.A]; x.nB = dim[x.B]; x.nC = dim[x.C];
    x.cell = info->cell;
    x.minA = info->min[x.A]; x.minB = info->min[x.B]; x.minC = info->min[x.C];
    x.nbB = x.nB < kBuckets ? x.nB : kBuckets;
    x.nbC = x.nC < kBuckets ? x.nC : kBuckets;
    x.kB = x.nbB / (x.nB * info->cell);
    x.kC = x.nbC / (x.nC * info->cell);
    auto stride = [&](int a) -> long long {
      return a == 0 ? 1 : (a == 1 ? dim[0] : (long long)dim[0] * dim[1]);
    };
    x.strideA = stride(x.A); x.strideB = stride(x.B); x.strideC = stride(x.C);
    const int nb = x.nbB * x.nbC;
    k_vox_ranges<<<(unsigned)std::min<long long>((ntri + 255) / 256, 4096), 256, 0, s>>>(
        P, ntri, x, rect);
    k_vox_bucket<<<(nb * 32 + 127) / 128, 128, 0, s>>>(rect, ntri, x.nbB, nb, 0, bcount,
                                                        nullptr, nullptr);
    k_vox_scan<<<1, 32, 0, s>>>(bcount, nb, bstart);
    int total = 0;
    cudaMemcpyAsync(&total, bstart + nb, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return done(WT_ERR_CUDA, "voxel bucketing failed");
    VoxBuffers items_mem;
    int* items = (int*)items_mem.get(sizeof(int) * (size_t)(total > 0 ? total : 1));
    if (!items) return done(WT_ERR_OOM, "cannot allocate the bucket lists");
    k_vox_bucket<<<(nb * 32 + 127) / 128, 128, 0, s>>>(rect, ntri, x.nbB, nb, 1, nullptr,
                                                        bstart, items);
    const long long cols = (long long)x.nB * x.nC;
    k_vox_rays<<<(unsigned)((cols + 127) / 128), 128, 0, s>>>(P, bstart, items, x, votes,
                                                              scratch);
    if (cudaStreamSynchronize(s) != cudaSuccess) return done(WT_ERR_CUDA, "voxel ray pass failed");
  }
  k_vox_combine<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, s>>>(
      votes, shell, n, gdev, counts);
  unsigned long long hc[2] = {0, 0};
  cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(grid, gdev, (size_t)n, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return done(WT_ERR_CUDA, "voxel build failed");
  info->solid = (int64_t)hc[0];
  info->openness = hc[0] ? (double)hc[1] / (double)hc[0] : 0.0;
  return done(WT_OK, "");
}

}  // extern "C"
