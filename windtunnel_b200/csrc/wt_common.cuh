// wt_common.cuh — D3Q19 lattice constants, storage formats and the
// parameter blocks shared by every kernel of libwt.so.
#pragma once

#include <utility>

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wt.h"

namespace wt {

constexpr int Q = 19;
constexpr int FLAG_SOLID_MASK = 3;  // low two bits: WT_FLUID / WT_SOLID_OBJ / WT_SOLID_WALL
constexpr int FLAG_NEAR = 4;        // bit 2: fluid interior cell with a solid neighbour

// Direction set of js/lbm.js:29-33 (the order is part of the f-buffer layout).
__host__ __device__ constexpr int ex(int q) {
  constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  return t[q];
}
__host__ __device__ constexpr int ey(int q) {
  constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
  return t[q];
}
__host__ __device__ constexpr int ez(int q) {
  constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  return t[q];
}
__host__ __device__ constexpr int opp(int q) {
  constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
  return t[q];
}
// Mirror images in y and in z (free-slip side planes).
__host__ __device__ constexpr int mirror_y(int q) {
  constexpr int t[Q] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
  return t[q];
}
__host__ __device__ constexpr int mirror_z(int q) {
  constexpr int t[Q] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
  return t[q];
}
// The opposite and mirror tables must be the index maps they claim to be.
constexpr bool direction_tables_consistent() {
  for (int q = 0; q < Q; q++) {
    if (ex(opp(q)) != -ex(q) || ey(opp(q)) != -ey(q) || ez(opp(q)) != -ez(q)) return false;
    const int my = mirror_y(q), mz = mirror_z(q);
    if (ex(my) != ex(q) || ey(my) != -ey(q) || ez(my) != ez(q)) return false;
    if (ex(mz) != ex(q) || ey(mz) != ey(q) || ez(mz) != -ez(q)) return false;
  }
  return true;
}
static_assert(direction_tables_consistent(), "D3Q19 opposite / mirror tables are inconsistent");

// Lattice weights (js/lbm.js:34-37), as the IEEE doubles 1/3, 1/18, 1/36.
__host__ __device__ constexpr double wq(int q) {
  return q == 0 ? 1.0 / 3 : (q <= 6 ? 1.0 / 18 : 1.0 / 36);
}

// ---- storage formats -------------------------------------------------------
// Each trait converts between the stored deviation and the arithmetic type.
template <class S>
struct Store;

template <>
struct Store<float> {
  static constexpr int kind = WT_STORE_F32;
  __device__ __forceinline__ static float load_f(float v) { return v; }
  __device__ __forceinline__ static double load_d(float v) { return (double)v; }
  __device__ __forceinline__ static float from_f(float v) { return v; }
  __device__ __forceinline__ static float from_d(double v) { return __double2float_rn(v); }
};

template <>
struct Store<double> {
  static constexpr int kind = WT_STORE_F64;
  __device__ __forceinline__ static float load_f(double v) { return (float)v; }
  __device__ __forceinline__ static double load_d(double v) { return v; }
  __device__ __forceinline__ static double from_f(float v) { return (double)v; }
  __device__ __forceinline__ static double from_d(double v) { return v; }
};

// Half-precision deviations, scaled by WT_F16_SCALE (a power of two, so the
// scaling itself is exact).
template <>
struct Store<__half> {
  static constexpr int kind = WT_STORE_F16DEV;
  __device__ __forceinline__ static float load_f(__half v) {
    return __half2float(v) * (float)(1.0 / WT_F16_SCALE);
  }
  __device__ __forceinline__ static double load_d(__half v) { return (double)load_f(v); }
  __device__ __forceinline__ static __half from_f(float v) {
    return __float2half_rn(v * (float)WT_F16_SCALE);
  }
  __device__ __forceinline__ static __half from_d(double v) {
    return __double2half(v * WT_F16_SCALE);
  }
};

// ---- per-launch parameter block of the fused step --------------------------
template <class S>
struct StepArgs {
  const S* F;          // populations read (current f)
  S* G;                // populations written (next f)
  const uint8_t* flags;
  const unsigned long long* nmask;  // per near-wall cell: solid neighbours (bits q), body (bits 32+q)
  float* ux;
  float* uy;
  float* uz;
  float* rho;
  const float* uwx;
  const float* uwy;
  const float* uwz;
  double* part;        // this step's force partials, 3 per warp slot
  const int* wslot;    // per warp of the grid: its partial slot, or -1 (no wall cell)
  unsigned* err;       // bit 0: non-finite / non-positive density; bit 1: stale slot table
  int nx, ny, nz;
  long long n;         // nx*ny*nz
  long long nxy;       // nx*ny
  long long src[Q];    // pull offset of direction q: q*n - (ex + nx*ey + nxy*ez)
  long long dst[Q];    // store offset of direction q: q*n
  // src[q] and dst[q] in bytes, when both buffers span < 2^31 bytes; both are
  // non-negative for every lattice of at least 3 cells per axis, and unsigned
  // so that adding one to a pointer needs no sign extension
  uint32_t srcb[Q];
  uint32_t dstb[Q];
  // float64 parameters (exact collision)
  double tau0, omega0, cs2, lam;
  // float32 parameters (fast collision), rounded once on the host
  float tau0f, omega0f, omm0f, les_cf, lamf, u0f;
  int les, trt, mov, freeslip, write_fields;
  int f16_sr;          // half storage: stochastic instead of nearest rounding
  unsigned sr_seed;    // per-step seed of the stochastic rounding
  int gx;              // x-segments (units) per row
  long long units;     // gx*ny*nz
  S eq[Q];             // equilibrium deviation at rho=1, u=(u0,0,0), rounded to S
  uint32_t eq2[Q];     // half storage: eq[q] in both halves of a 32-bit word
  const double* sfrac; // partial bounce-back: solid fraction on the box sb (x fastest), or null
  int sb[6];           // its half-open box x0, y0, z0, x1, y1, z1
  long long pf;        // L2 prefetch distance in cells (0: none), see prefetch_ahead
};

// Ask L2 for the populations that the warp pf cells further on in launch
// order will pull: lane q < 19 prefetches the line holding the first of that
// warp's 32 pulled values of direction q (the warp beside it covers the rest
// of a line its values straddle). Issued by a warp before its own loads, it
// keeps DRAM requests in flight for cells whose blocks have not started yet.
template <class S>
__device__ __forceinline__ void prefetch_ahead(const StepArgs<S>& a, long long warp_cell0) {
  const int lane = threadIdx.x & 31;
  if (a.pf <= 0 || lane >= 19) return;
  const long long e = warp_cell0 + a.pf + a.src[lane];
  if (e >= 0 && e < 19 * a.n) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.F + e));
}

// Programmatic dependent launch. A step kernel launched by launch_pdl (the
// programmatic stream-serialization attribute) may have its blocks
// dispatched into the SM slots the previous grid in the stream frees while
// that grid's last blocks still run; pdl_enter, the kernel's first
// statement, waits until the previous grid has completed and its stores are
// visible, then lets the next grid launch. Launched without the attribute
// both instructions return at once. A launch error is recorded for
// cudaGetLastError like that of any launch.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... P, class... A>
inline void launch_pdl(void (*k)(P...), dim3 grid, dim3 block, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// Block shape of the fused step: one thread per cell along x.
constexpr int STEP_BX = 128;
constexpr int STEP_WARPS = STEP_BX / 32;

inline dim3 step_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nx + STEP_BX - 1) / STEP_BX), (unsigned)ny, (unsigned)nz);
}

// Force-partial segment of cell (x, y, z): 32 consecutive cells of a row.
// Every step kernel reduces its momentum exchange per segment, so one slot
// table (built by voxelize for the segments holding a near-wall cell) serves
// them all.
__host__ __device__ inline long long seg_of(int x, int y, int z, int nx, int ny) {
  const int nseg = (nx + 31) / 32;
  return ((long long)z * ny + y) * nseg + x / 32;
}

}  // namespace wt
