// wt_kernels_fast.cu — float32-arithmetic instantiations of the fused step
// (float32 and half-deviation storage), plus the force reduction. Built with
// the default multiply-add contraction.
#include "wt_internal.h"
#include "wt_staged_launch.cuh"
#include "wt_pipe.cuh"
#include "wt_vec.cuh"
#include "wt_x2.cuh"
#include "wt_tma.cuh"
#include "wt_pbb.cuh"
#include "wt_lean.cuh"
#include "wt_h2.cuh"
#include "wt_tile.cuh"

#include <algorithm>

namespace wt {

void launch_step_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) k_step<float, false, long long><<<grid, STEP_BX, 0, s>>>(a);
  else k_step<float, false, int><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_step_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) k_step<__half, false, long long><<<grid, STEP_BX, 0, s>>>(a);
  else k_step<__half, false, int><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_vec_f32(const StepArgs<float>& a, bool wide, cudaStream_t s) {
  const dim3 g = vec_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_vec<float, long long><<<g, VEC_BX, 0, s>>>(a);
  else k_step_vec<float, int><<<g, VEC_BX, 0, s>>>(a);
}

void launch_vec_f16(const StepArgs<__half>& a, bool wide, cudaStream_t s) {
  const dim3 g = vec_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_vec<__half, long long><<<g, VEC_BX, 0, s>>>(a);
  else k_step_vec<__half, int><<<g, VEC_BX, 0, s>>>(a);
}

void launch_x2_f32(const StepArgs<float>& a, bool wide, cudaStream_t s) {
  const dim3 g = x2_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_x2<float, long long><<<g, X2_BX, 0, s>>>(a);
  else k_step_x2<float, int><<<g, X2_BX, 0, s>>>(a);
}

void launch_x2_f16(const StepArgs<__half>& a, bool wide, cudaStream_t s) {
  const dim3 g = x2_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_x2<__half, long long><<<g, X2_BX, 0, s>>>(a);
  else k_step_x2<__half, int><<<g, X2_BX, 0, s>>>(a);
}

void launch_lean_f32(const StepArgs<float>& a, dim3 grid, bool, cudaStream_t s) {
  k_step_lean<float><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_lean_f16(const StepArgs<__half>& a, dim3 grid, bool, cudaStream_t s) {
  k_step_lean<__half><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_tile_f32(const StepArgs<float>& a, dim3 grid, bool, cudaStream_t s) {
  k_step_tile<float><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_tile_f16(const StepArgs<__half>& a, dim3 grid, bool, cudaStream_t s) {
  k_step_tile<__half><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_pair_f16(const StepArgs<__half>& a, dim3, bool, cudaStream_t s) {
  const dim3 g((unsigned)((a.nx + 2 * H2_BX - 1) / (2 * H2_BX)), (unsigned)a.ny, (unsigned)a.nz);
  k_step_h2<true><<<g, H2_BX, 0, s>>>(a);
}

// ---- partial bounce-back and adjoint (float32 arithmetic) -------------------------

void launch_pbb_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) k_step_pbb<float, false, long long><<<grid, STEP_BX, 0, s>>>(a);
  else k_step_pbb<float, false, int><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_pbb_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s) {
  if (wide) k_step_pbb<__half, false, long long><<<grid, STEP_BX, 0, s>>>(a);
  else k_step_pbb<__half, false, int><<<grid, STEP_BX, 0, s>>>(a);
}

void launch_adj_f32(const StepArgs<float>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s) {
  launch_adjoint<float, float>(a, Tn, Tc, ds, wJ, comp, s);
}

void launch_adj_f16(const StepArgs<__half>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s) {
  launch_adjoint<__half, float>(a, Tn, Tc, ds, wJ, comp, s);
}

// ---- TMA tile kernel ------------------------------------------------------------

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, found through the runtime (libwt.so
// links only cudart).
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

template <class S>
bool encode_maps(void* const buf[2], int nx, int ny, int nz, TmaMaps* out) {
  using C = Tma<S>;
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const CUtensorMapDataType dt =
      sizeof(S) == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)Q};
  const cuuint64_t strides[3] = {(cuuint64_t)nx * sizeof(S), (cuuint64_t)nx * ny * sizeof(S),
                                 (cuuint64_t)nx * ny * nz * sizeof(S)};
  // Tile geometry. A row of at most 256 cells whose 32-cell segments pair up
  // in warps (nx a multiple of 64) is one tile wide: its boxes need no halo,
  // since the first and last cells of a row pull nothing. Otherwise tiles are
  // 128 cells wide and their boxes carry a 16-byte halo on each side.
  int tx, h;
  if (nx <= 256 && nx % 64 == 0) { tx = nx; h = 0; }
  else { tx = 128; h = C::HALO; }
  const int ty = C::CELLS / tx;
  const int bw = tx + 2 * h;
  const int pad = C::PAD;
  out->tx = tx; out->ty = ty; out->bw = bw; out->h = h;
  out->in_slot = (ty * bw + pad - 1) / pad * pad;
  out->out_slot = (ty * tx + pad - 1) / pad * pad;
  out->gx = (nx + tx - 1) / tx;
  out->gy = (ny + ty - 1) / ty;
  if (out->in_slot > C::IN_SLOT_MAX || out->out_slot > C::OUT_SLOT_MAX) return false;
  const cuuint32_t box_ld[4] = {(cuuint32_t)bw, (cuuint32_t)ty, 1, 1};
  const cuuint32_t box_st[4] = {(cuuint32_t)tx, (cuuint32_t)ty, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int b = 0; b < 2; b++) {
    if (fn(&out->ld[b], dt, 4, buf[b], dims, strides, box_ld, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    if (fn(&out->st[b], dt, 4, buf[b], dims, strides, box_st, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

template <class S>
void launch_tma(const StepArgs<S>& a, const TmaMaps& m, int ld_buf, cudaStream_t s) {
  using C = Tma<S>;
  constexpr int kMaxDevices = 64;
  static int grid_of[kMaxDevices] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  int& grid = grid_of[dev % kMaxDevices];
  if (grid == 0) {
    cudaFuncSetAttribute(k_step_tma<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)C::SMEM);
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_step_tma<S>, C::THREADS, C::SMEM);
    grid = std::max(1, sms * std::max(per, 1));
  }
  const long long ntiles = (long long)m.gx * m.gy * a.nz;
  const long long g = std::min<long long>(grid, ntiles);
  k_step_tma<S><<<(unsigned)g, C::THREADS, C::SMEM, s>>>(a, m, ld_buf, ld_buf ^ 1, ntiles);
}

}  // namespace

bool tma_supported(int storage, int nx) {
  if (storage == WT_STORE_F32) return nx % 4 == 0;
  if (storage == WT_STORE_F16DEV) return nx % 8 == 0;
  return false;
}

bool make_tma_maps(int storage, void* const buf[2], int nx, int ny, int nz, TmaMaps* out) {
  if (!tma_supported(storage, nx)) return false;
  if (storage == WT_STORE_F32) return encode_maps<float>(buf, nx, ny, nz, out);
  return encode_maps<__half>(buf, nx, ny, nz, out);
}

void launch_tma_f32(const StepArgs<float>& a, const TmaMaps& m, int ld_buf, cudaStream_t s) {
  launch_tma<float>(a, m, ld_buf, s);
}

void launch_tma_f16(const StepArgs<__half>& a, const TmaMaps& m, int ld_buf, cudaStream_t s) {
  launch_tma<__half>(a, m, ld_buf, s);
}

void launch_pipe_f32(const StepArgs<float>& a, bool wide, cudaStream_t s) {
  const dim3 g = pipe_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_pipe<float, long long><<<g, STEP_BX, 0, s>>>(a);
  else k_step_pipe<float, int><<<g, STEP_BX, 0, s>>>(a);
}

void launch_pipe_f16(const StepArgs<__half>& a, bool wide, cudaStream_t s) {
  const dim3 g = pipe_grid(a.nx, a.ny, a.nz);
  if (wide) k_step_pipe<__half, long long><<<g, STEP_BX, 0, s>>>(a);
  else k_step_pipe<__half, int><<<g, STEP_BX, 0, s>>>(a);
}

void launch_staged_f32_fast(const StepArgs<float>& a, cudaStream_t s) {
  launch_staged<float, false>(a, s);
}

void launch_staged_f16_fast(const StepArgs<__half>& a, cudaStream_t s) {
  launch_staged<__half, false>(a, s);
}

// Marks the 32-cell segments that hold at least one near-wall cell.
__global__ void k_mark_segments(const uint8_t* __restrict__ flags, int nx, int ny, int nz,
                             uint8_t* __restrict__ mark) {
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (flags[i] & FLAG_NEAR) {
      const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
      mark[seg_of(x, y, z, nx, ny)] = 1;
    }
  }
}

void launch_mark_segments(const uint8_t* flags, int nx, int ny, int nz, uint8_t* mark,
                          cudaStream_t s) {
  k_mark_segments<<<148 * 16, 256, 0, s>>>(flags, nx, ny, nz, mark);
}

// One block per step; each thread sums a fixed strided subset of the warp
// partials, then a fixed-shape tree combines them. The order never depends
// on timing, so the force series is reproducible run to run.
constexpr int RED_T = 256;

__global__ void __launch_bounds__(RED_T) k_force_reduce(const double* __restrict__ part,
                                                        unsigned nblocks,
                                                        double* __restrict__ out) {
  __shared__ double sm[3][RED_T];
  const double* p = part + (size_t)blockIdx.x * nblocks * 3;
  double ax = 0, ay = 0, az = 0;
  for (unsigned b = threadIdx.x; b < nblocks; b += RED_T) {
    ax += p[3 * (size_t)b];
    ay += p[3 * (size_t)b + 1];
    az += p[3 * (size_t)b + 2];
  }
  sm[0][threadIdx.x] = ax;
  sm[1][threadIdx.x] = ay;
  sm[2][threadIdx.x] = az;
  __syncthreads();
  for (int w = RED_T / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sm[0][threadIdx.x] += sm[0][threadIdx.x + w];
      sm[1][threadIdx.x] += sm[1][threadIdx.x + w];
      sm[2][threadIdx.x] += sm[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[3 * (size_t)blockIdx.x] = sm[0][0];
    out[3 * (size_t)blockIdx.x + 1] = sm[1][0];
    out[3 * (size_t)blockIdx.x + 2] = sm[2][0];
  }
}

void launch_force_reduce(const double* part, unsigned nslots, int nsteps, double* out,
                         cudaStream_t s) {
  k_force_reduce<<<nsteps, RED_T, 0, s>>>(part, nslots, out);
}

}  // namespace wt
