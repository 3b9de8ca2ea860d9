// wt_internal.h — the handle behind wt_lattice* and the kernel launchers
// shared by the translation units of libwt.so.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/wt.h"
#include "wt_common.cuh"

struct wt_lattice {
  int nx = 0, ny = 0, nz = 0, storage = 0;
  long long n = 0;
  int device = 0;
  long long pf = 0;              // L2 prefetch distance of the lean kernel (cells)
  size_t elem = 4;               // bytes per stored population
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;    // second stream of wt_adjoint (recomputation), made on first use
  void* buf[2] = {nullptr, nullptr};  // population buffers A and B (js/lbm.js:74-75)
  int parity = 0;                // js/lbm.js:80: f = parity ? B : A
  uint8_t* flags = nullptr;      // solid code (bits 0-1) | near bit (bit 2)
  unsigned long long* nmask = nullptr;  // near-wall cells: solid / body neighbour bits
  float* ux = nullptr;
  float* uy = nullptr;
  float* uz = nullptr;
  float* rho = nullptr;
  float* uwx = nullptr;          // wall velocities of solid cells (js/lbm.js:92-94)
  float* uwy = nullptr;
  float* uwz = nullptr;
  // per-step force reduction: one partial per 32-cell segment holding a near-wall cell
  long long nsegs = 0;           // 32-cell row segments of the lattice
  int* wslot = nullptr;          // per segment: partial slot or -1
  int nslots = 0;                // segments with a slot
  int part_cap = 0;              // slots that fit in `part` (per step of a chunk)
  double* part = nullptr;
  double* forces_dev = nullptr;
  double* forces_host = nullptr; // pinned
  int forces_cap = 0;            // steps that fit in forces_dev / forces_host
  unsigned* err_dev = nullptr;
  unsigned* err_host = nullptr;  // pinned
  double* sfrac = nullptr;       // partial bounce-back solid fraction on sbox (device), or null
  void* adj_pool = nullptr;      // device memory a wt_adjoint run with keep left for the next
  size_t adj_pool_bytes = 0;
  int sbox[6] = {0, 0, 0, 0, 0, 0};
  // voxelize statistics scratch
  uint8_t* col = nullptr;        // ny*nz frontal projection
  uint8_t* plan = nullptr;       // nx*nz planform projection
  int* low = nullptr;            // nx*nz lowest body cell per column
  int* counters = nullptr;       // [0] body cells, [1] wall velocity seen
  // host-side state
  wt_params p{};
  wt_body_stats stats{};
  double force[3] = {0, 0, 0};
  int64_t steps = 0;
  int64_t launches = 0;
  std::string err;
};

namespace wt {

// Step launchers (one per storage x arithmetic pair that is provided).
// `wide` selects 64-bit direction offsets (19*n beyond 31 bits).
void launch_step_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_step_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_step_f32_exact(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_step_f64_exact(const StepArgs<double>& a, dim3 grid, bool wide, cudaStream_t s);

// Partial bounce-back step (direct, one thread per cell) and one step of
// its discrete adjoint. The adjoint arithmetic is float64 for float64
// storage or the exact collision, float32 otherwise.
void launch_pbb_f32_fast(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_pbb_f16_fast(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_pbb_f32_exact(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_pbb_f64_exact(const StepArgs<double>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_adj_f32(const StepArgs<float>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s);
void launch_adj_f16(const StepArgs<__half>& a, const float* Tn, float* Tc, double* ds, double wJ,
                    int comp, cudaStream_t s);
void launch_adj_f32x(const StepArgs<float>& a, const double* Tn, double* Tc, double* ds,
                     double wJ, int comp, cudaStream_t s);
void launch_adj_f64(const StepArgs<double>& a, const double* Tn, double* Tc, double* ds,
                    double wJ, int comp, cudaStream_t s);

// One thread per cell with 32-bit byte offsets from one pointer per cell;
// float32 collision, buffers under 2^31 bytes (wide is ignored).
void launch_lean_f32(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_lean_f16(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s);

// Two adjacent cells per thread with the packed float32x2 collision; the
// lean kernel's conditions and an even nx (grid is ignored).
void launch_pair_f16(const StepArgs<__half>& a, dim3 grid, bool wide, cudaStream_t s);
void launch_pair_f32(const StepArgs<float>& a, dim3 grid, bool wide, cudaStream_t s);

// Launch attributes of the step kernels (the pair kernels' L1 carveout), set
// once per lattice creation.
cudaError_t configure_step_kernels();

// Load the device code of every step and reduction kernel a wt_step call can
// launch (cudaFuncGetAttributes on each), so that none is loaded lazily
// inside a later call. The exact variant covers the --fmad=false unit.
cudaError_t preload_step_kernels();
cudaError_t preload_exact_step_kernels();

// Deterministic per-step sum of the warp partials: out[3*s..3*s+2].
void launch_force_reduce(const double* part, unsigned nslots, int nsteps, double* out,
                         cudaStream_t s);

// mark[s] = 1 for every 32-cell segment s holding a near-wall cell.
void launch_mark_segments(const uint8_t* flags, int nx, int ny, int nz, uint8_t* mark,
                          cudaStream_t s);

// Equilibrium initialisation of both buffers and the fields:
// mode 0 = reset(), mode 1 = reset() + seeded noise.
void launch_init(wt_lattice* h, int mode, uint64_t seed, double amp);

// voxelize pieces (js/lbm.js:197-214, :225-246, :268-282).
void launch_clear_obj(wt_lattice* h);
void launch_floor(wt_lattice* h, int ground, double road_vel);
void launch_box_mask(wt_lattice* h, const int rg[6], const uint8_t* mask_dev,
                     const uint8_t* wall_set_dev, const double* wall_vel_dev);
void launch_box_grid(wt_lattice* h, const int rg[6], const uint8_t* grid_dev, int gnx, int gny,
                     int gnz, const double gmin[3], double ginv, const double M[9],
                     const double P[3], double scale);
void launch_near(wt_lattice* h);

// Population conversion to float32 / float64 deviations.
void launch_convert(const void* src, int storage, void* dst, int dtype, long long count,
                    cudaStream_t s);
void launch_convert_in(const void* src, int dtype, void* dst, int storage, long long count,
                       cudaStream_t s);

// Trilinear velocity sample of js/lbm.js:515-539 for npts points.
void launch_sample(wt_lattice* h, const double* xyz_dev, int npts, double* out_dev);

// Equilibrium deviation at rho=1, u=(u0,0,0) per direction, in float64 with
// the operation order of js/lbm.js:155-162.
void eq_u0_table(double u0, double out[19]);

}  // namespace wt
