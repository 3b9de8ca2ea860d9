/*
 * wt.h — C ABI of the B200 D3Q19 lattice-Boltzmann step (libwt.so).
 *
 * This is the drop-in boundary for windtunnel's solver core, js/lbm.js
 * (the `LBM` class, js/lbm.js:51-550) and its batched CPU executor
 * (`LBMPool.Pool.step`, js/pool.js:97-125). Every entry point below names
 * the reference member it replaces. Host bindings (the Python mirror in
 * windtunnel_b200/lbm.py, an N-API addon for Node) are thin layers over it.
 *
 * Conventions
 *   - Every call returns an int status: WT_OK (0) or a negative WT_ERR_*.
 *     The message of the last failure is kept per handle (wt_last_error).
 *   - Host pointers are borrowed for the duration of the call only. The
 *     library owns all device memory of a handle.
 *   - One handle is used by one host thread at a time (not locked). Each
 *     handle owns one CUDA stream; calls are synchronous unless stated.
 *   - Lattice layout (js/lbm.js:20-23, :142): cell i = x + nx*(y + ny*z);
 *     populations are structure-of-arrays, f[q*n + i], stored as deviations
 *     f_q - w_q from the rest state, in the 19-direction order of
 *     js/lbm.js:29-33.
 */
#ifndef WT_H
#define WT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WT_Q 19

/* Status codes. */
enum {
  WT_OK = 0,
  WT_ERR_ARG = -1,         /* bad argument: dims, sizes, null pointers, ranges */
  WT_ERR_OOM = -2,         /* device (or pinned host) allocation failed */
  WT_ERR_CUDA = -3,        /* a CUDA runtime call failed */
  WT_ERR_DIVERGED = -4,    /* a step produced a non-finite or non-positive density */
  WT_ERR_TIMEOUT = -5,     /* a bounded device-side wait gave up (no current kernel waits) */
  WT_ERR_STATE = -6,       /* call not valid in the handle's current state */
  WT_ERR_UNSUPPORTED = -7  /* option combination not provided */
};

/* Population storage formats. */
enum {
  WT_STORE_F32 = 0,    /* float32 deviations, as the reference's Float32Array (js/lbm.js:74-75) */
  WT_STORE_F16DEV = 1, /* IEEE half deviations, scaled by WT_F16_SCALE (a power of two) */
  WT_STORE_F64 = 2     /* float64 deviations (the FP64 oracle form) */
};

/* Scale applied to deviations before they are rounded to half precision:
 * 2^12 keeps the ~1e-6..1e-1 deviation range of a low-Mach flow inside
 * half's normal range (6.1e-5 .. 65504) without changing relative precision. */
#define WT_F16_SCALE 4096.0

/* Arithmetic inside the step kernel. */
enum {
  WT_MATH_FAST = 0,  /* float32 collision, re-associated for fewer instructions (FP32/FP16 forms) */
  WT_MATH_EXACT = 1  /* float64 collision in the reference's exact operation order, no FMA
                        contraction: with WT_STORE_F32 it reproduces js/lbm.js bit for bit */
};

/* Treatment of the side planes y=0, y=ny-1, z=0, z=nz-1. */
enum {
  WT_SIDE_EQ = 0,       /* reference behaviour: Dirichlet equilibrium (rho=1, u=(u0,0,0)),
                           js/lbm.js:488-503 */
  WT_SIDE_FREESLIP = 1  /* specular reflection off walls halfway outside the first interior
                           layer; the plane cells still hold the equilibrium for observers */
};

/* Which step kernel runs. The values 2-6 and 9 named step kernels that
 * measured slower than LEAN on B200 and were removed; they are not reused
 * and are rejected (WT_ERR_ARG). */
enum {
  WT_KERNEL_AUTO = 0,    /* the kernel measured fastest on B200 for the form: PAIR when it
                            can run, else LEAN when it can run, else DIRECT */
  WT_KERNEL_DIRECT = 1,  /* one thread per cell, populations gathered straight from HBM;
                            every storage, arithmetic and boundary option */
  WT_KERNEL_LEAN = 7,    /* one thread per cell, 32-bit byte offsets from one pointer per cell,
                            the collision in storage units with approximate reciprocal / square
                            root, and for half storage on lattices whose population buffer
                            fits in twice the L2 an L2 prefetch of the populations a fixed
                            distance ahead in launch order (environment WT_PREFETCH_CELLS
                            overrides the distance at wt_create, for any lattice; 0 turns it
                            off); float32 collision, buffers under 2 GiB, stationary walls */
  WT_KERNEL_PAIR = 8     /* two adjacent cells per thread, one aligned load and store of the
                            pair per direction (32-bit half pairs, 64-bit float32 pairs), both
                            cells collided at once in packed float32x2 instructions; LEAN's
                            conditions (half or float32 storage) and an even nx */
};

/* Rounding of half-precision stores. Stochastic rounding draws its random
 * bits from a hash of (cell, step), so a run is reproducible. */
enum { WT_ROUND_NEAREST = 0, WT_ROUND_STOCHASTIC = 1 };

/* Occupancy codes, js/lbm.js:39. */
enum { WT_FLUID = 0, WT_SOLID_OBJ = 1, WT_SOLID_WALL = 2 };

/* Which population buffer, js/lbm.js:131-132. */
enum { WT_BUF_F = 0, WT_BUF_G = 1 };

/* Solver parameters: the reference's public LBM fields (js/lbm.js:95, :106-111)
 * plus the two build options side_bc and math. */
typedef struct wt_params {
  double u0;         /* inlet / far-field speed, lattice units (LBM.u0, default 0.06) */
  double tau;        /* molecular relaxation time (LBM.tau, default 0.5035) */
  int32_t les;       /* Smagorinsky LES on/off (LBM.les, default 1) */
  int32_t trt;       /* two-relaxation-time collision on/off (LBM.trt, default 1) */
  double csm;        /* Smagorinsky constant (LBM.csm, default 0.14) */
  double lambda;     /* TRT magic parameter (LBM.lambda, default 1/4) */
  int32_t moving_walls; /* moving no-slip walls on/off (LBM.movingWalls; set by voxelize) */
  int32_t side_bc;   /* WT_SIDE_EQ (default) or WT_SIDE_FREESLIP */
  int32_t math;      /* WT_MATH_FAST (default) or WT_MATH_EXACT */
  int32_t kernel;    /* WT_KERNEL_* (default WT_KERNEL_AUTO) */
  int32_t f16_rounding; /* half storage: WT_ROUND_NEAREST (default) or WT_ROUND_STOCHASTIC */
  int32_t reserved;  /* must be 0 */
} wt_params;

/* Body statistics computed by voxelize, js/lbm.js:247-264. */
typedef struct wt_body_stats {
  int32_t frontal_area;   /* yz columns the body covers, at least 1 (LBM.frontalArea) */
  int32_t planform_area;  /* xz columns the body covers, at least 1 (LBM.planformArea) */
  int32_t solid_cells;    /* SOLID_OBJ cells set by the last voxelize (LBM.solidCells) */
  int32_t ride_height;    /* median non-zero underbody gap in cells (LBM.rideHeight) */
  int32_t ground;         /* road present (LBM.ground) */
  int32_t moving_walls;   /* LBM.movingWalls after voxelize */
} wt_body_stats;

typedef struct wt_lattice wt_lattice;

/* Reference defaults of js/lbm.js:106-111 (side_bc = WT_SIDE_EQ, math = WT_MATH_FAST,
 * kernel = WT_KERNEL_AUTO). */
void wt_default_params(wt_params* p);

/* new LBM(nx, ny, nz) — js/lbm.js:58-128. Allocates both population buffers,
 * occupancy and fields on the current CUDA device and runs reset().
 * nx, ny, nz >= 3. storage is a WT_STORE_* value. */
int wt_create(int nx, int ny, int nz, int storage, wt_lattice** out);

/* Frees every device allocation of the handle. NULL is accepted. */
int wt_destroy(wt_lattice* h);

/* Message of the handle's last failure ("" if none). With h == NULL, the
 * message of the last failed wt_create on this thread. */
const char* wt_last_error(const wt_lattice* h);

/* Lattice dims and storage format. */
int wt_get_dims(const wt_lattice* h, int* nx, int* ny, int* nz, int* storage);

/* Assign / read the public solver fields (js/lbm.js:95, :106-111). */
int wt_set_params(wt_lattice* h, const wt_params* p);
int wt_get_params(const wt_lattice* h, wt_params* p);

/* LBM.reset() — js/lbm.js:164-174: both buffers to the equilibrium at rho=1,
 * u=(u0,0,0) (u=0 in solid cells), fields to match, steps=0, force=0. */
int wt_reset(wt_lattice* h);

/* reset() followed by seeded velocity noise on every non-solid cell:
 * u = (u0 + amp*(2r-1), amp*(2r-1), amp*(2r-1)) with r the splitmix64 draws
 * 3i, 3i+1, 3i+2 of `seed` (draw k is mix(seed + (k+1)*0x9E3779B97F4A7C15),
 * r = (x >> 11) * 2^-53). No reference counterpart: the configs' initial state. */
int wt_init_eq_noise(wt_lattice* h, uint64_t seed, double amp);

/* Inclusive integer scan range of LBM.voxelize for a body box
 * {x0,y0,z0,x1,y1,z1} (js/lbm.js:216-218): range = {x0,x1,y0,y1,z0,z1}. */
int wt_voxel_range(const wt_lattice* h, const double box[6], int range[6]);

/* LBM.voxelize(inside, box, ground, wallVel, roadVel) — js/lbm.js:191-266.
 * `inside` holds inside(x+.5, y+.5, z+.5) for every cell of the scan range of
 * `box`, x fastest (len = product of the range extents). The closure is
 * evaluated by the host. wall_set / wall_vel (optional, same cell order;
 * wall_vel 3 doubles per cell) hold wallVel's return value and output.
 * Clears the previous body, sets the road row, marks the body, computes the
 * area statistics and rebuilds the near-wall flags. */
int wt_voxelize_mask(wt_lattice* h, const double box[6], const uint8_t* inside, size_t inside_len,
                     const uint8_t* wall_set, const double* wall_vel, int ground, double road_vel);

/* LBM.voxelize with the voxel-backed Body.makeTest() closure evaluated on the
 * device — js/shapes.js:365-388 (the custom-body lookup) inside
 * js/lbm.js:191-266. grid is the body-space Uint8 occupancy grid of
 * js/voxel.js:89-101 (gnx*gny*gnz bytes, index a + gnx*(b + gny*c)), gmin
 * and ginv its min corner and inverse cell size; M (row-major 3x3, the
 * Body._updateMat rotation of js/shapes.js:353-362), P (Body.pos) and scale
 * (Body.scale) place it. The lookup runs in float64 with no FMA contraction,
 * so the occupancy is bit-identical to the reference closure. */
int wt_voxelize_grid(wt_lattice* h, const uint8_t* grid, int gnx, int gny, int gnz,
                     const double gmin[3], double ginv, const double M[9], const double P[3],
                     double scale, const double box[6], int ground, double road_vel);

/* LBM.frontalArea / planformArea / solidCells / rideHeight / ground /
 * movingWalls — js/lbm.js:247-264. */
int wt_get_body_stats(const wt_lattice* h, wt_body_stats* out);

/* LBM.step() repeated nsteps times — js/lbm.js:285-291 — which is also
 * LBMPool.Pool.step(n) (js/pool.js:97-125). forces (optional) receives
 * 3*nsteps doubles: the momentum-exchange force [fx,fy,fz] of every step,
 * accumulated in float64. Fields (ux,uy,uz,rho) are current on return.
 * Returns WT_ERR_DIVERGED if any step met a non-finite or non-positive
 * density (the state is then left as computed). */
int wt_step(wt_lattice* h, int nsteps, double* forces);

/* wt_step without any device or pinned allocation. This entry point has no
 * counterpart in the reference; it is for callers that cannot let the
 * library allocate while they run: a host whose own memory pool has already
 * claimed the device's memory (so a cudaMalloc would fail), or a host
 * stepping inside a frame loop that must not stall, since cudaMalloc and
 * cudaFree may synchronise the whole device. wt_step may grow
 * its force-series buffers; this call keeps the force partials, the
 * per-step forces and the error word in one fixed device array of about
 * 3.2 MB instead (16384 wall segments x 8 steps of partials, 4096 steps of
 * forces), whose address it looks up with cudaGetSymbolAddress on every call.
 * Same results as wt_step: it runs the kernel wt_step picks.
 * Limits: nsteps in 0..4096 (else WT_ERR_ARG); a body with more than 16384
 * 32-cell wall segments, or a solid-fraction field, gives WT_ERR_UNSUPPORTED;
 * the lattice's device must be the current device (else WT_ERR_STATE).
 * A call with nsteps = 0 sets up: it looks the array up and loads the device
 * code of every step and reduction kernel a later call can launch (code
 * loading can need device memory); make it on each device before any stream
 * capture. The array is shared by every lattice on the device, so calls that
 * overlap in time, from two threads or on two lattices, race and give wrong
 * forces. forces (optional) receives 3*nsteps doubles as for wt_step. */
int wt_step_noalloc(wt_lattice* h, int nsteps, double* forces);

/* Partial bounce-back field (no reference counterpart; the differentiable
 * body of the adjoint): solid fraction s in [0, 1] for every cell of the
 * half-open box {x0, y0, z0, x1, y1, z1}, x fastest. A fluid cell with
 * fraction s stores g_q = (1 - s) gc_q + s f_opp(q) (gc collided, f pulled)
 * and adds s * sum_q c_q (gc_q - f_opp(q)) to the force. box == NULL clears
 * the field. While a field is set the step runs the direct kernel. */
int wt_set_solid_fraction(wt_lattice* h, const int box[6], const double* s);

/* Objective and checkpointing of wt_adjoint. */
typedef struct wt_adj_cfg {
  int32_t nsteps;      /* forward steps from the current state */
  int32_t window;      /* J = mean of the force component over the last `window` steps */
  int32_t component;   /* 0 = x (drag), 1 = y, 2 = z */
  int32_t checkpoint;  /* steps between stored states; 0 = every state when
                          (nsteps + 3) states fit in 3/4 of the free device
                          memory, else ceil(sqrt(nsteps)) */
  int32_t keep;        /* nonzero: leave this run's device memory (checkpoints, interval
                          store, adjoint buffers) in the lattice for the next wt_adjoint
                          call that fits in it, as an optimisation loop wants; 0: free it,
                          and any memory an earlier call kept, when the call ends.
                          wt_destroy frees kept memory. */
  int32_t reserved[3]; /* must be 0 */
} wt_adj_cfg;

typedef struct wt_adj_stats {
  double J;            /* the objective */
  double forward_ms;   /* forward sweep with checkpoint copies (CUDA events) */
  double backward_ms;  /* recomputation + adjoint steps (CUDA events) */
  int64_t device_bytes;/* device memory the run used (checkpoints, segment, adjoint) */
  int32_t checkpoints; /* checkpoint intervals */
  int32_t segment;     /* steps per checkpoint interval */
} wt_adj_stats;

/* d(J)/d(s) by the discrete adjoint of the step (no reference counterpart).
 * Runs cfg->nsteps steps from the current state (the lattice ends where
 * wt_step(h, nsteps) would leave it) storing a checkpoint every
 * cfg->checkpoint steps, then runs the adjoint backwards, recomputing each
 * interval's states from its checkpoint; the last interval's states are kept
 * from the forward sweep, so with checkpoint == nsteps nothing is recomputed. dJds receives one double per cell
 * of the solid-fraction box (x fastest). Adjoint arithmetic: float64 for
 * float64 storage or WT_MATH_EXACT, float32 otherwise. Stationary walls only
 * (WT_ERR_UNSUPPORTED with moving walls); WT_ERR_STATE without a field. */
int wt_adjoint(wt_lattice* h, const wt_adj_cfg* cfg, double* dJds, wt_adj_stats* stats);

/* Voxel.build (js/voxel.js:48-102): a triangle soup in body space becomes a
 * body-space occupancy grid for wt_voxelize_grid. The fields follow the
 * returned object of js/voxel.js:89-101. */
typedef struct wt_voxel_info {
  int32_t nx, ny, nz;   /* grid dims (2 cells of padding each side) */
  int32_t reserved;
  int64_t tris;         /* stats.tris */
  double cell, inv;     /* cell size and 1 / cell */
  double min[3];        /* grid min corner */
  double ext[3];        /* half extents of the mesh bounds */
  double centre[3];     /* centre of the mesh bounds */
  double bbox[6];       /* mesh bounds x0, y0, z0, x1, y1, z1 */
  int64_t solid;        /* stats.solid: occupied cells */
  double openness;      /* stats.openness: cells where the three parity votes disagree / solid */
} wt_voxel_info;

/* The grid dims, cell size and bounds for `res` cells along the longest
 * axis (js/voxel.js:48-71), without building: tris holds 9*ntri floats.
 * Errors (WT_ERR_ARG, message in wt_voxel_last_error): no triangles, a
 * degenerate mesh, a grid of more than 40e6 cells (js/voxel.js:51, :56, :71). */
int wt_voxel_dims(const float* tris, int64_t ntri, int res, wt_voxel_info* info);

/* Voxel.build(P, res) on the current CUDA device — js/voxel.js:48-232: the
 * surface shell OR'd with a two-of-three vote of ray-parity fills along x, y
 * and z, in float64 with the reference's operation order (bit-identical to
 * the reference). grid (grid_len = nx*ny*nz bytes, index x + nx*(y + ny*z))
 * receives 1 for solid cells. Allocates and frees its own device buffers. */
int wt_voxel_build(const float* tris, int64_t ntri, int res, uint8_t* grid, size_t grid_len,
                   wt_voxel_info* info);

/* Message of the last failed wt_voxel_* call on this thread. */
const char* wt_voxel_last_error(void);

/* LBM.force — js/lbm.js:113, :289: the force of the last step. */
int wt_get_force(const wt_lattice* h, double out[3]);

/* LBM.steps and LBM.parity. */
int wt_get_steps(const wt_lattice* h, int64_t* steps, int* parity);

/* LBM.ux / uy / uz / rho — js/lbm.js:85-88: n floats each, any may be NULL. */
int wt_get_fields(wt_lattice* h, float* ux, float* uy, float* uz, float* rho);

/* LBM.solid / LBM.near — js/lbm.js:82-83: n bytes each. */
int wt_get_solid(wt_lattice* h, uint8_t* out);
int wt_get_near(wt_lattice* h, uint8_t* out);

/* LBM.f / LBM.g getters — js/lbm.js:131-132. which = WT_BUF_F or WT_BUF_G.
 * dtype WT_STORE_F32 / WT_STORE_F64 converts the stored deviations to that
 * type (19*n elements); dtype equal to the handle's storage copies raw
 * elements (for WT_STORE_F16DEV: halves holding deviation * WT_F16_SCALE).
 * bytes must equal 19*n*sizeof(element). */
int wt_get_populations(wt_lattice* h, int which, int dtype, void* out, size_t bytes);
int wt_set_populations(wt_lattice* h, int which, int dtype, const void* in, size_t bytes);

/* Checkpoint / resume: both population buffers, fields, occupancy, wall
 * velocities, parity, step count and last force as one opaque blob. */
int wt_state_size(const wt_lattice* h, size_t* bytes);
int wt_get_state(wt_lattice* h, void* out, size_t bytes);
int wt_set_state(wt_lattice* h, const void* in, size_t bytes);

/* LBM.sample(x, y, z, out) — js/lbm.js:515-539 — for npts points (xyz holds
 * 3*npts doubles, out receives 3*npts doubles). Trilinear at cell centres,
 * (u0,0,0) outside the half-cell margin. */
int wt_sample(wt_lattice* h, const double* xyz, int npts, double* out);

/* LBM.isSolid(x, y, z) — js/lbm.js:541-545. */
int wt_is_solid(wt_lattice* h, double x, double y, double z, int* out);

/* The scalar the reference's slice view colours (js/main.js:925-968), for
 * every cell of one lattice plane: plane 0 is the xy plane z = k, plane 1
 * the xz plane y = k; field 0 = |u| / u0, 1 = pressure coefficient of the
 * 5-point averaged density ((rho - 1) / 3) / (u0^2 / 2), 2 = in-plane
 * vorticity / u0 (central differences). out holds nx * (ny or nz) floats,
 * x fastest; solid cells are NaN. The colour map itself is the caller's. */
int wt_slice(wt_lattice* h, int plane, int k, int field, float* out, size_t len);

/* One step of the reference's smoke particles (js/main.js:691-709) for n
 * particles: xyz (3n doubles, lattice coordinates) moves by the trilinear
 * velocity of LBM.sample times kstep; expired[p] (optional) = 1 when the
 * particle left the margins of js/main.js:701-702 or entered a solid cell;
 * speed[p] (optional) = |u| / u0 at its old position. Ages, respawning and
 * colours stay with the caller. */
int wt_advect(wt_lattice* h, double* xyz, int n, double kstep, uint8_t* expired, float* speed);

/* The handle's CUDA stream (a cudaStream_t), for timing with events. */
int wt_get_stream(const wt_lattice* h, void** stream);

/* Number of kernels the library has launched on this handle so far. */
int wt_get_launch_count(const wt_lattice* h, int64_t* count);

#ifdef __cplusplus
}
#endif

#endif /* WT_H */
