// wt_staged.cuh — the fused step with bulk-copy (TMA) staging of the pull rows.
//
// Same semantics as k_step (wt_step.cuh), different data movement. The
// lattice is cut into units: one x-segment of up to TX cells of one (y, z)
// row. A persistent CTA walks its units; for each interior unit one thread
// issues 19 cp.async.bulk copies -- the source row of every direction, i.e.
// row (y - ey, z - ez) shifted by -ex, with PAD elements of margin so every
// copy starts on a 16-byte boundary -- completing on a per-stage mbarrier.
// Units are prefetched D deep, so HBM traffic no longer waits for the
// collision arithmetic. The CTA is warp-specialised: one producer warp issues
// the copies, gated per stage by an "empty" mbarrier; four consumer warps run
// independently of one another -- each waits on the stage's "full" mbarrier,
// reads its 32 cells' pulled values from shared memory at fixed offsets,
// collides, stores the 19 outputs straight to HBM (coalesced) and arrives on
// "empty". No CTA-wide barrier is taken inside the loop.
//
// Preconditions (checked on the host): nx is a multiple of VEC = 16 bytes /
// sizeof(S), so every row, every direction block and every copy is 16-byte
// aligned. Each copy is additionally bounds- and alignment-checked on the
// device before it is issued; each wait is bounded by a clock budget and
// reports WT_ERR_TIMEOUT (bit 2 of the error word) instead of hanging.
#pragma once

#include "wt_step.cuh"

namespace wt {

template <class S>
struct Staged {
  static constexpr int TX = 128;                  // cells per unit = consumer threads
  static constexpr int NCONS = TX / 32;           // consumer warps
  static constexpr int THREADS = TX + 32;         // + one producer warp
  static constexpr int VEC = 16 / (int)sizeof(S); // elements per 16 bytes
  static constexpr int PAD = VEC;                 // margin each side of a staged row
  static constexpr int W = TX + 2 * PAD;          // staged elements per direction
  static constexpr int D = sizeof(S) == 8 ? 2 : 3;  // input stages
  static constexpr size_t IN_BYTES = (size_t)D * Q * W * sizeof(S);
  static constexpr size_t SMEM = IN_BYTES + 2 * D * sizeof(unsigned long long);
  // register budget: CTAs per SM the kernel is compiled to keep resident
  static constexpr int min_blocks(bool exact) { return exact ? 2 : 5; }
};

// ---- PTX wrappers ----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// One lane of the (converged) warp, chosen by the hardware.
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n .reg .b32 r;\n .reg .pred p;\n elect.sync r|p, 0xffffffff;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(pred));
  return pred != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Record the first rejected copy (kind 1 = load, 2 = store) for the host.
template <class S>
__device__ __forceinline__ void report_copy(const StepArgs<S>& a, int kind, int q, long long u,
                                            long long off) {
  atomicOr(a.err, 8u);
  if (atomicCAS((unsigned long long*)a.diag, 0ULL, (unsigned long long)kind) == 0ULL) {
    a.diag[1] = q;
    a.diag[2] = u;
    a.diag[3] = off;
  }
}

// Wait for `parity` on a stage barrier, giving up after ~`budget` cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity,
                                                  long long budget) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > budget) return false;
  }
  return true;
}

constexpr long long kWaitBudgetCycles = 4000000000LL;   // ~2 s at B200 clocks

// Position of a unit: x-segment `tile` of row (y, z). Units are numbered
// tile-fastest; a CTA walks a contiguous range, so the position advances
// without divisions.
struct UnitPos {
  long long u;
  int tile, y, z;
  __device__ __forceinline__ void start(long long u0, int gx, int ny) {
    u = u0;
    tile = (int)(u0 % gx);
    const long long row = u0 / gx;
    y = (int)(row % ny);
    z = (int)(row / ny);
  }
  __device__ __forceinline__ void next(int gx, int ny) {
    ++u;
    if (++tile == gx) {
      tile = 0;
      if (++y == ny) { y = 0; ++z; }
    }
  }
};

// Issue the loads of unit p into `stage` (one thread). Boundary rows need no
// loads; their stage barrier is completed with an empty transaction so the
// phase bookkeeping stays uniform.
template <class S>
__device__ __forceinline__ void issue_unit(const StepArgs<S>& a, const UnitPos& p, S* in_stage,
                                           uint32_t bar) {
  // Executed by the whole producer warp with uniform values; one elected
  // lane performs the barrier arrival and the copies.
  using C = Staged<S>;
  const bool interior = p.y >= 1 && p.y <= a.ny - 2 && p.z >= 1 && p.z <= a.nz - 2;
  const int x0 = p.tile * C::TX;
  const int w = min(C::TX, a.nx - x0);
  const uint32_t bytes = (uint32_t)((w + 2 * C::PAD) * sizeof(S));
  const long long rowbase = (long long)a.nx * p.y + a.nxy * p.z + x0 - C::PAD;
  int bad = -1;
  if (interior) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      // the row of direction q, unshifted in x: the -ex shift is applied when
      // the threads read the stage (index t + PAD - ex)
      const long long off = a.src[q] + ex(q) + rowbase;
      if ((uintptr_t)(a.F + off) % 16 != 0 || off < 0 || off + (w + 2 * C::PAD) > 19 * a.n)
        bad = q;
    }
  }
  if (elect_one()) {
    if (!interior) {
      mbar_arrive_expect_tx(bar, 0);
    } else if (bad >= 0) {
      report_copy(a, 1, bad, p.u, a.src[bad] + ex(bad) + rowbase);   // skipped, reported
      mbar_arrive_expect_tx(bar, 0);
    } else {
      mbar_arrive_expect_tx(bar, bytes * Q);
#pragma unroll
      for (int q = 0; q < Q; q++) {
        bulk_g2s(smem_addr(in_stage + q * C::W), a.F + a.src[q] + ex(q) + rowbase, bytes, bar);
      }
    }
  }
  __syncwarp();
}

// Writer of the collision outputs straight to HBM (the staged kernel's
// stores): direction q of cell i goes to base[q * n].
template <class S, class IDX>
struct GlobalOut {
  S* base;                   // G + i
  IDX n;                     // cells per direction block
  __device__ __forceinline__ void put(int q, S v) { base[(IDX)q * n] = v; }
};

template <class S, bool EXACT, class IDX>
__global__ void __launch_bounds__(Staged<S>::THREADS, Staged<S>::min_blocks(EXACT))
    k_step_staged(const __grid_constant__ StepArgs<S> a) {
  using C = Staged<S>;
  using M = typename std::conditional<EXACT, double, float>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S* in_s = reinterpret_cast<S*>(smem_raw);
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem_raw + C::IN_BYTES);
  unsigned long long* empty = full + C::D;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // this CTA's contiguous range of units
  const long long per = (a.units + gridDim.x - 1) / gridDim.x;
  const long long ubeg = (long long)blockIdx.x * per;
  const long long uend = min(a.units, ubeg + per);
  const long long count = uend - ubeg;
  if (count <= 0) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::D; s++) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), C::NCONS);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == C::NCONS) {
    // ---- producer warp: issues every unit's 19 row copies -------------------------
    UnitPos pf;
    pf.start(ubeg, a.gx, a.ny);
    for (long long k = 0; k < count; k++, pf.next(a.gx, a.ny)) {
      const int stage = (int)(k % C::D);
      if (k >= C::D &&
          !mbar_wait_bounded(smem_addr(&empty[stage]), (uint32_t)((k / C::D - 1) & 1),
                             kWaitBudgetCycles)) {
        if (lane == 0) atomicOr(a.err, 4u);   // consumers stopped: issue nothing more
        return;
      }
      issue_unit(a, pf, in_s + (size_t)stage * Q * C::W, smem_addr(&full[stage]));
    }
    return;
  }

  // ---- consumers: each warp owns 32 cells of every unit ----------------------------
  const int t = threadIdx.x;   // cell within the unit
  const int gx = a.gx, ny = a.ny, nz = a.nz, nx = a.nx;
  UnitPos p;
  p.start(ubeg, gx, ny);
  // the occupancy byte of this thread's cell in the next unit is loaded one
  // unit ahead, so its HBM round trip overlaps the current unit's collision
  auto flag_of = [&](const UnitPos& q) -> uint8_t {
    const int xq = q.tile * C::TX + t;
    if (xq >= nx) return 0;
    return a.flags[(long long)xq + (long long)nx * q.y + a.nxy * q.z];
  };
  uint8_t fl_next = flag_of(p);
  for (long long k = 0; k < count; k++, p.next(gx, ny)) {
    const uint8_t fl_cur = fl_next;
    if (k + 1 < count) {
      UnitPos pn = p;
      pn.next(gx, ny);
      fl_next = flag_of(pn);
    }
    const int stage = (int)(k % C::D);
    if (!mbar_wait_bounded(smem_addr(&full[stage]), (uint32_t)((k / C::D) & 1),
                           kWaitBudgetCycles)) {
      atomicOr(a.err, 4u);   // a row copy never completed: stop (the producer then stops too)
      return;
    }
    const S* in = in_s + (size_t)stage * Q * C::W;
    const int y = p.y, z = p.z;
    const int x0 = p.tile * C::TX;
    const int w = min(C::TX, nx - x0);
    const int x = x0 + t;
    const long long i = (long long)x + (long long)nx * y + a.nxy * z;
    const bool edge_row = z == 0 || z == nz - 1 || y == ny - 1;   // all equilibrium
    double Fx = 0, Fy = 0, Fz = 0;
    bool near_cell = false;

    if (t < w && x < nx - 1) {
      const bool dup = (x == nx - 2);
      S* Gi = a.G + i;
      int cat;
      uint8_t fl = 0;
      if (x == 0 || edge_row) {
        cat = CAT_EQ;
      } else {
        fl = fl_cur;
        if (fl & FLAG_SOLID_MASK) cat = CAT_KEEP;
        else if (y == 0) cat = CAT_EQ;
        else cat = CAT_FLUID;
      }
      if (cat == CAT_FLUID) {
        M f[Q];
#pragma unroll
        for (int q = 0; q < Q; q++) f[q] = ld<M>(in[q * C::W + t + C::PAD - ex(q)]);
        near_cell = (fl & FLAG_NEAR) != 0;
        const bool shell = a.freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
        if (near_cell || shell) patch_special<S, M>(a, i, x, y, z, shell, f, Fx, Fy, Fz);
        if (!dup) {
          if constexpr (EXACT) {
            collide_exact<S>(a, f, i, false, near_cell, GlobalOut<S, IDX>{Gi, (IDX)a.n});
          } else {
            collide_fast<S>(a, f, i, false, near_cell, GlobalOut<S, IDX>{Gi, (IDX)a.n});
          }
        } else {
          S o[Q];
          if constexpr (EXACT) {
            collide_exact<S>(a, f, i, true, near_cell, RegOut<S>{o});
          } else {
            collide_fast<S>(a, f, i, true, near_cell, RegOut<S>{o});
          }
#pragma unroll
          for (int q = 0; q < Q; q++) { Gi[(IDX)a.dst[q]] = o[q]; Gi[(IDX)a.dst[q] + 1] = o[q]; }
        }
      } else if (cat == CAT_EQ) {
#pragma unroll
        for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q]] = a.eq[q];
        if (dup) {
#pragma unroll
          for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = a.eq[q];
        }
        if (a.write_fields) {
          a.ux[i] = a.u0f; a.uy[i] = 0.0f; a.uz[i] = 0.0f; a.rho[i] = 1.0f;
          if (dup) { a.ux[i + 1] = a.u0f; a.uy[i + 1] = 0.0f; a.uz[i + 1] = 0.0f; a.rho[i + 1] = 1.0f; }
        }
      } else if (dup) {
        // outlet copy of a solid cell in column nx-2: its g is not written this step
#pragma unroll
        for (int q = 0; q < Q; q++) Gi[(IDX)a.dst[q] + 1] = Gi[(IDX)a.dst[q]];
        if (a.write_fields) {
          a.ux[i + 1] = a.ux[i]; a.uy[i + 1] = a.uy[i]; a.uz[i + 1] = a.uz[i]; a.rho[i + 1] = a.rho[i];
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[stage]));
    warp_force_partial_w(Fx, Fy, Fz, near_cell, a,
                         seg_of(x0 + (t & ~31), y, z, nx, ny));
  }
}

}  // namespace wt
