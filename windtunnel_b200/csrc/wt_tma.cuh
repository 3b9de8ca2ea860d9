// wt_tma.cuh — the fused step on tensor-map TMA tiles.
//
// Same semantics and per-cell rules as k_step (wt_step.cuh). The lattice is
// cut into tiles of TX cells along x by TY rows along y in one z plane. A
// persistent CTA walks its tiles with a warp-specialised pipeline:
//
//   load issuer (lane 0 of warp 0)  for every tile, 19 cp.async.bulk.tensor
//                                   loads -- direction q's box of (TX + 2H) x TY
//                                   source cells at (x0 - H, y0 - ey, z - ez, q)
//                                   -- into one of DI input stages, completing on
//                                   the stage's "full" mbarrier; a stage is
//                                   reloaded as soon as every consumer warp has
//                                   read it ("empty").
//   store issuer (lane 0 of warp 1) once the consumers have filled one of DO
//                                   output buffers ("ready"), 19 tensor stores of
//                                   TX x TY boxes at (x0, y0, z, q); the buffer is
//                                   released ("ofree") when the stores have read it.
//   consumers (NC warps)            read the pulled values of their two cells
//                                   per direction from the input stage at fixed
//                                   offsets (the -ex shift is an index offset,
//                                   the halo H covers x0-1 and x0+TX), release
//                                   the stage, collide both cells in packed
//                                   float32x2 arithmetic (collide_x2) and write
//                                   the 19 outputs into the output buffer, dense
//                                   TX x TY per direction.
//
// No address arithmetic per population remains in the consumers: every
// shared-memory access is a fixed offset from one base register. Boxes that
// reach outside the lattice are zero-filled by the TMA unit on load (those
// values are only read by cells that do not pull) and clipped on store.
// Solid cells keep their stale populations: their outputs are re-read from
// HBM, so the store rewrites the value already there.
//
// Preconditions (host): float32 or half storage, float32 collision, nx a
// multiple of 16 bytes / element size (tensor-map row pitch), nearest
// rounding for half storage. Every mbarrier wait is bounded by a clock
// budget; a timeout sets bit 2 of the error word (WT_ERR_TIMEOUT on the
// host), the role that saw it stops (consumer warps decide per warp, so a
// warp never splits), and the load issuer waits (bounded) for the loads it
// has in flight before it returns.
#pragma once

#include <cuda.h>

#include "wt_staged.cuh"
#include "wt_x2.cuh"

namespace wt {

template <class S>
struct Tma {
  static constexpr int CELLS = 512;                 // cells per tile (two per consumer thread)
  static constexpr int NC = 8;                      // consumer warps
  static constexpr int THREADS = 32 * (NC + 2);     // + load-issuer warp + store-issuer warp
  static constexpr int HALO = 16 / (int)sizeof(S);  // x halo when a tile is narrower than a row
  static constexpr int PAD = 128 / (int)sizeof(S);  // slot pitch rounding (128 bytes)
  static constexpr int IN_SLOT_MAX = CELLS + 8 * HALO + PAD;   // tx=128, ty=4 with halos
  static constexpr int OUT_SLOT_MAX = CELLS + PAD;
  static constexpr int DI = sizeof(S) == 2 ? 5 : 3; // input stages
  static constexpr int DO = 2;                      // output buffers
  static constexpr size_t IN_BYTES_MAX = (size_t)Q * IN_SLOT_MAX * sizeof(S);
  static constexpr size_t OUT_BYTES_MAX = (size_t)Q * OUT_SLOT_MAX * sizeof(S);
  static constexpr size_t OUT_OFF = (size_t)DI * IN_BYTES_MAX;
  static constexpr size_t BAR_OFF = OUT_OFF + (size_t)DO * OUT_BYTES_MAX;
  // + 128: the ring starts at the first 128-byte boundary of the dynamic allocation
  static constexpr size_t SMEM = BAR_OFF + 2 * (DI + DO) * sizeof(unsigned long long) + 16 + 128;
  static_assert(NC * 32 * 2 == CELLS, "two cells per consumer thread");
  static_assert(SMEM <= 227 * 1024, "stage ring exceeds the shared-memory limit");
  static_assert(IN_BYTES_MAX % 128 == 0 && OUT_BYTES_MAX % 128 == 0, "stages must stay aligned");
};

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            int z, int q, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(q), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int x, int y, int z, int q,
                                             uint32_t src) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::
          "l"(reinterpret_cast<uint64_t>(map)),
      "r"(x), "r"(y), "r"(z), "r"(q), "r"(src)
      : "memory");
}
__device__ __forceinline__ void bulk_wait_read_0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

struct TileCoord {
  int x0, y0, z;
};
__device__ __forceinline__ TileCoord tile_coord(long long t, int gx, int gy, int tx, int ty) {
  TileCoord c;
  const int xt = (int)(t % gx);
  const long long r = t / gx;
  c.x0 = xt * tx;
  c.y0 = (int)(r % gy) * ty;
  c.z = (int)(r / gy);
  return c;
}

// Bounded wait executed by every lane of a warp; true on all lanes only if
// every lane saw the phase complete (a uniform decision for the warp).
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity) {
  const bool ok = mbar_wait_bounded(bar, parity, kWaitBudgetCycles);
  return __all_sync(0xffffffffu, ok);
}

template <class S>
__global__ void __launch_bounds__(Tma<S>::THREADS, 1)
    k_step_tma(const __grid_constant__ StepArgs<S> a, const __grid_constant__ TmaMaps m,
               int ld_buf, int st_buf, long long ntiles) {
  using C = Tma<S>;
  using T = X2<S>;
  using P = Pair<S>;
  using V = typename T::V;
  constexpr float SC = T::SC;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_dyn + ((128u - (smem_addr(smem_dyn) & 127u)) & 127u);
  S* in_st = reinterpret_cast<S*>(smem_raw);
  S* out_st = reinterpret_cast<S*>(smem_raw + C::OUT_OFF);
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem_raw + C::BAR_OFF);
  unsigned long long* empty = full + C::DI;     // consumers have read the input stage
  unsigned long long* ready = empty + C::DI;    // consumers have written the output buffer
  unsigned long long* ofree = ready + C::DO;    // the tensor stores have read the output buffer
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // this CTA's contiguous range of tiles
  const long long per = (ntiles + gridDim.x - 1) / gridDim.x;
  const long long tbeg = (long long)blockIdx.x * per;
  const long long tend = min(ntiles, tbeg + per);
  const long long count = tend - tbeg;
  if (count <= 0) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::DI; s++) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), C::NC);
    }
    for (int o = 0; o < C::DO; o++) {
      mbar_init(smem_addr(&ready[o]), C::NC);
      mbar_init(smem_addr(&ofree[o]), 1);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == 0) {
    // ---------------------------------------------------------- load issuer
    if (lane != 0) return;
    const CUtensorMap* ldm = &m.ld[ld_buf];
    long long issued = 0;
    for (long long k = 0; k < count; k++) {
      const int s = (int)(k % C::DI);
      if (k >= C::DI &&
          !mbar_wait_bounded(smem_addr(&empty[s]), (uint32_t)((k / C::DI - 1) & 1),
                             kWaitBudgetCycles)) {
        atomicOr(a.err, 4u);   // consumers stopped
        break;
      }
      const TileCoord c = tile_coord(tbeg + k, m.gx, m.gy, m.tx, m.ty);
      const uint32_t bar = smem_addr(&full[s]);
      if (c.z == 0 || c.z == a.nz - 1) {
        mbar_arrive_expect_tx(bar, 0);   // end plane: every cell is the equilibrium
      } else {
        mbar_arrive_expect_tx(bar, (uint32_t)(Q * m.ty * m.bw * sizeof(S)));
        const uint32_t dst = smem_addr(in_st + (size_t)s * Q * m.in_slot);
#pragma unroll 1
        for (int q = 0; q < Q; q++)
          tma_load_4d(dst + (uint32_t)(q * m.in_slot * sizeof(S)), ldm, c.x0 - m.h, c.y0 - ey(q),
                      c.z - ez(q), q, bar);
      }
      issued = k + 1;
    }
    // loads still landing in the stages complete before the CTA may exit
    for (long long k = issued - 1; k >= 0 && k >= issued - C::DI; k--)
      mbar_wait_bounded(smem_addr(&full[k % C::DI]), (uint32_t)((k / C::DI) & 1),
                        kWaitBudgetCycles);
    return;
  }
  if (warp == 1) {
    // ---------------------------------------------------------- store issuer
    if (lane != 0) return;
    const CUtensorMap* stm = &m.st[st_buf];
    for (long long k = 0; k < count; k++) {
      const int o = (int)(k % C::DO);
      if (!mbar_wait_bounded(smem_addr(&ready[o]), (uint32_t)((k / C::DO) & 1),
                             kWaitBudgetCycles)) {
        atomicOr(a.err, 4u);
        break;
      }
      const TileCoord c = tile_coord(tbeg + k, m.gx, m.gy, m.tx, m.ty);
      const uint32_t src = smem_addr(out_st + (size_t)o * Q * m.out_slot);
#pragma unroll 1
      for (int q = 0; q < Q; q++)
        tma_store_4d(stm, c.x0, c.y0, c.z, q, src + (uint32_t)(q * m.out_slot * sizeof(S)));
      bulk_commit();
      bulk_wait_read_0();   // the buffer may be rewritten once the stores have read it
      mbar_arrive(smem_addr(&ofree[o]));
    }
    bulk_wait_all();
    return;
  }

  // -------------------------------------------------------------- consumers
  const int t = threadIdx.x - 64;                 // 0 .. NC*32-1
  const int pr = t % (m.tx / 2), ty = t / (m.tx / 2);   // rows ty >= m.ty hold no cells
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  for (long long k = 0; k < count; k++) {
    const int s = (int)(k % C::DI), o = (int)(k % C::DO);
    const TileCoord c = tile_coord(tbeg + k, m.gx, m.gy, m.tx, m.ty);
    const int x0 = c.x0 + 2 * pr, y = c.y0 + ty, z = c.z;
    const bool active = x0 < nx && y < ny && ty < m.ty;
    const long long i0 = (long long)x0 + (long long)nx * y + a.nxy * z;
    const bool edge_row = z == 0 || z == nz - 1 || y == ny - 1;
    uint8_t flA = 0, flB = 0;
    if (active && !edge_row) {
      const uint16_t fl2 = *reinterpret_cast<const uint16_t*>(a.flags + i0);
      flA = (uint8_t)fl2;
      flB = (uint8_t)(fl2 >> 8);
    }
    const int catA = edge_row ? CAT_EQ : cell_category(a, x0, y, flA);
    const int catB = edge_row ? CAT_EQ
                              : ((x0 + 1 == nx - 1) ? CAT_NONE : cell_category(a, x0 + 1, y, flB));
    const bool interior = active && !edge_row && y >= 1;
    if (!warp_wait(smem_addr(&full[s]), (uint32_t)((k / C::DI) & 1))) {
      atomicOr(a.err, 4u);
      break;
    }
    f2 f[Q];
    if (interior) {
      const S* in = in_st + (size_t)s * Q * m.in_slot + ty * m.bw + 2 * pr + m.h;
#pragma unroll
      for (int q = 0; q < Q; q++) {
        const S* p = in + q * m.in_slot - ex(q);
        f[q] = make_float2(T::raw(p[0]), T::raw(p[1]));
      }
    } else {
#pragma unroll
      for (int q = 0; q < Q; q++) f[q] = pk(0.0f);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));   // this warp is done with the stage

    double Fx = 0, Fy = 0, Fz = 0;
    bool near_any = false;
    const bool fluidA = interior && catA == CAT_FLUID, fluidB = interior && catB == CAT_FLUID;
    f2 r = pk(SC), vx = pk(0.0f), vy = pk(0.0f), vz = pk(0.0f);
    if (fluidA || fluidB) {
      const bool shell = a.freeslip && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
      const bool nearA = fluidA && (flA & FLAG_NEAR) != 0;
      const bool nearB = fluidB && (flB & FLAG_NEAR) != 0;
      near_any = nearA || nearB;
      if (fluidA && (nearA || shell)) patch_raw<S, 0>(a, i0, x0, y, z, nearA, shell, f, Fx, Fy, Fz);
      if (fluidB && (nearB || shell))
        patch_raw<S, 1>(a, i0 + 1, x0 + 1, y, z, nearB, shell, f, Fx, Fy, Fz);
      collide_x2<S>(a, f, r, vx, vy, vz);
      if ((fluidA && !(r.x > 0.0f && r.x < 3.0e38f)) || (fluidB && !(r.y > 0.0f && r.y < 3.0e38f)))
        atomicOr(a.err, 1u);
      if (a.mov && !a.write_fields) {
        if (nearA) a.rho[i0] = r.x * (1.0f / SC);
        if (nearB) a.rho[i0 + 1] = r.y * (1.0f / SC);
      }
    }

    // outputs of the pair, dense TX x TY per direction, once the buffer is free
    if (k >= C::DO && !warp_wait(smem_addr(&ofree[o]), (uint32_t)((k / C::DO - 1) & 1))) {
      atomicOr(a.err, 4u);
      break;
    }
    S* out = out_st + (size_t)o * Q * m.out_slot + ty * m.tx + 2 * pr;
    if (active) {
      const bool eqA = catA == CAT_EQ, eqB = catB == CAT_EQ;
      const bool keepA = catA == CAT_KEEP, keepB = catB == CAT_KEEP;
      const bool outB = catB == CAT_NONE;
      if (!eqA && !eqB && !keepA && !keepB && !outB) {
#pragma unroll
        for (int q = 0; q < Q; q++)
          *reinterpret_cast<V*>(out + q * m.out_slot) = T::pack(f[q]);
      } else {
        const S* Gi = a.G + i0;
#pragma unroll
        for (int q = 0; q < Q; q++) {
          const V pv = T::pack(f[q]);
          S sa = eqA ? a.eq[q] : P::lo(pv);
          S sb = eqB ? a.eq[q] : P::hi(pv);
          if (keepA) sa = Gi[q * a.n];
          if (keepB) sb = Gi[q * a.n + 1];
          if (outB) sb = sa;
          *reinterpret_cast<V*>(out + q * m.out_slot) = P::make(sa, sb);
        }
      }
      if (a.write_fields) {
        float ra = 1.0f, xa = a.u0f, ya = 0.0f, za = 0.0f;
        if (fluidA) { ra = r.x * (1.0f / SC); xa = vx.x; ya = vy.x; za = vz.x; }
        if (keepA) { ra = a.rho[i0]; xa = a.ux[i0]; ya = a.uy[i0]; za = a.uz[i0]; }
        else { a.rho[i0] = ra; a.ux[i0] = xa; a.uy[i0] = ya; a.uz[i0] = za; }
        if (outB) {
          a.rho[i0 + 1] = ra; a.ux[i0 + 1] = xa; a.uy[i0 + 1] = ya; a.uz[i0 + 1] = za;
        } else if (fluidB) {
          a.rho[i0 + 1] = r.y * (1.0f / SC); a.ux[i0 + 1] = vx.y; a.uy[i0 + 1] = vy.y;
          a.uz[i0 + 1] = vz.y;
        } else if (eqB) {
          a.rho[i0 + 1] = 1.0f; a.ux[i0 + 1] = a.u0f; a.uy[i0 + 1] = 0.0f; a.uz[i0 + 1] = 0.0f;
        }
      }
    }
    fence_proxy_async_smem();   // generic-proxy writes become visible to the tensor stores
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&ready[o]));
    constexpr double inv_sc = 1.0 / (double)SC;
    pair_force_partial(Fx * inv_sc, Fy * inv_sc, Fz * inv_sc, near_any, a, x0 & ~31, y, z);
  }
}

}  // namespace wt
