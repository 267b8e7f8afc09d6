// sweep_tma.cuh -- TMA-pipelined E and H sweeps (sm_100a).
//
// The bulk Yee updates (src/grid.c:709-888) and the UPML updates
// (src/pml.c:859-1176) as persistent marching sweeps.  The host cuts each
// update region into tiles of KW (k) x JH (j) columns and a run of i planes
// (JH = 256 / KW); a block owns a strided subset of the tiles and walks
// their planes in order.  One thread per (j,k) column.
//
// Data movement: every plane a tile needs is brought into shared memory by
// cp.async.bulk.tensor (TMA) loads -- the updated component boxes, the
// curl's component boxes with a one-row / one-column halo, the coefficient
// index (or the coefficient volumes), and for UPML tiles the auxiliary
// fields -- into a ring of S stages, each with an mbarrier that completes
// when its bytes have landed.  Thread 0 keeps the ring full across tile
// boundaries, so the loads of the next S-2 planes are in flight while a
// plane is computed.  Stores go straight to global memory, predicated on the
// component's update box, one coalesced row per warp.
//
// Plane bookkeeping: a tile with planes i0..i1 (n planes) uses n + 1
// stages.  The E sweep marches up: stage 0 holds only Hy, Hz of plane
// i0 - 1 (the x-derivative's lower neighbour) and stage q >= 1 plane
// i0 - 1 + q.  The H sweep marches down: stage 0 holds only Ey, Ez of plane
// i1 + 1 and stage q >= 1 plane i1 + 1 - q.  Plane p of the march reads
// stage p + 1; the neighbour plane's two values come from stage 0 for
// p = 0 and from the previous plane (kept in registers) after that.  Every
// thread waits on the stages it reads; a block-wide vote then releases the
// stages before it to the producer, so three stages suffice.
//
// Every mbarrier wait is bounded.  A wait that runs out records an error
// code in *err, waits (bounded) for the loads the block still has in
// flight, and leaves the block; the host reports VGPU_ETIMEOUT.
//
// UPML auxiliaries live in full-volume arrays indexed like the fields.  The
// update regions of one component never overlap (the engine checks this at
// set-up), so each point keeps exactly the auxiliary state the reference's
// per-region arrays hold.
#pragma once

#include <cuda.h>

#include "kernels.cuh"

namespace vgpu_dev {

// Bound on mbarrier polls; each poll may suspend for up to the hint below,
// so a lost transfer ends the block after about a second.
constexpr uint32_t kSpinLimit = 1u << 20;
constexpr uint32_t kSuspendHintNs = 1000;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
  for (uint32_t it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
// No multicast: the source is always this GPU's own memory.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Tensor maps of one sweep and tile shape.  own: the three updated
// components, box (W, JH); oth: the curl's three components, box (W, JH+1);
// coef: alpha/beta (E) or gamma (H) volumes, box (W, JH); idx: the one-byte
// coefficient index, box (32 bytes, JH); aux: PP0..2, P0..2 (E) or B0..2 (H).
struct SweepMaps {
  CUtensorMap own[3];
  CUtensorMap oth[3];
  CUtensorMap coef[6];
  CUtensorMap idx;
  CUtensorMap aux[6];
};

// Full-volume UPML state and 1-D profiles for the sweeps.
template <typename T>
struct PmlFull {
  const T *ad[3], *bd[3], *ah[3], *bh[3], *ibd[3], *ibh[3];
  T *aux[6];           // PP0..2, P0..2 (E sweep) or B0..2 (H sweep)
  Box lim[6][3];       // [region][component of this sweep]
};

struct SweepTile {
  int region;          // -1 bulk, else PML region ordinal
  int i0, i1;          // planes (inclusive)
  int j0, k0;          // first column
};

__host__ __device__ constexpr uint32_t round128(uint32_t b) { return (b + 127u) / 128u * 128u; }

template <typename T, int KW, bool ESWEEP, bool PML>
struct SweepLayout {
  static constexpr int JH = 256 / KW;
  static constexpr int HALO = 16 / (int)sizeof(T);   // elements per 16 bytes
  static constexpr int W = KW + HALO;                // box width in elements
  static constexpr int NCOEF = ESWEEP ? 6 : 3;
  static constexpr int NAUX = PML ? (ESWEEP ? 6 : 3) : 0;
  static constexpr int S = (sizeof(T) == 8 && PML) ? 3 : 4;   // >= 3 (see above)
  static constexpr uint32_t OWN_B = (uint32_t)(W * JH * sizeof(T));
  static constexpr uint32_t OTH_B = (uint32_t)(W * (JH + 1) * sizeof(T));
  static constexpr uint32_t IDX_B = 32u * JH;
  static constexpr uint32_t OFF_OWN = 0;
  static constexpr uint32_t OFF_OTH = OFF_OWN + 3 * round128(OWN_B);
  static constexpr uint32_t OFF_AUX = OFF_OTH + 3 * round128(OTH_B);
  static constexpr uint32_t OFF_CF = OFF_AUX + NAUX * round128(OWN_B);
  __host__ __device__ static constexpr uint32_t stage_bytes(bool compressed)
  {
    return OFF_CF + (compressed ? round128(IDX_B) : NCOEF * round128(OWN_B));
  }
  // Bytes a full stage receives, and a partial one (two curl components).
  __host__ __device__ static constexpr uint32_t full_tx(bool compressed)
  {
    return 3 * OWN_B + 3 * OTH_B + NAUX * OWN_B + (compressed ? IDX_B : NCOEF * OWN_B);
  }
  static constexpr uint32_t PARTIAL_TX = 2 * OTH_B;
  __host__ __device__ static constexpr uint32_t smem_bytes(bool compressed) { return S * stage_bytes(compressed); }
};

template <typename T, int KW, bool ESWEEP, bool PML>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && !PML) ? 4 : 2)
    k_sweep_tma(const __grid_constant__ SweepMaps maps, Grid<T> g, const SweepTile *__restrict__ tiles, int ntiles,
                Box b0in, Box b1in, Box b2in, PmlFull<T> pf, CoefIndex ci, int *err)
{
  using L = SweepLayout<T, KW, ESWEEP, PML>;
  constexpr int S = L::S, W = L::W, HALO = L::HALO;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t full[S];
  __shared__ T tab[256 * L::NCOEF];
  __shared__ int sh_err;

  const bool compressed = ci.idx != nullptr;
  const uint32_t stage_b = L::stage_bytes(compressed);
  const uint32_t full_tx = L::full_tx(compressed);
  const int tid = threadIdx.x;
  const int kl = tid % KW, jl = tid / KW;

  if (tid == 0) {
    // After an earlier pipeline failure the run is lost: skip the work.
    sh_err = *(volatile int *)err;
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  if (compressed) {
    const T *src = (const T *)ci.table;
    for (int q = tid; q < ci.ntab * L::NCOEF; q += 256) tab[q] = src[q];
  }
  __syncthreads();
  if (sh_err) return;

  // Producer cursor (thread 0): next tile ordinal and stage within it.
  int pm = 0, pq = 0;
  int64_t issued = 0, waited = 0;

  auto produce_one = [&]() -> bool {
    const int tile_id = blockIdx.x + pm * gridDim.x;
    if (tile_id >= ntiles) return false;
    const SweepTile tt = tiles[tile_id];
    const int n = tt.i1 - tt.i0 + 1;
    const int slot = (int)(issued % S);
    unsigned char *st = smem + (size_t)slot * stage_b;
    uint64_t *bar = &full[slot];
    const int xs_e = tt.k0 & ~(HALO - 1);
    const int xs_o = ESWEEP ? ((tt.k0 - 1) & ~(HALO - 1)) : xs_e;
    const int yo = ESWEEP ? tt.j0 - 1 : tt.j0;
    const int i = ESWEEP ? tt.i0 - 1 + pq : tt.i1 + 1 - pq;
    const bool partial = pq == 0;
    if (partial) {
      mbar_arrive_expect_tx(bar, L::PARTIAL_TX);
      for (int c = 1; c < 3; c++) tma_load_3d(st + L::OFF_OTH + c * round128(L::OTH_B), &maps.oth[c], bar, xs_o, yo, i);
    } else {
      mbar_arrive_expect_tx(bar, full_tx);
      for (int c = 0; c < 3; c++) tma_load_3d(st + L::OFF_OWN + c * round128(L::OWN_B), &maps.own[c], bar, xs_e, tt.j0, i);
      for (int c = 0; c < 3; c++) tma_load_3d(st + L::OFF_OTH + c * round128(L::OTH_B), &maps.oth[c], bar, xs_o, yo, i);
      for (int c = 0; c < L::NAUX; c++)
        tma_load_3d(st + L::OFF_AUX + c * round128(L::OWN_B), &maps.aux[c], bar, xs_e, tt.j0, i);
      if (compressed)
        tma_load_3d(st + L::OFF_CF, &maps.idx, bar, tt.k0 & ~15, tt.j0, i);
      else
        for (int c = 0; c < L::NCOEF; c++)
          tma_load_3d(st + L::OFF_CF + c * round128(L::OWN_B), &maps.coef[c], bar, xs_e, tt.j0, i);
    }
    issued++;
    if (++pq > n) { pq = 0; pm++; }
    return true;
  };

  if (tid == 0)
    while (issued < S && produce_one()) {}

  T *__restrict__ F0 = g.F[ESWEEP ? EX : HX];
  T *__restrict__ F1 = g.F[ESWEEP ? EY : HY];
  T *__restrict__ F2 = g.F[ESWEEP ? EZ : HZ];

  int64_t cg = 0;  // stage index of the current tile's stage 0
  bool failed = false;
  for (int m = 0; !failed; m++) {
    const int tile_id = blockIdx.x + m * gridDim.x;
    if (tile_id >= ntiles) break;
    const SweepTile t = tiles[tile_id];
    const int n = t.i1 - t.i0 + 1;
    Box b0 = b0in, b1 = b1in, b2 = b2in;
    if (PML) {
      b0 = pf.lim[t.region][0];
      b1 = pf.lim[t.region][1];
      b2 = pf.lim[t.region][2];
    }
    const int k = t.k0 + kl;
    const int j = t.j0 + jl;
    const bool jok = j < g.n1;
    const int xs_e = t.k0 & ~(HALO - 1);
    const int xs_o = ESWEEP ? ((t.k0 - 1) & ~(HALO - 1)) : xs_e;
    const int io = jl * W + (k - xs_e);                        // own boxes
    const int ih = (ESWEEP ? jl + 1 : jl) * W + (k - xs_o);    // curl boxes
    const int ii = jl * 32 + (k - (t.k0 & ~15));              // index box
    const int jc = jok ? j : g.n1 - 1;
    const int kc = min(k, (int)g.s1 - 1);
    const T d1 = ld((ESWEEP ? g.idh[1] : g.ide[1]) + jc);
    const T d2 = ld((ESWEEP ? g.idh[2] : g.ide[2]) + kc);
    // The neighbour plane's two curl components at this column: Hy, Hz of
    // plane i-1 (E sweep) or Ey, Ez of plane i+1 (H sweep).
    T nb1 = 0, nb2 = 0;

    for (int p = 0; p < n; p++) {
      const int64_t A = cg + p + 1;
      bool ok = true;
      if (p == 0) {
        ok = mbar_wait(&full[cg % S], (uint32_t)((cg / S) & 1));
        if (ok) {
          const unsigned char *s0p = smem + (size_t)(cg % S) * stage_b;
          nb1 = ((const T *)(s0p + L::OFF_OTH + round128(L::OTH_B)))[ih];
          nb2 = ((const T *)(s0p + L::OFF_OTH + 2 * round128(L::OTH_B)))[ih];
        }
      }
      if (ok) ok = mbar_wait(&full[A % S], (uint32_t)((A / S) & 1));
      if (tid == 0 && ok) waited = A + 1;
      // Uniform decision, and every thread is done with the stages before A.
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      if (tid == 0)
        while (issued < A + S && produce_one()) {}

      const int i = ESWEEP ? t.i0 + p : t.i1 - p;
      const unsigned char *sc = smem + (size_t)(A % S) * stage_b;
      const T *own0 = (const T *)(sc + L::OFF_OWN);
      const T *own1 = (const T *)(sc + L::OFF_OWN + round128(L::OWN_B));
      const T *own2 = (const T *)(sc + L::OFF_OWN + 2 * round128(L::OWN_B));
      const T *oth0 = (const T *)(sc + L::OFF_OTH);
      const T *oth1 = (const T *)(sc + L::OFF_OTH + round128(L::OTH_B));
      const T *oth2 = (const T *)(sc + L::OFF_OTH + 2 * round128(L::OTH_B));

      T cf[L::NCOEF];
      if (compressed) {
        const uint8_t *ix = (const uint8_t *)(sc + L::OFF_CF);
        const T *cw = tab + L::NCOEF * (int)ix[ii];
#pragma unroll
        for (int c = 0; c < L::NCOEF; c++) cf[c] = cw[c];
      } else {
#pragma unroll
        for (int c = 0; c < L::NCOEF; c++) cf[c] = ((const T *)(sc + L::OFF_CF + c * round128(L::OWN_B)))[io];
      }
      const T v0 = own0[io], v1 = own1[io], v2 = own2[io];
      const bool s0 = jok && b0.contains(i, j, k);
      const bool s1 = jok && b1.contains(i, j, k);
      const bool s2 = jok && b2.contains(i, j, k);
      const int64_t x = g.at(i, jc, kc);
      T c0, c1, c2;
      if (ESWEEP) {
        // curl H (src/grid.h:139-167): hz_jm = Hz(j-1), hy_km = Hy(k-1),
        // hx_km = Hx(k-1), hx_jm = Hx(j-1); nb = H of plane i-1.
        const T idhx = ld(g.idh[0] + i);
        const T hx = oth0[ih], hy = oth1[ih], hz = oth2[ih];
        c0 = d1 * (hz - oth2[ih - W]) + d2 * (oth1[ih - 1] - hy);
        c1 = d2 * (hx - oth0[ih - 1]) + idhx * (nb2 - hz);
        c2 = idhx * (hy - nb1) + d1 * (oth0[ih - W] - hx);
        nb1 = hy;
        nb2 = hz;
      } else {
        // curl E (src/grid.h:264-283): neighbours at j+1, k+1; nb = E of
        // plane i+1.
        const T idex = ld(g.ide[0] + i);
        const T ex = oth0[ih], ey = oth1[ih], ez = oth2[ih];
        c0 = d2 * (oth1[ih + 1] - ey) + d1 * (ez - oth2[ih + W]);
        c1 = idex * (nb2 - ez) + d2 * (ex - oth0[ih + 1]);
        c2 = d1 * (oth0[ih + W] - ex) + idex * (ey - nb1);
        nb1 = ey;
        nb2 = ez;
      }
      if (!PML) {
        if (ESWEEP) {
          if (s0) F0[x] = cf[0] * v0 + cf[3] * c0;
          if (s1) F1[x] = cf[1] * v1 + cf[4] * c1;
          if (s2) F2[x] = cf[2] * v2 + cf[5] * c2;
        } else {
          if (s0) F0[x] = v0 + cf[0] * c0;
          if (s1) F1[x] = v1 + cf[1] * c1;
          if (s2) F2[x] = v2 + cf[2] * c2;
        }
      } else {
        const T *ax = (const T *)(sc + L::OFF_AUX);
        const int ab = (int)(round128(L::OWN_B) / sizeof(T));  // elements between aux boxes
        const T ad0 = ld(pf.ad[0] + i), bd0 = ld(pf.bd[0] + i), ah0 = ld(pf.ah[0] + i);
        const T ad1 = ld(pf.ad[1] + jc), bd1 = ld(pf.bd[1] + jc), ah1 = ld(pf.ah[1] + jc);
        const T ad2 = ld(pf.ad[2] + kc), bd2 = ld(pf.bd[2] + kc), ah2 = ld(pf.ah[2] + kc);
        if (ESWEEP) {
          // src/pml.c:859-1023: PP = alpha PP + beta curl; P from PP's
          // change; E from P's change.
          const T ibh0 = ld(pf.ibh[0] + i), ibh1 = ld(pf.ibh[1] + jc), ibh2 = ld(pf.ibh[2] + kc);
          if (s0) {
            const T oPP = ax[io], oP = ax[3 * ab + io];
            const T nPP = cf[0] * oPP + cf[3] * c0;
            pf.aux[0][x] = nPP;
            const T nP = ad1 * oP + bd1 * (nPP - oPP);
            pf.aux[3][x] = nP;
            F0[x] = ad2 * v0 + bd2 * ibh0 * (nP - ah0 * oP);
          }
          if (s1) {
            const T oPP = ax[ab + io], oP = ax[4 * ab + io];
            const T nPP = cf[1] * oPP + cf[4] * c1;
            pf.aux[1][x] = nPP;
            const T nP = ad2 * oP + bd2 * (nPP - oPP);
            pf.aux[4][x] = nP;
            F1[x] = ad0 * v1 + bd0 * ibh1 * (nP - ah1 * oP);
          }
          if (s2) {
            const T oPP = ax[2 * ab + io], oP = ax[5 * ab + io];
            const T nPP = cf[2] * oPP + cf[5] * c2;
            pf.aux[2][x] = nPP;
            const T nP = ad0 * oP + bd0 * (nPP - oPP);
            pf.aux[5][x] = nP;
            F2[x] = ad1 * v2 + bd1 * ibh2 * (nP - ah2 * oP);
          }
        } else {
          // src/pml.c:1026-1176: B = ah B + gamma bh curl; H from B's change.
          const T bh0 = ld(pf.bh[0] + i), bh1 = ld(pf.bh[1] + jc), bh2 = ld(pf.bh[2] + kc);
          const T ibd0 = ld(pf.ibd[0] + i), ibd1 = ld(pf.ibd[1] + jc), ibd2 = ld(pf.ibd[2] + kc);
          if (s0) {
            const T oB = ax[io];
            const T nB = ah1 * oB + cf[0] * bh1 * c0;
            pf.aux[0][x] = nB;
            F0[x] = ah2 * v0 + bh2 * ibd0 * (nB - ad0 * oB);
          }
          if (s1) {
            const T oB = ax[ab + io];
            const T nB = ah2 * oB + cf[1] * bh2 * c1;
            pf.aux[1][x] = nB;
            F1[x] = ah0 * v1 + bh0 * ibd1 * (nB - ad1 * oB);
          }
          if (s2) {
            const T oB = ax[2 * ab + io];
            const T nB = ah0 * oB + cf[2] * bh0 * c2;
            pf.aux[2][x] = nB;
            F2[x] = ah1 * v2 + bh1 * ibd2 * (nB - ad2 * oB);
          }
        }
      }
    }
    cg += n + 1;
  }

  if (failed && tid == 0) {
    // Record the failure, then let the loads still in flight land before
    // the block's shared memory is released.
    atomicCAS(err, 0, 1);
    for (int64_t q = waited; q < issued; q++) (void)mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
  }
}

}  // namespace vgpu_dev
