// sweep_tma.cuh -- TMA-pipelined E and H sweeps (sm_100a).
//
// The bulk Yee updates (src/grid.c:709-888) and the UPML updates
// (src/pml.c:859-1176) as persistent marching sweeps.  The host cuts the
// grid into tiles of 32 (k) x 8 (j) columns and a run of i planes; a block
// owns a strided subset of the tiles and walks their planes in order.
// Eight compute warps hold one (j,k) column per thread; lane 0 of a ninth
// warp issues the loads.
//
// Data movement: every plane a tile needs is brought into shared memory by
// cp.async.bulk.tensor (TMA) loads -- the updated component boxes, the
// curl's component boxes with a one-row / 16-byte halo, the coefficient
// index (or the coefficient volumes), and for tiles with UPML points the
// auxiliary fields -- into a ring of S stages.  Each stage has an mbarrier
// that completes when its bytes have landed and a second one that completes
// when the compute warps have read it.  The producer keeps the ring full
// across tile boundaries, so the next planes' loads are in flight while a
// plane is computed.  Stores go straight to global memory, predicated on
// the point's update box, one coalesced row per warp.
//
// One launch per half step.  Without UPML regions the bulk kernel (PML =
// false) takes every tile.  With them the UPML kernel does: the bulk tiles,
// the X and Y regions' tiles and the bulk-footprint tiles whose k rows reach
// into a Z region, interleaved; each point picks the bulk or the UPML update
// from the boxes it lies in, so the thin Z slabs ride in the same 32-wide
// rows as the bulk next to them, with their auxiliaries in narrow boxes over
// the slab's columns, and bulk-only tiles load no auxiliaries.
//
// Plane bookkeeping: a tile with planes i0..i1 (n planes) uses n + 1
// stages.  The E sweep marches up: stage 0 holds only Hy, Hz of plane
// i0 - 1 (the x-derivative's lower neighbour) and stage q >= 1 plane
// i0 - 1 + q.  The H sweep marches down: stage 0 holds only Ey, Ez of plane
// i1 + 1 and stage q >= 1 plane i1 + 1 - q.  Plane p of the march reads
// stage p + 1; the neighbour plane's two values come from stage 0 for
// p = 0 and from the previous plane (kept in registers) after that.
// Stage 0 also brings the tile's header (SweepHeader), built on the host,
// so the compute warps read nothing from global memory.
//
// Every mbarrier wait is bounded.  A wait that runs out records an error
// code in *err and ends the warp; the producer, the block's last thread,
// first waits (bounded) for the loads it has in flight.  The host reports
// VGPU_ETIMEOUT, and later launches of the run return at once.
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
// so a lost transfer ends the warp after about a second.
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

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t polls = kSpinLimit)
{
  for (uint32_t it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Polls a compute warp makes on a stage's data barrier before it gives up.
// kSpinLimit unless a test lowers it (vgpu_set_sweep_wait_limit) to make the
// wait run out; the producer's waits always keep kSpinLimit, so a block
// whose compute warps left still waits for every load it issued.
__device__ uint32_t g_full_wait_polls = kSpinLimit;

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

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Tensor maps of one sweep.  own: the three updated components, box
// (32, 8); oth: the curl's three components, box (32 + halo, 9); coef:
// alpha/beta (E) or gamma (H) volumes, box (32, 8); idx: the one-byte
// coefficient index, box (32 bytes, 8); aux: PP0..2, P0..2 (E) or B0..2
// (H), box (32, 8); auxn: the same volumes, box (wn, 8), over a Z slab's
// columns only.
struct SweepMaps {
  CUtensorMap own[3];
  CUtensorMap oth[3];
  CUtensorMap coef[6];
  CUtensorMap idx;
  CUtensorMap aux[6];
  CUtensorMap auxn[6];
  int wn;              // width of the auxn boxes in elements (0: unused)
};

// Full-volume UPML auxiliaries of one sweep.
template <typename T>
struct PmlFull {
  T *aux[6];           // PP0..2, P0..2 (E sweep) or B0..2 (H sweep)
};

// A tile: planes i0..i1 of the 32 x 8 columns starting at (j0, k0), k0 a
// multiple of 32.  Its points update with the bulk formula where `bulk` is
// set and they lie in the bulk box, and with the UPML formula where they lie
// in the box of region reg[0] or reg[1] (-1: none).  UPML auxiliaries come
// in full-width boxes (ax < 0) or, for a tile whose only UPML points are
// one Z slab, in narrow boxes starting at column ax.
struct SweepTile {
  int reg[2];
  int bulk;
  int i0, i1;
  int j0, k0;
  int ax;
};

constexpr int kSweepKW = 32;   // k columns per tile (one warp row)
constexpr int kSweepJH = 8;    // j rows per tile (one per compute warp)
constexpr int kSweepMaxPlanes = 32;
constexpr int kSweepThreads = 288;

// Per-tile values, built on the host and copied into shared memory with the
// tile's stage 0: the tile, per-plane line lengths and UPML x profiles
// (entry p = plane p of the march), per-row and per-column ones, and
// box-membership masks (bit c: bulk box of component c, bit 3+c: region
// reg[0], bit 6+c: region reg[1]); a point's mask is
// row_mask[j] & col_mask[k] & plane_mask[p].  UPML profiles are ordered
// (a, b, c, d) = (ad, bd, ah, ibh) for E and (ah, bh, ad, ibd) for H.
template <typename T, bool PML>
struct alignas(16) SweepHeader {
  SweepTile t;
  uint32_t plane_mask[kSweepMaxPlanes];
  uint32_t row_mask[kSweepJH];
  uint32_t col_mask[kSweepKW];
  T dx[kSweepMaxPlanes];
  T dy[kSweepJH];
  T dz[kSweepKW];
  T px[PML ? 4 : 1][kSweepMaxPlanes];
  T py[PML ? 4 : 1][kSweepJH];
  T pz[PML ? 4 : 1][kSweepKW];
};

__host__ __device__ constexpr uint32_t round128(uint32_t b) { return (b + 127u) / 128u * 128u; }

// What k_headers needs beside the tiles: the sweep's components' bulk boxes
// and UPML region boxes, the line lengths (E sweep: idh; H sweep: ide) and
// the four UPML profiles (a, b, c, d) per axis, all in the storage type.
struct HeaderBoxes {
  Box bulk[3];
  Box reg[6][3];   // [region][component]
};

template <typename T>
struct HeaderLines {
  const T *line[3];
  const T *prof[4][3];
  int n[3];
};

// The headers of a tile list (SweepHeader), one warp per tile: lane l fills
// plane l of the march, row l (l < 8) and column l.  A value outside the
// grid is 0; a plane past the tile's last has an empty mask.
template <typename T, bool ES, bool PML>
__global__ void k_headers(const SweepTile *__restrict__ tiles, int ntiles, HeaderBoxes hb, HeaderLines<T> hl,
                          SweepHeader<T, PML> *__restrict__ out)
{
  const int q = blockIdx.x, l = threadIdx.x;
  if (q >= ntiles) return;
  const SweepTile t = tiles[q];
  SweepHeader<T, PML> &h = out[q];
  auto bits = [&](int v, int axis) {
    auto in = [&](const Box &b) -> uint32_t {
      const int lo = axis == 0 ? b.i0 : axis == 1 ? b.j0 : b.k0, hi = axis == 0 ? b.i1 : axis == 1 ? b.j1 : b.k1;
      return (v >= lo && v <= hi) ? 1u : 0u;
    };
    uint32_t m = 0;
    for (int c = 0; c < 3; c++) {
      if (t.bulk) m |= in(hb.bulk[c]) << c;
      if (PML && t.reg[0] >= 0) m |= in(hb.reg[t.reg[0]][c]) << (3 + c);
      if (PML && t.reg[1] >= 0) m |= in(hb.reg[t.reg[1]][c]) << (6 + c);
    }
    return m;
  };
  auto at = [&](const T *a, int axis, int v) { return (a && v >= 0 && v < hl.n[axis]) ? a[v] : (T)0; };
  if (l == 0) h.t = t;
  const int n = t.i1 - t.i0 + 1;
  const int i = ES ? t.i0 + l : t.i1 - l;
  h.plane_mask[l] = l < n ? bits(i, 0) : 0u;
  h.dx[l] = at(hl.line[0], 0, i);
  if (PML)
    for (int a = 0; a < 4; a++) h.px[a][l] = at(hl.prof[a][0], 0, i);
  if (l < kSweepJH) {
    const int j = t.j0 + l;
    h.row_mask[l] = j < hl.n[1] ? bits(j, 1) : 0u;
    h.dy[l] = at(hl.line[1], 1, j);
    if (PML)
      for (int a = 0; a < 4; a++) h.py[a][l] = at(hl.prof[a][1], 1, j);
  }
  const int k = t.k0 + l;
  h.col_mask[l] = bits(k, 2);
  h.dz[l] = at(hl.line[2], 2, k);
  if (PML)
    for (int a = 0; a < 4; a++) h.pz[a][l] = at(hl.prof[a][2], 2, k);
}

// ---- grouped sweeps: one launch over the tiles of many meshes ------------
//
// A group launch takes a list of tiles drawn from many independent meshes of
// one precision (the batched form of the solver's propagate() loop).  Each
// tile names its mesh and its header; the mesh's descriptor in global memory
// holds its tensor maps, the per-mesh values the compute warps need and its
// coefficient table.  The producer brings the mesh values and, when the
// tile's mesh differs from the one last loaded into that buffer, the
// coefficient table into shared memory with the tile's stage 0.  Blocks
// take chunks of consecutive list positions from a counter as they go (the
// next chunk is requested while the current one issues), so the launch ends
// evenly however uneven its tiles' costs; the list runs mesh by mesh, so
// the tiles in flight at one time are neighbours in a few meshes (their
// halo rows meet in L2) and a block changes mesh at most once per chunk.
// After its last tile the producer hands the compute warps a stage 0 whose
// header holds no planes, which ends their loop.

constexpr int kGroupTab = 64;   // coefficient tuples a grouped mesh may have

// Per-mesh values the compute warps read, copied into shared memory with a
// tile's stage 0.
template <typename T>
struct alignas(16) GroupMeshCompute {
  T *F[3];          // the three updated components
  T *aux[6];        // full-volume UPML auxiliaries (PmlFull)
  int64_t s0, s1;   // strides of i and j
  int n1, wn;       // j extent; width of the narrow auxiliary boxes
  int pad[2];
};

// One mesh of a group.  Tensor maps in global memory are copied to the
// device by a stream-ordered copy before the launch; the producer fences
// them (tensormap proxy acquire, GPU scope) when it moves to the mesh, so
// its TMA loads read the maps as copied, not a descriptor cached from
// earlier contents of the same address.
template <typename T>
struct alignas(64) GroupMesh {
  SweepMaps maps;
  GroupMeshCompute<T> mc;
  const void *headers;   // SweepHeader<T, PML>[this mesh's tiles]
  const T *table;        // coefficient tuples, 16-byte aligned
  uint32_t tab_bytes;    // the table's bytes, a multiple of 16
  int pad;
};

struct GroupTile {
  SweepTile t;
  int mesh;            // index into the group's GroupMesh array
  const void *hdr;     // the tile's SweepHeader<T, PML>
  const void *table;   // the mesh's coefficient tuples (16-byte aligned)
  uint32_t tab_bytes;  // the table's bytes, a multiple of 16
  int wn;              // the mesh's narrow auxiliary box width
};

__device__ __forceinline__ void fence_tensormap(const CUtensorMap *m)
{
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((uint64_t)m) : "memory");
}

template <typename T, bool ESWEEP, bool PML>
struct SweepLayout {
  static constexpr int JH = kSweepJH;
  static constexpr int HALO = 16 / (int)sizeof(T);   // elements per 16 bytes
  static constexpr int W = kSweepKW + HALO;          // curl boxes: the tile row plus a halo
  static constexpr int NCOEF = ESWEEP ? 6 : 3;
  static constexpr int NAUX = PML ? (ESWEEP ? 6 : 3) : 0;
  static constexpr int S = (sizeof(T) == 8 && PML) ? 3 : 4;   // ring depth
  // The tile header has two buffers: tile m + 2's stage 0 rewrites tile m's,
  // and the producer may issue it once stage g - S is released, g being its
  // place in the ring.  A tile takes at least two stages (stage 0 and one
  // plane), so g - S reaches tile m's stage 0 -- whose release ends every
  // read of tile m's header -- only while S <= 4.
  static_assert(S <= 4, "two header buffers hold only for rings of at most four stages");
  static constexpr int MIN_BLOCKS = sizeof(T) == 4 ? (PML ? 3 : 4) : 2;
  static constexpr uint32_t OWN_B = (uint32_t)(kSweepKW * JH * sizeof(T));
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
  // Bytes a full stage receives, with full-width auxiliaries.
  __host__ __device__ static constexpr uint32_t full_tx(bool compressed)
  {
    return 3 * OWN_B + 3 * OTH_B + NAUX * OWN_B + (compressed ? IDX_B : NCOEF * OWN_B);
  }
  // Stage 0: two curl components and the header.
  static constexpr uint32_t PARTIAL_TX = 2 * OTH_B + (uint32_t)sizeof(SweepHeader<T, PML>);
  __host__ __device__ static constexpr uint32_t smem_bytes(bool compressed) { return S * stage_bytes(compressed); }
};

// Block: warps 0..7 compute, warp 8 lane 0 produces.  GROUP: the ntiles
// tiles gtiles of many meshes (gm), taken `chunk` at a time from *counter
// (zero at launch); maps, g, tiles, headers, pf and ci are unused.  Every
// grouped mesh has a coefficient index of at most kGroupTab tuples.
template <typename T, bool ESWEEP, bool PML, bool GROUP = false>
__global__ void __launch_bounds__(kSweepThreads, SweepLayout<T, ESWEEP, PML>::MIN_BLOCKS)
    k_sweep_tma(const __grid_constant__ SweepMaps maps, Grid<T> g, const SweepTile *__restrict__ tiles,
                const SweepHeader<T, PML> *__restrict__ headers, int ntiles, PmlFull<T> pf, CoefIndex ci, int *err,
                const GroupMesh<T> *__restrict__ gm = nullptr, const GroupTile *__restrict__ gtiles = nullptr,
                int *counter = nullptr, int chunk = 1)
{
  using L = SweepLayout<T, ESWEEP, PML>;
  using Hdr = SweepHeader<T, PML>;
  using MC = GroupMeshCompute<T>;
  constexpr int S = L::S, W = L::W, HALO = L::HALO, KW = kSweepKW;
  constexpr int TAB = (GROUP ? kGroupTab : 256) * L::NCOEF;   // one table buffer
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t full[S], empty[S];
  __shared__ uint64_t tdone[2];   // GROUP: every compute warp has finished a tile that used buffer b
  __shared__ __align__(16) T tab[(GROUP ? 2 : 1) * TAB];
  __shared__ Hdr hdr[2];
  __shared__ MC mcs[GROUP ? 2 : 1];
  __shared__ int sh_err;

  const bool compressed = GROUP || ci.idx != nullptr;
  const uint32_t stage_b = L::stage_bytes(compressed);
  const int tid = threadIdx.x;
  const int warp = tid / 32, lane = tid % 32;

  if (tid == 0) {
    // After an earlier pipeline failure the run is lost: skip the work.
    sh_err = *(volatile int *)err;
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 8);
    }
    if (GROUP)
      for (int b = 0; b < 2; b++) mbar_init(&tdone[b], 8);
    mbar_fence_init();
  }
  if (!GROUP && compressed) {
    const T *src = (const T *)ci.table;
    for (int q = tid; q < ci.ntab * L::NCOEF; q += kSweepThreads) tab[q] = src[q];
  }
  __syncthreads();
  if (sh_err) return;

  if (warp == 8) {
    // ---- producer ----
    if (lane != 0) return;
    const uint32_t full_tx = L::full_tx(compressed);
    uint32_t gs = 0;
    bool ok = true;
    // Solo: positions blockIdx.x, + gridDim.x, ...  GROUP: the current
    // chunk [.., cend) and the start of the next one, already requested.
    int id = (int)blockIdx.x, cend = 0, pend = 0;
    if (GROUP) {
      id = atomicAdd(counter, chunk);
      cend = min(id + chunk, ntiles);
      pend = id < ntiles ? atomicAdd(counter, chunk) : ntiles;
    }
    auto next_pos = [&](int cur) {
      if (!GROUP) return cur + (int)gridDim.x;
      if (cur + 1 < cend) return cur + 1;
      const int n0 = pend;
      cend = min(n0 + chunk, ntiles);
      pend = n0 < ntiles ? atomicAdd(counter, chunk) : ntiles;
      return n0;
    };
    SweepTile tt{};
    GroupTile gt{};
    if (id < ntiles) {
      if (GROUP) gt = gtiles[id];
      else tt = tiles[id];
    }
    // GROUP: the mesh of the previous tile (its maps fenced) and the meshes
    // whose tables the two table buffers hold.  Buffer b (m & 1) of the
    // header, mesh values and table is rewritten for tile m only once every
    // compute warp has finished tile m - 2 (tdone[b]): a warp reads the mesh
    // values while it stores, after it has released the tile's last stage.
    int cur_mesh = -1, tab_mesh0 = -1, tab_mesh1 = -1;
    uint32_t fenced = 0;   // map sets of cur_mesh fenced: 1 own/oth/idx, 2 aux, 4 auxn
    uint32_t m = 0;
    for (; ok && id < ntiles; m++) {
      // The next tile's record loads while this one issues.
      const int id_next = next_pos(id);
      SweepTile nt{};
      GroupTile ngt{};
      if (id_next < ntiles) {
        if (GROUP) ngt = gtiles[id_next];
        else nt = tiles[id_next];
      }
      if (GROUP) tt = gt.t;
      const SweepMaps *mp = &maps;
      if (GROUP) {
        // Each set of the mesh's maps is fenced before its first use since
        // the block moved to the mesh.
        mp = &gm[gt.mesh].maps;
        if (gt.mesh != cur_mesh) {
          cur_mesh = gt.mesh;
          fenced = 0;
        }
        const uint32_t need = 1u | (PML && tt.reg[0] >= 0 ? (tt.ax < 0 ? 2u : 4u) : 0u);
        if (need & ~fenced & 1u) {
          for (int c = 0; c < 3; c++) {
            fence_tensormap(&mp->own[c]);
            fence_tensormap(&mp->oth[c]);
          }
          fence_tensormap(&mp->idx);
        }
        if (need & ~fenced & 2u)
          for (int c = 0; c < L::NAUX; c++) fence_tensormap(&mp->aux[c]);
        if (need & ~fenced & 4u)
          for (int c = 0; c < L::NAUX; c++) fence_tensormap(&mp->auxn[c]);
        fenced |= need;
      }
      const int wn = GROUP ? gt.wn : maps.wn;
      const uint32_t narrow_tx = full_tx - L::NAUX * L::OWN_B + L::NAUX * (uint32_t)(wn * L::JH * sizeof(T));
      const int n = tt.i1 - tt.i0 + 1;
      const int xs_o = ESWEEP ? tt.k0 - HALO : tt.k0;
      const int yo = ESWEEP ? tt.j0 - 1 : tt.j0;
      for (int q = 0; q <= n; q++) {
        const uint32_t slot = gs % S;
        if (gs >= S && !mbar_wait(&empty[slot], ((gs / S) - 1) & 1)) {
          ok = false;
          break;
        }
        unsigned char *st = smem + slot * stage_b;
        uint64_t *bar = &full[slot];
        const int i = ESWEEP ? tt.i0 - 1 + q : tt.i1 + 1 - q;
        if (q == 0) {
          if (GROUP) {
            const int b = (int)(m & 1);
            const bool need_tab = (b ? tab_mesh1 : tab_mesh0) != gt.mesh;
            if (m >= 2 && !mbar_wait(&tdone[b], ((m >> 1) - 1) & 1)) {
              ok = false;
              break;
            }
            const uint32_t tb = need_tab ? gt.tab_bytes : 0u;
            mbar_arrive_expect_tx(bar, L::PARTIAL_TX + (uint32_t)sizeof(MC) + tb);
            bulk_load(&hdr[b], gt.hdr, (uint32_t)sizeof(Hdr), bar);
            bulk_load(&mcs[b], &gm[gt.mesh].mc, (uint32_t)sizeof(MC), bar);
            if (need_tab) {
              bulk_load(tab + b * TAB, gt.table, tb, bar);
              if (b) tab_mesh1 = gt.mesh;
              else tab_mesh0 = gt.mesh;
            }
          } else {
            mbar_arrive_expect_tx(bar, L::PARTIAL_TX);
            bulk_load(&hdr[m & 1], headers + id, (uint32_t)sizeof(Hdr), bar);
          }
          for (int c = 1; c < 3; c++)
            tma_load_3d(st + L::OFF_OTH + c * round128(L::OTH_B), &mp->oth[c], bar, xs_o, yo, i);
        } else {
          // Tiles of bulk points only (reg[0] < 0) load no auxiliaries.
          const bool has_aux = tt.reg[0] >= 0;
          mbar_arrive_expect_tx(bar, !has_aux ? full_tx - L::NAUX * L::OWN_B : (tt.ax < 0 ? full_tx : narrow_tx));
          for (int c = 0; c < 3; c++)
            tma_load_3d(st + L::OFF_OWN + c * round128(L::OWN_B), &mp->own[c], bar, tt.k0, tt.j0, i);
          for (int c = 0; c < 3; c++)
            tma_load_3d(st + L::OFF_OTH + c * round128(L::OTH_B), &mp->oth[c], bar, xs_o, yo, i);
          for (int c = 0; c < (has_aux ? L::NAUX : 0); c++) {
            if (tt.ax < 0)
              tma_load_3d(st + L::OFF_AUX + c * round128(L::OWN_B), &mp->aux[c], bar, tt.k0, tt.j0, i);
            else
              tma_load_3d(st + L::OFF_AUX + c * round128(L::OWN_B), &mp->auxn[c], bar, tt.ax, tt.j0, i);
          }
          if (compressed)
            tma_load_3d(st + L::OFF_CF, &mp->idx, bar, tt.k0, tt.j0, i);
          else
            for (int c = 0; c < L::NCOEF; c++)
              tma_load_3d(st + L::OFF_CF + c * round128(L::OWN_B), &mp->coef[c], bar, tt.k0, tt.j0, i);
        }
        gs++;
      }
      id = id_next;
      if (GROUP) gt = ngt;
      else tt = nt;
    }
    // GROUP: a stage 0 whose header holds no planes ends the compute warps'
    // loop.  Written by this thread into the header buffer, then released
    // by a plain arrival (the barrier expects one arrival and no bytes).
    if (GROUP && ok) {
      const uint32_t slot = gs % S;
      if ((gs >= S && !mbar_wait(&empty[slot], ((gs / S) - 1) & 1)) ||
          (m >= 2 && !mbar_wait(&tdone[m & 1], ((m >> 1) - 1) & 1))) {
        ok = false;
      } else {
        hdr[m & 1].t.i0 = 1;
        hdr[m & 1].t.i1 = 0;
        mbar_arrive(&full[slot]);
        gs++;
      }
    }
    if (!ok) atomicCAS(err, 0, 1);
    // No load may still be in flight when the block's last thread leaves.
    for (uint32_t q = gs > S ? gs - S : 0; q < gs; q++) (void)mbar_wait(&full[q % S], (q / S) & 1);
    return;
  }

  // ---- compute warps ----
  const uint32_t full_polls = *(volatile uint32_t *)&g_full_wait_polls;
  const int kl = tid % KW, jl = tid / KW;
  const int io = jl * KW + kl;                        // row-wide boxes
  const int ih = (ESWEEP ? jl + 1 : jl) * W + (ESWEEP ? kl + HALO : kl);   // curl boxes
  uint32_t gs = 0;
  for (uint32_t m = 0;; m++) {
    if (!GROUP && (int)(blockIdx.x + m * gridDim.x) >= ntiles) return;
    // Stage 0 of the tile, with its header.
    uint32_t slot = gs % S;
    bool ok = mbar_wait(&full[slot], (gs / S) & 1, full_polls);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicCAS(err, 0, 1);
      return;
    }
    const Hdr &h = hdr[m & 1];
    const SweepTile t = h.t;
    if (GROUP && t.i1 < t.i0) return;   // the producer's end mark
    // The tile's mesh: the launch's own (solo) or the one stage 0 brought.
    const MC &mc = mcs[GROUP ? (m & 1) : 0];
    T *__restrict__ F0 = GROUP ? mc.F[0] : g.F[ESWEEP ? EX : HX];
    T *__restrict__ F1 = GROUP ? mc.F[1] : g.F[ESWEEP ? EY : HY];
    T *__restrict__ F2 = GROUP ? mc.F[2] : g.F[ESWEEP ? EZ : HZ];
    const int64_t s0 = GROUP ? mc.s0 : g.s0, s1 = GROUP ? mc.s1 : g.s1;
    const int n1 = GROUP ? mc.n1 : g.n1;
    const int wn = GROUP ? mc.wn : maps.wn;
    const T *tabm = tab + (GROUP ? (int)(m & 1) * TAB : 0);
    const int n = t.i1 - t.i0 + 1;
    const int k = t.k0 + kl;
    const int j = t.j0 + jl;
    // UPML auxiliaries: full-width boxes share the row-wide layout.
    const int ia = t.ax < 0 ? io : jl * wn + (k - t.ax);
    const int jc = min(j, n1 - 1);
    const int kc = min(k, (int)s1 - 1);
    const int64_t x0 = (int64_t)jc * s1 + kc;
    const uint32_t col = h.row_mask[jl] & h.col_mask[kl];
    const uint32_t pm_l = h.plane_mask[lane];
    const T d1 = h.dy[jl], d2 = h.dz[kl], dx_l = h.dx[lane];
    T pa_l = 0, pb_l = 0, pc_l = 0, pd_l = 0;   // x profiles of plane = lane
    T q1a = 0, q1b = 0, q1c = 0, q1d = 0;       // y profiles of this row
    T q2a = 0, q2b = 0, q2c = 0, q2d = 0;       // z profiles of this column
    if (PML) {
      pa_l = h.px[0][lane]; pb_l = h.px[1][lane]; pc_l = h.px[2][lane]; pd_l = h.px[3][lane];
      q1a = h.py[0][jl]; q1b = h.py[1][jl]; q1c = h.py[2][jl]; q1d = h.py[3][jl];
      q2a = h.pz[0][kl]; q2b = h.pz[1][kl]; q2c = h.pz[2][kl]; q2d = h.pz[3][kl];
    }
    // The neighbour plane's two curl components at this column -- Hy, Hz of
    // plane i0-1 (E sweep) or Ey, Ez of plane i1+1 (H sweep).
    T nb1, nb2;
    {
      const unsigned char *st = smem + slot * stage_b;
      nb1 = ((const T *)(st + L::OFF_OTH + round128(L::OTH_B)))[ih];
      nb2 = ((const T *)(st + L::OFF_OTH + 2 * round128(L::OTH_B)))[ih];
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      gs++;
    }

    for (int p = 0; p < n; p++) {
      slot = gs % S;
      ok = mbar_wait(&full[slot], (gs / S) & 1, full_polls);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicCAS(err, 0, 1);
        return;
      }
      const int i = ESWEEP ? t.i0 + p : t.i1 - p;
      const T dx = __shfl_sync(0xffffffffu, dx_l, p);
      const uint32_t m9 = col & __shfl_sync(0xffffffffu, pm_l, p);
      // Which update each component takes: bit c bulk, bit 3+c UPML.
      const uint32_t sel = (m9 & 7u) | ((m9 | (m9 >> 3)) & 56u);
      const unsigned char *sc = smem + slot * stage_b;
      const T *own0 = (const T *)(sc + L::OFF_OWN);
      const T *own1 = (const T *)(sc + L::OFF_OWN + round128(L::OWN_B));
      const T *own2 = (const T *)(sc + L::OFF_OWN + 2 * round128(L::OWN_B));
      const T *oth0 = (const T *)(sc + L::OFF_OTH);
      const T *oth1 = (const T *)(sc + L::OFF_OTH + round128(L::OTH_B));
      const T *oth2 = (const T *)(sc + L::OFF_OTH + 2 * round128(L::OTH_B));

      T cf[L::NCOEF];
      if (compressed) {
        const uint8_t *ix = (const uint8_t *)(sc + L::OFF_CF);
        const T *cw = tabm + L::NCOEF * (int)ix[io];
#pragma unroll
        for (int c = 0; c < L::NCOEF; c++) cf[c] = cw[c];
      } else {
#pragma unroll
        for (int c = 0; c < L::NCOEF; c++) cf[c] = ((const T *)(sc + L::OFF_CF + c * round128(L::OWN_B)))[io];
      }
      const T v0 = own0[io], v1 = own1[io], v2 = own2[io];
      T c0, c1, c2;
      if (ESWEEP) {
        // curl H (src/grid.h:139-167): Hz(j-1), Hy(k-1), Hx(k-1), Hx(j-1),
        // and the i-1 plane's Hy, Hz from the previous plane.
        const T hx = oth0[ih], hy = oth1[ih], hz = oth2[ih];
        c0 = d1 * (hz - oth2[ih - W]) + d2 * (oth1[ih - 1] - hy);
        c1 = d2 * (hx - oth0[ih - 1]) + dx * (nb2 - hz);
        c2 = dx * (hy - nb1) + d1 * (oth0[ih - W] - hx);
        nb1 = hy;
        nb2 = hz;
      } else {
        // curl E (src/grid.h:264-283): neighbours at j+1, k+1, and the i+1
        // plane's Ey, Ez from the previous (higher) plane.
        const T ex = oth0[ih], ey = oth1[ih], ez = oth2[ih];
        c0 = d2 * (oth1[ih + 1] - ey) + d1 * (ez - oth2[ih + W]);
        c1 = dx * (nb2 - ez) + d2 * (ex - oth0[ih + 1]);
        c2 = d1 * (oth0[ih + W] - ex) + dx * (ey - nb1);
        nb1 = ey;
        nb2 = ez;
      }
      T ax0 = 0, ax1 = 0, ax2 = 0, ax3 = 0, ax4 = 0, ax5 = 0;
      if (PML && (sel & 56u)) {
        // Narrow boxes cover exactly the UPML points' columns.
        const T *ax = (const T *)(sc + L::OFF_AUX);
        constexpr int ab = (int)(round128(L::OWN_B) / sizeof(T));  // elements between aux boxes
        ax0 = ax[ia];
        ax1 = ax[ab + ia];
        ax2 = ax[2 * ab + ia];
        if (ESWEEP) {
          ax3 = ax[3 * ab + ia];
          ax4 = ax[4 * ab + ia];
          ax5 = ax[5 * ab + ia];
        }
      }
      // Every read of this stage is done: hand it back to the producer.
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      gs++;

      const int64_t x = x0 + (int64_t)i * s0;
      // UPML-region tiles hold no bulk points: the branch is uniform.
      if (!PML || t.bulk) {
        if (ESWEEP) {
          if (sel & 1u) F0[x] = cf[0] * v0 + cf[3] * c0;
          if (sel & 2u) F1[x] = cf[1] * v1 + cf[4] * c1;
          if (sel & 4u) F2[x] = cf[2] * v2 + cf[5] * c2;
        } else {
          if (sel & 1u) F0[x] = v0 + cf[0] * c0;
          if (sel & 2u) F1[x] = v1 + cf[1] * c1;
          if (sel & 4u) F2[x] = v2 + cf[2] * c2;
        }
      }
      // Bulk-only tiles (reg[0] < 0, the same for the whole block) skip the
      // UPML part, profile shuffles included.
      if (PML && t.reg[0] >= 0) {
#define AUX(c) (GROUP ? mc.aux[c] : pf.aux[c])
        const T xa = __shfl_sync(0xffffffffu, pa_l, p), xb = __shfl_sync(0xffffffffu, pb_l, p);
        const T xc = __shfl_sync(0xffffffffu, pc_l, p), xd = __shfl_sync(0xffffffffu, pd_l, p);
        if (ESWEEP) {
          // src/pml.c:859-1023: PP = alpha PP + beta curl; P from PP's
          // change; E from P's change.  (a, b, c, d) = (ad, bd, ah, ibh).
          if (sel & 8u) {
            const T nPP = cf[0] * ax0 + cf[3] * c0;
            AUX(0)[x] = nPP;
            const T nP = q1a * ax3 + q1b * (nPP - ax0);
            AUX(3)[x] = nP;
            F0[x] = q2a * v0 + q2b * xd * (nP - xc * ax3);
          }
          if (sel & 16u) {
            const T nPP = cf[1] * ax1 + cf[4] * c1;
            AUX(1)[x] = nPP;
            const T nP = q2a * ax4 + q2b * (nPP - ax1);
            AUX(4)[x] = nP;
            F1[x] = xa * v1 + xb * q1d * (nP - q1c * ax4);
          }
          if (sel & 32u) {
            const T nPP = cf[2] * ax2 + cf[5] * c2;
            AUX(2)[x] = nPP;
            const T nP = xa * ax5 + xb * (nPP - ax2);
            AUX(5)[x] = nP;
            F2[x] = q1a * v2 + q1b * q2d * (nP - q2c * ax5);
          }
        } else {
          // src/pml.c:1026-1176: B = ah B + gamma bh curl; H from B's
          // change.  (a, b, c, d) = (ah, bh, ad, ibd).
          if (sel & 8u) {
            const T nB = q1a * ax0 + cf[0] * q1b * c0;
            AUX(0)[x] = nB;
            F0[x] = q2a * v0 + q2b * xd * (nB - xc * ax0);
          }
          if (sel & 16u) {
            const T nB = q2a * ax1 + cf[1] * q2b * c1;
            AUX(1)[x] = nB;
            F1[x] = xa * v1 + xb * q1d * (nB - q1c * ax1);
          }
          if (sel & 32u) {
            const T nB = xa * ax2 + cf[2] * xb * c2;
            AUX(2)[x] = nB;
            F2[x] = q1a * v2 + q1b * q2d * (nB - q2c * ax2);
          }
        }
#undef AUX
      }
    }
    if (GROUP) {
      // Every read of buffer m & 1 by this warp is done.
      __syncwarp();
      if (lane == 0) mbar_arrive(&tdone[m & 1]);
    }
  }
}

}  // namespace vgpu_dev
