// kernels.cuh -- device kernels of the vulture_b200 FDTD engine (sm_100a).
//
// Every kernel restates one update routine of the reference time loop
// (src/simulation.c:156-222) with the same arithmetic expressions in the same
// order; the engine is built with --fmad=false so that in FP64 each value is
// bit-identical to the reference's real=double solver.  T is the storage and
// arithmetic type of fields and coefficients (double or float); DFT
// accumulators, Debye currents, SIBC filter state and the analytic incident
// field phase are always double.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "vgpu.h"

namespace vgpu_dev {

enum { EX = 0, EY, EZ, HX, HY, HZ };

// Inclusive index box.
struct Box {
  int i0, i1, j0, j1, k0, k1;
  __host__ __device__ bool contains(int i, int j, int k) const {
    return i >= i0 && i <= i1 && j >= j0 && j <= j1 && k >= k0 && k <= k1;
  }
  __host__ __device__ int ni() const { return i1 - i0 + 1; }
  __host__ __device__ int nj() const { return j1 - j0 + 1; }
  __host__ __device__ int nk() const { return k1 - k0 + 1; }
  __host__ __device__ bool empty() const { return i1 < i0 || j1 < j0 || k1 < k0; }
  __host__ __device__ int64_t count() const { return empty() ? 0 : (int64_t)ni() * nj() * nk(); }
};

static inline Box box_from(const int32_t l[6]) { return Box{ l[0], l[1], l[2], l[3], l[4], l[5] }; }

// Device view of the grid: fields, coefficients and line arrays.  Volumes are
// [n0][n1][n2p] with the k rows padded to a multiple of 32 elements.  The E
// (alpha, beta) and H (gamma) coefficients come either from full volumes
// (cf) or, for meshes with at most 256 distinct tuples, from a one-byte
// index per point and a table (cidx, ctab); coef() reads whichever is set.
template <typename T>
struct Grid {
  T *F[6];
  const T *cf[9];
  const uint8_t *cidx[2];   // E, H coefficient index (null: volumes)
  const T *ctab[2];         // tables: 6 values per E tuple, 3 per H tuple
  const T *ide[3];
  const T *idh[3];
  int n0, n1, n2;
  int64_t s0, s1;  // strides of i and j
  __device__ __forceinline__ int64_t at(int i, int j, int k) const { return (int64_t)i * s0 + (int64_t)j * s1 + k; }
  // Coefficient q (0..5 alpha/beta E x,y,z; 6..8 gamma H x,y,z) at point x.
  __device__ __forceinline__ T coef(int q, int64_t x) const
  {
    if (q < 6) return cidx[0] ? ctab[0][6 * (int)cidx[0][x] + q] : cf[q][x];
    return cidx[1] ? ctab[1][3 * (int)cidx[1][x] + (q - 6)] : cf[q][x];
  }
};

// ---------------------------------------------------------------------------
// UPML state (src/pml.c:44-84): 1-D profiles per axis and each region's
// field limits.  The auxiliary fields live in full volumes (sweep_tma.cuh).
// ---------------------------------------------------------------------------

template <typename T>
struct PmlView {
  const T *ad[3], *bd[3], *ah[3], *bh[3], *ibd[3], *ibh[3];
  int nreg;
  Box lim[6][6];       // [region][field]
};

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// Coefficient compression: when a mesh has at most 256 distinct coefficient
// tuples, idx[x] indexes a table of (alpha_x, alpha_y, alpha_z, beta_x,
// beta_y, beta_z) for E or (gamma_x, gamma_y, gamma_z) for H.  The table
// holds the same values as the full volumes, so results are unchanged.
struct CoefIndex {
  const uint8_t *idx;   // null: use the full coefficient volumes
  const void *table;    // ntab * (6 or 3) values of type T
  int ntab;
};


// ---------------------------------------------------------------------------
// Mur first-order ABC (src/mur.c:135-555).  A list of planar work items; each
// thread updates one tangential E (before the bulk update, reading the
// neighbour's pre-update value) or one normal H.
// ---------------------------------------------------------------------------

struct MurItem {
  Box b;            // the face plane for component c
  int c;            // field component
  int axis, dir;    // neighbour offset along axis (E items)
  int face;
  int64_t first;    // first flattened thread of the item
};

struct MurView {
  int nitems;
  MurItem it[12];
  double zeta[6];
};

template <typename T>
__device__ __forceinline__ T bulk_e_value(const Grid<T> &g, int c, int i, int j, int k)
{
  const int64_t x = g.at(i, j, k);
  const T *Hx = g.F[HX], *Hy = g.F[HY], *Hz = g.F[HZ];
  if (c == EX) return g.coef(0, x) * g.F[EX][x] + g.coef(3, x) * (g.idh[1][j] * (Hz[x] - Hz[x - g.s1]) + g.idh[2][k] * (Hy[x - 1] - Hy[x]));
  if (c == EY) return g.coef(1, x) * g.F[EY][x] + g.coef(4, x) * (g.idh[2][k] * (Hx[x] - Hx[x - 1]) + g.idh[0][i] * (Hz[x - g.s0] - Hz[x]));
  return g.coef(2, x) * g.F[EZ][x] + g.coef(5, x) * (g.idh[0][i] * (Hy[x] - Hy[x - g.s0]) + g.idh[1][j] * (Hx[x - g.s1] - Hx[x]));
}

// A Mur item is one face plane (fewer than 2^31 points, checked at set-up):
// its coordinates decode in 32-bit arithmetic.
template <typename T>
__device__ __forceinline__ void item_coords(const MurItem &m, int64_t t, int &i, int &j, int &k)
{
  const unsigned nj = (unsigned)m.b.nj(), nk = (unsigned)m.b.nk(), u = (unsigned)t;
  const unsigned q = u / nk, r = q / nj;
  k = m.b.k0 + (int)(u - q * nk);
  j = m.b.j0 + (int)(q - r * nj);
  i = m.b.i0 + (int)r;
}

// One launch covers every item: blockIdx.y is the item, threads walk its
// face box (k fastest), so no thread searches the item list.
template <typename T>
__global__ void k_mur_e(Grid<T> g, const __grid_constant__ MurView mv)
{
  const MurItem &m = mv.it[blockIdx.y];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.b.count()) return;
  int i, j, k;
  item_coords<T>(m, t, i, j, k);
  const int ni = i + (m.axis == 0 ? m.dir : 0), nj = j + (m.axis == 1 ? m.dir : 0), nk = k + (m.axis == 2 ? m.dir : 0);
  T tmp = bulk_e_value(g, m.c, ni, nj, nk);
  const int64_t x = g.at(i, j, k), xn = g.at(ni, nj, nk);
  T *F = g.F[m.c];
  F[x] = F[xn] + (T)mv.zeta[m.face] * (tmp - F[x]);
}

template <typename T>
__global__ void k_mur_h(Grid<T> g, const __grid_constant__ MurView mv)
{
  const MurItem &m = mv.it[blockIdx.y];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.b.count()) return;
  int i, j, k;
  item_coords<T>(m, t, i, j, k);
  const int64_t x = g.at(i, j, k);
  const T *Ex = g.F[EX], *Ey = g.F[EY], *Ez = g.F[EZ];
  if (m.c == HX)
    g.F[HX][x] = g.F[HX][x] + g.coef(6, x) * (g.ide[2][k] * (Ey[x + 1] - Ey[x]) + g.ide[1][j] * (Ez[x] - Ez[x + g.s1]));
  else if (m.c == HY)
    g.F[HY][x] = g.F[HY][x] + g.coef(7, x) * (g.ide[0][i] * (Ez[x + g.s0] - Ez[x]) + g.ide[2][k] * (Ex[x] - Ex[x + 1]));
  else
    g.F[HZ][x] = g.F[HZ][x] + g.coef(8, x) * (g.ide[1][j] * (Ex[x + g.s1] - Ex[x]) + g.ide[0][i] * (Ey[x] - Ey[x + g.s0]));
}

// ---------------------------------------------------------------------------
// Debye blocks (src/debye.c:243-307).
// ---------------------------------------------------------------------------

struct DebyeItem {
  Box b;
  int c, np;
  int64_t first;     // first flattened thread
  int64_t jofs;      // offset of this item's currents (complex) in J
  int64_t eofs;      // offset of this item's cells in lastE
  int coef_ofs;      // offset of dalpha/dbeta (complex, np each) in coefs
};

// One (item, cell) of the Debye update, thread index t over all items.  The
// independent loads (the field, its last value, the update coefficient, the
// currents) are issued before any arithmetic; the expressions are the
// reference's: E = E - beta * sum((1 + dalpha) J) rounded once to T, then
// J = dalpha J + dbeta (E - lastE).
template <typename T>
__device__ __forceinline__ void debye_point(const Grid<T> &g, const DebyeItem *__restrict__ items, int nitems,
                                            int64_t t, double2 *__restrict__ J, T *__restrict__ lastE,
                                            const double2 *__restrict__ coefs)
{
  int q = 0;
  while (q + 1 < nitems && t >= items[q + 1].first) q++;
  const DebyeItem m = items[q];
  const int64_t cell = t - m.first;
  // A block holds fewer than 2^31 cells (checked at set-up): 32-bit decode.
  const unsigned nj = (unsigned)m.b.nj(), nk = (unsigned)m.b.nk(), u = (unsigned)cell;
  const unsigned qk = u / nk, qj = qk / nj;
  const int i = m.b.i0 + (int)qj, j = m.b.j0 + (int)(qk - qj * nj), k = m.b.k0 + (int)(u - qk * nk);
  const int64_t x = g.at(i, j, k);
  T *E = g.F[m.c];
  const int64_t le = m.eofs + cell;
  const T e_old = E[x];
  const T last = lastE[le];
  const T beta = g.coef(3 + m.c, x);
  const double2 *da = coefs + m.coef_ofs, *db = da + m.np;
  double2 *Jc = J + m.jofs + cell * m.np;
  // Jsum = sum (1 + dalpha) * J, complex arithmetic as C99 (no contraction).
  double sr = 0.0, si = 0.0;
  for (int p = 0; p < m.np; p++) {
    double ar = 1 + da[p].x, ai = da[p].y;
    double2 v = Jc[p];
    sr = sr + (ar * v.x - ai * v.y);
    si = si + (ar * v.y + ai * v.x);
  }
  const T e_new = e_old - beta * sr;
  E[x] = e_new;
  const T diff = e_new - last;
  for (int p = 0; p < m.np; p++) {
    double2 v = Jc[p];
    double nr = (da[p].x * v.x - da[p].y * v.y) + db[p].x * (double)diff;
    double ni = (da[p].x * v.y + da[p].y * v.x) + db[p].y * (double)diff;
    Jc[p] = make_double2(nr, ni);
  }
  lastE[le] = e_new;
}

// Debye blocks (src/debye.c:243-307): one thread per (block, component, cell).
template <typename T>
__global__ void k_debye(Grid<T> g, const DebyeItem *items, int nitems, int64_t total, double2 *J, T *lastE,
                        const double2 *coefs)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total) debye_point(g, items, nitems, t, J, lastE, coefs);
}

// ---------------------------------------------------------------------------
// Sources (src/source.c:602-753).
// ---------------------------------------------------------------------------

// Point t of source box b at step n.
template <typename T>
__device__ __forceinline__ void source_point(const Grid<T> &g, const Box &b, int c, int kind, T soft,
                                             const T *values, uint64_t n, int64_t t)
{
  if (t >= b.count()) return;
  int64_t nj = b.nj(), nk = b.nk();
  int i = b.i0 + (int)(t / (nj * nk)), j = b.j0 + (int)((t / nk) % nj), k = b.k0 + (int)(t % nk);
  const int64_t x = g.at(i, j, k);
  T v = values[n];
  T *F = g.F[c];
  if (kind == VGPU_SRC_FIELD) F[x] = soft * F[x] + v;
  else F[x] = soft * F[x] - g.coef(c <= EZ ? 3 + c : 6 + c - HX, x) * v;
}

template <typename T>
__global__ void k_source(Grid<T> g, Box b, int c, int kind, T soft, const T *values, const uint64_t *step_base,
                         int step_rel)
{
  source_point(g, b, c, kind, soft, values, *step_base + step_rel, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Ghost layer (src/surface.c:569-812).  One launch per field type.  E: each
// component belongs to one axis.  H: each component is written by the faces of
// two axes in the reference's order (X, Y, Z); a point on two ghost planes
// takes the composition of both copies, which equals the reference's
// sequential result because every copy reads interior values.
// ---------------------------------------------------------------------------

struct GhostView {
  int mode[6];        // VGPU_GHOST_* per face
  int go_lo[3], go_hi[3];
};

__device__ __forceinline__ bool ghost_src(const GhostView &gv, int axis, int idx, int &src, int &neg)
{
  int lo = gv.go_lo[axis], hi = gv.go_hi[axis];
  int face;
  if (idx == lo - 1) face = 2 * axis;
  else if (idx == hi) face = 2 * axis + 1;
  else return false;
  int mode = gv.mode[face];
  if (mode == VGPU_GHOST_NONE) return false;
  bool is_lo = (face % 2) == 0;
  if (mode == VGPU_GHOST_PERIODIC) src = is_lo ? hi - 1 : lo;
  else src = is_lo ? lo : hi - 1;
  neg = mode == VGPU_GHOST_PMC;
  return true;
}

template <typename T>
__global__ void k_ghost(Grid<T> g, GhostView gv, int efield, int nb_all)
{
  // blockIdx.y: which (component, axis, side) plane; threads: points on it.
  int plane = blockIdx.y;
  int comp, axis, side;
  if (efield) {
    axis = plane / 2;
    side = plane % 2;
    comp = axis;
  } else {
    // H: 3 components x 2 writer axes x 2 sides.
    comp = HX + plane / 4;
    int w = (plane / 2) % 2;
    int ca = comp - HX;
    axis = (w == 0) ? (ca == 0 ? 1 : 0) : (ca == 2 ? 1 : 2);
    side = plane % 2;
  }
  int face = 2 * axis + side;
  if (gv.mode[face] == VGPU_GHOST_NONE) return;
  int b = (axis + 1) % 3, c = (axis + 2) % 3;
  int nbp = gv.go_hi[b] - gv.go_lo[b] + 2, ncp = gv.go_hi[c] - gv.go_lo[c] + 2;
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nbp * ncp) return;
  int ib = gv.go_lo[b] - 1 + (int)(t / ncp), ic = gv.go_lo[c] - 1 + (int)(t % ncp);
  int p[3];
  p[axis] = side == 0 ? gv.go_lo[axis] - 1 : gv.go_hi[axis];
  p[b] = ib;
  p[c] = ic;
  T *F = g.F[comp];
  if (efield) {
    int src, neg;
    ghost_src(gv, axis, p[axis], src, neg);
    int s[3] = { p[0], p[1], p[2] };
    s[axis] = src;
    T v = F[g.at(s[0], s[1], s[2])];
    F[g.at(p[0], p[1], p[2])] = neg ? -v : v;
    return;
  }
  // H: the writer axes of comp, in reference order.
  int ca = comp - HX;
  int A = ca == 0 ? 1 : 0;          // first writer axis
  int Bx = ca == 2 ? 1 : 2;         // second writer axis
  int srcA, negA, srcB, negB;
  bool onA = ghost_src(gv, A, p[A], srcA, negA);
  bool onB = ghost_src(gv, Bx, p[Bx], srcB, negB);
  // A point on both planes is handled by the thread of the later axis only.
  if (axis == A && onB) return;
  int s[3] = { p[0], p[1], p[2] };
  bool neg = false;
  if (onB) { s[Bx] = srcB; neg = negB; }
  if (onA) { s[A] = srcA; neg = neg != (bool)negA; }
  T v = F[g.at(s[0], s[1], s[2])];
  F[g.at(p[0], p[1], p[2])] = neg ? -v : v;
  (void)nb_all;
}

// ---------------------------------------------------------------------------
// Observers (src/observer.c:622-650, 857-899).
// ---------------------------------------------------------------------------

// Binary observers (src/observer.c:1164-1198): at the top of step n inside
// the output window, node q's six components go to row n % chunk of ring
// block (n / chunk) % 2, as float.
template <typename T>
__global__ void k_bin_observe(Grid<T> g, const int *__restrict__ pts, int64_t npts, float *__restrict__ ring,
                              const uint64_t *step_base, int step_rel, uint64_t out_start, uint64_t out_stop,
                              int chunk)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * 6) return;
  const uint64_t n = *step_base + step_rel;
  if (n < out_start || n > out_stop) return;
  const int64_t q = t / 6;
  const int c = (int)(t - q * 6);
  const int64_t x = g.at(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
  const int64_t row = (int64_t)((n / chunk) & 1) * chunk + (int64_t)(n % chunk);
  ring[row * npts * 6 + t] = (float)g.F[c][x];
}

// Samples of step n at thread t: TD points' six components into the TD
// buffer (row n - out_start), then FD points' into staging row
// (n - out_start) % tblock.
template <typename T>
__device__ __forceinline__ void observe_point(const Grid<T> &g, const int *td_pts, int num_td, const int *fd_pts,
                                              int num_fd, T *td_buf, double *fd_stage, uint64_t n,
                                              uint64_t out_start, uint64_t out_stop, int tblock, int t)
{
  if (n < out_start || n > out_stop) return;
  uint64_t row = n - out_start;
  if (t < num_td * 6) {
    int p = t / 6, c = t % 6;
    const int *pt = td_pts + 3 * p;
    td_buf[(row * num_td + p) * 6 + c] = g.F[c][g.at(pt[0], pt[1], pt[2])];
    return;
  }
  t -= num_td * 6;
  if (t < num_fd * 6) {
    int p = t / 6, c = t % 6;
    const int *pt = fd_pts + 3 * p;
    fd_stage[(row % tblock) * (int64_t)num_fd * 6 + t] = (double)g.F[c][g.at(pt[0], pt[1], pt[2])];
  }
}

template <typename T>
__global__ void k_observe(Grid<T> g, const int *td_pts, int num_td, const int *fd_pts, int num_fd, T *td_buf,
                          double *fd_stage, const uint64_t *step_base, int step_rel, uint64_t out_start,
                          uint64_t out_stop, int tblock)
{
  observe_point(g, td_pts, num_td, fd_pts, num_fd, td_buf, fd_stage, *step_base + step_rel, out_start, out_stop,
                tblock, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

// ---------------------------------------------------------------------------
// Side work of a grouped step (many meshes in one launch): each item is one
// mesh's observer samples or one of its source boxes, with its own step
// counter; block b works on the item whose block range holds b.
// ---------------------------------------------------------------------------

template <typename T>
struct GroupSide {
  const Grid<T> *g;        // the mesh's grid (device copy)
  const uint64_t *step;    // the mesh's step counter
  int first_block;         // blocks of the items before this one
  int kind;                // 0: observer samples, 1: a source box
  // source box
  Box b;
  int c, skind;
  T soft;
  const T *values;
  // observers
  const int *td_pts, *fd_pts;
  int num_td, num_fd;
  T *td_buf;
  double *fd_stage;
  uint64_t out_start, out_stop;
  int tblock;
};

template <typename T>
__global__ void k_group_side(const GroupSide<T> *__restrict__ items, int nitems, int step_rel)
{
  int lo = 0, hi = nitems - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (items[mid].first_block <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GroupSide<T> &it = items[lo];
  const int64_t t = (int64_t)(blockIdx.x - it.first_block) * blockDim.x + threadIdx.x;
  const uint64_t n = *it.step + step_rel;
  if (it.kind == 0)
    observe_point(*it.g, it.td_pts, it.num_td, it.fd_pts, it.num_fd, it.td_buf, it.fd_stage, n, it.out_start,
                  it.out_stop, it.tblock, (int)t);
  else
    source_point(*it.g, it.b, it.c, it.skind, it.soft, it.values, n, t);
}

// Advance the step counters of a group's meshes by nsteps.
__global__ void k_group_advance(uint64_t *const *steps, int n, int nsteps)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) *steps[t] += nsteps;
}

// Twiddles cos/sin(omega_f * t_n) for the rows of one DFT block.
__global__ void k_twiddle(const double *omega, int nf, double dt, uint64_t out_start, uint64_t row0, int nrows,
                          double2 *tw)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrows * nf) return;
  int r = t / nf, f = t % nf;
  double time = (double)(out_start + row0 + r) * dt;
  double wt = omega[f] * time;
  double s, c;
  sincos(wt, &s, &c);
  tw[t] = make_double2(c, s);
}

// re[pc][f] += v*cos, im[pc][f] -= v*sin for each buffered row in order, one
// thread per (pc, f): the same sequence of additions as the reference's
// per-step accumulation.
__global__ void k_dft_accumulate(const double *stage, int npc, int nf, int nrows, int row_offset, int tblock,
                                 const double2 *tw, double *re, double *im)
{
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  int pc = blockIdx.y * blockDim.y + threadIdx.y;
  extern __shared__ double sm[];
  double *vs = sm;  // [blockDim.y][nrows]
  for (int q = threadIdx.y * blockDim.x + threadIdx.x; q < blockDim.y * nrows; q += blockDim.x * blockDim.y) {
    int py = q / nrows, r = q % nrows;
    int pcq = blockIdx.y * blockDim.y + py;
    vs[q] = pcq < npc ? stage[((row_offset + r) % tblock) * (int64_t)npc + pcq] : 0.0;
  }
  __syncthreads();
  if (f >= nf || pc >= npc) return;
  double ar = re[(int64_t)pc * nf + f], ai = im[(int64_t)pc * nf + f];
  const double *v = vs + threadIdx.y * nrows;
  for (int r = 0; r < nrows; r++) {
    double2 w = tw[(int64_t)r * nf + f];
    ar = ar + v[r] * w.x;
    ai = ai - v[r] * w.y;
  }
  re[(int64_t)pc * nf + f] = ar;
  im[(int64_t)pc * nf + f] = ai;
}

// The same fold as a GEMM on the FP64 tensor cores (the tcgen05 MMA kinds
// have no f64 form; the FP64 MMA is mma.sync, here its m16n8k4 shape, which
// timed 2.6x faster than the scalar kernel above on a 98,352-series x
// 500-frequency block and 1.5x faster than the m8n8k4 shape).  For a block
// of rows r = 0..nrows-1 and a tile of 64 point-components x 32 frequencies:
//   re[pc][f] += sum_r v[r][pc] * cos(w_f t_r)
//   im[pc][f] += sum_r v[r][pc] * (-sin(w_f t_r))
// i.e. D[pc][2f + {0,1}] = A[pc][r] x B[r][2f + {0,1}] with the twiddle
// columns interleaved (cos, -sin), so each pair of a thread's accumulators
// is the re and im of one (pc, f).  The rows' sum is formed in FP64 FMAs and
// then added to the running sums (src/observer.c:857-899 adds row by row; the
// two orders agree to rounding).  Rows are taken 32 at a time through shared
// memory; rows past nrows read as zero.
constexpr int kDftTileM = 64;          // point-components per block (4 warps x 16)
constexpr int kDftTileF = 32;          // frequencies per block (64 twiddle columns)
constexpr int kDftTileK = 32;          // rows per shared-memory pass
constexpr int kDftPad = 4;             // row padding: conflict-free fragment loads

// D (16x8) += A (16x4) x B (4x8).  Fragments, g = lane / 4, t = lane % 4:
// a = {A[g][t], A[g+8][t]}, b = B[t][g], d = {D[g][2t], D[g][2t+1],
// D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void mma_f64_m16n8k4(double (&d)[4], double a0, double a1, double b)
{
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, {%0, %1, %2, %3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(b));
}

__global__ void __launch_bounds__(128) k_dft_mma(const double *__restrict__ stage, int npc, int nf, int nrows,
                                                 int row_offset, int tblock, const double2 *__restrict__ tw,
                                                 double *__restrict__ re, double *__restrict__ im, int pc0)
{
  __shared__ double As[kDftTileK][kDftTileM + kDftPad];        // [row][pc]
  __shared__ double Bs[kDftTileK][2 * kDftTileF + kDftPad];    // [row][2f + (cos, -sin)]
  // Launches cover at most 65535 tiles of point-components; pc0 is the
  // first one of this launch.
  const int m0 = pc0 + blockIdx.y * kDftTileM, f0 = blockIdx.x * kDftTileF;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, t = lane & 3;   // fragment row group and column in group
  double acc[8][4];
#pragma unroll
  for (int ni = 0; ni < 8; ni++) acc[ni][0] = acc[ni][1] = acc[ni][2] = acc[ni][3] = 0.0;
  // Each thread loads the same tile column c of rows r = tid / 64 + 2q (A)
  // and tid / 32 + 4q (B): the ring row is found once per row, not per value.
  const int ca = tid % kDftTileM, cb = tid % kDftTileF;
  for (int r0 = 0; r0 < nrows; r0 += kDftTileK) {
    const int kr = min(kDftTileK, nrows - r0);
    for (int r = tid / kDftTileM; r < kDftTileK; r += 128 / kDftTileM) {
      const int pc = m0 + ca;
      As[r][ca] = (r < kr && pc < npc) ? stage[(int64_t)((row_offset + r0 + r) % tblock) * npc + pc] : 0.0;
    }
    for (int r = tid / kDftTileF; r < kDftTileK; r += 128 / kDftTileF) {
      const int f = f0 + cb;
      const double2 w = (r < kr && f < nf) ? tw[(int64_t)(r0 + r) * nf + f] : make_double2(0.0, 0.0);
      Bs[r][2 * cb] = w.x;
      Bs[r][2 * cb + 1] = -w.y;
    }
    __syncthreads();
    // A full pass of kDftTileK rows, unrolled; rows past nrows are zeros.
#pragma unroll
    for (int k = 0; k < kDftTileK; k += 4) {
      const double a0 = As[k + t][16 * warp + g], a1 = As[k + t][16 * warp + g + 8];
      double b[8];
#pragma unroll
      for (int ni = 0; ni < 8; ni++) b[ni] = Bs[k + t][8 * ni + g];
#pragma unroll
      for (int ni = 0; ni < 8; ni++) mma_f64_m16n8k4(acc[ni], a0, a1, b[ni]);
    }
    __syncthreads();
  }
  // acc[ni][2h + j] = D[16 warp + g + 8h][8 ni + 2t + j]: column pair
  // (8 ni + 2t, +1) is frequency 4 ni + t of the tile, (re, im).
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int pc = m0 + 16 * warp + g + 8 * h;
    if (pc >= npc) continue;
#pragma unroll
    for (int ni = 0; ni < 8; ni++) {
      const int f = f0 + 4 * ni + t;
      if (f >= nf) continue;
      const int64_t x = (int64_t)pc * nf + f;
      re[x] = re[x] + acc[ni][2 * h];
      im[x] = im[x] + acc[ni][2 * h + 1];
    }
  }
}

// ---------------------------------------------------------------------------
// Waveforms on the device (src/waveform.c:412-638), used by the analytic
// plane-wave incident field.  Evaluated in double.
// ---------------------------------------------------------------------------

struct DevWaveform {
  int type, table_size;
  double size, delay, width, frequency;
  const double *table;
};

__device__ inline double dev_spline(const DevWaveform &w, double t)
{
  const double *tab = w.table;
  unsigned long n = (unsigned long)w.table_size, klo = 0, khi = n - 1, k;
  while (khi - klo > 1UL) {
    k = (khi + klo) >> 1;
    if (tab[3 * k] > t) khi = k;
    else klo = k;
  }
  double h = tab[3 * khi] - tab[3 * klo];
  double a = (tab[3 * khi] - t) / h, b = (t - tab[3 * klo]) / h;
  return a * tab[3 * klo + 1] + b * tab[3 * khi + 1] +
         ((a * a * a - a) * tab[3 * klo + 2] + (b * b * b - b) * tab[3 * khi + 2]) * (h * h) / 6.0;
}

// The reference squares with pow(v, 2.0); v * v is the correctly rounded
// square, which a correctly rounded pow also returns, at a fraction of the
// cost.
__device__ __forceinline__ double sq(double v) { return v * v; }

__device__ inline double dev_waveform(const DevWaveform &w, double t, double delay)
{
  const double pi = 3.14159265358979311600;  // 4*atan(1) in double
  double x = t - delay - w.delay, W = w.width, f = w.frequency, env;
  switch (w.type) {
    case VGPU_WF_GAUSSIAN_PULSE:
    case VGPU_WF_NARROW_GAUSSIAN_PULSE: return w.size * exp(-0.5 * sq(x / W));
    case VGPU_WF_DIFF_GAUSSIAN_PULSE: return w.size * (-x / W * exp(-0.5 * sq(x / W)));
    case VGPU_WF_RICKER_WAVELET: return w.size * ((1.0 - sq(x / W)) * exp(-0.5 * sq(x / W)));
    case VGPU_WF_MOD_GAUSSIAN_PULSE: return w.size * (exp(-0.5 * sq(x / W)) * sin(2.0 * pi * f * x));
    case VGPU_WF_COMPACT_PULSE:
    case VGPU_WF_MOD_COMPACT_PULSE:
      if (x <= 0.0) env = 0.0;
      else if (x < 2.0 * W)
        env = 1.0 / 32.0 * (10.0 - 15.0 * cos(pi / W * x) + 6.0 * cos(2.0 * pi / W * x) - cos(3.0 * pi / W * x));
      else env = 0.0;
      return w.type == VGPU_WF_COMPACT_PULSE ? w.size * env : w.size * (env * sin(2.0 * pi * f * x));
    case VGPU_WF_DIFF_COMPACT_PULSE:
      if (x <= 0.0 || x >= 2.0 * W) return w.size * 0.0;
      return w.size * (1.0 / 32.0 * (15.0 * sin(pi / W * x) - 12.0 * sin(2.0 * pi / W * x) + 3.0 * sin(3.0 * pi / W * x)));
    case VGPU_WF_RAMPED_SINUSOID:
      if (x <= 0.0) env = 0.0;
      else if (x < 1.0 * W)
        env = 1.0 / 32.0 * (10.0 - 15.0 * cos(pi / W * x) + 6.0 * cos(2.0 * pi / W * x) - cos(3.0 * pi / W * x));
      else env = 1.0;
      return w.size * (env * sin(2.0 * pi * f * x));
    case VGPU_WF_EXTERNAL:
      if (x < w.table[0] || x > w.table[3 * (w.table_size - 1)]) return w.size * 0.0;
      return w.size * dev_spline(w, x);
    default: return 0.0;
  }
}

// ---------------------------------------------------------------------------
// TFSF plane waves (src/planewave.c:576-1007, 1226-1419).
// ---------------------------------------------------------------------------

template <typename T>
struct PwView {
  int use_aux;
  DevWaveform wf;
  double delay, phase_velocity;
  double kinc[3], finc[6], r0[3], ijk0[3];
  const double *pos_node[3], *pos_half[3];
  // auxiliary grid
  T *Eyi, *Hzi, *PPyi, *Pyi, *Bzi;
  const T *adx, *bdx, *ahx, *bhx;
  const T *source;
  int nx, xb;
  T beta, gamma, eta0;
};

struct TfsfItem {
  Box b;          // corrected points of this face for component c
  int c, inc, sign, axis, shift;
  int64_t first;
};

struct TfsfView {
  int n;
  TfsfItem it[12];
};

// Auxiliary 1-D grid, one block (src/planewave.c:1318-1374).
template <typename T>
__global__ void k_aux_e(PwView<T> pw, const uint64_t *step_base, int step_rel)
{
  for (int i = 1 + threadIdx.x; i < pw.xb; i += blockDim.x) pw.Eyi[i] = pw.Eyi[i] + pw.beta * (pw.Hzi[i - 1] - pw.Hzi[i]);
  for (int i = pw.xb + threadIdx.x; i < pw.nx; i += blockDim.x) {
    int L = i - pw.xb;
    T oPP = pw.PPyi[L];
    pw.PPyi[L] = pw.PPyi[L] + pw.beta * (pw.Hzi[i - 1] - pw.Hzi[i]);
    T oP = pw.Pyi[L];
    pw.Pyi[L] = pw.Pyi[L] + (pw.PPyi[L] - oPP);
    pw.Eyi[i] = pw.adx[L] * pw.Eyi[i] + pw.bdx[L] * (pw.Pyi[L] - oP);
  }
  if (threadIdx.x == 0) pw.Eyi[0] = pw.source[*step_base + step_rel];
}

template <typename T>
__global__ void k_aux_h(PwView<T> pw)
{
  for (int i = threadIdx.x; i < pw.xb; i += blockDim.x) pw.Hzi[i] = pw.Hzi[i] + pw.gamma * (pw.Eyi[i] - pw.Eyi[i + 1]);
  for (int i = pw.xb + threadIdx.x; i < pw.nx; i += blockDim.x) {
    int L = i - pw.xb;
    T oB = pw.Bzi[L];
    pw.Bzi[L] = pw.ahx[L] * pw.Bzi[L] + pw.gamma * pw.bhx[L] * (-pw.Eyi[i + 1] + pw.Eyi[i]);
    pw.Hzi[i] = pw.Hzi[i] + (pw.Bzi[L] - oB);
  }
}

// Face corrections from a precomputed point list.  Each entry is one
// (face, point) correction of the reference's loops.  Points corrected by
// one face only come first, one entry each; the entries of a point on
// several faces (the Huygens box's edges) follow, contiguous and in the
// reference's face order, and one thread applies them in sequence.  What
// does not change between steps is computed once by k_tfsf_prepare: the
// analytic field's phase term d / v, or the auxiliary-grid cell and
// fraction.  The line length and update coefficients are copies of the
// grid's values.
template <typename T>
struct alignas(16) TfsfEntry {
  int64_t x;    // field index of the corrected point
  double dv;    // analytic field: d / phase velocity; auxiliary grid: the fraction
  T idv;        // line length
  T ca, cb;     // alpha and beta (E) or -, gamma (H)
  int meta;     // item (face, component) in bits 0-7; auxiliary-grid cell above
  __host__ __device__ int q() const { return meta & 255; }
  __host__ __device__ int cell() const { return meta >> 8; }
};

template <typename T>
struct TfsfList {
  TfsfEntry<T> *ent;
  const int64_t *seed_x;   // set-up only: each entry's field index ...
  const uint8_t *seed_q;   // ... and item, from which k_tfsf_prepare fills it
  const int *mstart;       // multi-entry points: entry starts, nmulti + 1 values
  int64_t nentries;
  int nsingle, nmulti;
};

template <typename T>
__global__ void k_tfsf_prepare(Grid<T> g, PwView<T> pw, TfsfView tv, TfsfList<T> tl, int efield)
{
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= tl.nentries) return;
  TfsfEntry<T> &en = tl.ent[e];
  en.x = tl.seed_x[e];
  en.meta = tl.seed_q[e];
  const TfsfItem &item = tv.it[en.q()];
  const int c = item.inc;
  // The corrected point (i, j, k) from its field index, and the incident
  // field's position: the point shifted along the item's axis.
  const int pi = (int)(en.x / g.s0);
  const int pj = (int)((en.x - (int64_t)pi * g.s0) / g.s1);
  const int pk = (int)(en.x - (int64_t)pi * g.s0 - (int64_t)pj * g.s1);
  const int i = pi + (item.axis == 0 ? item.shift : 0), j = pj + (item.axis == 1 ? item.shift : 0),
            k = pk + (item.axis == 2 ? item.shift : 0);
  // The corrected point's line length and coefficients, as the sweeps read
  // them.
  {
    const int gi = item.axis == 0 ? pi : item.axis == 1 ? pj : pk;
    en.idv = efield ? g.idh[item.axis][gi] : g.ide[item.axis][gi];
    en.ca = efield ? g.coef(item.c, en.x) : (T)0;
    en.cb = efield ? g.coef(3 + item.c, en.x) : g.coef(6 + item.c - HX, en.x);
  }
  if (!pw.use_aux) {
    // Phase term of the analytic incident field (src/planewave.c:450-554):
    // d = kinc . (r - r0), r at the component's node or mid-edge position.
    int gg[3] = { i, j, k };
    double r[3];
    for (int a = 0; a < 3; a++) {
      bool half = c <= EZ ? (c == a) : (c - HX != a);
      r[a] = half ? pw.pos_half[a][gg[a]] : pw.pos_node[a][gg[a]];
    }
    double d = pw.kinc[0] * (r[0] - pw.r0[0]) + pw.kinc[1] * (r[1] - pw.r0[1]) + pw.kinc[2] * (r[2] - pw.r0[2]);
    en.dv = d / pw.phase_velocity;
    return;
  }
  T rc[3] = { (T)i, (T)j, (T)k };
  if (c <= EZ) rc[c] = rc[c] + (T)0.5;
  else
    for (int a = 0; a < 3; a++)
      if (a != c - HX) rc[a] = rc[a] + (T)0.5;
  T d = (T)pw.kinc[0] * (rc[0] - (T)pw.ijk0[0]) + (T)pw.kinc[1] * (rc[1] - (T)pw.ijk0[1]) +
        (T)pw.kinc[2] * (rc[2] - (T)pw.ijk0[2]);
  // The fraction is a T; stored as a double it round-trips exactly.
  int id;
  T frac;
  if (c <= EZ) {
    id = (int)floor((double)d);
    frac = d - (T)id;
  } else {
    id = (int)floor((double)d + 0.5);
    frac = (T)((double)d + 0.5 - id);
  }
  en.meta = (en.meta & 255) | (int)((unsigned)id << 8);
  en.dv = (double)frac;
}

// One correction of `v` (src/planewave.c:576-1007, the expression of the
// item's face and component).
template <typename T>
__device__ __forceinline__ T tfsf_apply(const PwView<T> &pw, const TfsfView &tv, const TfsfEntry<T> &en, T v,
                                        double time, int efield)
{
  const TfsfItem &it = tv.it[en.q()];
  T inc;
  if (!pw.use_aux) {
    inc = (T)(pw.finc[it.inc] * dev_waveform(pw.wf, time - en.dv, pw.delay));
  } else {
    const int id = en.cell();
    const T dp = (T)en.dv;
    T value;
    if (it.inc <= EZ) value = (1 - dp) * pw.Eyi[2 + id] + dp * pw.Eyi[2 + id + 1];
    else value = pw.eta0 * ((1 - dp) * pw.Hzi[2 - 1 + id] + dp * pw.Hzi[2 + id]);
    inc = (T)pw.finc[it.inc] * value;
  }
  if (efield) {
    if (it.sign > 0) return en.ca * v + en.cb * (en.idv * inc);
    return en.ca * v - en.cb * (en.idv * inc);
  }
  if (it.sign > 0) return v + en.cb * (en.idv * inc);
  return v - en.cb * (en.idv * inc);
}

// Threads [0, ceil(nsingle / 2)) take two single entries each, spaced
// ceil(nsingle / 2) apart so each load is coalesced across the warp, with
// both loads issued before the first use (two per thread timed faster than
// one or four on the graded 200x160x120 UPML mesh); the threads after them take one multi-entry
// run each.
constexpr int kTfsfPerThread = 2;

template <typename T>
__device__ __forceinline__ void tfsf_point(const Grid<T> &g, const PwView<T> &pw, const TfsfView &tv,
                                           const TfsfList<T> &tl, double dt, uint64_t n, int efield, int t)
{
  const int ns4 = (tl.nsingle + kTfsfPerThread - 1) / kTfsfPerThread;
  if (t >= ns4 + tl.nmulti) return;
  const double time = efield ? n * dt : (n + 0.5) * dt;
  if (t < ns4) {
    TfsfEntry<T> en[kTfsfPerThread];
    T v[kTfsfPerThread];
#pragma unroll
    for (int m = 0; m < kTfsfPerThread; m++)
      if (t + m * ns4 < tl.nsingle) en[m] = tl.ent[t + m * ns4];
#pragma unroll
    for (int m = 0; m < kTfsfPerThread; m++)
      if (t + m * ns4 < tl.nsingle) v[m] = g.F[tv.it[en[m].q()].c][en[m].x];
#pragma unroll
    for (int m = 0; m < kTfsfPerThread; m++)
      if (t + m * ns4 < tl.nsingle) g.F[tv.it[en[m].q()].c][en[m].x] = tfsf_apply(pw, tv, en[m], v[m], time, efield);
    return;
  }
  const int r = t - ns4;
  const int e0 = tl.mstart[r], e1 = tl.mstart[r + 1];
  const TfsfEntry<T> first = tl.ent[e0];
  T *F = g.F[tv.it[first.q()].c];
  T v = F[first.x];
  for (int e = e0; e < e1; e++) v = tfsf_apply(pw, tv, tl.ent[e], v, time, efield);
  F[first.x] = v;
}

template <typename T>
__global__ void k_tfsf_list(Grid<T> g, const __grid_constant__ PwView<T> pw, const __grid_constant__ TfsfView tv,
                            const __grid_constant__ TfsfList<T> tl, double dt, const uint64_t *step_base,
                            int step_rel, int efield)
{
  tfsf_point(g, pw, tv, tl, dt, *step_base + step_rel, efield, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

// Parts of a step that touch disjoint points, run as one launch so their
// latency-bound chains overlap (the engine checks disjointness at set-up):
// blocks [0, nb_debye) take the Debye cells, the next nb_tfsf blocks one
// plane wave's corrections of the step, and the last nb_obs blocks the
// observer samples of the step after it.  Each job does exactly what its own
// kernel does (k_debye, k_tfsf_list, k_observe).
template <typename T>
struct SideLaunch {
  int nb_debye, nb_tfsf, nb_obs;
  const DebyeItem *debye;
  int n_debye;
  int64_t debye_total;
  double2 *J;
  T *lastE;
  const double2 *dcoef;
  PwView<T> pw;
  TfsfView tv;
  TfsfList<T> tl;
  double dt;
  int efield;
  const int *td_pts, *fd_pts;
  int num_td, num_fd;
  T *td_buf;
  double *fd_stage;
  uint64_t out_start, out_stop;
  int tblock;
};

template <typename T>
__global__ void k_side(Grid<T> g, const __grid_constant__ SideLaunch<T> L, const uint64_t *step_base, int step_rel)
{
  int b = blockIdx.x;
  const uint64_t n = *step_base + step_rel;
  if (b < L.nb_debye) {
    const int64_t t = (int64_t)b * blockDim.x + threadIdx.x;
    if (t < L.debye_total) debye_point(g, L.debye, L.n_debye, t, L.J, L.lastE, L.dcoef);
    return;
  }
  b -= L.nb_debye;
  if (b < L.nb_tfsf) {
    tfsf_point(g, L.pw, L.tv, L.tl, L.dt, n, L.efield, (int)(b * blockDim.x + threadIdx.x));
    return;
  }
  b -= L.nb_tfsf;
  observe_point(g, L.td_pts, L.num_td, L.fd_pts, L.num_fd, L.td_buf, L.fd_stage, n + 1, L.out_start, L.out_stop,
                L.tblock, (int)(b * blockDim.x + threadIdx.x));
}

// ---------------------------------------------------------------------------
// SIBC (src/sibc.c:444-776, src/filter.c:309-327).
// ---------------------------------------------------------------------------

struct SibcSurf {
  Box g;              // faces: cells [i0, i1) etc. stored as inclusive i0..i1-1
  int normal, model;
  int64_t first;      // first global face index
  double A[4][4], B[4][4];
};

struct SibcModelDev {
  int np[4][4], off[4][4];
  double asymp[4][4];
  int poles;          // total poles of the model
};

template <typename T>
__global__ void k_sibc_e(Grid<T> g, const SibcSurf *surfs, int nsurf, const SibcModelDev *models,
                         const double2 *q0, const double2 *q1, const double2 *q2, const uint8_t *adjA,
                         const uint8_t *adjB, const int64_t *zofs, double2 *zeta, double *old, T *etan,
                         int64_t total)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  int s = 0;
  while (s + 1 < nsurf && t >= surfs[s + 1].first) s++;
  const SibcSurf &sf = surfs[s];
  const SibcModelDev &m = models[sf.model];
  int64_t f = t - sf.first;
  // A surface holds fewer than 2^31 faces (checked at set-up): 32-bit decode.
  const unsigned nj = (unsigned)sf.g.nj(), nk = (unsigned)sf.g.nk(), u = (unsigned)f;
  const unsigned qk = u / nk, qj = qk / nj;
  int i = sf.g.i0 + (int)qj, j = sf.g.j0 + (int)(qk - qj * nj), k = sf.g.k0 + (int)(u - qk * nk);
  const uint8_t *A = adjA + 4 * t, *B = adjB + 4 * t;
  T *Ex = g.F[EX], *Ey = g.F[EY], *Ez = g.F[EZ];
  const T *Hx = g.F[HX], *Hy = g.F[HY], *Hz = g.F[HZ];
  T Ht[4], Hin[4], Eout[4];
  if (sf.normal == 0) {
    Ey[g.at(i, j, k)] = 0.0; Ey[g.at(i, j, k + 1)] = 0.0;
    Ez[g.at(i, j, k)] = 0.0; Ez[g.at(i, j + 1, k)] = 0.0;
    Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hy[g.at(i - 1, j, k)] + Hy[g.at(i - 1, j + 1, k)]);
    Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hy[g.at(i, j, k)] + Hy[g.at(i, j + 1, k)]);
    Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hz[g.at(i - 1, j, k)] + Hz[g.at(i - 1, j, k + 1)]);
    Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hz[g.at(i, j, k)] + Hz[g.at(i, j, k + 1)]);
  } else if (sf.normal == 1) {
    Ez[g.at(i, j, k)] = 0.0; Ez[g.at(i + 1, j, k)] = 0.0;
    Ex[g.at(i, j, k)] = 0.0; Ex[g.at(i, j, k + 1)] = 0.0;
    Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hz[g.at(i, j - 1, k)] + Hz[g.at(i, j - 1, k + 1)]);
    Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hz[g.at(i, j, k)] + Hz[g.at(i, j, k + 1)]);
    Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hx[g.at(i, j - 1, k)] + Hx[g.at(i + 1, j - 1, k)]);
    Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hx[g.at(i, j, k)] + Hx[g.at(i + 1, j, k)]);
  } else {
    Ex[g.at(i, j, k)] = 0.0; Ex[g.at(i, j + 1, k)] = 0.0;
    Ey[g.at(i, j, k)] = 0.0; Ey[g.at(i + 1, j, k)] = 0.0;
    Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hx[g.at(i, j, k - 1)] + Hx[g.at(i + 1, j, k - 1)]);
    Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hx[g.at(i, j, k)] + Hx[g.at(i + 1, j, k)]);
    Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hy[g.at(i, j, k - 1)] + Hy[g.at(i, j + 1, k - 1)]);
    Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hy[g.at(i, j, k)] + Hy[g.at(i, j + 1, k)]);
  }
  for (int a = 0; a < 4; a++) {
    Hin[a] = 0.0;
    for (int b = 0; b < 4; b++) Hin[a] = Hin[a] + (T)sf.A[a][b] * Ht[b];
  }
  double2 *z = zeta + zofs[s] + f * m.poles;
  double *o = old + 16 * t;
  for (int a = 0; a < 4; a++) {
    Eout[a] = 0.0;
    for (int b = 0; b < 4; b++) {
      double xin = Hin[b];
      double y = m.asymp[a][b] * xin;
      int off = m.off[a][b];
      double2 *zz = z + (off - m.off[0][0]);
      // A filter entry without poles is its constant term alone: its input
      // history feeds only the pole recursion, so it is neither read nor
      // kept (nothing else reads it).
      if (m.np[a][b] == 0) {
        Eout[a] = Eout[a] + y;
        continue;
      }
      double po = o[4 * a + b];
      for (int r = 0; r < m.np[a][b]; r++) {
        double2 a0 = q0[off + r], a1 = q1[off + r], a2 = q2[off + r], zv = zz[r];
        double re = (a0.x * zv.x - a0.y * zv.y) + a1.x * po;
        double im = (a0.x * zv.y + a0.y * zv.x) + a1.y * po;
        re = re + a2.x * xin;
        im = im + a2.y * xin;
        zz[r] = make_double2(re, im);
        y = y + re;
      }
      o[4 * a + b] = xin;
      Eout[a] = Eout[a] + y;
    }
  }
  T *et = etan + 4 * t;
  for (int a = 0; a < 4; a++) {
    T v = 0.0;
    for (int b = 0; b < 4; b++) v = v + (T)sf.B[a][b] * Eout[b];
    et[a] = v;
  }
}

// One thread per corrected H value: apply its operations in order.  The
// operation's coefficients are stored in T, the type the correction
// computes in (the values are rounded to T once, at set-up, where the
// update rounded them at each use), and its tangential-E indices in 32 bits.
template <typename T>
struct SibcOp {
  int32_t e1, e2;     // indices into etan
  int32_t kind, pad;
  T c, d1, d2, n1, n2;
};

template <typename T>
__global__ void k_sibc_h(Grid<T> g, const int64_t *__restrict__ tgt_index, const int *__restrict__ tgt_comp,
                         const int64_t *__restrict__ tgt_start, int64_t ntgt, const SibcOp<T> *__restrict__ ops,
                         const T *__restrict__ etan)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntgt) return;
  T *F = g.F[tgt_comp[t]];
  const int64_t x = tgt_index[t];
  T h = F[x];
  for (int64_t q = tgt_start[t]; q < tgt_start[t + 1]; q++) {
    const SibcOp<T> o = ops[q];
    if (o.kind == 0) { h = 0.0; continue; }
    const T e1 = etan[o.e1];
    if (o.kind == 1) {
      h = h + o.c * (o.d1 * e1);
    } else {
      const T e2 = etan[o.e2];
      h = h + o.c * (o.n1 * (o.d1 * e1) + o.n2 * (o.d2 * e2));
    }
  }
  F[x] = h;
}

// Finiteness scan of all field volumes.
template <typename T>
__global__ void k_finite(Grid<T> g, int64_t vol_padded, int *flag)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; t < vol_padded; t += stride)
    for (int c = 0; c < 6; c++)
      if (!isfinite((double)g.F[c][t])) { atomicExch(flag, 1); return; }
}

// Stability check (FP64): sums of squares of the three E and of the three H
// components over every stored point, added into out[0] and out[1].  Not the
// physical energy (no permittivity, permeability or cell-volume weights) but
// a norm of the fields that grows without bound once the update is unstable
// and turns non-finite with any field value.  The reference's only guard is
// the Courant-number check before the loop (src/simulation.c:64-84).  One
// atomic add per block and quantity.
template <typename T>
__global__ void k_energy(Grid<T> g, int64_t vol_padded, double *out)
{
  double e = 0.0, h = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < vol_padded; t += stride) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double v = (double)g.F[c][t];
      e = e + v * v;
    }
#pragma unroll
    for (int c = 3; c < 6; c++) {
      const double v = (double)g.F[c][t];
      h = h + v * v;
    }
  }
  __shared__ double se[32], sh[32];
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    h += __shfl_down_sync(0xffffffffu, h, o);
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) {
    se[w] = e;
    sh[w] = h;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (int)(blockDim.x / 32);
    e = l < nw ? se[l] : 0.0;
    h = l < nw ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      e += __shfl_down_sync(0xffffffffu, e, o);
      h += __shfl_down_sync(0xffffffffu, h, o);
    }
    if (l == 0) {
      atomicAdd(&out[0], e);
      atomicAdd(&out[1], h);
    }
  }
}

}  // namespace vgpu_dev
