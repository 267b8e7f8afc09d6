/*
 * vh_grid.c -- grid, media and boundary set-up for vulture_b200.
 *
 * Restates the reference's initialisation of the Yee grid and of everything
 * painted into its coefficient volumes, in the order src/vulture.c:95-136
 * calls them.  Each function cites the reference code it follows; arithmetic
 * is in double with the reference's operation order (its real=double build).
 */
#include <assert.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <unistd.h>

#include "vh.h"

typedef struct {
  void (*fn)(void *, int, int);
  void *ctx;
  int lo, hi;
} vh_range_job;

static void *range_main(void *arg)
{
  vh_range_job *j = arg;
  j->fn(j->ctx, j->lo, j->hi);
  return NULL;
}

void vh_parallel_for(int begin, int end, int64_t work, void (*fn)(void *ctx, int lo, int hi), void *ctx)
{
  const int n = end - begin;
  long cores = sysconf(_SC_NPROCESSORS_ONLN);
  int nt = cores > 16 ? 16 : (cores < 1 ? 1 : (int)cores);
  if (work < (1 << 18) || n < 2) nt = 1;
  if (nt > n) nt = n;
  if (nt <= 1) {
    if (n > 0) fn(ctx, begin, end);
    return;
  }
  pthread_t th[16];
  vh_range_job jobs[16];
  int started[16] = { 0 };
  for (int t = 0; t < nt; t++) {
    jobs[t] = (vh_range_job){ fn, ctx, begin + (int)((int64_t)n * t / nt), begin + (int)((int64_t)n * (t + 1) / nt) };
    /* The first range runs here; a thread that fails to start runs its
     * range here as well. */
    if (t > 0) started[t] = pthread_create(&th[t], NULL, range_main, &jobs[t]) == 0;
  }
  range_main(&jobs[0]);
  for (int t = 1; t < nt; t++) {
    if (started[t]) pthread_join(th[t], NULL);
    else range_main(&jobs[t]);
  }
}

static double *alloc_volume(size_t n);
static uint8_t *alloc_bytes(size_t n);

int vh_outer_type(const vh_ctx *c, int face) { return c->bnds[c->ext_bnd[face]].type; }

static int outer_layers(const vh_ctx *c, int face) { return c->bnds[c->ext_bnd[face]].num_layers; }

/* External surface defaults and checks (src/surface.c:271-335). */
static int init_external_surface_parameters(vh_ctx *c)
{
  for (int f = XLO; f <= ZHI; f++) {
    int b = vh_find_boundary(c, VH_FACE_STR[f]);
    if (b < 0) {
      int layers, order;
      double n_eff, rc, kmax;
      vh_pml_defaults(&layers, &order, &n_eff, &rc, &kmax);
      b = vh_add_boundary(c, VH_FACE_STR[f], BT_PML, layers, order, n_eff, rc, kmax, "", NULL, NULL);
    }
    c->ext_bnd[f] = b;
  }
  for (int f = XLO; f <= ZHI; f++) {
    vh_boundary *b = &c->bnds[c->ext_bnd[f]];
    switch (b->type) {
      case BT_PEC:
      case BT_PMC:
      case BT_MUR:
        b->num_layers = 0;
        break;
      case BT_PERIODIC: {
        b->num_layers = 0;
        int opp = f - 2 * (f % 2) + 1;
        if (c->bnds[c->ext_bnd[opp]].type != BT_PERIODIC)
          return vh_fail(c, "PERIODIC boundary on %s surface doesn't match that on surface %s",
                         VH_FACE_STR[f], VH_FACE_STR[opp]);
        break;
      }
      case BT_PML:
        if (b->num_layers < 1)
          return vh_fail(c, "PML on %s surface has less than one (%d) layers", VH_FACE_STR[f], b->num_layers);
        break;
      default:
        /* FREE_SPACE or SIBC on an external face: the reference asserts
         * (src/surface.c:330), which its release build compiles out, and then
         * runs with the face unterminated; the same happens here. */
        vh_log(c, 0, "*** Warning: %s boundary type is not supported on external surface %s\n",
               b->name, VH_FACE_STR[f]);
        break;
    }
  }
  return 0;
}

/* src/grid.c:357-387 */
static void set_grid_extents(vh_ctx *c)
{
  c->ggbox[XLO] = c->ggbox[YLO] = c->ggbox[ZLO] = 0;
  c->gobox[XLO] = c->gobox[YLO] = c->gobox[ZLO] = 1;
  for (int a = 0; a < 3; a++) {
    c->gibox[2 * a] = c->gobox[2 * a] + outer_layers(c, 2 * a);
    c->gibox[2 * a + 1] = c->gibox[2 * a] + c->num_lines[a] - 1;
    c->gobox[2 * a + 1] = c->gibox[2 * a + 1] + outer_layers(c, 2 * a + 1);
    c->ggbox[2 * a + 1] = c->gobox[2 * a + 1] + 1;
    c->n[a] = c->gobox[2 * a + 1] - c->gobox[2 * a] + 2;
  }
}

/* src/grid.c:390-411 */
static void init_field_array_limits(vh_ctx *c)
{
  bool inner[6], outer[6];
  for (int f = 0; f < 6; f++) {
    inner[f] = vh_outer_type(c, f) != BT_MUR;
    outer[f] = true;
  }
  vh_set_field_limits(c->gibox, c->gfilim, inner);
  vh_set_field_limits(c->gobox, c->gfolim, outer);
}

/* Cell edge lengths and the time step (src/grid.c:583-679). */
static void init_cell_edges(vh_ctx *c)
{
  for (int a = 0; a < 3; a++) {
    int lo = 2 * a, hi = 2 * a + 1, nn = c->n[a];
    double *de = c->de[a] = calloc(nn, sizeof(double));
    double *dh = c->dh[a] = calloc(nn, sizeof(double));
    double *ide = c->ide[a] = calloc(nn, sizeof(double));
    double *idh = c->idh[a] = calloc(nn, sizeof(double));
    const double *ln = c->lines[a];
    int gi0 = c->gibox[lo], gi1 = c->gibox[hi], go0 = c->gobox[lo], go1 = c->gobox[hi];
    c->dmin[a] = 1.79769313486231570815e+308; /* REAL_MAX of the real=double build */
    c->dmax[a] = 0.0;
    for (int i = go0; i <= gi0 - 1; i++) de[i] = ln[1] - ln[0];
    for (int i = gi0; i <= gi1 - 1; i++) de[i] = ln[i - gi0 + 1] - ln[i - gi0];
    for (int i = gi1; i <= go1 - 1; i++) de[i] = ln[gi1 - gi0] - ln[gi1 - gi0 - 1];
    de[go0 - 1] = de[go0];
    de[go1] = de[go1 - 1];
    for (int i = go0 - 1; i <= go1; i++) {
      ide[i] = 1.0 / de[i];
      if (de[i] < c->dmin[a]) c->dmin[a] = de[i];
      if (de[i] > c->dmax[a]) c->dmax[a] = de[i];
    }
    for (int i = go0; i <= go1; i++) dh[i] = 0.5 * (de[i] + de[i - 1]);
    dh[go0 - 1] = dh[go0];
    for (int i = go0; i <= go1; i++) {
      idh[i] = 1.0 / dh[i];
      if (dh[i] < c->dmin[a]) c->dmin[a] = dh[i];
      if (dh[i] > c->dmax[a]) c->dmax[a] = dh[i];
    }
    idh[go0 - 1] = idh[go0];
  }
  c->dt = c->courant / c->c0 /
          sqrt((1.0 / c->dmin[0]) * (1.0 / c->dmin[0]) + (1.0 / c->dmin[1]) * (1.0 / c->dmin[1]) +
               (1.0 / c->dmin[2]) * (1.0 / c->dmin[2]));
}

/* Grid classification with the reference's one-sided test (src/grid.c:1505-1549). */
static void set_grid_type(vh_ctx *c)
{
  bool uni[3] = { true, true, true };
  for (int a = 0; a < 3; a++)
    for (int i = c->gibox[2 * a] + 1; i <= c->gibox[2 * a + 1] - 1; i++)
      if (c->de[a][i] - c->de[a][i - 1] > 1e-5) uni[a] = false;
  if (uni[0] && uni[1] && uni[2]) {
    if (fabs(c->de[0][c->gibox[XLO]] - c->de[1][c->gibox[YLO]]) < 1e-5 &&
        fabs(c->de[1][c->gibox[YLO]] - c->de[2][c->gibox[ZLO]]) < 1e-5)
      c->grid_type = GT_CUBIC;
    else
      c->grid_type = GT_UNIFORM;
    for (int a = 0; a < 3; a++) c->duni[a] = c->de[a][c->gibox[2 * a]];
  } else {
    c->grid_type = GT_NONUNIFORM;
    c->duni[0] = c->duni[1] = c->duni[2] = -1.0;
  }
}

int vh_init_grid(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising the grid...\n\n");
  if (init_external_surface_parameters(c)) return -1;
  set_grid_extents(c);
  init_field_array_limits(c);
  int64_t vol = (int64_t)c->n[0] * c->n[1] * c->n[2];
  for (int q = 0; q < 9; q++) {
    c->coef[q] = alloc_volume((size_t)vol);
    if (!c->coef[q]) return vh_fail(c, "Failed to allocate grid coefficient arrays (%lld cells)", (long long)vol);
  }
  /* Tags are an aid, not state: without memory for them the engine scans
   * the volumes instead. */
  for (int f = 0; f < 6; f++) c->ctag[f] = alloc_bytes((size_t)vol);
  if (!c->ctag[0] || !c->ctag[1] || !c->ctag[2] || !c->ctag[3] || !c->ctag[4] || !c->ctag[5]) vh_free_tags(c);
  init_cell_edges(c);
  set_grid_type(c);
  return 0;
}

/* Newton iteration for the numerical phase velocity (src/grid.c:1552-1617). */
static double num_phase_velocity_func(const vh_ctx *c, double k, const double A[3], double B)
{
  double t[3];
  for (int a = 0; a < 3; a++) t[a] = sin(A[a] * k) / c->duni[a];
  double func = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] - B * B;
  double der = A[0] * sin(2 * A[0] * k) / (c->duni[0] * c->duni[0]) +
               A[1] * sin(2 * A[1] * k) / (c->duni[1] * c->duni[1]) +
               A[2] * sin(2 * A[2] * k) / (c->duni[2] * c->duni[2]);
  return func / der;
}

double vh_numerical_phase_velocity(vh_ctx *c, double theta, double phi)
{
  double A[3], B, w, k;
  w = 2.0 * c->pi * (1.0 / c->dt / 23);
  A[0] = 0.5 * c->duni[0] * sin(theta) * cos(phi);
  A[1] = 0.5 * c->duni[1] * sin(theta) * sin(phi);
  A[2] = 0.5 * c->duni[2] * cos(theta);
  B = (sin(0.5 * w * c->dt) / (c->c0 * c->dt));
  k = w / c->c0;
  for (int i = 0; i < 10; i++) k = k - num_phase_velocity_func(c, k, A, B);
  return w / k;
}

/* Physical position of a field point (src/grid.c:1429-1476). */
void vh_field_physical_location(const vh_ctx *c, double r[3], int field, int ig, int jg, int kg)
{
  int g[3] = { ig, jg, kg };
  for (int a = 0; a < 3; a++) {
    int m = g[a] - c->gibox[2 * a];
    bool half;
    if (field <= EZ) half = (field == a);
    else half = (field - HX) != a;
    double node;
    int nl = c->num_lines[a];
    /* Outside the mesh lines the reference reads past its line array; here
     * the first/last mesh step is extended instead. */
    if (m < 0) node = c->lines[a][0] + m * (c->lines[a][1] - c->lines[a][0]);
    else if (m > nl - 1) node = c->lines[a][nl - 1] + (m - nl + 1) * (c->lines[a][nl - 1] - c->lines[a][nl - 2]);
    else node = c->lines[a][m];
    r[a] = half ? node + 0.5 * c->de[a][g[a]] : node;
  }
}

/* ---- media ---- */

/* Update coefficients from material parameters (src/medium.c:482-504). */
void vh_calc_coeff(vh_ctx *c, vh_medium *m)
{
  double dt = c->dt, sum = 0.0;
  for (int p = 0; p < m->num_poles; p++) {
    m->dalpha[p] = (1 + 0.5 * dt * m->pole[p]) / (1 - 0.5 * dt * m->pole[p]);
    m->dbeta[p] = c->eps0 * m->res[p] / (1 - 0.5 * dt * m->pole[p]);
    sum = sum + creal(m->dbeta[p]);
  }
  m->alpha = (2.0 * m->eps_r * c->eps0 + 2.0 * sum * dt - dt * m->sigma) /
             (2.0 * m->eps_r * c->eps0 + 2.0 * sum * dt + dt * m->sigma);
  m->beta = (2.0 * dt) / (2.0 * m->eps_r * c->eps0 + 2.0 * sum * dt + dt * m->sigma);
  m->gamma = dt / (m->mu_r * c->mu0);
}

/* src/medium.c:381-441 */
int vh_init_media(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising media...\n\n");
  for (int i = 0; i < c->num_media; i++) {
    vh_medium *m = &c->media[i];
    if (m->type == MT_DEBYE) {
      m->dalpha = calloc(m->num_poles ? m->num_poles : 1, sizeof(double complex));
      m->dbeta = calloc(m->num_poles ? m->num_poles : 1, sizeof(double complex));
    }
    vh_calc_coeff(c, m);
  }
  c->media[MT_FREE_SPACE].alpha = 1.0;
  c->media[MT_FREE_SPACE].beta = c->dt / c->eps0;
  c->media[MT_FREE_SPACE].gamma = c->dt / c->mu0;
  c->media[MT_PEC].alpha = -1.0;
  c->media[MT_PEC].beta = 0.0;
  c->media[MT_PEC].gamma = c->dt / c->mu0;
  return 0;
}

typedef struct {
  vh_ctx *c;
  const vh_medium *m;
  int flim[6][6];
  uint8_t tag;        /* the painted triple's tag; unused without tags */
} paint_job;

/* Planes lo..hi-1 of every component's limits. */
static void paint_range(void *ctx, int lo, int hi)
{
  paint_job *p = ctx;
  vh_ctx *c = p->c;
  const vh_medium *m = p->m;
  for (int f = EX; f <= HZ; f++) {
    double *a = f <= EZ ? c->coef[f] : NULL;
    double *b = f <= EZ ? c->coef[3 + f] : c->coef[6 + f - HX];
    uint8_t *t = c->ctag[f];
    const int ia = p->flim[f][XLO] > lo ? p->flim[f][XLO] : lo;
    const int ib = p->flim[f][XHI] < hi - 1 ? p->flim[f][XHI] : hi - 1;
    for (int i = ia; i <= ib; i++)
      for (int j = p->flim[f][YLO]; j <= p->flim[f][YHI]; j++)
        for (int k = p->flim[f][ZLO]; k <= p->flim[f][ZHI]; k++) {
          int64_t q = vh_idx(c, i, j, k);
          if (a) { a[q] = m->alpha; b[q] = m->beta; }
          else b[q] = m->gamma;
          if (t) t[q] = p->tag;
        }
  }
}

size_t vh_volume_bytes(size_t n)
{
  const size_t huge = (size_t)1 << 21;
  return n ? (n * sizeof(double) + huge - 1) / huge * huge : huge;
}

/* A zeroed volume of n doubles: anonymous pages, which the kernel hands out
 * zeroed on first touch (the painting threads touch them in parallel), so
 * nothing writes the volume twice; advised for huge pages.  Freed by
 * vh_free_volume. */
static size_t tag_bytes(size_t n)
{
  const size_t huge = (size_t)1 << 21;
  return n ? (n + huge - 1) / huge * huge : huge;
}

/* A zeroed volume of n bytes, allocated like the double volumes. */
static uint8_t *alloc_bytes(size_t n)
{
  const size_t bytes = tag_bytes(n);
  void *p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) return NULL;
#ifdef MADV_HUGEPAGE
  madvise(p, bytes, MADV_HUGEPAGE);
#endif
  return p;
}

void vh_free_tags(vh_ctx *c)
{
  const size_t n = (size_t)c->n[0] * c->n[1] * c->n[2];
  for (int f = 0; f < 6; f++) {
    if (c->ctag[f]) munmap(c->ctag[f], tag_bytes(n));
    c->ctag[f] = NULL;
  }
  c->num_ctags = 0;
}

/* The tag of a medium's current (alpha, beta, gamma): the triple's place in
 * the painted list, plus one.  A medium's coefficients may change between
 * paintings (a lumped source's), so the tag names the values painted, not
 * the medium.  A 256th distinct triple drops the tags. */
static uint8_t medium_tag(vh_ctx *c, const vh_medium *m)
{
  if (!c->ctag[0]) return 0;
  const double v[3] = { m->alpha, m->beta, m->gamma };
  for (int t = 0; t < c->num_ctags; t++)
    if (memcmp(c->ctag_coef[t], v, sizeof v) == 0) return (uint8_t)(t + 1);
  if (c->num_ctags == 255) {
    vh_free_tags(c);
    return 0;
  }
  memcpy(c->ctag_coef[c->num_ctags], v, sizeof v);
  return (uint8_t)++c->num_ctags;
}

static double *alloc_volume(size_t n)
{
  const size_t bytes = vh_volume_bytes(n);
  void *p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) return NULL;
#ifdef MADV_HUGEPAGE
  madvise(p, bytes, MADV_HUGEPAGE);
#endif
  return p;
}

void vh_free_volume(double *p, size_t n)
{
  if (p) munmap(p, vh_volume_bytes(n));
}

/* Paint a medium's coefficients over a box (src/grid.c:1726-1873). */
void vh_set_medium_on_grid(vh_ctx *c, const int gbbox[6], int medium, unsigned char mask)
{
  bool incl[6];
  int flim[6][6];
  vh_mask_to_bool(incl, mask);
  if (vh_bbox_type(gbbox) == BB_POINT) return;
  vh_set_field_limits(gbbox, flim, incl);
  paint_job job = { c, &c->media[medium], { 0 }, 0 };
  memcpy(job.flim, flim, sizeof flim);
  job.tag = medium_tag(c, job.m);
  int64_t work = 0;
  for (int f = EX; f <= HZ; f++)
    work += (int64_t)(flim[f][XHI] - flim[f][XLO] + 1) * (flim[f][YHI] - flim[f][YLO] + 1) *
            (flim[f][ZHI] - flim[f][ZLO] + 1);
  int i0 = flim[EX][XLO], i1 = flim[EX][XHI];
  for (int f = EY; f <= HZ; f++) {
    if (flim[f][XLO] < i0) i0 = flim[f][XLO];
    if (flim[f][XHI] > i1) i1 = flim[f][XHI];
  }
  vh_parallel_for(i0, i1 + 1, work, paint_range, &job);
}

/* src/grid.c:1146-1162 */
void vh_init_media_arrays(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising grid media arrays ...\n\n");
  vh_set_medium_on_grid(c, c->ggbox, MT_FREE_SPACE, VH_FACE_MASKS[XLO] | VH_FACE_MASKS[YLO] | VH_FACE_MASKS[ZLO]);
}

/* Material blocks and Debye block limits (src/block.c:148-228, src/debye.c:76-196). */
int vh_init_blocks(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising blocks...\n\n");
  int num_debye = 0;
  for (int b = 0; b < c->num_blocks; b++) {
    vh_block *blk = &c->blocks[b];
    int g[6];
    vh_bbox_offset(g, blk->mbbox, c->gibox);
    vh_set_medium_on_grid(c, g, blk->medium, blk->mask);
    if (c->media[blk->medium].type == MT_DEBYE) num_debye++;
  }
  c->num_debye = num_debye;
  c->debye_flim = calloc(num_debye ? num_debye : 1, sizeof *c->debye_flim);
  c->debye_medium = calloc(num_debye ? num_debye : 1, sizeof(int));
  int d = 0;
  for (int b = 0; b < c->num_blocks; b++) {
    vh_block *blk = &c->blocks[b];
    if (c->media[blk->medium].type != MT_DEBYE) continue;
    int g[6], flim[6][6];
    bool incl[6];
    vh_bbox_offset(g, blk->mbbox, c->gibox);
    vh_mask_to_bool(incl, blk->mask);
    vh_set_field_limits(g, flim, incl);
    for (int f = EX; f <= EZ; f++)
      for (int face = 0; face < 6; face++) c->debye_flim[d][f][face] = flim[f][face];
    c->debye_medium[d] = blk->medium;
    d++;
  }
  return 0;
}

/* Thin wires become PEC (or free-space) edges (src/line.c:165-204). */
int vh_init_lines(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising lines...\n\n");
  for (int l = 0; l < c->num_lns; l++) {
    vh_line *ln = &c->lns[l];
    vh_bbox_offset(ln->gbbox, ln->mbbox, c->gibox);
    int type = c->wires[ln->wire].type;
    vh_set_medium_on_grid(c, ln->gbbox, type == TW_PEC ? MT_PEC : MT_FREE_SPACE, VH_FACE_MASK_ALL);
  }
  return 0;
}

/* Internal surfaces (src/surface.c:350-405). */
int vh_init_internal_surfaces(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising internal surfaces...\n\n");
  int num_sibc = 0;
  for (int s = 0; s < c->num_surfs; s++) {
    vh_surface *sf = &c->surfs[s];
    int type = c->bnds[sf->boundary].type;
    vh_bbox_offset(sf->gbbox, sf->mbbox, c->gibox);
    switch (type) {
      case BT_PEC: vh_set_medium_on_grid(c, sf->gbbox, MT_PEC, VH_FACE_MASK_ALL); break;
      case BT_FREE_SPACE: vh_set_medium_on_grid(c, sf->gbbox, MT_FREE_SPACE, VH_FACE_MASK_ALL); break;
      case BT_SIBC: vh_set_medium_on_grid(c, sf->gbbox, MT_PEC, VH_FACE_MASK_ALL); num_sibc++; break;
      default: break;
    }
  }
  c->num_sibcs = num_sibc;
  return vh_init_sibc_surfaces(c);
}

/* PEC backing of PML and PEC external faces (src/surface.c:407-458). */
static void init_external_pec_pmc(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising PEC/PMC surfaces...\n\n");
  for (int f = XLO; f <= ZHI; f++) {
    int type = vh_outer_type(c, f);
    /* BOUNDARY_MEDIUM_TYPE (src/boundary.c:48): PML, PEC and SIBC map to PEC. */
    if (type == BT_PML || type == BT_PEC || type == BT_SIBC) {
      int b[6];
      vh_face_of_bbox(b, c->gobox, f);
      vh_set_medium_on_grid(c, b, MT_PEC, VH_FACE_MASK_ALL);
    }
  }
}

/* ---- UPML (src/pml.c) ---- */

static double pml_sigma_profile(const vh_ctx *c, double x, double depth, double mesh, int order, double n_eff,
                                double rc)
{
  double smax;
  if (rc > 0) smax = -(order + 1.0) / (2.0 * c->eta0 * n_eff * depth) * log(rc);
  else smax = 4.0 * (order + 1.0) / (5.0 * c->eta0 * n_eff * mesh);
  return smax * pow(x, order);
}

static double pml_kappa_profile(double x, int order, double kmax)
{
  return 1.0 + (kmax - 1.0) * pow(x, order);
}

/* Graded loss profiles of one face (src/pml.c:198-262). */
static void set_profile(vh_ctx *c, int a, int low, int high, int dir, int order, double n_eff, double rc,
                        double kmax)
{
  double *de = c->de[a], *dh = c->dh[a];
  double *gd = c->pml_gd[a], *kd = c->pml_kd[a], *bd = c->pml_bd[a], *ad = c->pml_ad[a];
  double *gh = c->pml_gh[a], *kh = c->pml_kh[a], *bh = c->pml_bh[a], *ah = c->pml_ah[a];
  double *ibd = c->pml_ibd[a], *ibh = c->pml_ibh[a];
  double total = 0.0, depthE, depthH, sprof, kprof, dt = c->dt;
  for (int i = low; i <= high; i++) total = total + de[i];
  if (dir == -1) {
    depthE = total;
    depthH = total - 0.5 * de[low];
  } else {
    depthE = 0.0;
    depthH = 0.5 * de[low];
  }
  for (int i = low; i <= high; i++) {
    sprof = 0.5 * dt / c->eps0 * pml_sigma_profile(c, depthE / total, total, de[low], order, n_eff, rc);
    kprof = pml_kappa_profile(depthE / total, order, kmax);
    gh[i] = sprof;
    kh[i] = kprof;
    bd[i] = 1.0 / (kprof + sprof);
    ibd[i] = kprof + sprof;
    ad[i] = (kprof - sprof) / (kprof + sprof);
    depthE = depthE + dir * de[i];
  }
  if (dir == +1) {
    sprof = 0.5 * dt / c->eps0 * pml_sigma_profile(c, depthE / total, total, de[low], order, n_eff, rc);
    kprof = pml_kappa_profile(depthE / total, order, kmax);
    gh[high + 1] = sprof;
    kh[high + 1] = kprof;
    bd[high + 1] = 1.0 / (kprof + sprof);
    ibd[high + 1] = kprof + sprof;
    ad[high + 1] = (kprof - sprof) / (kprof + sprof);
  }
  for (int i = low; i <= high; i++) {
    sprof = 0.5 * dt / c->eps0 * pml_sigma_profile(c, depthH / total, total, de[low], order, n_eff, rc);
    kprof = pml_kappa_profile(depthH / total, order, kmax);
    gd[i] = sprof;
    kd[i] = kprof;
    bh[i] = 1.0 / (kprof + sprof);
    ibh[i] = kprof + sprof;
    ah[i] = (kprof - sprof) / (kprof + sprof);
    depthH = depthH + dir * dh[i];
  }
}

/* src/pml.c:124-195 */
static void set_pml_limits(vh_ctx *c)
{
  static const bool incl[6][6] = { { 1, 0, 1, 1, 1, 1 }, { 0, 1, 1, 1, 1, 1 }, { 1, 1, 1, 0, 1, 1 },
                                   { 1, 1, 0, 1, 1, 1 }, { 1, 1, 1, 1, 1, 0 }, { 1, 1, 1, 1, 0, 1 } };
  int *gi = c->gibox, *go = c->gobox;
  for (int r = 0; r < 6; r++) {
    int a = r / 2;
    for (int b = 0; b < 3; b++) {
      if (b == a) {
        if (r % 2 == 0) { c->pbox[r][2 * b] = go[2 * b]; c->pbox[r][2 * b + 1] = gi[2 * b]; }
        else { c->pbox[r][2 * b] = gi[2 * b + 1]; c->pbox[r][2 * b + 1] = go[2 * b + 1]; }
      } else if (b < a) {
        /* Axes handled by an earlier region pair stay inside the inner box. */
        c->pbox[r][2 * b] = gi[2 * b];
        c->pbox[r][2 * b + 1] = gi[2 * b + 1];
      } else {
        c->pbox[r][2 * b] = go[2 * b];
        c->pbox[r][2 * b + 1] = go[2 * b + 1];
      }
    }
    vh_set_field_limits(c->pbox[r], c->fplim[r], incl[r]);
  }
}

/* src/pml.c:265-424 */
static void set_pml_parameters(vh_ctx *c)
{
  for (int a = 0; a < 3; a++) {
    for (int i = c->gobox[2 * a] - 1; i <= c->gobox[2 * a + 1]; i++) {
      c->pml_kd[a][i] = 1.0; c->pml_kh[a][i] = 1.0;
      c->pml_gd[a][i] = 0.0; c->pml_gh[a][i] = 0.0;
      c->pml_bd[a][i] = 1.0; c->pml_bh[a][i] = 1.0;
      c->pml_ibd[a][i] = 1.0; c->pml_ibh[a][i] = 1.0;
      c->pml_ad[a][i] = 1.0; c->pml_ah[a][i] = 1.0;
    }
  }
  for (int f = XLO; f <= ZHI; f++) {
    if (vh_outer_type(c, f) != BT_PML) continue;
    const vh_boundary *b = &c->bnds[c->ext_bnd[f]];
    int a = f / 2;
    if (f % 2 == 0)
      set_profile(c, a, c->gobox[f], c->gibox[f] - 1, -1, b->order, b->n_eff, b->ref_coeff, b->kmax);
    else
      set_profile(c, a, c->gibox[f], c->gobox[f] - 1, +1, b->order, b->n_eff, b->ref_coeff, b->kmax);
  }
}

typedef struct {
  vh_ctx *c;
  int r;
  int lim[6][6];
} pml_copy_job;

/* Region r's copies for split-axis coordinates lo..hi-1 (axis j for the X
 * regions, i for the others). */
static void pml_copy_range(void *ctx, int lo, int hi)
{
  pml_copy_job *p = ctx;
  vh_ctx *c = p->c;
  const int r = p->r, a = r / 2, off = (r % 2 == 0) ? +1 : -1, d = a == 0 ? 1 : 0;
  const int plane = c->gibox[r];
  for (int f = EX; f <= HZ; f++) {
    /* Components normal to the region's axis (E) or tangential (H) read one
     * layer inside the inner box; the others read on the boundary plane. */
    int src_off;
    if (f <= EZ) src_off = (f == a) ? off : 0;
    else src_off = (f - HX == a) ? 0 : off;
    const int src = plane + src_off;
    int l[6];
    memcpy(l, p->lim[f], sizeof l);
    if (l[2 * d] < lo) l[2 * d] = lo;
    if (l[2 * d + 1] > hi - 1) l[2 * d + 1] = hi - 1;
    for (int i = l[XLO]; i <= l[XHI]; i++)
      for (int j = l[YLO]; j <= l[YHI]; j++)
        for (int k = l[ZLO]; k <= l[ZHI]; k++) {
          int s[3] = { i, j, k };
          s[a] = src;
          int64_t qd = vh_idx(c, i, j, k), qs = vh_idx(c, s[0], s[1], s[2]);
          if (f <= EZ) {
            c->coef[f][qd] = c->coef[f][qs];
            c->coef[3 + f][qd] = c->coef[3 + f][qs];
          } else {
            c->coef[6 + f - HX][qd] = c->coef[6 + f - HX][qs];
          }
          if (c->ctag[f]) c->ctag[f][qd] = c->ctag[f][qs];
        }
  }
}

/* Carry inner-boundary media into the PML, Z then Y then X (src/pml.c:445-629). */
static void init_pml_material_arrays(vh_ctx *c)
{
  static const bool incl[6][6] = { { 0, 0, 1, 1, 1, 1 }, { 0, 0, 1, 1, 1, 1 }, { 1, 1, 0, 0, 1, 1 },
                                   { 1, 1, 0, 0, 1, 1 }, { 1, 1, 1, 1, 0, 0 }, { 1, 1, 1, 1, 0, 0 } };
  int lim[6][6][6];
  for (int r = 0; r < 6; r++) vh_set_field_limits(c->pbox[r], lim[r], incl[r]);
  static const int order[6] = { ZLO, ZHI, YLO, YHI, XLO, XHI };
  for (int o = 0; o < 6; o++) {
    const int r = order[o];
    pml_copy_job job = { c, r, { { 0 } } };
    memcpy(job.lim, lim[r], sizeof job.lim);
    /* Split along an axis other than the copy axis, so no range reads a
     * plane another range writes. */
    const int d = r / 2 == 0 ? 1 : 0;
    int lo = 1 << 30, hi = -(1 << 30);
    int64_t work = 0;
    for (int f = EX; f <= HZ; f++) {
      if (lim[r][f][2 * d] < lo) lo = lim[r][f][2 * d];
      if (lim[r][f][2 * d + 1] > hi) hi = lim[r][f][2 * d + 1];
      work += (int64_t)(lim[r][f][XHI] - lim[r][f][XLO] + 1) * (lim[r][f][YHI] - lim[r][f][YLO] + 1) *
              (lim[r][f][ZHI] - lim[r][f][ZLO] + 1);
    }
    vh_parallel_for(lo, hi + 1, work, pml_copy_range, &job);
  }
}

static void init_pml(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising PML...\n\n");
  set_pml_limits(c);
  for (int a = 0; a < 3; a++) {
    int nn = c->n[a];
    c->pml_ad[a] = calloc(nn, sizeof(double)); c->pml_bd[a] = calloc(nn, sizeof(double));
    c->pml_gd[a] = calloc(nn, sizeof(double)); c->pml_kd[a] = calloc(nn, sizeof(double));
    c->pml_ah[a] = calloc(nn, sizeof(double)); c->pml_bh[a] = calloc(nn, sizeof(double));
    c->pml_gh[a] = calloc(nn, sizeof(double)); c->pml_kh[a] = calloc(nn, sizeof(double));
    c->pml_ibd[a] = calloc(nn, sizeof(double)); c->pml_ibh[a] = calloc(nn, sizeof(double));
  }
  set_pml_parameters(c);
  init_pml_material_arrays(c);
}

/* ---- Mur (src/mur.c:101-131) ---- */

static void init_mur(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising Mur boundaries...\n\n");
  memset(c->murbox, 0, sizeof c->murbox);
  for (int f = XLO; f <= ZHI; f++) {
    if (vh_outer_type(c, f) != BT_MUR) continue;
    bool incl[6] = { true, true, true, true, true, true };
    vh_face_of_bbox(c->murbox[f], c->gibox, f);
    for (int g = 0; g < 6; g++)
      if (g / 2 != f / 2 && vh_outer_type(c, g) == BT_MUR) incl[g] = false;
    vh_set_field_limits(c->murbox[f], c->fmlim[f], incl);
  }
  for (int f = XLO; f <= ZHI; f++) {
    int a = f / 2;
    /* Both faces of an axis read the edge at the box's low index entry. */
    double d = c->de[a][c->murbox[f][2 * a]];
    c->zeta[f] = (c->c0 * c->dt - d) / (c->c0 * c->dt + d);
  }
}

int vh_init_external_surfaces(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising non-PEC/PMC external surfaces...\n\n");
  init_external_pec_pmc(c);
  init_pml(c);
  init_mur(c);
  return 0;
}

bool vh_is_pmc_edge(const vh_ctx *c, int dir, int index)
{
  int lo = 2 * dir, hi = lo + 1;
  int tl = vh_outer_type(c, lo), th = vh_outer_type(c, hi);
  return ((tl == BT_PMC || tl == BT_PERIODIC) && index == c->gibox[lo]) ||
         ((th == BT_PMC || th == BT_PERIODIC) && index == c->gibox[hi]);
}
