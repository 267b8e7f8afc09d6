/*
 * vh_problem.c -- the host entry points: load a mesh, run the set-up in the
 * reference's order (src/vulture.c:77-148) and assemble the vgpu_problem.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "vh.h"

void vh_sibc_matrices(const vh_sibc *s, double A[4][4], double B[4][4]);
void vh_set_tls_error(const char *msg);

/* src/physical.c:37-48 */
static void physical_constants(vh_ctx *c)
{
  c->pi = 4.0 * atan(1.0);
  c->c0 = 299792458;
  c->mu0 = 4.0 * c->pi * 1e-7;
  c->eps0 = 1.0 / (c->mu0 * c->c0 * c->c0);
  c->eta0 = sqrt(c->mu0 / c->eps0);
}

/* Predefined boundaries, wires and media (src/mesh.c:246-266). */
static void init_mesh(vh_ctx *c)
{
  vh_add_boundary(c, "PEC", BT_PEC, 0, 0, 1.0, -1.0, 1.0, "", NULL, NULL);
  vh_add_boundary(c, "PMC", BT_PMC, 0, 0, 1.0, +1.0, 1.0, "", NULL, NULL);
  vh_add_boundary(c, "FREE_SPACE", BT_FREE_SPACE, 0, 0, 1.0, 0.0, 1.0, "", NULL, NULL);
  vh_wire *w;
  c->wires = calloc(16, sizeof(vh_wire));
  c->cap_wires = 16;
  w = &c->wires[c->num_wires++];
  snprintf(w->name, VH_TAG, "PEC");
  w->type = TW_PEC;
  w = &c->wires[c->num_wires++];
  snprintf(w->name, VH_TAG, "FREE_SPACE");
  w->type = TW_FREE_SPACE;
  vh_add_medium(c, "FREE_SPACE", MT_SIMPLE, 1.0, 0.0, 1.0, 0, NULL, NULL, "");
  vh_add_medium(c, "PEC", MT_PEC, 1.0, 1e8, 1.0, 0, NULL, NULL, "");
}

static void report_grid(vh_ctx *c)
{
  static const char *gt[3] = { "CUBIC", "UNIFORM", "NONUNIFORM" };
  vh_log(c, 0, "\nGrid characteristics:\n\n");
  vh_log(c, 0, "  Grid is %s\n", gt[c->grid_type]);
  vh_log(c, 0, "  Number of lines x: %d y: %d z: %d\n", c->num_lines[0], c->num_lines[1], c->num_lines[2]);
  vh_log(c, 0, "  Mesh BBOX=[%d,%d,%d,%d,%d,%d]\n", c->mbox[0], c->mbox[1], c->mbox[2], c->mbox[3], c->mbox[4],
         c->mbox[5]);
  vh_log(c, 0, "  Grid dimensions [cells]: %d x %d x %d\n", c->n[0], c->n[1], c->n[2]);
  vh_log(c, 0, "  Grid size: %lu cells\n", (unsigned long)vhost_num_cells(c));
  vh_log(c, 0, "  Inner grid: BBOX=[%d,%d,%d,%d,%d,%d]\n", c->gibox[0], c->gibox[1], c->gibox[2], c->gibox[3],
         c->gibox[4], c->gibox[5]);
  vh_log(c, 0, "  Outer grid: BBOX=[%d,%d,%d,%d,%d,%d]\n", c->gobox[0], c->gobox[1], c->gobox[2], c->gobox[3],
         c->gobox[4], c->gobox[5]);
  vh_log(c, 0, "  Ghost grid: BBOX=[%d,%d,%d,%d,%d,%d]\n", c->ggbox[0], c->ggbox[1], c->ggbox[2], c->ggbox[3],
         c->ggbox[4], c->ggbox[5]);
  vh_log(c, 0, "  Minimum edge lengths: DXMIN = %e, DYMIN = %e, DZMIN = %e\n", c->dmin[0], c->dmin[1], c->dmin[2]);
  vh_log(c, 0, "  Maximum edge lengths: DXMAX = %e, DYMAX = %e, DZMAX = %e\n", c->dmax[0], c->dmax[1], c->dmax[2]);
  vh_log(c, 0, "  Time step [s]: %e\n", c->dt);
  vh_log(c, 0, "  CFLN [-]: %e\n", c->courant);
  for (int r = 0; r < 6; r++)
    vh_log(c, 0, "  PML %s Region: BBOX=[%d,%d,%d,%d,%d,%d]\n", VH_FACE_STR[r], c->pbox[r][0], c->pbox[r][1] - 1,
           c->pbox[r][2], c->pbox[r][3] - 1, c->pbox[r][4], c->pbox[r][5] - 1);
}

static void report_mesh(vh_ctx *c)
{
  vh_log(c, 0, "\nMesh characteristics:\n\n");
  vh_log(c, 0, "  Mesh version: %d.%d.%d\n", c->version[0], c->version[1], c->version[2]);
  vh_log(c, 0, "  Mesh title: %s\n", c->comment);
  vh_log(c, 0, "  Number of time steps: %lu\n", c->num_steps);
  vh_log(c, 0, "  Courant number: %g\n", c->courant);
  vh_log(c, 0, "  Number of boundaries: %lu\n", (unsigned long)c->num_bnds);
  vh_log(c, 0, "  Number of media: %lu\n", (unsigned long)c->num_media);
  vh_log(c, 0, "  Number of wires: %lu\n", (unsigned long)c->num_wires);
  vh_log(c, 0, "  Number of external surfaces: 6\n");
  vh_log(c, 0, "  Number of internal surfaces: %lu\n", (unsigned long)c->num_surfs);
  vh_log(c, 0, "  Number of blocks: %lu\n", (unsigned long)c->num_blocks);
  vh_log(c, 0, "  Number of lines: %lu\n", (unsigned long)c->num_lns);
  vh_log(c, 0, "  Number of waveforms: %lu\n", (unsigned long)c->num_wfs);
  vh_log(c, 0, "  Number of sources: %lu\n", (unsigned long)c->num_srcs);
  vh_log(c, 0, "  Number of plane waves: %lu\n", (unsigned long)c->num_pws);
  vh_log(c, 0, "  Number of observers: %lu\n", (unsigned long)c->num_obs);
}

/* With VHOST_TRACE set, vhost_load prints the time of each set-up phase to
 * stderr. */
typedef struct {
  int on, len;
  struct timespec t;
  char buf[512];
} load_clock;

static void load_mark(load_clock *lc, const char *name)
{
  if (!lc->on) return;
  struct timespec now;
  clock_gettime(CLOCK_MONOTONIC, &now);
  const double ms = (now.tv_sec - lc->t.tv_sec) * 1e3 + (now.tv_nsec - lc->t.tv_nsec) * 1e-6;
  lc->t = now;
  if (lc->len < (int)sizeof lc->buf - 40) lc->len += snprintf(lc->buf + lc->len, sizeof lc->buf - lc->len, " %s %.2f", name, ms);
}

int vhost_load(const char *mesh_path, const char *log_path, int verbose, vhost **out)
{
  load_clock lc = { getenv("VHOST_TRACE") != NULL, 0, { 0, 0 }, { 0 } };
  if (lc.on) clock_gettime(CLOCK_MONOTONIC, &lc.t);
  *out = NULL;
  vh_ctx *c = calloc(1, sizeof(vh_ctx));
  if (!c) { vh_set_tls_error("out of memory"); return VGPU_ENOMEM; }
  c->verbose = verbose;
  c->courant = -1.0;
  if (log_path) {
    c->log = fopen(log_path, "w");
    if (!c->log) {
      vh_fail(c, "Failed to open log file %s", log_path);
      vhost_free(c);
      return VGPU_EINVAL;
    }
    fprintf(c->log, "\n *** %s version %d.%d.%d *** \n\n", "Vulture", 0, 7, 1);
  }
  physical_constants(c);
  init_mesh(c);
  int rc = vh_read_mesh(c, mesh_path);
  if (!rc) {
    /* initSimulation's default (src/simulation.c:111-122). */
    if (c->courant < 0.0) c->courant = sqrt(3.0) / 2.0;
    report_mesh(c);
  }
  load_mark(&lc, "read");
  if (!rc) rc = vh_init_grid(c);
  if (!rc) {
    for (int b = 0; b < c->num_bnds && !rc; b++)
      if (c->bnds[b].type == BT_SIBC) rc = vh_init_sibc_boundary(c, &c->bnds[b]);
  }
  load_mark(&lc, "grid");
  if (!rc) rc = vh_init_media(c);
  if (!rc) vh_init_media_arrays(c);
  load_mark(&lc, "media");
  if (!rc) rc = vh_init_blocks(c);
  if (!rc) rc = vh_init_lines(c);
  if (!rc) rc = vh_init_internal_surfaces(c);
  if (!rc) rc = vh_init_external_surfaces(c);
  load_mark(&lc, "blocks-lines-surfaces");
  if (!rc) rc = vh_init_waveforms(c);
  if (!rc) rc = vh_init_sources(c);
  if (!rc) rc = vh_init_planewaves(c);
  load_mark(&lc, "sources-planewaves");
  if (!rc) rc = vh_init_observers(c);
  load_mark(&lc, "observers");
  if (rc) {
    vh_set_tls_error(c->err);
    vhost_free(c);
    return VGPU_EINVAL;
  }
  report_grid(c);
  load_mark(&lc, "report");
  if (lc.on) fprintf(stderr, "vhost load (ms):%s\n", lc.buf);
  *out = c;
  return 0;
}

/* ---- problem assembly ---- */

/* The assembled problem's medium tags: the painted ones, unless the host
 * asked for none (vhost_use_tags). */
static void set_problem_tags(vh_ctx *c)
{
  vgpu_problem *p = &c->prob;
  const int on = c->ctag[0] && c->num_ctags > 0 && !c->tags_off;
  for (int f = 0; f < 6; f++) p->coef_tag[f] = on ? c->ctag[f] : NULL;
  p->num_tags = on ? c->num_ctags : 0;
  p->tag_coef = on ? &c->ctag_coef[0][0] : NULL;
}

int vh_build_problem(vh_ctx *c, int precision)
{
  vgpu_problem *p = &c->prob;
  memset(p, 0, sizeof *p);
  p->abi_version = VGPU_ABI_VERSION;
  p->precision = precision;
  memcpy(p->n, c->n, sizeof p->n);
  memcpy(p->gibox, c->gibox, sizeof p->gibox);
  memcpy(p->gobox, c->gobox, sizeof p->gobox);
  memcpy(p->gfilim, c->gfilim, sizeof p->gfilim);
  p->num_steps = c->num_steps;
  p->dt = c->dt;
  for (int a = 0; a < 3; a++) {
    p->ide[a] = c->ide[a];
    p->idh[a] = c->idh[a];
  }
  for (int q = 0; q < 9; q++) p->coef[q] = c->coef[q];
  set_problem_tags(c);
  for (int f = 0; f < 6; f++) {
    int t = vh_outer_type(c, f);
    p->ghost[f] = t == BT_PEC ? VGPU_GHOST_PEC : t == BT_PMC ? VGPU_GHOST_PMC
                : t == BT_PERIODIC ? VGPU_GHOST_PERIODIC : VGPU_GHOST_NONE;
    p->pml_present[f] = t == BT_PML;
    p->mur_present[f] = t == BT_MUR;
    p->mur_zeta[f] = c->zeta[f];
  }
  memcpy(p->pml_flim, c->fplim, sizeof p->pml_flim);
  memcpy(p->mur_flim, c->fmlim, sizeof p->mur_flim);
  for (int a = 0; a < 3; a++) {
    p->pml_ad[a] = c->pml_ad[a];
    p->pml_bd[a] = c->pml_bd[a];
    p->pml_ah[a] = c->pml_ah[a];
    p->pml_bh[a] = c->pml_bh[a];
    p->pml_ibd[a] = c->pml_ibd[a];
    p->pml_ibh[a] = c->pml_ibh[a];
  }

  /* Debye blocks. */
  p->num_debye = c->num_debye;
  if (c->num_debye) {
    int tot = 0;
    for (int d = 0; d < c->num_debye; d++) tot += c->media[c->debye_medium[d]].num_poles;
    c->p_debye = calloc(c->num_debye, sizeof(vgpu_debye));
    c->p_debye_coef = calloc(4 * (size_t)(tot ? tot : 1), sizeof(double));
    int off = 0;
    for (int d = 0; d < c->num_debye; d++) {
      const vh_medium *m = &c->media[c->debye_medium[d]];
      vgpu_debye *db = &c->p_debye[d];
      memcpy(db->flim, c->debye_flim[d], sizeof db->flim);
      db->num_poles = m->num_poles;
      double *da = c->p_debye_coef + 4 * off, *dbb = da + 2 * m->num_poles;
      for (int q = 0; q < m->num_poles; q++) {
        da[2 * q] = creal(m->dalpha[q]);
        da[2 * q + 1] = cimag(m->dalpha[q]);
        dbb[2 * q] = creal(m->dbeta[q]);
        dbb[2 * q + 1] = cimag(m->dbeta[q]);
      }
      db->dalpha = da;
      db->dbeta = dbb;
      off += m->num_poles;
    }
    p->debye = c->p_debye;
  }

  /* SIBC. */
  p->num_sibc_models = c->num_sibc_models;
  p->sibc_models = c->sibc_rc;
  p->num_sibc = c->num_sibcs;
  if (c->num_sibcs) {
    c->p_sibc = calloc(c->num_sibcs, sizeof(vgpu_sibc_surface));
    for (int s = 0; s < c->num_sibcs; s++) {
      vgpu_sibc_surface *o = &c->p_sibc[s];
      const vh_sibc *sb = &c->sibcs[s];
      o->normal = sb->normal;
      o->model = sb->model;
      memcpy(o->gbbox, sb->gbbox, sizeof o->gbbox);
      vh_sibc_matrices(sb, o->A, o->B);
      o->adjA = sb->adjA;
      o->adjB = sb->adjB;
    }
    p->sibc = c->p_sibc;
  }
  p->num_sibc_hops = c->num_hops;
  p->sibc_hops = c->hops;

  /* Sources with their per-step amplitudes (src/source.c:602-753). */
  uint64_t nt = c->num_steps;
  p->num_sources = 0;
  c->p_srcs = calloc(c->num_srcs ? c->num_srcs : 1, sizeof(vgpu_source));
  c->p_src_vals = calloc((size_t)(c->num_srcs ? c->num_srcs : 1) * (nt ? nt : 1), sizeof(double));
  for (int s = 0; s < c->num_srcs; s++) {
    vh_source *it = &c->srcs[s];
    int kind;
    if (it->type == ST_EFIELD || it->type == ST_HFIELD) kind = VGPU_SRC_FIELD;
    else if (it->type == ST_ELEC_CURR_DENSITY || it->type == ST_MAGN_CURR_DENSITY) kind = VGPU_SRC_CURRENT;
    else continue;
    /* The reference only applies E types in the E pass and H types in the H
     * pass; a type/field mismatch cannot arise after init. */
    bool efield = it->field <= EZ;
    vgpu_source *o = &c->p_srcs[p->num_sources];
    double *vals = c->p_src_vals + (size_t)p->num_sources * (nt ? nt : 1);
    o->field = it->field;
    o->kind = kind;
    o->soft = it->soft;
    memcpy(o->flim, it->flim[it->field], sizeof o->flim);
    for (uint64_t n = 0; n < nt; n++) {
      double t = efield ? n * c->dt : (n + 0.5) * c->dt;
      vals[n] = it->size * vh_waveform_value(c, t, it->wf, it->delay);
    }
    o->values = vals;
    p->num_sources++;
  }
  p->sources = c->p_srcs;

  /* Waveforms for device evaluation. */
  p->num_waveforms = c->num_wfs;
  c->p_wfs = calloc(c->num_wfs ? c->num_wfs : 1, sizeof(vgpu_waveform));
  for (int w = 0; w < c->num_wfs; w++) {
    vgpu_waveform *o = &c->p_wfs[w];
    o->type = c->wfs[w].type;
    o->size = c->wfs[w].size;
    o->delay = c->wfs[w].delay;
    o->width = c->wfs[w].width;
    o->frequency = c->wfs[w].frequency;
    o->table_size = c->wfs[w].table_size;
    o->table = c->wfs[w].table;
  }
  p->waveforms = c->p_wfs;

  /* Plane waves. */
  p->num_planewaves = c->num_pws;
  c->p_pws = calloc(c->num_pws ? c->num_pws : 1, sizeof(vgpu_planewave));
  c->p_pw_vals = calloc((size_t)(c->num_pws ? c->num_pws : 1) * (nt ? nt : 1) + 64 * (size_t)(c->num_pws + 1),
                        sizeof(double));
  for (int q = 0; q < c->num_pws; q++) {
    vh_planewave *it = &c->pws[q];
    vgpu_planewave *o = &c->p_pws[q];
    memcpy(o->active, it->active, sizeof o->active);
    memcpy(o->flim, it->flim, sizeof o->flim);
    o->waveform = it->wf;
    o->use_aux_grid = c->grid_type == GT_CUBIC;
    o->delay = it->delay;
    memcpy(o->kinc, it->kinc, sizeof o->kinc);
    memcpy(o->finc, it->finc, sizeof o->finc);
    memcpy(o->r0, it->r0, sizeof o->r0);
    memcpy(o->ijk0, it->ijk0, sizeof o->ijk0);
    o->phase_velocity = it->phase_velocity;
    if (o->use_aux_grid) {
      double *base = c->p_pw_vals + (size_t)q * ((nt ? nt : 1) + 64);
      o->aux_nx = it->nx;
      o->aux_xb = it->xb;
      o->aux_npml = 10;
      o->aux_beta = it->beta_eyi;
      o->aux_gamma = it->gamma_hzi;
      memcpy(base, it->adx, 10 * sizeof(double));
      memcpy(base + 10, it->bdx, 10 * sizeof(double));
      memcpy(base + 20, it->ahx, 10 * sizeof(double));
      memcpy(base + 30, it->bhx, 10 * sizeof(double));
      o->aux_adx = base;
      o->aux_bdx = base + 10;
      o->aux_ahx = base + 20;
      o->aux_bhx = base + 30;
      double *src = base + 64;
      for (uint64_t n = 0; n < nt; n++) src[n] = vh_waveform_value(c, n * c->dt, it->wf, it->delay);
      o->aux_source = src;
    }
  }
  p->planewaves = c->p_pws;
  for (int a = 0; a < 3; a++) {
    c->pos_node[a] = calloc(c->n[a], sizeof(double));
    c->pos_half[a] = calloc(c->n[a], sizeof(double));
    for (int i = 0; i < c->n[a]; i++) {
      double r[3];
      int ijk[3] = { c->gibox[XLO], c->gibox[YLO], c->gibox[ZLO] };
      ijk[a] = i;
      vh_field_physical_location(c, r, HX + a, ijk[0], ijk[1], ijk[2]);
      c->pos_node[a][i] = r[a];
      vh_field_physical_location(c, r, EX + a, ijk[0], ijk[1], ijk[2]);
      c->pos_half[a][i] = r[a];
    }
    p->pos_node[a] = c->pos_node[a];
    p->pos_half[a] = c->pos_half[a];
  }

  /* Observers. */
  p->out_start = c->out_start;
  p->out_stop = c->out_stop;
  p->num_td = c->num_td;
  p->td_points = c->td_points;
  p->num_fd = c->num_fd;
  p->fd_points = c->fd_points;
  p->num_bin = c->num_bin;
  p->bin_points = c->bin_points;
  p->num_freq = (int32_t)c->num_freq;
  p->omega = c->omega;
  c->prob_ready = 1;
  return 0;
}

int vhost_problem(vhost *h, int32_t precision, const vgpu_problem **out)
{
  if (!h || !out) { vh_set_tls_error("null argument"); return VGPU_EINVAL; }
  if (precision != VGPU_FP64 && precision != VGPU_FP32) { vh_set_tls_error("invalid precision"); return VGPU_EINVAL; }
  if (!h->prob_ready) vh_build_problem(h, precision);
  h->prob.precision = precision;
  *out = &h->prob;
  return 0;
}

int vhost_use_tags(vhost *h, int32_t use)
{
  if (!h) { vh_set_tls_error("null argument"); return VGPU_EINVAL; }
  h->tags_off = !use;
  if (h->prob_ready) set_problem_tags(h);
  return 0;
}

int64_t vhost_check_tags(const vhost *h)
{
  if (!h || !h->ctag[0] || h->num_ctags == 0) return -1;
  const int64_t vol = (int64_t)h->n[0] * h->n[1] * h->n[2];
  const double zero = 0.0;
  int64_t bad = 0;
  for (int f = EX; f <= HZ; f++) {
    const double *a = f <= EZ ? h->coef[f] : NULL;
    const double *b = f <= EZ ? h->coef[3 + f] : h->coef[6 + f - HX];
    const uint8_t *t = h->ctag[f];
    for (int64_t q = 0; q < vol; q++) {
      if (t[q] > h->num_ctags) { bad++; continue; }
      const double *v = t[q] ? h->ctag_coef[t[q] - 1] : NULL;
      const double *ea = v ? &v[0] : &zero, *eb = v ? &v[f <= EZ ? 1 : 2] : &zero;
      if ((a && memcmp(&a[q], ea, sizeof(double)) != 0) || memcmp(&b[q], eb, sizeof(double)) != 0) bad++;
    }
  }
  return bad;
}

uint64_t vhost_num_steps(const vhost *h) { return h->num_steps; }
uint64_t vhost_num_output_steps(const vhost *h)
{
  if (h->num_steps == 0 || h->out_start >= h->num_steps) return 0;
  uint64_t stop = h->out_stop < h->num_steps - 1 ? h->out_stop : h->num_steps - 1;
  return stop - h->out_start + 1;
}
int32_t vhost_num_td(const vhost *h) { return h->num_td; }
int32_t vhost_num_fd(const vhost *h) { return h->num_fd; }
int64_t vhost_num_bin(const vhost *h) { return h->num_bin; }
int32_t vhost_num_freq(const vhost *h) { return (int32_t)h->num_freq; }
double vhost_dt(const vhost *h) { return h->dt; }
uint64_t vhost_num_cells(const vhost *h)
{
  return (uint64_t)(h->gobox[XHI] - h->gobox[XLO]) * (uint64_t)(h->gobox[YHI] - h->gobox[YLO]) *
         (uint64_t)(h->gobox[ZHI] - h->gobox[ZLO]);
}

const char *vhost_observer_name(const vhost *h, int32_t fd, int32_t slot)
{
  int kind = fd ? OBS_FD_ASCII : OBS_TD_ASCII;
  for (int o = 0; o < h->num_obs; o++)
    if (h->obs[o].kind == kind && h->obs[o].slot == slot) return h->obs[o].name;
  return NULL;
}

void vhost_free(vhost *c)
{
  if (!c) return;
  if (c->log) fclose(c->log);
  for (int a = 0; a < 3; a++) {
    free(c->lines[a]);
    free(c->de[a]); free(c->dh[a]); free(c->ide[a]); free(c->idh[a]);
    free(c->pml_ad[a]); free(c->pml_bd[a]); free(c->pml_gd[a]); free(c->pml_kd[a]);
    free(c->pml_ah[a]); free(c->pml_bh[a]); free(c->pml_gh[a]); free(c->pml_kh[a]);
    free(c->pml_ibd[a]); free(c->pml_ibh[a]);
    free(c->pos_node[a]); free(c->pos_half[a]);
  }
  for (int q = 0; q < 9; q++) vh_free_volume(c->coef[q], (size_t)c->n[0] * c->n[1] * c->n[2]);
  vh_free_tags(c);
  for (int m = 0; m < c->num_media; m++) {
    free(c->media[m].res); free(c->media[m].pole); free(c->media[m].dalpha); free(c->media[m].dbeta);
  }
  for (int w = 0; w < c->num_wfs; w++) free(c->wfs[w].table);
  for (int s = 0; s < c->num_sibcs; s++) { free(c->sibcs[s].adjA); free(c->sibcs[s].adjB); }
  for (int m = 0; m < c->num_sibc_models; m++)
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < 4; q++) { free(c->sibc_pr[m].poles[p][q]); free(c->sibc_pr[m].residues[p][q]); }
  free(c->media); free(c->bnds); free(c->wires); free(c->blocks); free(c->surfs); free(c->lns);
  free(c->wfs); free(c->srcs); free(c->pws); free(c->obs);
  free(c->debye_flim); free(c->debye_medium);
  free(c->sibc_pr); free(c->sibcs); free(c->sibc_rc); free(c->sibc_q); free(c->hops);
  free(c->omega); free(c->td_points); free(c->fd_points); free(c->bin_points);
  if (c->impulse) fclose(c->impulse);
  free(c->p_srcs); free(c->p_src_vals); free(c->p_debye); free(c->p_debye_coef);
  free(c->p_pws); free(c->p_pw_vals); free(c->p_wfs); free(c->p_sibc);
  free(c);
}
