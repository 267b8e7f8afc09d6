/*
 * vh_parse.c -- .mesh reader for vulture_b200.
 *
 * Restates the card grammar of the reference's readMesh() (src/mesh.c:269-405):
 * four sections, two-letter cards, '#' comments, required and singleton cards,
 * and each module's parse* function.  Field-by-field scanning follows the
 * reference's sscanf formats so the same files parse to the same values; the
 * reference reads PML and SIBC numbers into `real` with %e, here they are read
 * as double as in its real=double build.
 */
#define _GNU_SOURCE
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include "vh.h"

const unsigned char VH_FACE_MASKS[6] = { 0x20, 0x10, 0x8, 0x4, 0x2, 0x1 };
const char *VH_FACE_STR[6] = { "XLO", "XHI", "YLO", "YHI", "ZLO", "ZHI" };
const char *VH_FIELD_STR[6] = { "EX", "EY", "EZ", "HX", "HY", "HZ" };

static __thread char vh_tls_err[1024];

int vh_fail(vh_ctx *c, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(c->err, sizeof c->err, fmt, ap);
  va_end(ap);
  snprintf(vh_tls_err, sizeof vh_tls_err, "%s", c->err);
  if (c->log) {
    fprintf(c->log, "*** Error: %s\n", c->err);
    fflush(c->log);
  }
  return -1;
}

void vh_set_tls_error(const char *msg)
{
  snprintf(vh_tls_err, sizeof vh_tls_err, "%s", msg);
}

const char *vhost_last_error(void) { return vh_tls_err; }

void vh_log(vh_ctx *c, int verbose_only, const char *fmt, ...)
{
  if (!c->log || (verbose_only && !c->verbose)) return;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(c->log, fmt, ap);
  va_end(ap);
}

/* ---- bounding boxes (src/bounding_box.c) ---- */

int vh_bbox_type(const int b[6])
{
  static const int type[8] = { BB_VOLUME, BB_SURFACE, BB_SURFACE, BB_LINE, BB_SURFACE, BB_LINE,
                               BB_LINE, BB_POINT };
  int m = (b[XLO] == b[XHI]) + 2 * (b[YLO] == b[YHI]) + 4 * (b[ZLO] == b[ZHI]);
  return type[m];
}

int vh_bbox_direction(const int b[6])
{
  static const int dir[8] = { CA_UNDEF, XDIR, YDIR, ZDIR, ZDIR, YDIR, XDIR, CA_UNDEF };
  int m = (b[XLO] == b[XHI]) + 2 * (b[YLO] == b[YHI]) + 4 * (b[ZLO] == b[ZHI]);
  return dir[m];
}

/* The reference compares bbox[ZLO] <= bbox[ZLO] (src/bounding_box.h:31),
 * so the z extent is never checked; kept as is. */
bool vh_bbox_is_normal(const int b[6])
{
  return b[XLO] <= b[XHI] && b[YLO] <= b[YHI];
}

bool vh_bbox_is_within(const int b1[6], const int b2[6])
{
  return b1[XLO] >= b2[XLO] && b1[XHI] <= b2[XHI] && b1[YLO] >= b2[YLO] && b1[YHI] <= b2[YHI] &&
         b1[ZLO] >= b2[ZLO] && b1[ZHI] <= b2[ZHI];
}

void vh_bbox_offset(int out[6], const int b[6], const int off[6])
{
  out[XLO] = b[XLO] + off[XLO];
  out[YLO] = b[YLO] + off[YLO];
  out[ZLO] = b[ZLO] + off[ZLO];
  out[XHI] = b[XHI] + off[XLO];
  out[YHI] = b[YHI] + off[YLO];
  out[ZHI] = b[ZHI] + off[ZLO];
}

void vh_face_of_bbox(int out[6], const int b[6], int face)
{
  for (int f = 0; f < 6; f++) out[f] = b[f];
  int axis = face / 2;
  int v = b[face];
  out[2 * axis] = v;
  out[2 * axis + 1] = v;
}

/* Tangential E or normal H on a face (src/bounding_box.c:162-210). */
bool vh_field_in_boundary(int field, int face)
{
  int axis = face / 2;
  if (field <= EZ) return field != axis;
  return (field - HX) == axis;
}

bool vh_field_parallel_to_boundary(int field, int face)
{
  return (field % 3) != face / 2;
}

/* Field limits of a volume with each face's boundary fields included or not
 * (src/grid.c:414-454). */
void vh_set_field_limits(const int bbox[6], int flim[6][6], const bool incl[6])
{
  for (int field = EX; field <= HZ; field++) {
    for (int face = XLO; face <= ZHI; face++) {
      bool lo = (face % 2) == 0;
      if (vh_field_in_boundary(field, face)) {
        if (incl[face]) flim[field][face] = bbox[face];
        else flim[field][face] = lo ? bbox[face] + 1 : bbox[face] - 1;
      } else {
        flim[field][face] = lo ? bbox[face] : bbox[face] - 1;
      }
    }
  }
}

unsigned char vh_face_mask_from_string(const char *s)
{
  char *end = NULL;
  long v = strtol(s, &end, 2);
  if (v < 0 || v > 63L || *end) return VH_FACE_MASK_ERROR;
  return (unsigned char)v;
}

void vh_mask_to_bool(bool incl[6], unsigned char mask)
{
  for (int f = 0; f < 6; f++) incl[f] = (mask & VH_FACE_MASKS[f]) != 0;
}

/* ---- growable lists ---- */

#define VH_PUSH(c, arr, num, cap, type)                                         \
  ({                                                                            \
    if ((c)->num == (c)->cap) {                                                 \
      int ncap = (c)->cap ? 2 * (c)->cap : 16;                                  \
      type *na = realloc((c)->arr, (size_t)ncap * sizeof(type));                \
      if (!na) abort();                                                         \
      (c)->arr = na;                                                            \
      (c)->cap = ncap;                                                          \
    }                                                                           \
    memset(&(c)->arr[(c)->num], 0, sizeof(type));                               \
    &(c)->arr[(c)->num++];                                                      \
  })

int vh_find_medium(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_media; i++)
    if (strncmp(c->media[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

int vh_find_boundary(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_bnds; i++)
    if (strncmp(c->bnds[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

int vh_find_waveform(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_wfs; i++)
    if (strncmp(c->wfs[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

static int find_wire(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_wires; i++)
    if (strncmp(c->wires[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

static int find_source(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_srcs; i++)
    if (strncmp(c->srcs[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

static int find_planewave(const vh_ctx *c, const char *name)
{
  for (int i = 0; i < c->num_pws; i++)
    if (strncmp(c->pws[i].name, name, VH_TAG) == 0) return i;
  return -1;
}

/* Observer names are looked up in a hash table: plane observers come as
 * thousands of point cards. */
typedef struct {
  uint64_t *keys;
  int *vals;
  size_t cap, used;
} name_hash;

static __thread name_hash *obs_hash_tls;

static uint64_t hash_name(const char *s)
{
  uint64_t h = 1469598103934665603ull;
  for (; *s; s++) h = (h ^ (unsigned char)*s) * 1099511628211ull;
  return h ? h : 1;
}

static int obs_lookup(const vh_ctx *c, name_hash *h, const char *name, int insert_as)
{
  if (h->cap == 0 || (h->used + 1) * 2 > h->cap) {
    size_t ncap = h->cap ? 2 * h->cap : 1024;
    uint64_t *nk = calloc(ncap, sizeof(uint64_t));
    int *nv = calloc(ncap, sizeof(int));
    for (size_t i = 0; i < h->cap; i++) {
      if (!h->keys[i]) continue;
      size_t p = h->keys[i] & (ncap - 1);
      while (nk[p]) p = (p + 1) & (ncap - 1);
      nk[p] = h->keys[i];
      nv[p] = h->vals[i];
    }
    free(h->keys);
    free(h->vals);
    h->keys = nk;
    h->vals = nv;
    h->cap = ncap;
  }
  uint64_t key = hash_name(name);
  size_t p = key & (h->cap - 1);
  while (h->keys[p]) {
    if (h->keys[p] == key && strncmp(c->obs[h->vals[p]].name, name, VH_TAG) == 0) return h->vals[p];
    p = (p + 1) & (h->cap - 1);
  }
  if (insert_as >= 0) {
    h->keys[p] = key;
    h->vals[p] = insert_as;
    h->used++;
  }
  return -1;
}

/* ---- model additions ---- */

int vh_add_medium(vh_ctx *c, const char *name, int type, double eps_r, double sigma, double mu_r,
                  int num_poles, const double *res, const double *poles, const char *file)
{
  vh_medium *m = VH_PUSH(c, media, num_media, cap_media, vh_medium);
  snprintf(m->name, VH_TAG, "%s", name);
  m->type = type;
  m->eps_r = eps_r;
  m->sigma = sigma;
  m->mu_r = mu_r;
  if (type == MT_DEBYE) {
    if (!file || !file[0]) {
      m->num_poles = num_poles;
      m->res = calloc(num_poles ? num_poles : 1, sizeof(double complex));
      m->pole = calloc(num_poles ? num_poles : 1, sizeof(double complex));
      for (int p = 0; p < num_poles; p++) {
        m->res[p] = (double complex)res[p];
        m->pole[p] = (double complex)poles[p];
      }
    } else {
      /* Debye parameter file (src/medium.c:325-379). */
      FILE *fp = fopen(file, "r");
      if (!fp) return vh_fail(c, "Cannot open Debye parameter file %s", file);
      double t1, t2, t3, t4;
      int np;
      if (fscanf(fp, "%d %lf %lf %lf", &np, &t1, &t2, &t3) != 4) {
        fclose(fp);
        return vh_fail(c, "Failed to read first line of Debye parameter file %s", file);
      }
      if (np < 0) { fclose(fp); return vh_fail(c, "Number of poles in %s must be >=0", file); }
      if (t1 < 1.0) { fclose(fp); return vh_fail(c, "High frequency rel. permittivity in %s must be >=1", file); }
      if (t2 < 0.0) { fclose(fp); return vh_fail(c, "Conductivity in %s must be >=0", file); }
      if (t3 < 1.0) { fclose(fp); return vh_fail(c, "Rel. permeability in %s must be >=1", file); }
      m->eps_r = t1;
      m->sigma = t2;
      m->mu_r = t3;
      m->num_poles = np;
      m->res = calloc(np ? np : 1, sizeof(double complex));
      m->pole = calloc(np ? np : 1, sizeof(double complex));
      for (int p = 0; p < np; p++) {
        if (fscanf(fp, "%lf %lf %lf %lf", &t1, &t2, &t3, &t4) != 4) {
          fclose(fp);
          return vh_fail(c, "Failed to read parameters from Debye parameter file %s", file);
        }
        m->res[p] = t1 + I * t2;
        if (t3 > 0.0) { fclose(fp); return vh_fail(c, "Unstable pole in file %s", file); }
        m->pole[p] = t3 + I * t4;
      }
      fclose(fp);
    }
  }
  return (int)(m - c->media);
}

int vh_add_boundary(vh_ctx *c, const char *name, int type, int num_layers, int order, double n_eff,
                    double ref_coeff, double kmax, const char *file, double S_TM[2][2], double S_TE[2][2])
{
  vh_boundary *b = VH_PUSH(c, bnds, num_bnds, cap_bnds, vh_boundary);
  snprintf(b->name, VH_TAG, "%s", name);
  b->type = type;
  b->num_layers = num_layers;
  b->order = order;
  b->n_eff = n_eff;
  b->ref_coeff = ref_coeff;
  b->kmax = kmax;
  snprintf(b->file, VH_PATH, "%s", file ? file : "");
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      if (S_TM) b->S_TM[i][j] = S_TM[i][j];
      if (S_TE) b->S_TE[i][j] = S_TE[i][j];
    }
  b->sibc_model = -1;
  return (int)(b - c->bnds);
}

static void add_wire(vh_ctx *c, const char *name, int type)
{
  vh_wire *w = VH_PUSH(c, wires, num_wires, cap_wires, vh_wire);
  snprintf(w->name, VH_TAG, "%s", name);
  w->type = type;
}

void vh_pml_defaults(int *num_layers, int *order, double *n_eff, double *ref_coeff, double *kmax)
{
  /* src/pml.c:1326-1337 */
  *num_layers = 6;
  *order = 4;
  *n_eff = 1.0;
  *ref_coeff = -1.0;
  *kmax = 1.0;
}

/* Copy a quoted file name relative to the mesh directory when not absolute. */
static void resolve_path(const vh_ctx *c, char out[VH_PATH], const char *name)
{
  if (name[0] == '/' || !c->mesh_dir[0]) snprintf(out, VH_PATH, "%s", name);
  else snprintf(out, VH_PATH, "%s/%s", c->mesh_dir, name);
  FILE *fp = fopen(out, "r");
  if (fp) { fclose(fp); return; }
  snprintf(out, VH_PATH, "%s", name);
}

/* ---- card parsers (one per reference parse* function) ---- */

static bool parse_VM(vh_ctx *c, char *l)
{
  if (sscanf(l, "%d.%d.%d", &c->version[0], &c->version[1], &c->version[2]) != 3) return false;
  if (c->version[0] >= 2000 || c->version[1] >= 1000 || c->version[2] >= 1000) return false;
  return true;
}

static bool parse_CE(vh_ctx *c, char *l)
{
  snprintf(c->comment, sizeof c->comment, "%s", l);
  return true;
}

static bool parse_DM(vh_ctx *c, char *l)
{
  if (sscanf(l, "%d %d %d", &c->mesh_cells[0], &c->mesh_cells[1], &c->mesh_cells[2]) != 3) return false;
  for (int d = 0; d < 3; d++) {
    if (c->mesh_cells[d] < 1) return false;
    c->num_lines[d] = c->mesh_cells[d] + 1;
  }
  c->mbox[XLO] = 0; c->mbox[XHI] = c->mesh_cells[0];
  c->mbox[YLO] = 0; c->mbox[YHI] = c->mesh_cells[1];
  c->mbox[ZLO] = 0; c->mbox[ZHI] = c->mesh_cells[2];
  return true;
}

/* Obsolete external boundary card (src/surface.c:160-211). */
static bool parse_BR(vh_ctx *c, char *l)
{
  int t[6];
  if (sscanf(l, "%d %d %d %d %d %d", &t[0], &t[1], &t[2], &t[3], &t[4], &t[5]) != 6) return false;
  for (int f = 0; f < 6; f++) {
    int type, layers = 0, order = 0;
    double n_eff = 0, rc = 0, kmax = 0;
    switch (t[f]) {
      case -1: type = BT_PEC; rc = -1.0; break;
      case 0: type = BT_PML; vh_pml_defaults(&layers, &order, &n_eff, &rc, &kmax); break;
      case 1: type = BT_PMC; rc = 1.0; break;
      default: return false;
    }
    vh_add_boundary(c, VH_FACE_STR[f], type, layers, order, n_eff, rc, kmax, "", NULL, NULL);
  }
  return true;
}

/* PML depths (src/boundary.c:74-102).  A face without a boundary yet resolves
 * to boundary 0, as the reference's isBoundary() leaves number = 0. */
static bool parse_BE(vh_ctx *c, char *l)
{
  int d[6];
  if (sscanf(l, "%d %d %d %d %d %d", &d[0], &d[1], &d[2], &d[3], &d[4], &d[5]) != 6) return false;
  for (int f = 0; f < 6; f++) {
    if (d[f] < 0) return false;
    int b = vh_find_boundary(c, VH_FACE_STR[f]);
    if (b < 0) b = 0;
    c->bnds[b].num_layers = d[f];
  }
  return true;
}

static bool parse_MT(vh_ctx *c, char *l)
{
  char name[VH_TAG] = "", type_str[VH_TAG] = "", file[VH_PATH] = "";
  static const char *types[4] = { "FREE_SPACE", "PEC", "SIMPLE", "DEBYE" };
  double eps_r = 1.0, sigma = 0.0, mu_r = 1.0, res[3] = { 0 }, poles[3] = { 0 };
  int np = 0;
  if (sscanf(l, "%31s %31s", name, type_str) < 2) return false;
  if (vh_find_medium(c, name) >= 0) return false;
  int type = -1;
  for (int t = 0; t < 4; t++)
    if (strncmp(type_str, types[t], VH_TAG) == 0) type = t;
  if (type < 0) return false;
  int ns;
  switch (type) {
    case MT_SIMPLE:
      ns = sscanf(l, "%31s %31s %lf %lf %lf", name, type_str, &eps_r, &sigma, &mu_r);
      if (ns >= 3 && eps_r < 1.0) return false;
      if (ns >= 4 && sigma < 0.0) return false;
      if (ns >= 5 && mu_r < 1.0) return false;
      break;
    case MT_DEBYE:
      ns = sscanf(l, "%31s %31s %lf %lf %lf %lf %lf %lf %lf %lf %lf", name, type_str, &eps_r, &sigma,
                  &mu_r, &res[0], &poles[0], &res[1], &poles[1], &res[2], &poles[2]);
      if (ns >= 3 && eps_r < 1.0) return false;
      if (ns >= 4 && sigma < 0.0) return false;
      if (ns >= 5 && mu_r < 1.0) return false;
      if (ns == 7 || ns == 9 || ns == 11) {
        np = (ns - 5) / 2;
      } else {
        char raw[VH_PATH] = "";
        if (sscanf(l, "%31s %31s \"%1023[^\"]\"", name, type_str, raw) != 3) return false;
        resolve_path(c, file, raw);
      }
      break;
    default:
      break;
  }
  return vh_add_medium(c, name, type, eps_r, sigma, mu_r, np, res, poles, file) >= 0;
}

static bool parse_BT(vh_ctx *c, char *l)
{
  char name[VH_TAG] = "", type_str[VH_TAG] = "", file[VH_PATH] = "";
  static const char *types[7] = { "PMC", "PML", "PEC", "FREE_SPACE", "PERIODIC", "MUR", "SIBC" };
  double S_TM[2][2] = { { -1.0, 0.0 }, { 0.0, -1.0 } };
  double S_TE[2][2] = { { -1.0, 0.0 }, { 0.0, -1.0 } };
  int layers = 0, order = 0;
  double n_eff = 0, rc = 0, kmax = 0;
  if (sscanf(l, "%31s %31s", name, type_str) < 2) return false;
  if (vh_find_boundary(c, name) >= 0) return false;
  int type = -1;
  for (int t = 0; t < 7; t++)
    if (strncmp(type_str, types[t], VH_TAG) == 0) type = t;
  if (type < 0) return false;
  switch (type) {
    case BT_PEC: rc = -1.0; break;
    case BT_PMC: rc = 1.0; break;
    case BT_FREE_SPACE: rc = 0.0; break;
    case BT_PERIODIC: rc = 1.0; break;
    case BT_MUR: rc = 0.0; break;
    case BT_PML:
      vh_pml_defaults(&layers, &order, &n_eff, &rc, &kmax);
      sscanf(l, "%31s %31s %d %d %le %le %le", name, type_str, &layers, &order, &n_eff, &rc, &kmax);
      break;
    case BT_SIBC: {
      int ns = sscanf(l, "%31s %31s %le %le %le %le %le %le %le %le", name, type_str, &S_TM[0][0],
                      &S_TM[0][1], &S_TM[1][0], &S_TM[1][1], &S_TE[0][0], &S_TE[0][1], &S_TE[1][0],
                      &S_TE[1][1]);
      if (ns == 10) {
      } else if (ns == 6) {
        for (int i = 0; i < 2; i++)
          for (int j = 0; j < 2; j++) S_TE[i][j] = S_TM[i][j];
      } else {
        char raw[VH_PATH] = "";
        if (sscanf(l, "%31s %31s \"%1023[^\"]\"", name, type_str, raw) != 3) return false;
        resolve_path(c, file, raw);
      }
      break;
    }
  }
  vh_add_boundary(c, name, type, layers, order, n_eff, rc, kmax, file, S_TM, S_TE);
  return true;
}

static bool parse_WT(vh_ctx *c, char *l)
{
  char name[VH_TAG] = "", type_str[VH_TAG] = "";
  if (sscanf(l, "%31s %31s", name, type_str) < 2) return false;
  if (find_wire(c, name) >= 0) return false;
  /* The reference accepts only PEC wires here (src/wire.c:120-128). */
  if (strncmp(type_str, "PEC", VH_TAG) != 0) return false;
  add_wire(c, name, TW_PEC);
  return true;
}

static bool parse_MB(vh_ctx *c, char *l)
{
  char medium[VH_TAG] = "", mask_str[VH_TAG] = "111111";
  int b[6];
  if (sscanf(l, "%d %d %d %d %d %d %31s %31s", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], medium,
             mask_str) < 7)
    return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  if (vh_bbox_type(b) != BB_VOLUME) return false;
  int m = vh_find_medium(c, medium);
  if (m < 0) return false;
  unsigned char mask = vh_face_mask_from_string(mask_str);
  if (mask == VH_FACE_MASK_ERROR) return false;
  vh_block *blk = VH_PUSH(c, blocks, num_blocks, cap_blocks, vh_block);
  memcpy(blk->mbbox, b, sizeof b);
  blk->medium = m;
  blk->mask = mask;
  return true;
}

static bool parse_TB(vh_ctx *c, char *l)
{
  char bname[VH_TAG] = "";
  int b[6], orient = 1;
  double angle = 0.0;
  if (sscanf(l, "%d %d %d %d %d %d %31s %d %lf", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], bname,
             &orient, &angle) < 7)
    return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  if (vh_bbox_type(b) != BB_SURFACE) return false;
  int bi = vh_find_boundary(c, bname);
  if (bi < 0) return false;
  if (orient != 1 && orient != -1) return false;
  if (angle < -180.0 || angle > 180.0) return false;
  vh_surface *s = VH_PUSH(c, surfs, num_surfs, cap_surfs, vh_surface);
  memcpy(s->mbbox, b, sizeof b);
  s->boundary = bi;
  s->orient = orient;
  s->angle = angle;
  return true;
}

static bool parse_TW(vh_ctx *c, char *l)
{
  char wname[VH_TAG] = "", lo[VH_TAG] = "", hi[VH_TAG] = "";
  static const char *ends[3] = { "THRU", "END", "CORNER" };
  int b[6];
  int ns = sscanf(l, "%d %d %d %d %d %d %31s %31s %31s", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5],
                  wname, lo, hi);
  if (ns < 7) return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  if (vh_bbox_type(b) != BB_LINE) return false;
  int w = find_wire(c, wname);
  if (w < 0) return false;
  if (ns >= 8) {
    int ok = 0;
    for (int e = 0; e < 3; e++) ok |= strncmp(ends[e], lo, VH_TAG) == 0;
    if (!ok) return false;
  }
  if (ns >= 9) {
    int ok = 0;
    for (int e = 0; e < 3; e++) ok |= strncmp(ends[e], hi, VH_TAG) == 0;
    if (!ok) return false;
  }
  vh_line *ln = VH_PUSH(c, lns, num_lns, cap_lns, vh_line);
  memcpy(ln->mbbox, b, sizeof b);
  ln->wire = w;
  return true;
}

static bool parse_WF(vh_ctx *c, char *l)
{
  static const char *types[10] = { "GAUSSIAN_PULSE", "NARROW_GAUSSIAN_PULSE", "DIFF_GAUSSIAN_PULSE",
                                   "RICKER_WAVELET", "MOD_GAUSSIAN_PULSE", "COMPACT_PULSE",
                                   "DIFF_COMPACT_PULSE", "MOD_COMPACT_PULSE", "RAMPED_SINUSOID",
                                   "EXTERNAL" };
  char name[VH_TAG] = "", type_str[VH_TAG] = "", file[VH_PATH] = "";
  double size = -1.0, delay = -1.0, width = -1.0, freq = -1.0;
  if (sscanf(l, "%31s %31s", name, type_str) < 2) return false;
  if (vh_find_waveform(c, name) >= 0) return false;
  int type = -1;
  for (int t = 0; t < 10; t++)
    if (strncmp(type_str, types[t], VH_TAG) == 0) type = t;
  if (type < 0) return false;
  if (type == VGPU_WF_EXTERNAL) {
    char raw[VH_PATH] = "";
    int ns = sscanf(l, "%31s %31s \"%1023[^\"]\" %lf %lf", name, type_str, raw, &size, &delay);
    if (ns < 3) return false;
    if (ns >= 4 && size < 0.0) return false;
    resolve_path(c, file, raw);
  } else {
    int ns = sscanf(l, "%31s %31s %lf %lf %lf %lf", name, type_str, &size, &delay, &width, &freq);
    if (ns >= 3 && size < 0.0) return false;
    if (ns >= 5 && width <= 0.0) return false;
    if (ns == 6 && freq <= 0.0) return false;
  }
  vh_waveform *w = VH_PUSH(c, wfs, num_wfs, cap_wfs, vh_waveform);
  snprintf(w->name, VH_TAG, "%s", name);
  w->type = type;
  w->size = size;
  w->delay = delay;
  w->width = width;
  w->frequency = freq;
  snprintf(w->file, VH_PATH, "%s", file);
  return true;
}

/* Source tag table: the 84 tags of src/source.c:130-280 grouped in triples
 * (X, Y, Z polarisation).  Each row: base tag, type, field of the X member,
 * soft flag, surface normals of the X/Y/Z members (-1 when not a surface
 * current). */
typedef struct {
  const char *tag;
  int type, field0, soft, normal[3];
} src_tag_row;

static const src_tag_row SRC_TAGS[] = {
  { "E", ST_EFIELD, EX, 1, { -1, -1, -1 } },
  { "H", ST_HFIELD, HX, 1, { -1, -1, -1 } },
  { "=E", ST_EFIELD, EX, 0, { -1, -1, -1 } },
  { "=H", ST_HFIELD, HX, 0, { -1, -1, -1 } },
  { "J", ST_ELEC_CURR_DENSITY, EX, 1, { -1, -1, -1 } },
  { "JM", ST_MAGN_CURR_DENSITY, HX, 1, { -1, -1, -1 } },
  { "=J", ST_ELEC_CURR_DENSITY, EX, 0, { -1, -1, -1 } },
  { "=JM", ST_MAGN_CURR_DENSITY, HX, 0, { -1, -1, -1 } },
  { "JS", ST_ELEC_SURF_CURR_DENSITY, EX, 1, { -1, -1, -1 } },
  { "JMS", ST_MAGN_SURF_CURR_DENSITY, HX, 1, { -1, -1, -1 } },
  { "=JS", ST_ELEC_SURF_CURR_DENSITY, EX, 0, { -1, -1, -1 } },
  { "=JMS", ST_MAGN_SURF_CURR_DENSITY, HX, 0, { -1, -1, -1 } },
  { "I", ST_ELEC_CURRENT, EX, 1, { -1, -1, -1 } },
  { "IM", ST_MAGN_CURRENT, HX, 1, { -1, -1, -1 } },
  { "=I", ST_ELEC_CURRENT, EX, 0, { -1, -1, -1 } },
  { "=IM", ST_MAGN_CURRENT, HX, 0, { -1, -1, -1 } },
  { "ID", ST_ELEC_CURRENT_MOMENT, EX, 1, { -1, -1, -1 } },
  { "IMD", ST_MAGN_CURRENT_MOMENT, HX, 1, { -1, -1, -1 } },
  { "=ID", ST_ELEC_CURRENT_MOMENT, EX, 0, { -1, -1, -1 } },
  { "=IMD", ST_MAGN_CURRENT_MOMENT, HX, 0, { -1, -1, -1 } },
  { "V", ST_VOLTAGE, EX, 1, { -1, -1, -1 } },
  { "=V", ST_VOLTAGE, EX, 0, { -1, -1, -1 } },
  { "VR", ST_THEVENIN_VOLTAGE, EX, 1, { -1, -1, -1 } },
  { "IG", ST_NORTON_CURRENT, EX, 1, { -1, -1, -1 } },
};

/* Surface-current tags carry two axis letters: polarisation then a second
 * letter; JSXY (pol X, normal Y), JSYZ (Y, Z), JSZX (Z, X), JSXZ (X, Z),
 * JSYX (Y, X), JSZY (Z, Y) (src/source.c:206-231). */
static bool decode_source_tag(const char *tag, int *type, int *pol, int *norm, int *field, int *soft)
{
  size_t len = strlen(tag);
  if (len < 2) return false;
  for (size_t r = 0; r < sizeof SRC_TAGS / sizeof SRC_TAGS[0]; r++) {
    const src_tag_row *row = &SRC_TAGS[r];
    size_t bl = strlen(row->tag);
    bool surf = row->type == ST_ELEC_SURF_CURR_DENSITY || row->type == ST_MAGN_SURF_CURR_DENSITY;
    size_t want = bl + (surf ? 2 : 1);
    if (len != want || strncmp(tag, row->tag, bl) != 0) continue;
    int p = tag[bl] - 'X';
    if (p < 0 || p > 2) continue;
    int nrm = -1;
    if (surf) {
      int n2 = tag[bl + 1] - 'X';
      if (n2 < 0 || n2 > 2 || n2 == p) continue;
      nrm = n2;
    }
    *type = row->type;
    *pol = p;
    *norm = nrm;
    *field = row->field0 + p;
    *soft = row->soft;
    return true;
  }
  return false;
}

static bool parse_EX(vh_ctx *c, char *l)
{
  char name[VH_TAG] = "", tag[VH_TAG] = "", wfname[VH_TAG] = "";
  int b[6];
  double size = 1.0, delay = 0.0, resist = 0.0;
  if (sscanf(l, "%d %d %d %d %d %d %31s %31s %31s", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], name, tag,
             wfname) < 9)
    return false;
  if (find_source(c, name) >= 0) return false;
  int type, pol, norm, field, soft;
  if (!decode_source_tag(tag, &type, &pol, &norm, &field, &soft)) return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  if (type == ST_THEVENIN_VOLTAGE || type == ST_NORTON_CURRENT) {
    sscanf(l, "%d %d %d %d %d %d %31s %31s %31s %lf %lf %lf", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5],
           name, tag, wfname, &resist, &size, &delay);
    /* Lumped sources must be one edge (src/source.c:430-434). */
    if (vh_bbox_type(b) != BB_LINE) return false;
    char rname[VH_TAG];
    snprintf(rname, VH_TAG, "__VR_RS_%d__", c->num_srcs + 1);
    vh_add_medium(c, rname, MT_SIMPLE, 1.0, 0.0, 1.0, 0, NULL, NULL, "");
  } else {
    sscanf(l, "%d %d %d %d %d %d %31s %31s %31s %lf %lf", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], name,
           tag, wfname, &size, &delay);
  }
  int wf = vh_find_waveform(c, wfname);
  if (wf < 0) return false;
  vh_source *s = VH_PUSH(c, srcs, num_srcs, cap_srcs, vh_source);
  snprintf(s->name, VH_TAG, "%s", name);
  s->type = type;
  s->pol = pol;
  s->norm = norm;
  s->field = field;
  s->soft = soft;
  memcpy(s->mbbox, b, sizeof b);
  s->wf = wf;
  s->size = size;
  s->delay = delay;
  s->resistance = resist;
  return true;
}

static bool parse_PW(vh_ctx *c, char *l)
{
  char name[VH_TAG] = "", wfname[VH_TAG] = "", mask[VH_TAG] = "111111";
  int b[6];
  double theta = 0, phi = 0, eta = 0, size = 1.0, delay = 0.0;
  int act[6] = { 1, 1, 1, 1, 1, 1 };
  int ns = sscanf(l, "%d %d %d %d %d %d %31s %31s %lf %lf %lf %31s %lf %lf", &b[0], &b[1], &b[2], &b[3],
                  &b[4], &b[5], name, wfname, &theta, &phi, &eta, mask, &size, &delay);
  if (ns < 11) return false;
  if (find_planewave(c, name) >= 0) return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  int wf = vh_find_waveform(c, wfname);
  if (wf < 0) return false;
  if (theta < 0.0 || theta > 180.0) return false;
  if (phi < 0.0 || phi > 360.0) return false;
  if (eta < 0 || eta >= 360.0) return false;
  if (ns >= 12) {
    if (strlen(mask) != 6) return false;
    for (int f = 0; f < 6; f++) {
      if (mask[f] == '0') act[f] = 0;
      else if (mask[f] == '1') act[f] = 1;
      else return false;
    }
  }
  if (ns >= 13 && size < 0.0) return false;
  vh_planewave *p = VH_PUSH(c, pws, num_pws, cap_pws, vh_planewave);
  snprintf(p->name, VH_TAG, "%s", name);
  memcpy(p->mbbox, b, sizeof b);
  p->wf = wf;
  memcpy(p->active, act, sizeof act);
  p->theta = theta;
  p->phi = phi;
  p->eta = eta;
  p->size = size;
  p->delay = delay;
  return true;
}

static bool parse_OP(vh_ctx *c, char *l)
{
  static const char *types[3] = { "TDOM_ASCII", "FDOM_ASCII", "TDOM_BINARY" };
  char name[VH_TAG] = "", type_str[VH_TAG] = "", wfname[VH_TAG] = "";
  int b[6] = { 0 }, step[3] = { 1, 1, 1 };
  if (sscanf(l, "%d %d %d %d %d %d %31s %31s", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], name,
             type_str) < 8)
    return false;
  if (obs_lookup(c, obs_hash_tls, name, -1) >= 0) return false;
  if (!vh_bbox_is_normal(b) || !vh_bbox_is_within(b, c->mbox)) return false;
  int kind = -1;
  for (int t = 0; t < 3; t++)
    if (strncmp(type_str, types[t], VH_TAG) == 0) kind = t;
  if (kind < 0) return false;
  if (kind != OBS_TD_BINARY) {
    if (vh_bbox_type(b) != BB_POINT) return false;
    sscanf(l, "%d %d %d %d %d %d %31s %31s %31s", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], name,
           type_str, wfname);
  } else {
    sscanf(l, "%d %d %d %d %d %d %31s %31s %d %d %d", &b[0], &b[1], &b[2], &b[3], &b[4], &b[5], name,
           type_str, &step[0], &step[1], &step[2]);
    if (step[0] < 0 || step[1] < 0 || step[2] < 0) return false;
  }
  int wf = 0;
  if (wfname[0]) {
    wf = vh_find_waveform(c, wfname);
    if (wf < 0) return false;
  }
  vh_observer *o = VH_PUSH(c, obs, num_obs, cap_obs, vh_observer);
  snprintf(o->name, VH_TAG, "%s", name);
  o->kind = kind;
  memcpy(o->mbbox, b, sizeof b);
  memcpy(o->step, step, sizeof step);
  o->wf = wf;
  obs_lookup(c, obs_hash_tls, name, (int)(o - c->obs));
  return true;
}

static bool parse_FF(vh_ctx *c, char *l)
{
  (void)l;
  vh_log(c, 0, "*** Warning: Parsing of boundary far-fields not implemeneted yet - ignoring FF card.\n");
  return true;
}

static bool parse_NT(vh_ctx *c, char *l)
{
  unsigned long n = 0;
  if (sscanf(l, "%lu", &n) != 1) return false;
  c->num_steps = n;
  return true;
}

static bool parse_OT(vh_ctx *c, char *l)
{
  if (sscanf(l, "%lu %lu", &c->ot_start, &c->ot_stop) != 2) return false;
  if (c->ot_stop < c->ot_start) return false;
  c->has_ot = 1;
  return true;
}

static bool parse_OF(vh_ctx *c, char *l)
{
  double a = -1.0, b = -1.0;
  unsigned long n = 0;
  if (sscanf(l, "%lf %lf %lu", &a, &b, &n) != 3) return false;
  if (a < 0) return false;
  if (b < a) return false;
  if (n < 1UL) return false;
  c->of_start = a;
  c->of_stop = b;
  c->of_num = n;
  c->has_of = 1;
  return true;
}

static bool parse_CN(vh_ctx *c, char *l)
{
  double cn;
  if (sscanf(l, "%lf", &cn) != 1) return false;
  if (cn >= 1.0) return false;
  c->courant = cn;
  return true;
}

static bool parse_MS(vh_ctx *c, char *l)
{
  double d[3];
  int ns = sscanf(l, "%lf %lf %lf", &d[0], &d[1], &d[2]);
  if (ns == 1) d[1] = d[2] = d[0];
  else if (ns != 3) return false;
  for (int a = 0; a < 3; a++)
    if (d[a] <= 0.0) return false;
  for (int a = 0; a < 3; a++) {
    c->lines[a] = malloc(sizeof(double) * c->num_lines[a]);
    for (int i = 0; i < c->num_lines[a]; i++) c->lines[a][i] = i * d[a];
  }
  return true;
}

static bool read_lines(vh_ctx *c, FILE *fp, int axis)
{
  c->lines[axis] = malloc(sizeof(double) * c->num_lines[axis]);
  for (int k = 0; k < c->num_lines[axis]; k++) {
    double v;
    if (fscanf(fp, "%lf", &v) != 1) return false;
    c->lines[axis][k] = v;
  }
  return true;
}

/* ---- card dispatcher (src/mesh.c:48-191, 269-405) ---- */

enum { CT_VM, CT_CE, CT_DM, CT_BR, CT_BE, CT_GS, CT_MT, CT_BT, CT_WT, CT_MB, CT_TB, CT_TW, CT_WF, CT_EX,
       CT_PW, CT_OP, CT_FF, CT_GE, CT_NT, CT_OT, CT_OF, CT_CN, CT_MS, CT_XL, CT_YL, CT_ZL, CT_EN, CT_NUM };

static const char *CARD[CT_NUM] = { "VM", "CE", "DM", "BR", "BE", "GS", "MT", "BT", "WT", "MB",
                                    "TB", "TW", "WF", "EX", "PW", "OP", "FF", "GE", "NT", "OT",
                                    "OF", "CN", "MS", "XL", "YL", "ZL", "EN" };
static const int SECTION_OF[CT_NUM] = { 0, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2,
                                        2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3 };
static const bool REQUIRED[CT_NUM] = { 1, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0,
                                       0, 0, 0, 1, 1, 0, 0, 0, 0, 0, 0, 0, 1 };
static const bool SINGLETON[CT_NUM] = { 1, 0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0,
                                        0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1 };
static const bool END_OF_SECTION[CT_NUM] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0,
                                             0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 1 };

static void trim(char *s)
{
  char *p = s;
  while (*p && isspace((unsigned char)*p)) p++;
  if (p != s) memmove(s, p, strlen(p) + 1);
  size_t n = strlen(s);
  while (n > 0 && isspace((unsigned char)s[n - 1])) s[--n] = '\0';
}

int vh_read_mesh(vh_ctx *c, const char *path)
{
  FILE *fp = fopen(path, "r");
  if (!fp) return vh_fail(c, "Cannot open input mesh file %s", path);
  {
    const char *slash = strrchr(path, '/');
    if (slash) snprintf(c->mesh_dir, sizeof c->mesh_dir, "%.*s", (int)(slash - path), path);
  }
  name_hash hash = { 0 };
  obs_hash_tls = &hash;

  bool found[CT_NUM] = { 0 };
  bool found_source = false, found_output = false;
  char raw[1024], line[1024];
  unsigned long line_no = 0;
  int section = 0;
  int rc = 0;

  vh_log(c, 0, "\n  Reading input mesh file %s...\n\n", path);
  while (!feof(fp)) {
    if (!fgets(raw, sizeof raw - 1, fp)) {
      if (feof(fp)) break;
      rc = vh_fail(c, "Error reading %s after line number %lu", path, line_no);
      goto done;
    }
    line_no++;
    snprintf(line, sizeof line, "%s", raw);
    char *hash_pos = strchr(line, '#');
    if (hash_pos) *hash_pos = '\0';
    trim(line);
    if (!line[0]) continue;
    int card = -1;
    if (strlen(line) >= 2)
      for (int t = 0; t < CT_NUM; t++)
        if (strncmp(line, CARD[t], 2) == 0) { card = t; break; }
    if (card < 0) { rc = vh_fail(c, "Invalid card on line %lu: %s", line_no, raw); goto done; }
    if (SECTION_OF[card] != section) {
      rc = vh_fail(c, "Card type %s on line %lu is invalid in mesh section %d", CARD[card], line_no, section);
      goto done;
    }
    if (found[card] && SINGLETON[card]) {
      rc = vh_fail(c, "Card type %s on line %lu is has already been found", CARD[card], line_no);
      goto done;
    }
    found[card] = true;
    char *arg = line + 2;
    bool ok = true;
    switch (card) {
      case CT_VM: ok = parse_VM(c, arg); break;
      case CT_CE: ok = parse_CE(c, arg); break;
      case CT_DM: ok = parse_DM(c, arg); break;
      case CT_BR: ok = parse_BR(c, arg); break;
      case CT_BE: ok = parse_BE(c, arg); break;
      case CT_MT: ok = parse_MT(c, arg); break;
      case CT_BT: ok = parse_BT(c, arg); break;
      case CT_WT: ok = parse_WT(c, arg); break;
      case CT_MB: ok = parse_MB(c, arg); break;
      case CT_TB: ok = parse_TB(c, arg); break;
      case CT_TW: ok = parse_TW(c, arg); break;
      case CT_WF: ok = parse_WF(c, arg); break;
      case CT_EX: ok = parse_EX(c, arg); break;
      case CT_PW: ok = parse_PW(c, arg); break;
      case CT_OP: ok = parse_OP(c, arg); break;
      case CT_FF: ok = parse_FF(c, arg); break;
      case CT_NT: ok = parse_NT(c, arg); break;
      case CT_OT: ok = parse_OT(c, arg); break;
      case CT_OF: ok = parse_OF(c, arg); break;
      case CT_CN: ok = parse_CN(c, arg); break;
      case CT_MS: ok = parse_MS(c, arg); break;
      case CT_XL: ok = read_lines(c, fp, XDIR); break;
      case CT_YL: ok = read_lines(c, fp, YDIR); break;
      case CT_ZL: ok = read_lines(c, fp, ZDIR); break;
      default: break;
    }
    if (!ok) { rc = vh_fail(c, "Failed to parse %s card on line %lu: %s", CARD[card], line_no, raw); goto done; }
    switch (card) {
      case CT_EX: case CT_PW: found_source = true; break;
      case CT_OP: case CT_FF: found_output = true; break;
      case CT_GE:
        if (!found_source) { rc = vh_fail(c, "No source found in section 2 of mesh file!"); goto done; }
        if (!found_output) vh_log(c, 0, "*** Warning: No outputs found in section 2 of mesh file!\n");
        break;
      case CT_MS: found[CT_MS] = found[CT_XL] = found[CT_YL] = found[CT_ZL] = true; break;
      case CT_XL: found[CT_MS] = found[CT_XL] = true; break;
      case CT_YL: found[CT_MS] = found[CT_YL] = true; break;
      case CT_ZL: found[CT_MS] = found[CT_ZL] = true; break;
      case CT_EN:
        if (!found[CT_MS] || !(found[CT_XL] && found[CT_YL] && found[CT_ZL])) {
          rc = vh_fail(c, "No mesh lines found in section 3 of mesh file!");
          goto done;
        }
        break;
      default: break;
    }
    if (END_OF_SECTION[card]) {
      for (int t = 0; t < CT_NUM; t++)
        if (SECTION_OF[t] == section && REQUIRED[t] && !found[t]) {
          rc = vh_fail(c, "Required card %s not found in Section %d", CARD[t], section);
          goto done;
        }
      vh_log(c, 0, "  Processed Section %d\n\n", section);
      section++;
    }
  }
  /* A file that stops before EN never closes section 3. */
  if (section < 4) rc = vh_fail(c, "Mesh file %s ends in section %d", path, section);
done:
  fclose(fp);
  free(hash.keys);
  free(hash.vals);
  obs_hash_tls = NULL;
  return rc;
}
