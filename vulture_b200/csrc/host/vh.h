/*
 * vh.h -- internal header of the host side of vulture_b200.
 *
 * The host side reads a Vulture .mesh file and performs the solver's set-up
 * (everything the reference does in src/vulture.c:95-148 before calling
 * propagate()), producing a vgpu_problem for the device engine, and writes the
 * observer files afterwards.  Unlike the reference, which keeps its model in
 * file-scope globals, all state lives in one vh_ctx so that many problems can
 * be set up in one process (batching and serving).
 *
 * All set-up arithmetic is done in double with the reference's operation
 * order, so the arrays equal those of the reference built with real=double
 * (the FP64 oracle) bit for bit.
 */
#ifndef VH_H
#define VH_H

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <complex.h>

#include "vgpu.h"
#include "vhost.h"

#define VH_TAG 32
#define VH_PATH 1024

enum { XLO = 0, XHI, YLO, YHI, ZLO, ZHI };
enum { XDIR = 0, YDIR, ZDIR, CA_UNDEF };
enum { EX = 0, EY, EZ, HX, HY, HZ };
enum { BB_INVALID = 0, BB_POINT, BB_LINE, BB_SURFACE, BB_VOLUME };

/* Medium types (src/medium.h:50-59). */
enum { MT_FREE_SPACE = 0, MT_PEC = 1, MT_SIMPLE = 2, MT_DEBYE = 3, MT_UNDEFINED = 4 };
/* Boundary types (src/boundary.h:50-62). */
enum { BT_PMC = 0, BT_PML = 1, BT_PEC = 2, BT_FREE_SPACE = 3, BT_PERIODIC = 4, BT_MUR = 5,
       BT_SIBC = 6, BT_UNDEFINED = 7 };
/* Wire types (src/wire.h). */
enum { TW_PEC = 0, TW_FREE_SPACE = 1 };
/* Source types (src/source.h:40-56). */
enum { ST_EFIELD = 0, ST_HFIELD, ST_ELEC_CURR_DENSITY, ST_MAGN_CURR_DENSITY,
       ST_ELEC_SURF_CURR_DENSITY, ST_MAGN_SURF_CURR_DENSITY, ST_ELEC_CURRENT,
       ST_MAGN_CURRENT, ST_ELEC_CURRENT_MOMENT, ST_MAGN_CURRENT_MOMENT, ST_VOLTAGE,
       ST_THEVENIN_VOLTAGE, ST_NORTON_CURRENT };
/* Grid types (src/grid.h:43-52). */
enum { GT_CUBIC = 0, GT_UNIFORM = 1, GT_NONUNIFORM = 2 };
/* Observer kinds (src/observer.c:177-281). */
enum { OBS_TD_ASCII = 0, OBS_FD_ASCII = 1, OBS_TD_BINARY = 2 };

typedef struct {
  char name[VH_TAG];
  int type;
  double eps_r, sigma, mu_r;
  int num_poles;
  double complex *res, *pole;
  double alpha, beta, gamma;
  double complex *dalpha, *dbeta;
} vh_medium;

typedef struct {
  char name[VH_TAG];
  int type;
  int num_layers, order;
  double n_eff, ref_coeff, kmax;
  char file[VH_PATH];
  double S_TM[2][2], S_TE[2][2];
  int sibc_model;             /* index into ctx->sibc_models, -1 if none */
} vh_boundary;

typedef struct { char name[VH_TAG]; int type; } vh_wire;

typedef struct {
  int mbbox[6];
  int medium;
  unsigned char mask;
} vh_block;

typedef struct {
  int mbbox[6];
  int boundary;
  int orient;
  double angle;
  int gbbox[6];
} vh_surface;

typedef struct {
  int mbbox[6];
  int wire;
  int gbbox[6];
} vh_line;

typedef struct {
  char name[VH_TAG];
  int type;
  double size, delay, width, frequency;
  char file[VH_PATH];
  int table_size;
  double *table;              /* [table_size][3] */
  unsigned long last_idx;     /* spline search cache */
} vh_waveform;

typedef struct {
  char name[VH_TAG];
  int type, pol, norm, field, soft;
  int mbbox[6];
  int wf;
  double size, delay, resistance;
  int gbbox[6];
  int flim[6][6];
} vh_source;

typedef struct {
  char name[VH_TAG];
  int mbbox[6];
  int wf;
  int active[6];
  double theta, phi, eta, size, delay;
  int gbbox[6];
  int flim[6][6][6];
  double kinc[3], finc[6], ijk0[3], r0[3];
  double phase_velocity;
  /* auxiliary grid */
  int nx, xb;
  double beta_eyi, gamma_hzi;
  double adx[10], bdx[10], ahx[10], bhx[10];
} vh_planewave;

typedef struct {
  char name[VH_TAG];
  int kind;                   /* OBS_* */
  int mbbox[6];
  int step[3];
  int wf;                     /* reference waveform for FD normalisation */
  int gbbox[6];
  int slot;                   /* index into td_points / fd_points */
} vh_observer;

typedef struct {
  int normal, orient, model;
  double cosa, sina;
  int gbbox[6];
  int nfaces[3];
  uint8_t *adjA, *adjB;       /* [faces][4] */
} vh_sibc;

typedef struct {
  int m, n;
  int num_poles[4][4];
  double asymp[4][4];
  double complex *poles[4][4], *residues[4][4];
} vh_pole_residue;

struct vhost {
  char err[1024];
  FILE *log;
  int verbose;

  /* Parser state (src/mesh.c). */
  int version[3];
  char comment[VH_PATH];
  int mesh_cells[3];
  int num_lines[3];
  int mbox[6];
  double *lines[3];
  double courant;
  unsigned long num_steps;
  int has_ot, has_of;
  unsigned long ot_start, ot_stop;
  double of_start, of_stop;
  unsigned long of_num;
  char mesh_dir[VH_PATH];

  /* Model lists in definition order. */
  vh_medium *media; int num_media, cap_media;
  vh_boundary *bnds; int num_bnds, cap_bnds;
  vh_wire *wires; int num_wires, cap_wires;
  vh_block *blocks; int num_blocks, cap_blocks;
  vh_surface *surfs; int num_surfs, cap_surfs;
  vh_line *lns; int num_lns, cap_lns;
  vh_waveform *wfs; int num_wfs, cap_wfs;
  vh_source *srcs; int num_srcs, cap_srcs;
  vh_planewave *pws; int num_pws, cap_pws;
  vh_observer *obs; int num_obs, cap_obs;

  /* External surfaces: boundary index per face. */
  int ext_bnd[6];

  /* Grid (src/grid.c). */
  int n[3];
  int gibox[6], gobox[6], ggbox[6];
  int gfilim[6][6], gfolim[6][6];
  double *de[3], *dh[3], *ide[3], *idh[3];
  double dmin[3], dmax[3], duni[3];
  int grid_type;
  double dt;
  double *coef[9];
  /* Medium tags of the six components (vgpu_problem.coef_tag): the painted
   * (alpha, beta, gamma) triples in first-painted order; NULL once more than
   * 255 distinct triples were painted. */
  uint8_t *ctag[6];
  int num_ctags;
  double ctag_coef[255][3];
  int tags_off;               /* vhost_use_tags(h, 0) */
  double pi, c0, mu0, eps0, eta0;

  /* PML (src/pml.c). */
  int pbox[6][6];
  int fplim[6][6][6];
  double *pml_ad[3], *pml_bd[3], *pml_gd[3], *pml_kd[3];
  double *pml_ah[3], *pml_bh[3], *pml_gh[3], *pml_kh[3];
  double *pml_ibd[3], *pml_ibh[3];

  /* Mur (src/mur.c). */
  int murbox[6][6];
  int fmlim[6][6][6];
  double zeta[6];

  /* Debye blocks. */
  int num_debye;
  int (*debye_flim)[3][6];
  int *debye_medium;

  /* SIBC. */
  vh_pole_residue *sibc_pr; int num_sibc_models;
  vh_sibc *sibcs; int num_sibcs;
  vgpu_sibc_model *sibc_rc;
  double *sibc_q;             /* packed q0,q1,q2 for all models */
  vgpu_sibc_hop *hops; int64_t num_hops, cap_hops;

  /* Observers. */
  unsigned long out_start, out_stop;
  double start_freq, stop_freq, step_freq;
  unsigned long num_freq;
  double *omega;
  int num_td, num_fd;
  int32_t *td_points, *fd_points;
  int64_t num_bin;            /* nodes of all TDOM_BINARY observers */
  int32_t *bin_points;
  FILE *impulse;              /* impulse.dat while binary rows stream in */
  int impulse_failed;

  /* Assembled problem (owned). */
  vgpu_problem prob;
  vgpu_source *p_srcs;
  double *p_src_vals;
  vgpu_debye *p_debye;
  double *p_debye_coef;
  vgpu_planewave *p_pws;
  double *p_pw_vals;
  vgpu_waveform *p_wfs;
  vgpu_sibc_surface *p_sibc;
  double *pos_node[3], *pos_half[3];
  int prob_ready;
};

typedef struct vhost vh_ctx;

/* Errors: record a message and return -1. */
int vh_fail(vh_ctx *c, const char *fmt, ...);
void vh_log(vh_ctx *c, int verbose_only, const char *fmt, ...);

/* Grid volumes of n doubles (the coefficient arrays): bytes mapped, and
 * their release. */
size_t vh_volume_bytes(size_t n);
void vh_free_volume(double *p, size_t n);
void vh_free_tags(vh_ctx *c);

/* Runs fn(ctx, lo, hi) over [begin, end) split into contiguous ranges on
 * up to 16 threads; one call on the calling thread when work (the points
 * the whole range touches) is small.  The ranges must touch disjoint
 * memory. */
void vh_parallel_for(int begin, int end, int64_t work, void (*fn)(void *ctx, int lo, int hi), void *ctx);

/* Indexing helpers. */
static inline int64_t vh_idx(const vh_ctx *c, int i, int j, int k)
{
  return ((int64_t)i * c->n[1] + j) * c->n[2] + k;
}

/* bounding_box.c equivalents (src/bounding_box.c:36-357). */
int vh_bbox_type(const int b[6]);
int vh_bbox_direction(const int b[6]);
bool vh_bbox_is_normal(const int b[6]);
bool vh_bbox_is_within(const int b1[6], const int b2[6]);
void vh_bbox_offset(int out[6], const int b[6], const int off[6]);
void vh_face_of_bbox(int out[6], const int b[6], int face);
bool vh_field_in_boundary(int field, int face);
bool vh_field_parallel_to_boundary(int field, int face);
void vh_set_field_limits(const int bbox[6], int flim[6][6], const bool incl[6]);
unsigned char vh_face_mask_from_string(const char *s);
void vh_mask_to_bool(bool incl[6], unsigned char mask);
extern const unsigned char VH_FACE_MASKS[6];
#define VH_FACE_MASK_ALL 0x3F
#define VH_FACE_MASK_ERROR 0xFF
extern const char *VH_FACE_STR[6];
extern const char *VH_FIELD_STR[6];

/* Parser (src/mesh.c and the parse* functions of each module). */
int vh_read_mesh(vh_ctx *c, const char *path);
int vh_find_medium(const vh_ctx *c, const char *name);
int vh_find_boundary(const vh_ctx *c, const char *name);
int vh_find_waveform(const vh_ctx *c, const char *name);
int vh_add_medium(vh_ctx *c, const char *name, int type, double eps_r, double sigma, double mu_r,
                  int num_poles, const double *res, const double *poles, const char *file);
int vh_add_boundary(vh_ctx *c, const char *name, int type, int num_layers, int order, double n_eff,
                    double ref_coeff, double kmax, const char *file, double S_TM[2][2], double S_TE[2][2]);

/* Set-up stages, in the reference's order (src/vulture.c:95-148). */
int vh_init_grid(vh_ctx *c);
int vh_init_boundaries(vh_ctx *c);
int vh_init_media(vh_ctx *c);
void vh_init_media_arrays(vh_ctx *c);
int vh_init_blocks(vh_ctx *c);
int vh_init_lines(vh_ctx *c);
int vh_init_internal_surfaces(vh_ctx *c);
int vh_init_external_surfaces(vh_ctx *c);
int vh_init_waveforms(vh_ctx *c);
int vh_init_sources(vh_ctx *c);
int vh_init_planewaves(vh_ctx *c);
int vh_init_observers(vh_ctx *c);
int vh_build_problem(vh_ctx *c, int precision);

/* Grid and media helpers. */
void vh_set_medium_on_grid(vh_ctx *c, const int gbbox[6], int medium, unsigned char mask);
void vh_calc_coeff(vh_ctx *c, vh_medium *m);
double vh_numerical_phase_velocity(vh_ctx *c, double theta, double phi);
void vh_field_physical_location(const vh_ctx *c, double r[3], int field, int i, int j, int k);
int vh_outer_type(const vh_ctx *c, int face);
bool vh_is_pmc_edge(const vh_ctx *c, int dir, int index);

/* Waveforms. */
double vh_waveform_value(vh_ctx *c, double t, int wf, double delay);
void vh_pml_defaults(int *num_layers, int *order, double *n_eff, double *ref_coeff, double *kmax);

/* SIBC. */
int vh_init_sibc_boundary(vh_ctx *c, vh_boundary *b);
int vh_init_sibc_surfaces(vh_ctx *c);

/* Outputs. */
int vh_write_observers(vh_ctx *c, const double *td, uint64_t td_steps, const double *re,
                       const double *im, int full_precision);

#endif
