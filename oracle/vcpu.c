/*
 * vcpu.c -- ORACLE (test infrastructure only).
 *
 * A plain-C, single-threaded restatement of the Vulture time loop
 * (propagate(), src/simulation.c:136-231, and every update routine it calls)
 * acting on a vgpu_problem.  It is the checker for the CUDA engine: only
 * tests/, the smoke check and bench.py's CPU-baseline leg load it.  The
 * product never calls it.
 *
 * It is compiled twice: with VCPU_REAL=double (prefix vcpu64_) it is the
 * reference's real=double solver; with VCPU_REAL=float (prefix vcpu32_) it is
 * the FP32-storage mode of the engine (float fields/coefficients, double DFT,
 * Debye recursion, SIBC filter and analytic incident-field phase).
 *
 * Pinned against the reference itself: tests run the reference binaries
 * built by oracle/build_ref.sh on the same meshes and require identical
 * FP64 observer values (tests/test_oracle_reference.py).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vgpu.h"

#ifndef VCPU_REAL
#define VCPU_REAL double
#define VCPU_PREFIX vcpu64_
#endif

typedef VCPU_REAL real;

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define API(name) CAT(VCPU_PREFIX, name)

enum { EX = 0, EY, EZ, HX, HY, HZ };
enum { XLO = 0, XHI, YLO, YHI, ZLO, ZHI };

typedef struct {
  int32_t lim[6];
  int32_t nx, ny, nz;
} box_t;

typedef struct {
  const vgpu_problem *p;
  int32_t n0, n1, n2;
  int64_t vol;
  real *F[6];
  real *coef[9];
  real *ide[3], *idh[3];
  real *ad[3], *bd[3], *ah[3], *bh[3], *ibd[3], *ibh[3];
  real zeta[6];
  /* UPML auxiliary fields per region: PP, P for E and B for H. */
  real *PP[6][3], *P[6][3], *B[6][3];
  /* Debye: J[block][comp] complex per cell per pole, lastE per cell. */
  double complex **J[3];
  real **lastE[3];
  /* SIBC: filter state per face (16 filters, poles), previous input, Etan. */
  double complex **sz;
  double **sold;
  real **etan;
  /* Plane-wave auxiliary grids. */
  real **Eyi, **Hzi, **PPyi, **Pyi, **Bzi;
  /* Outputs. */
  double *td;
  float *bin;
  double *dre, *dim;
  uint64_t step;
} vcpu;

static inline int64_t IX(const vcpu *s, int i, int j, int k) { return ((int64_t)i * s->n1 + j) * s->n2 + k; }

static real *to_real(const double *src, int64_t n)
{
  real *d = malloc(sizeof(real) * (n ? n : 1));
  for (int64_t q = 0; q < n; q++) d[q] = (real)src[q];
  return d;
}

static int64_t lim_count(const int32_t l[6])
{
  if (l[1] < l[0] || l[3] < l[2] || l[5] < l[4]) return 0;
  return (int64_t)(l[1] - l[0] + 1) * (l[3] - l[2] + 1) * (l[5] - l[4] + 1);
}

void *API(create)(const vgpu_problem *p)
{
  vcpu *s = calloc(1, sizeof(vcpu));
  s->p = p;
  s->n0 = p->n[0];
  s->n1 = p->n[1];
  s->n2 = p->n[2];
  s->vol = (int64_t)s->n0 * s->n1 * s->n2;
  for (int f = 0; f < 6; f++) s->F[f] = calloc(s->vol, sizeof(real));
  for (int q = 0; q < 9; q++) s->coef[q] = to_real(p->coef[q], s->vol);
  for (int a = 0; a < 3; a++) {
    s->ide[a] = to_real(p->ide[a], p->n[a]);
    s->idh[a] = to_real(p->idh[a], p->n[a]);
    if (p->pml_ad[a]) {
      s->ad[a] = to_real(p->pml_ad[a], p->n[a]);
      s->bd[a] = to_real(p->pml_bd[a], p->n[a]);
      s->ah[a] = to_real(p->pml_ah[a], p->n[a]);
      s->bh[a] = to_real(p->pml_bh[a], p->n[a]);
      s->ibd[a] = to_real(p->pml_ibd[a], p->n[a]);
      s->ibh[a] = to_real(p->pml_ibh[a], p->n[a]);
    }
  }
  for (int f = 0; f < 6; f++) s->zeta[f] = (real)p->mur_zeta[f];
  for (int r = 0; r < 6; r++) {
    if (!p->pml_present[r]) continue;
    for (int c = 0; c < 3; c++) {
      s->PP[r][c] = calloc(lim_count(p->pml_flim[r][c]) + 1, sizeof(real));
      s->P[r][c] = calloc(lim_count(p->pml_flim[r][c]) + 1, sizeof(real));
      s->B[r][c] = calloc(lim_count(p->pml_flim[r][3 + c]) + 1, sizeof(real));
    }
  }
  for (int c = 0; c < 3; c++) {
    s->J[c] = calloc(p->num_debye + 1, sizeof(double complex *));
    s->lastE[c] = calloc(p->num_debye + 1, sizeof(real *));
    for (int b = 0; b < p->num_debye; b++) {
      int64_t cells = lim_count(p->debye[b].flim[c]);
      s->J[c][b] = calloc(cells * p->debye[b].num_poles + 1, sizeof(double complex));
      s->lastE[c][b] = calloc(cells + 1, sizeof(real));
    }
  }
  s->sz = calloc(p->num_sibc + 1, sizeof(double complex *));
  s->sold = calloc(p->num_sibc + 1, sizeof(double *));
  s->etan = calloc(p->num_sibc + 1, sizeof(real *));
  for (int q = 0; q < p->num_sibc; q++) {
    const vgpu_sibc_surface *sf = &p->sibc[q];
    const vgpu_sibc_model *m = &p->sibc_models[sf->model];
    int64_t faces = (int64_t)(sf->gbbox[1] - sf->gbbox[0]) * (sf->gbbox[3] - sf->gbbox[2]) * (sf->gbbox[5] - sf->gbbox[4]);
    int poles = 0;
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) poles += m->num_poles[a][b];
    s->sz[q] = calloc(faces * poles + 1, sizeof(double complex));
    s->sold[q] = calloc(faces * 16 + 1, sizeof(double));
    s->etan[q] = calloc(faces * 4 + 1, sizeof(real));
  }
  int npw = p->num_planewaves;
  s->Eyi = calloc(npw + 1, sizeof(real *));
  s->Hzi = calloc(npw + 1, sizeof(real *));
  s->PPyi = calloc(npw + 1, sizeof(real *));
  s->Pyi = calloc(npw + 1, sizeof(real *));
  s->Bzi = calloc(npw + 1, sizeof(real *));
  for (int q = 0; q < npw; q++) {
    const vgpu_planewave *pw = &p->planewaves[q];
    if (!pw->use_aux_grid) continue;
    s->Eyi[q] = calloc(pw->aux_nx + 2, sizeof(real));
    s->Hzi[q] = calloc(pw->aux_nx + 2, sizeof(real));
    s->PPyi[q] = calloc(pw->aux_npml + 1, sizeof(real));
    s->Pyi[q] = calloc(pw->aux_npml + 1, sizeof(real));
    s->Bzi[q] = calloc(pw->aux_npml + 1, sizeof(real));
  }
  uint64_t nout = 0;
  if (p->num_steps > 0 && p->out_start < p->num_steps)
    nout = (p->out_stop < p->num_steps - 1 ? p->out_stop : p->num_steps - 1) - p->out_start + 1;
  s->td = calloc((size_t)(nout + 1) * (p->num_td + 1) * 6, sizeof(double));
  s->bin = calloc((size_t)(nout + 1) * (p->num_bin + 1) * 6, sizeof(float));
  s->dre = calloc((size_t)(p->num_fd + 1) * 6 * (p->num_freq + 1), sizeof(double));
  s->dim = calloc((size_t)(p->num_fd + 1) * 6 * (p->num_freq + 1), sizeof(double));
  return s;
}

void API(destroy)(void *h)
{
  vcpu *s = h;
  if (!s) return;
  const vgpu_problem *p = s->p;
  for (int f = 0; f < 6; f++) free(s->F[f]);
  for (int q = 0; q < 9; q++) free(s->coef[q]);
  for (int a = 0; a < 3; a++) {
    free(s->ide[a]); free(s->idh[a]);
    free(s->ad[a]); free(s->bd[a]); free(s->ah[a]); free(s->bh[a]); free(s->ibd[a]); free(s->ibh[a]);
  }
  for (int r = 0; r < 6; r++)
    for (int c = 0; c < 3; c++) { free(s->PP[r][c]); free(s->P[r][c]); free(s->B[r][c]); }
  for (int c = 0; c < 3; c++) {
    for (int b = 0; b < p->num_debye; b++) { free(s->J[c][b]); free(s->lastE[c][b]); }
    free(s->J[c]); free(s->lastE[c]);
  }
  for (int q = 0; q < p->num_sibc; q++) { free(s->sz[q]); free(s->sold[q]); free(s->etan[q]); }
  free(s->sz); free(s->sold); free(s->etan);
  for (int q = 0; q < p->num_planewaves; q++) { free(s->Eyi[q]); free(s->Hzi[q]); free(s->PPyi[q]); free(s->Pyi[q]); free(s->Bzi[q]); }
  free(s->Eyi); free(s->Hzi); free(s->PPyi); free(s->Pyi); free(s->Bzi);
  free(s->td); free(s->bin); free(s->dre); free(s->dim);
  free(s);
}

/* ---- observers (src/observer.c:622-650, 760-798, 857-899) ---- */

static void update_observers(vcpu *s, uint64_t n)
{
  const vgpu_problem *p = s->p;
  if (n < p->out_start || n > p->out_stop) return;
  double t = n * p->dt;
  uint64_t row = n - p->out_start;
  for (int q = 0; q < p->num_td; q++) {
    const int32_t *pt = &p->td_points[3 * q];
    int64_t x = IX(s, pt[0], pt[1], pt[2]);
    for (int c = 0; c < 6; c++) s->td[(row * p->num_td + q) * 6 + c] = (double)s->F[c][x];
  }
  /* Binary observers store float (src/observer.c:1168-1185). */
  for (int64_t q = 0; q < p->num_bin; q++) {
    const int32_t *pt = &p->bin_points[3 * q];
    int64_t x = IX(s, pt[0], pt[1], pt[2]);
    for (int c = 0; c < 6; c++) s->bin[(row * p->num_bin + q) * 6 + c] = (float)s->F[c][x];
  }
  for (int q = 0; q < p->num_fd; q++) {
    const int32_t *pt = &p->fd_points[3 * q];
    int64_t x = IX(s, pt[0], pt[1], pt[2]);
    for (int c = 0; c < 6; c++) {
      double v = (double)s->F[c][x];
      double *re = &s->dre[((size_t)q * 6 + c) * p->num_freq], *im = &s->dim[((size_t)q * 6 + c) * p->num_freq];
      for (int f = 0; f < p->num_freq; f++) {
        double wt = p->omega[f] * t;
        re[f] += v * cos(wt);
        im[f] -= v * sin(wt);
      }
    }
  }
}

/* ---- bulk Yee updates (src/grid.c:709-888) ---- */

static void update_grid_E(vcpu *s)
{
  const int32_t(*L)[6] = s->p->gfilim;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  real *idhx = s->idh[0], *idhy = s->idh[1], *idhz = s->idh[2];
  for (int i = L[EX][XLO]; i <= L[EX][XHI]; i++)
    for (int j = L[EX][YLO]; j <= L[EX][YHI]; j++)
      for (int k = L[EX][ZLO]; k <= L[EX][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Ex[x] = s->coef[0][x] * Ex[x] + s->coef[3][x] * (idhy[j] * (Hz[x] - Hz[IX(s, i, j - 1, k)]) +
                                                          idhz[k] * (Hy[x - 1] - Hy[x]));
      }
  for (int i = L[EY][XLO]; i <= L[EY][XHI]; i++)
    for (int j = L[EY][YLO]; j <= L[EY][YHI]; j++)
      for (int k = L[EY][ZLO]; k <= L[EY][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Ey[x] = s->coef[1][x] * Ey[x] + s->coef[4][x] * (idhz[k] * (Hx[x] - Hx[x - 1]) +
                                                          idhx[i] * (Hz[IX(s, i - 1, j, k)] - Hz[x]));
      }
  for (int i = L[EZ][XLO]; i <= L[EZ][XHI]; i++)
    for (int j = L[EZ][YLO]; j <= L[EZ][YHI]; j++)
      for (int k = L[EZ][ZLO]; k <= L[EZ][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Ez[x] = s->coef[2][x] * Ez[x] + s->coef[5][x] * (idhx[i] * (Hy[x] - Hy[IX(s, i - 1, j, k)]) +
                                                          idhy[j] * (Hx[IX(s, i, j - 1, k)] - Hx[x]));
      }
}

static void update_grid_H(vcpu *s)
{
  const int32_t(*L)[6] = s->p->gfilim;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  real *idex = s->ide[0], *idey = s->ide[1], *idez = s->ide[2];
  for (int i = L[HX][XLO]; i <= L[HX][XHI]; i++)
    for (int j = L[HX][YLO]; j <= L[HX][YHI]; j++)
      for (int k = L[HX][ZLO]; k <= L[HX][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Hx[x] = Hx[x] + s->coef[6][x] * (idez[k] * (Ey[x + 1] - Ey[x]) + idey[j] * (Ez[x] - Ez[IX(s, i, j + 1, k)]));
      }
  for (int i = L[HY][XLO]; i <= L[HY][XHI]; i++)
    for (int j = L[HY][YLO]; j <= L[HY][YHI]; j++)
      for (int k = L[HY][ZLO]; k <= L[HY][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Hy[x] = Hy[x] + s->coef[7][x] * (idex[i] * (Ez[IX(s, i + 1, j, k)] - Ez[x]) + idez[k] * (Ex[x] - Ex[x + 1]));
      }
  for (int i = L[HZ][XLO]; i <= L[HZ][XHI]; i++)
    for (int j = L[HZ][YLO]; j <= L[HZ][YHI]; j++)
      for (int k = L[HZ][ZLO]; k <= L[HZ][ZHI]; k++) {
        int64_t x = IX(s, i, j, k);
        Hz[x] = Hz[x] + s->coef[8][x] * (idey[j] * (Ex[IX(s, i, j + 1, k)] - Ex[x]) + idex[i] * (Ey[x] - Ey[IX(s, i + 1, j, k)]));
      }
}

/* ---- UPML (src/pml.c:859-1176) ---- */

static void update_pml_E(vcpu *s)
{
  const vgpu_problem *p = s->p;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  real *idhx = s->idh[0], *idhy = s->idh[1], *idhz = s->idh[2];
  for (int r = 0; r < 6; r++) {
    if (!p->pml_present[r]) continue;
    const int32_t *l;
    l = p->pml_flim[r][EX];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *PP = s->PP[r][0], *P = s->P[r][0];
          real oPP = PP[a];
          PP[a] = s->coef[0][x] * PP[a] + s->coef[3][x] * (idhy[j] * (Hz[x] - Hz[IX(s, i, j - 1, k)]) +
                                                            idhz[k] * (Hy[x - 1] - Hy[x]));
          real oP = P[a];
          P[a] = s->ad[1][j] * P[a] + s->bd[1][j] * (PP[a] - oPP);
          Ex[x] = s->ad[2][k] * Ex[x] + s->bd[2][k] * s->ibh[0][i] * (P[a] - s->ah[0][i] * oP);
        }
    l = p->pml_flim[r][EY];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *PP = s->PP[r][1], *P = s->P[r][1];
          real oPP = PP[a];
          PP[a] = s->coef[1][x] * PP[a] + s->coef[4][x] * (idhz[k] * (Hx[x] - Hx[x - 1]) +
                                                            idhx[i] * (Hz[IX(s, i - 1, j, k)] - Hz[x]));
          real oP = P[a];
          P[a] = s->ad[2][k] * P[a] + s->bd[2][k] * (PP[a] - oPP);
          Ey[x] = s->ad[0][i] * Ey[x] + s->bd[0][i] * s->ibh[1][j] * (P[a] - s->ah[1][j] * oP);
        }
    l = p->pml_flim[r][EZ];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *PP = s->PP[r][2], *P = s->P[r][2];
          real oPP = PP[a];
          PP[a] = s->coef[2][x] * PP[a] + s->coef[5][x] * (idhx[i] * (Hy[x] - Hy[IX(s, i - 1, j, k)]) +
                                                            idhy[j] * (Hx[IX(s, i, j - 1, k)] - Hx[x]));
          real oP = P[a];
          P[a] = s->ad[0][i] * P[a] + s->bd[0][i] * (PP[a] - oPP);
          Ez[x] = s->ad[1][j] * Ez[x] + s->bd[1][j] * s->ibh[2][k] * (P[a] - s->ah[2][k] * oP);
        }
  }
}

static void update_pml_H(vcpu *s)
{
  const vgpu_problem *p = s->p;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  real *idex = s->ide[0], *idey = s->ide[1], *idez = s->ide[2];
  for (int r = 0; r < 6; r++) {
    if (!p->pml_present[r]) continue;
    const int32_t *l;
    l = p->pml_flim[r][HX];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *B = s->B[r][0];
          real oB = B[a];
          B[a] = s->ah[1][j] * B[a] + s->coef[6][x] * s->bh[1][j] *
                                          (idez[k] * (Ey[x + 1] - Ey[x]) + idey[j] * (Ez[x] - Ez[IX(s, i, j + 1, k)]));
          Hx[x] = s->ah[2][k] * Hx[x] + s->bh[2][k] * s->ibd[0][i] * (B[a] - s->ad[0][i] * oB);
        }
    l = p->pml_flim[r][HY];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *B = s->B[r][1];
          real oB = B[a];
          B[a] = s->ah[2][k] * B[a] + s->coef[7][x] * s->bh[2][k] *
                                          (idex[i] * (Ez[IX(s, i + 1, j, k)] - Ez[x]) + idez[k] * (Ex[x] - Ex[x + 1]));
          Hy[x] = s->ah[0][i] * Hy[x] + s->bh[0][i] * s->ibd[1][j] * (B[a] - s->ad[1][j] * oB);
        }
    l = p->pml_flim[r][HZ];
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          int64_t a = ((int64_t)(i - l[0]) * (l[3] - l[2] + 1) + (j - l[2])) * (l[5] - l[4] + 1) + (k - l[4]);
          real *B = s->B[r][2];
          real oB = B[a];
          B[a] = s->ah[0][i] * B[a] + s->coef[8][x] * s->bh[0][i] *
                                          (idey[j] * (Ex[IX(s, i, j + 1, k)] - Ex[x]) + idex[i] * (Ey[x] - Ey[IX(s, i + 1, j, k)]));
          Hz[x] = s->ah[1][j] * Hz[x] + s->bh[1][j] * s->ibd[2][k] * (B[a] - s->ad[2][k] * oB);
        }
  }
}

/* ---- Mur (src/mur.c:135-555) ---- */

/* Bulk-formula E value at (i,j,k) from the current (pre-update) fields. */
static real bulk_E(vcpu *s, int c, int i, int j, int k)
{
  real *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  int64_t x = IX(s, i, j, k);
  switch (c) {
    case EX:
      return s->coef[0][x] * s->F[EX][x] + s->coef[3][x] * (s->idh[1][j] * (Hz[x] - Hz[IX(s, i, j - 1, k)]) +
                                                              s->idh[2][k] * (Hy[x - 1] - Hy[x]));
    case EY:
      return s->coef[1][x] * s->F[EY][x] + s->coef[4][x] * (s->idh[2][k] * (Hx[x] - Hx[x - 1]) +
                                                              s->idh[0][i] * (Hz[IX(s, i - 1, j, k)] - Hz[x]));
    default:
      return s->coef[2][x] * s->F[EZ][x] + s->coef[5][x] * (s->idh[0][i] * (Hy[x] - Hy[IX(s, i - 1, j, k)]) +
                                                              s->idh[1][j] * (Hx[IX(s, i, j - 1, k)] - Hx[x]));
  }
}

static void update_mur_E(vcpu *s)
{
  const vgpu_problem *p = s->p;
  for (int f = 0; f < 6; f++) {
    if (!p->mur_present[f]) continue;
    int a = f / 2, dir = (f % 2 == 0) ? +1 : -1;
    /* Tangential components of face f, in the reference's order. */
    int comps[2];
    if (a == 0) { comps[0] = EY; comps[1] = EZ; }
    else if (a == 1) { comps[0] = EX; comps[1] = EZ; }
    else { comps[0] = EY; comps[1] = EX; }
    for (int cc = 0; cc < 2; cc++) {
      int c = comps[cc];
      const int32_t *l = p->mur_flim[f][c];
      for (int i = l[0]; i <= l[1]; i++)
        for (int j = l[2]; j <= l[3]; j++)
          for (int k = l[4]; k <= l[5]; k++) {
            int g[3] = { i, j, k };
            g[a] += dir;
            real tmp = bulk_E(s, c, g[0], g[1], g[2]);
            int64_t x = IX(s, i, j, k), xn = IX(s, g[0], g[1], g[2]);
            s->F[c][x] = s->F[c][xn] + s->zeta[f] * (tmp - s->F[c][x]);
          }
    }
  }
}

static void update_mur_H(vcpu *s)
{
  const vgpu_problem *p = s->p;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  real *idex = s->ide[0], *idey = s->ide[1], *idez = s->ide[2];
  for (int f = 0; f < 6; f++) {
    if (!p->mur_present[f]) continue;
    int a = f / 2;
    int c = HX + a;
    const int32_t *l = p->mur_flim[f][c];
    /* The normal H sits on the face plane: the low limit for LO faces and,
     * for XHI, the XLO entry of the face box (src/mur.c:433). */
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int g[3] = { i, j, k };
          if (a == 0 && g[0] != l[0]) continue;
          if (a == 1 && g[1] != (f == YLO ? l[2] : l[3])) continue;
          if (a == 2 && g[2] != (f == ZLO ? l[4] : l[5])) continue;
          int64_t x = IX(s, i, j, k);
          if (a == 0)
            Hx[x] = Hx[x] + s->coef[6][x] * (idez[k] * (Ey[x + 1] - Ey[x]) + idey[j] * (Ez[x] - Ez[IX(s, i, j + 1, k)]));
          else if (a == 1)
            Hy[x] = Hy[x] + s->coef[7][x] * (idex[i] * (Ez[IX(s, i + 1, j, k)] - Ez[x]) + idez[k] * (Ex[x] - Ex[x + 1]));
          else
            Hz[x] = Hz[x] + s->coef[8][x] * (idey[j] * (Ex[IX(s, i, j + 1, k)] - Ex[x]) + idex[i] * (Ey[x] - Ey[IX(s, i + 1, j, k)]));
        }
  }
}

/* ---- Debye (src/debye.c:243-307) ---- */

static void update_debye_E(vcpu *s)
{
  const vgpu_problem *p = s->p;
  for (int b = 0; b < p->num_debye; b++) {
    const vgpu_debye *d = &p->debye[b];
    int np = d->num_poles;
    for (int c = 0; c < 3; c++) {
      const int32_t *l = d->flim[c];
      real *E = s->F[c];
      int64_t cell = 0;
      for (int i = l[0]; i <= l[1]; i++)
        for (int j = l[2]; j <= l[3]; j++)
          for (int k = l[4]; k <= l[5]; k++, cell++) {
            int64_t x = IX(s, i, j, k);
            double complex *J = &s->J[c][b][cell * np];
            double complex Jsum = 0.0 + I * 0.0;
            for (int q = 0; q < np; q++) {
              double complex da = d->dalpha[2 * q] + I * d->dalpha[2 * q + 1];
              Jsum = Jsum + (1 + da) * J[q];
            }
            E[x] = E[x] - s->coef[3 + c][x] * creal(Jsum);
            for (int q = 0; q < np; q++) {
              double complex da = d->dalpha[2 * q] + I * d->dalpha[2 * q + 1];
              double complex db = d->dbeta[2 * q] + I * d->dbeta[2 * q + 1];
              J[q] = da * J[q] + db * (E[x] - s->lastE[c][b][cell]);
            }
            s->lastE[c][b][cell] = E[x];
          }
    }
  }
}

/* ---- SIBC (src/sibc.c:444-776, src/filter.c:309-327) ---- */

static void update_sibc_E(vcpu *s)
{
  const vgpu_problem *p = s->p;
  real *Ex = s->F[EX], *Ey = s->F[EY], *Ez = s->F[EZ], *Hx = s->F[HX], *Hy = s->F[HY], *Hz = s->F[HZ];
  for (int q = 0; q < p->num_sibc; q++) {
    const vgpu_sibc_surface *sf = &p->sibc[q];
    const vgpu_sibc_model *m = &p->sibc_models[sf->model];
    const int32_t *g = sf->gbbox;
    int nj = g[3] - g[2], nk = g[5] - g[4];
    int poles = 0;
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) poles += m->num_poles[a][b];
    for (int i = g[0], ii = 0; i < g[1]; i++, ii++)
      for (int j = g[2], jj = 0; j < g[3]; j++, jj++)
        for (int k = g[4], kk = 0; k < g[5]; k++, kk++) {
          int64_t f = ((int64_t)ii * nj + jj) * nk + kk;
          const uint8_t *A = &sf->adjA[4 * f], *B = &sf->adjB[4 * f];
          real Ht[4], Hin[4], Eout[4];
          switch (sf->normal) {
            case 0:
              Ey[IX(s, i, j, k)] = 0.0; Ey[IX(s, i, j, k + 1)] = 0.0;
              Ez[IX(s, i, j, k)] = 0.0; Ez[IX(s, i, j + 1, k)] = 0.0;
              Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hy[IX(s, i - 1, j, k)] + Hy[IX(s, i - 1, j + 1, k)]);
              Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hy[IX(s, i, j, k)] + Hy[IX(s, i, j + 1, k)]);
              Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hz[IX(s, i - 1, j, k)] + Hz[IX(s, i - 1, j, k + 1)]);
              Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hz[IX(s, i, j, k)] + Hz[IX(s, i, j, k + 1)]);
              break;
            case 1:
              Ez[IX(s, i, j, k)] = 0.0; Ez[IX(s, i + 1, j, k)] = 0.0;
              Ex[IX(s, i, j, k)] = 0.0; Ex[IX(s, i, j, k + 1)] = 0.0;
              Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hz[IX(s, i, j - 1, k)] + Hz[IX(s, i, j - 1, k + 1)]);
              Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hz[IX(s, i, j, k)] + Hz[IX(s, i, j, k + 1)]);
              Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hx[IX(s, i, j - 1, k)] + Hx[IX(s, i + 1, j - 1, k)]);
              Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hx[IX(s, i, j, k)] + Hx[IX(s, i + 1, j, k)]);
              break;
            default:
              Ex[IX(s, i, j, k)] = 0.0; Ex[IX(s, i, j + 1, k)] = 0.0;
              Ey[IX(s, i, j, k)] = 0.0; Ey[IX(s, i + 1, j, k)] = 0.0;
              Ht[0] = 0.5 * (1 + A[0] + A[1]) * (Hx[IX(s, i, j, k - 1)] + Hx[IX(s, i + 1, j, k - 1)]);
              Ht[1] = 0.5 * (1 + B[0] + B[1]) * (Hx[IX(s, i, j, k)] + Hx[IX(s, i + 1, j, k)]);
              Ht[2] = 0.5 * (1 + A[2] + A[3]) * (Hy[IX(s, i, j, k - 1)] + Hy[IX(s, i, j + 1, k - 1)]);
              Ht[3] = 0.5 * (1 + B[2] + B[3]) * (Hy[IX(s, i, j, k)] + Hy[IX(s, i, j + 1, k)]);
              break;
          }
          for (int a = 0; a < 4; a++) {
            Hin[a] = 0.0;
            for (int b = 0; b < 4; b++) Hin[a] = Hin[a] + (real)sf->A[a][b] * Ht[b];
          }
          for (int a = 0; a < 4; a++) {
            Eout[a] = 0.0;
            for (int b = 0; b < 4; b++) {
              double x = Hin[b];
              double y = m->asymp[a][b] * x;
              int off = m->pole_offset[a][b];
              double complex *z = &s->sz[q][f * poles + (off - m->pole_offset[0][0])];
              double *old = &s->sold[q][f * 16 + a * 4 + b];
              for (int r = 0; r < m->num_poles[a][b]; r++) {
                double complex q0 = m->q0[2 * (off + r)] + I * m->q0[2 * (off + r) + 1];
                double complex q1 = m->q1[2 * (off + r)] + I * m->q1[2 * (off + r) + 1];
                double complex q2 = m->q2[2 * (off + r)] + I * m->q2[2 * (off + r) + 1];
                z[r] = q0 * z[r] + q1 * *old + q2 * x;
                y = y + z[r];
              }
              *old = x;
              Eout[a] = Eout[a] + y;
            }
          }
          real *et = &s->etan[q][f * 4];
          for (int a = 0; a < 4; a++) {
            et[a] = 0.0;
            for (int b = 0; b < 4; b++) et[a] = et[a] + (real)sf->B[a][b] * Eout[b];
          }
        }
  }
}

static void update_sibc_H(vcpu *s)
{
  const vgpu_problem *p = s->p;
  for (int64_t h = 0; h < p->num_sibc_hops; h++) {
    const vgpu_sibc_hop *o = &p->sibc_hops[h];
    real *H = s->F[o->comp];
    if (o->kind == 0) { H[o->index] = 0.0; continue; }
    real e1 = s->etan[o->s1][4 * (int64_t)o->f1 + o->slot1];
    real c = (real)o->c, d1 = (real)o->d1;
    if (o->kind == 1) {
      H[o->index] = H[o->index] + c * (d1 * e1);
    } else {
      real e2 = s->etan[o->s2][4 * (int64_t)o->f2 + o->slot2];
      real d2 = (real)o->d2, n1 = (real)o->n1, n2 = (real)o->n2;
      H[o->index] = H[o->index] + c * (n1 * (d1 * e1) + n2 * (d2 * e2));
    }
  }
}

/* ---- sources (src/source.c:602-753) ---- */

static void update_sources(vcpu *s, int efield, uint64_t n)
{
  const vgpu_problem *p = s->p;
  for (int q = 0; q < p->num_sources; q++) {
    const vgpu_source *src = &p->sources[q];
    if ((src->field <= EZ) != efield) continue;
    real v = (real)src->values[n];
    real soft = (real)src->soft;
    real *F = s->F[src->field];
    real *cf = src->field <= EZ ? s->coef[3 + src->field] : s->coef[6 + src->field - HX];
    const int32_t *l = src->flim;
    for (int i = l[0]; i <= l[1]; i++)
      for (int j = l[2]; j <= l[3]; j++)
        for (int k = l[4]; k <= l[5]; k++) {
          int64_t x = IX(s, i, j, k);
          if (src->kind == VGPU_SRC_FIELD) F[x] = soft * F[x] + v;
          else F[x] = soft * F[x] - cf[x] * v;
        }
  }
}

/* ---- waveforms and plane waves (src/waveform.c:412-638, src/planewave.c:557-1419) ---- */

static double spline(const vgpu_waveform *w, double t)
{
  const double(*tab)[3] = (const double(*)[3])w->table;
  unsigned long n = (unsigned long)w->table_size, klo = 0, khi = n - 1, k;
  while (khi - klo > 1UL) {
    k = (khi + klo) >> 1;
    if (tab[k][0] > t) khi = k;
    else klo = k;
  }
  double h = tab[khi][0] - tab[klo][0];
  double a = (tab[khi][0] - t) / h, b = (t - tab[klo][0]) / h;
  return a * tab[klo][1] + b * tab[khi][1] + ((a * a * a - a) * tab[klo][2] + (b * b * b - b) * tab[khi][2]) * (h * h) / 6.0;
}

static double waveform_value(const vgpu_waveform *w, double t, double delay)
{
  const double pi = 4.0 * atan(1.0);
  double x = t - delay - w->delay, W = w->width, f = w->frequency, env;
  switch (w->type) {
    case VGPU_WF_GAUSSIAN_PULSE:
    case VGPU_WF_NARROW_GAUSSIAN_PULSE: return w->size * exp(-0.5 * (pow(x / W, 2.0)));
    case VGPU_WF_DIFF_GAUSSIAN_PULSE: return w->size * (-x / W * exp(-0.5 * (pow(x / W, 2.0))));
    case VGPU_WF_RICKER_WAVELET: return w->size * ((1.0 - pow(x / W, 2)) * exp(-0.5 * (pow(x / W, 2.0))));
    case VGPU_WF_MOD_GAUSSIAN_PULSE: return w->size * (exp(-0.5 * (pow(x / W, 2.0))) * sin(2.0 * pi * f * x));
    case VGPU_WF_COMPACT_PULSE:
    case VGPU_WF_MOD_COMPACT_PULSE:
      if (x <= 0.0) env = 0.0;
      else if (x < 2.0 * W)
        env = 1.0 / 32.0 * (10.0 - 15.0 * cos(pi / W * x) + 6.0 * cos(2.0 * pi / W * x) - cos(3.0 * pi / W * x));
      else env = 0.0;
      return w->type == VGPU_WF_COMPACT_PULSE ? w->size * env : w->size * (env * sin(2.0 * pi * f * x));
    case VGPU_WF_DIFF_COMPACT_PULSE:
      if (x <= 0.0 || x >= 2.0 * W) return w->size * 0.0;
      return w->size * (1.0 / 32.0 * (15.0 * sin(pi / W * x) - 12.0 * sin(2.0 * pi / W * x) + 3.0 * sin(3.0 * pi / W * x)));
    case VGPU_WF_RAMPED_SINUSOID:
      if (x <= 0.0) env = 0.0;
      else if (x < 1.0 * W)
        env = 1.0 / 32.0 * (10.0 - 15.0 * cos(pi / W * x) + 6.0 * cos(2.0 * pi / W * x) - cos(3.0 * pi / W * x));
      else env = 1.0;
      return w->size * (env * sin(2.0 * pi * f * x));
    case VGPU_WF_EXTERNAL: {
      const double(*tab)[3] = (const double(*)[3])w->table;
      if (x < tab[0][0] || x > tab[w->table_size - 1][0]) return w->size * 0.0;
      return w->size * spline(w, x);
    }
    default: return 0.0;
  }
}

/* Incident field of component c at (i,j,k) (src/planewave.c:557-573, 1378-1418). */
static real incident(vcpu *s, int q, int c, int i, int j, int k, double time)
{
  const vgpu_problem *p = s->p;
  const vgpu_planewave *pw = &p->planewaves[q];
  if (!pw->use_aux_grid) {
    int g[3] = { i, j, k };
    double r[3];
    for (int a = 0; a < 3; a++) {
      int half = c <= EZ ? (c == a) : (c - HX != a);
      r[a] = half ? p->pos_half[a][g[a]] : p->pos_node[a][g[a]];
    }
    double d = pw->kinc[0] * (r[0] - pw->r0[0]) + pw->kinc[1] * (r[1] - pw->r0[1]) + pw->kinc[2] * (r[2] - pw->r0[2]);
    return (real)(pw->finc[c] * waveform_value(&p->waveforms[pw->waveform], time - d / pw->phase_velocity, pw->delay));
  }
  real rc[3] = { (real)i, (real)j, (real)k };
  if (c <= EZ) rc[c] = (real)(c == 0 ? i : c == 1 ? j : k) + (real)0.5;
  else for (int a = 0; a < 3; a++) if (a != c - HX) rc[a] = rc[a] + (real)0.5;
  real k0 = (real)pw->kinc[0], k1 = (real)pw->kinc[1], k2 = (real)pw->kinc[2];
  real d = k0 * (rc[0] - (real)pw->ijk0[0]) + k1 * (rc[1] - (real)pw->ijk0[1]) + k2 * (rc[2] - (real)pw->ijk0[2]);
  real value;
  if (c <= EZ) {
    int id = (int)floor(d);
    real dp = d - id;
    value = (1 - dp) * s->Eyi[q][2 + id] + dp * s->Eyi[q][2 + id + 1];
  } else {
    /* d + 0.5 is a double expression in the reference (src/planewave.c:1406-1407). */
    int id = (int)floor((double)d + 0.5);
    real dp = (real)((double)d + 0.5 - id);
    const double mu0 = 4.0 * (4.0 * atan(1.0)) * 1e-7;
    const double eta0 = sqrt(mu0 / (1.0 / (mu0 * 299792458.0 * 299792458.0)));
    value = (real)eta0 * ((1 - dp) * s->Hzi[q][2 - 1 + id] + dp * s->Hzi[q][2 + id]);
  }
  return (real)pw->finc[c] * value;
}

static void aux_grid_E(vcpu *s, int q, uint64_t n)
{
  const vgpu_planewave *pw = &s->p->planewaves[q];
  real *E = s->Eyi[q], *H = s->Hzi[q];
  real beta = (real)pw->aux_beta;
  for (int i = 1; i < pw->aux_xb; i++) E[i] = E[i] + beta * (H[i - 1] - H[i]);
  for (int i = pw->aux_xb; i < pw->aux_nx; i++) {
    int L = i - pw->aux_xb;
    real oPP = s->PPyi[q][L];
    s->PPyi[q][L] = s->PPyi[q][L] + beta * (H[i - 1] - H[i]);
    real oP = s->Pyi[q][L];
    s->Pyi[q][L] = s->Pyi[q][L] + (s->PPyi[q][L] - oPP);
    E[i] = (real)pw->aux_adx[L] * E[i] + (real)pw->aux_bdx[L] * (s->Pyi[q][L] - oP);
  }
  E[0] = (real)pw->aux_source[n];
}

static void aux_grid_H(vcpu *s, int q)
{
  const vgpu_planewave *pw = &s->p->planewaves[q];
  real *E = s->Eyi[q], *H = s->Hzi[q];
  real gamma = (real)pw->aux_gamma;
  for (int i = 0; i < pw->aux_xb; i++) H[i] = H[i] + gamma * (E[i] - E[i + 1]);
  for (int i = pw->aux_xb; i < pw->aux_nx; i++) {
    int L = i - pw->aux_xb;
    real oB = s->Bzi[q][L];
    s->Bzi[q][L] = (real)pw->aux_ahx[L] * s->Bzi[q][L] + gamma * (real)pw->aux_bhx[L] * (-E[i + 1] + E[i]);
    H[i] = H[i] + (s->Bzi[q][L] - oB);
  }
}

/* One face correction: F = alpha*F + sign*beta*(id*inc) for E (alpha
 * applied again as the reference does), F = F + sign*gamma*(id*inc) for H. */
static void tfsf_face(vcpu *s, int q, int face, int c, int inc_c, int sign, double time)
{
  const vgpu_planewave *pw = &s->p->planewaves[q];
  const int32_t *l = pw->flim[face][c];
  int a = face / 2;
  int lo = face % 2 == 0;
  /* E corrections read H one cell outside on LO faces; H corrections read E
   * one cell inside on LO faces. */
  int shift = c <= EZ ? (lo ? -1 : 0) : (lo ? +1 : 0);
  real *F = s->F[c];
  real *idv = c <= EZ ? s->idh[a] : s->ide[a];
  for (int i = l[0]; i <= l[1]; i++)
    for (int j = l[2]; j <= l[3]; j++)
      for (int k = l[4]; k <= l[5]; k++) {
        int g[3] = { i, j, k };
        g[a] += shift;
        real inc = incident(s, q, inc_c, g[0], g[1], g[2], time);
        int64_t x = IX(s, i, j, k);
        int gi = a == 0 ? i : a == 1 ? j : k;
        if (c <= EZ) {
          real al = s->coef[c][x], be = s->coef[3 + c][x];
          if (sign > 0) F[x] = al * F[x] + be * (idv[gi] * inc);
          else F[x] = al * F[x] - be * (idv[gi] * inc);
        } else {
          real ga = s->coef[6 + c - HX][x];
          if (sign > 0) F[x] = F[x] + ga * (idv[gi] * inc);
          else F[x] = F[x] - ga * (idv[gi] * inc);
        }
      }
}

static void update_planewaves_E(vcpu *s, uint64_t n)
{
  const vgpu_problem *p = s->p;
  double t = n * p->dt;
  for (int q = 0; q < p->num_planewaves; q++) {
    const vgpu_planewave *pw = &p->planewaves[q];
    if (pw->use_aux_grid) aux_grid_E(s, q, n);
    if (pw->active[YLO]) { tfsf_face(s, q, YLO, EX, HZ, -1, t); tfsf_face(s, q, YLO, EZ, HX, +1, t); }
    if (pw->active[YHI]) { tfsf_face(s, q, YHI, EX, HZ, +1, t); tfsf_face(s, q, YHI, EZ, HX, -1, t); }
    if (pw->active[ZLO]) { tfsf_face(s, q, ZLO, EX, HY, +1, t); tfsf_face(s, q, ZLO, EY, HX, -1, t); }
    if (pw->active[ZHI]) { tfsf_face(s, q, ZHI, EX, HY, -1, t); tfsf_face(s, q, ZHI, EY, HX, +1, t); }
    if (pw->active[XLO]) { tfsf_face(s, q, XLO, EY, HZ, +1, t); tfsf_face(s, q, XLO, EZ, HY, -1, t); }
    if (pw->active[XHI]) { tfsf_face(s, q, XHI, EY, HZ, -1, t); tfsf_face(s, q, XHI, EZ, HY, +1, t); }
  }
}

static void update_planewaves_H(vcpu *s, uint64_t n)
{
  const vgpu_problem *p = s->p;
  double t = (n + 0.5) * p->dt;
  for (int q = 0; q < p->num_planewaves; q++) {
    const vgpu_planewave *pw = &p->planewaves[q];
    if (pw->use_aux_grid) aux_grid_H(s, q);
    if (pw->active[YLO]) { tfsf_face(s, q, YLO, HZ, EX, -1, t); tfsf_face(s, q, YLO, HX, EZ, +1, t); }
    if (pw->active[YHI]) { tfsf_face(s, q, YHI, HZ, EX, +1, t); tfsf_face(s, q, YHI, HX, EZ, -1, t); }
    if (pw->active[ZLO]) { tfsf_face(s, q, ZLO, HY, EX, +1, t); tfsf_face(s, q, ZLO, HX, EY, -1, t); }
    if (pw->active[ZHI]) { tfsf_face(s, q, ZHI, HY, EX, -1, t); tfsf_face(s, q, ZHI, HX, EY, +1, t); }
    if (pw->active[XLO]) { tfsf_face(s, q, XLO, HZ, EY, +1, t); tfsf_face(s, q, XLO, HY, EZ, -1, t); }
    if (pw->active[XHI]) { tfsf_face(s, q, XHI, HZ, EY, -1, t); tfsf_face(s, q, XHI, HY, EZ, +1, t); }
  }
}

/* ---- ghost layer (src/surface.c:569-812) ---- */

static void ghost_copy(vcpu *s, int c, int face, int mode, int fields_are_e)
{
  const vgpu_problem *p = s->p;
  int a = face / 2, lo = face % 2 == 0;
  int go_lo = p->gobox[2 * a], go_hi = p->gobox[2 * a + 1];
  int dst = lo ? go_lo - 1 : go_hi;
  int src;
  real sgn = 1;
  if (mode == VGPU_GHOST_PERIODIC) src = lo ? go_hi - 1 : go_lo;
  else src = lo ? go_lo : go_hi - 1;
  if (fields_are_e) {
    if (mode == VGPU_GHOST_PMC) sgn = -1;
  } else {
    if (mode == VGPU_GHOST_PMC) sgn = -1;
  }
  int b = (a + 1) % 3, cc = (a + 2) % 3;
  for (int u = p->gobox[2 * b] - 1; u <= p->gobox[2 * b + 1]; u++)
    for (int v = p->gobox[2 * cc] - 1; v <= p->gobox[2 * cc + 1]; v++) {
      int gd[3], gs[3];
      gd[a] = dst; gd[b] = u; gd[cc] = v;
      gs[a] = src; gs[b] = u; gs[cc] = v;
      real val = s->F[c][IX(s, gs[0], gs[1], gs[2])];
      s->F[c][IX(s, gd[0], gd[1], gd[2])] = sgn < 0 ? -val : val;
    }
}

static void update_ghost_E(vcpu *s)
{
  for (int f = 0; f < 6; f++) {
    int mode = s->p->ghost[f];
    if (mode == VGPU_GHOST_NONE) continue;
    ghost_copy(s, f / 2, f, mode, 1);
  }
}

static void update_ghost_H(vcpu *s)
{
  static const int comps[3][2] = { { HY, HZ }, { HZ, HX }, { HX, HY } };
  for (int f = 0; f < 6; f++) {
    int mode = s->p->ghost[f];
    if (mode == VGPU_GHOST_NONE) continue;
    int a = f / 2;
    /* The reference loops over the face once, copying both components per
     * point; the two components are independent, so copying one component
     * after the other gives the same values. */
    ghost_copy(s, comps[a][0], f, mode, 0);
    ghost_copy(s, comps[a][1], f, mode, 0);
  }
}

/* ---- the time loop (src/simulation.c:156-222) ---- */

int API(run)(void *h, uint64_t nsteps)
{
  vcpu *s = h;
  for (uint64_t it = 0; it < nsteps; it++) {
    uint64_t n = s->step;
    update_observers(s, n);
    update_pml_E(s);
    update_mur_E(s);
    update_grid_E(s);
    update_debye_E(s);
    update_sibc_E(s);
    update_sources(s, 1, n);
    update_planewaves_E(s, n);
    update_ghost_E(s);
    update_pml_H(s);
    update_mur_H(s);
    update_grid_H(s);
    update_sibc_H(s);
    update_sources(s, 0, n);
    update_planewaves_H(s, n);
    update_ghost_H(s);
    s->step++;
  }
  return 0;
}

int API(read_td)(void *h, double *out, uint64_t steps)
{
  vcpu *s = h;
  memcpy(out, s->td, sizeof(double) * steps * s->p->num_td * 6);
  return 0;
}

int API(read_bin)(void *h, float *out, uint64_t steps)
{
  vcpu *s = h;
  memcpy(out, s->bin, sizeof(float) * steps * s->p->num_bin * 6);
  return 0;
}

int API(read_dft)(void *h, double *re, double *im)
{
  vcpu *s = h;
  size_t n = (size_t)s->p->num_fd * 6 * s->p->num_freq;
  memcpy(re, s->dre, n * sizeof(double));
  memcpy(im, s->dim, n * sizeof(double));
  return 0;
}

int API(read_field)(void *h, int32_t c, double *out)
{
  vcpu *s = h;
  for (int64_t q = 0; q < s->vol; q++) out[q] = (double)s->F[c][q];
  return 0;
}

int API(write_field)(void *h, int32_t c, const double *in)
{
  vcpu *s = h;
  for (int64_t q = 0; q < s->vol; q++) s->F[c][q] = (real)in[q];
  return 0;
}
