/*
 * vh_sibc.c -- surface-impedance boundary (SIBC) set-up.
 *
 * Restates initSibcBoundary (src/sibc.c:120-196), the two-port S->Z
 * conversion and passivity test (src/sibc.c:790-827), the pole-residue ->
 * recursive-convolution conversion (src/filter.c:347-387), the pole-residue
 * matrix reader (src/filter.c:142-188) and initSibcSurfaces
 * (src/sibc.c:199-388).  It also turns the magnetic-field correction of
 * updateSibcSurfacesHfield (src/sibc.c:616-776) into an ordered list of
 * per-target operations (vgpu_sibc_hop) so the device can apply it with one
 * thread per corrected H value and the reference's order of additions.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vh.h"

/* src/sibc.c:790-803 */
static void tport_s2z(const vh_ctx *c, double Z[2][2], double S[2][2])
{
  double dS = (1.0 - S[0][0]) * (1.0 - S[1][1]) - S[0][1] * S[1][0];
  Z[0][0] = ((1.0 + S[0][0]) * (1.0 - S[1][1]) + S[0][1] * S[1][0]) / dS * c->eta0;
  Z[0][1] = 2.0 * S[0][1] * c->eta0 / dS;
  Z[1][0] = 2.0 * S[1][0] * c->eta0 / dS;
  Z[1][1] = ((1.0 - S[0][0]) * (1.0 + S[1][1]) + S[0][1] * S[1][0]) / dS * c->eta0;
}

/* src/sibc.c:806-827 */
static bool is_passive(double S[2][2])
{
  bool e00 = (1 - (S[0][0] * S[0][0] + S[1][0] * S[1][0])) >= 0.0;
  bool e01 = (S[0][0] * S[0][1] - S[1][0] * S[1][1]) >= 0.0;
  bool e10 = (S[0][1] * S[0][0] - S[1][1] * S[1][0]) >= 0.0;
  bool e11 = (1 - (S[0][1] * S[0][1] + S[1][1] * S[1][1])) >= 0.0;
  return e00 && e01 && e10 && e11;
}

static void pr_set(vh_pole_residue *pr, int p, int q, int np, double asymp, const double complex *poles,
                   const double complex *res)
{
  pr->num_poles[p][q] = np;
  pr->asymp[p][q] = asymp;
  pr->poles[p][q] = calloc(np ? np : 1, sizeof(double complex));
  pr->residues[p][q] = calloc(np ? np : 1, sizeof(double complex));
  for (int k = 0; k < np; k++) {
    if (poles) pr->poles[p][q][k] = poles[k];
    if (res) pr->residues[p][q][k] = res[k];
  }
}

int vh_init_sibc_boundary(vh_ctx *c, vh_boundary *b)
{
  vh_pole_residue pr;
  memset(&pr, 0, sizeof pr);
  pr.m = pr.n = 4;
  if (!b->file[0]) {
    double Ztm[2][2], Zte[2][2];
    if (!is_passive(b->S_TM) || !is_passive(b->S_TE))
      return vh_fail(c, "Passivity violation for SIBC boundary %s", b->name);
    tport_s2z(c, Ztm, b->S_TM);
    tport_s2z(c, Zte, b->S_TE);
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        pr_set(&pr, i, j, 0, Ztm[i][j], NULL, NULL);
        pr_set(&pr, i + 2, j, 0, 0.0, NULL, NULL);
        pr_set(&pr, i, j + 2, 0, 0.0, NULL, NULL);
        pr_set(&pr, i + 2, j + 2, 0, Zte[i][j], NULL, NULL);
      }
  } else {
    FILE *fp = fopen(b->file, "r");
    if (!fp) return vh_fail(c, "cannot open pole-residue matrix file %s.", b->file);
    int m, n;
    if (fscanf(fp, "%d %d", &m, &n) != 2) { fclose(fp); return vh_fail(c, "error reading extents from %s.", b->file); }
    if (!((m == 4 && n == 4) || (m == 2 && n == 2))) {
      fclose(fp);
      return vh_fail(c, "Pole-residue model must be 2x2 or 4x4!");
    }
    vh_pole_residue rd;
    memset(&rd, 0, sizeof rd);
    for (int row = 0; row < m; row++)
      for (int col = 0; col < n; col++) {
        int np = 0;
        double asymp = 0.0;
        if (fscanf(fp, "%d", &np) != 1 || fscanf(fp, "%lf", &asymp) != 1 || np < 0) {
          fclose(fp);
          return vh_fail(c, "error reading pole-residue matrix file %s.", b->file);
        }
        double complex *po = calloc(np ? np : 1, sizeof(double complex));
        double complex *re = calloc(np ? np : 1, sizeof(double complex));
        for (int k = 0; k < np; k++) {
          double pr_, pi_, rr, ri;
          if (fscanf(fp, "%lf %lf %lf %lf", &pr_, &pi_, &rr, &ri) != 4) {
            fclose(fp);
            return vh_fail(c, "error reading pole-residue matrix file %s.", b->file);
          }
          po[k] = pr_ + I * pi_;
          re[k] = rr + I * ri;
        }
        pr_set(&rd, row, col, np, asymp, po, re);
        free(po);
        free(re);
      }
    fclose(fp);
    if (m == 4) {
      pr = rd;
      pr.m = pr.n = 4;
    } else {
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          pr_set(&pr, i, j, rd.num_poles[i][j], rd.asymp[i][j], rd.poles[i][j], rd.residues[i][j]);
          pr_set(&pr, i + 2, j, 0, 0.0, NULL, NULL);
          pr_set(&pr, i, j + 2, 0, 0.0, NULL, NULL);
          pr_set(&pr, i + 2, j + 2, rd.num_poles[i][j], rd.asymp[i][j], rd.poles[i][j], rd.residues[i][j]);
        }
    }
  }
  int mi = c->num_sibc_models++;
  c->sibc_pr = realloc(c->sibc_pr, sizeof(vh_pole_residue) * c->num_sibc_models);
  c->sibc_pr[mi] = pr;
  b->sibc_model = mi;
  return 0;
}

/* Recursive-convolution coefficients of all models (src/filter.c:347-387),
 * packed for the problem description. */
static int build_rc_models(vh_ctx *c)
{
  int total = 0;
  for (int m = 0; m < c->num_sibc_models; m++)
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < 4; q++) total += c->sibc_pr[m].num_poles[p][q];
  c->sibc_rc = calloc(c->num_sibc_models ? c->num_sibc_models : 1, sizeof(vgpu_sibc_model));
  c->sibc_q = calloc(6 * (size_t)(total ? total : 1), sizeof(double));
  double *q0 = c->sibc_q, *q1 = q0 + 2 * (total ? total : 1), *q2 = q1 + 2 * (total ? total : 1);
  int off = 0;
  double T = c->dt;
  for (int m = 0; m < c->num_sibc_models; m++) {
    vgpu_sibc_model *rc = &c->sibc_rc[m];
    rc->q0 = q0;
    rc->q1 = q1;
    rc->q2 = q2;
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < 4; q++) {
        const vh_pole_residue *pr = &c->sibc_pr[m];
        rc->num_poles[p][q] = pr->num_poles[p][q];
        rc->pole_offset[p][q] = off;
        rc->asymp[p][q] = pr->asymp[p][q];
        for (int k = 0; k < pr->num_poles[p][q]; k++) {
          double complex alpha = pr->residues[p][q][k] / pr->poles[p][q][k];
          double complex beta = pr->poles[p][q][k] * T;
          double complex a0 = cexp(beta);
          double complex a1 = alpha / beta * (1.0 + (beta - 1.0) * cexp(beta));
          double complex a2 = alpha / beta * (cexp(beta) - beta - 1.0);
          q0[2 * off] = creal(a0); q0[2 * off + 1] = cimag(a0);
          q1[2 * off] = creal(a1); q1[2 * off + 1] = cimag(a1);
          q2[2 * off] = creal(a2); q2[2 * off + 1] = cimag(a2);
          off++;
        }
      }
  }
  return 0;
}

/* Orientation matrices (src/sibc.c:62-108). */
static const double Acp[4][4] = { { 0, 0, 1, 0 }, { 0, 0, 0, -1 }, { -1, 0, 0, 0 }, { 0, 1, 0, 0 } };
static const double Acm[4][4] = { { 0, 0, 0, -1 }, { 0, 0, 1, 0 }, { 0, 1, 0, 0 }, { -1, 0, 0, 0 } };
static const double Asp[4][4] = { { -1, 0, 0, 0 }, { 0, 1, 0, 0 }, { 0, 0, -1, 0 }, { 0, 0, 0, 1 } };
static const double Asm[4][4] = { { 0, 1, 0, 0 }, { -1, 0, 0, 0 }, { 0, 0, 0, 1 }, { 0, 0, -1, 0 } };
static const double Bcp[4][4] = { { 1, 0, 0, 0 }, { 0, 1, 0, 0 }, { 0, 0, 1, 0 }, { 0, 0, 0, 1 } };
static const double Bcm[4][4] = { { 0, 1, 0, 0 }, { 1, 0, 0, 0 }, { 0, 0, 0, 1 }, { 0, 0, 1, 0 } };
static const double Bsp[4][4] = { { 0, 0, -1, 0 }, { 0, 0, 0, -1 }, { 1, 0, 0, 0 }, { 0, 1, 0, 0 } };
static const double Bsm[4][4] = { { 0, 0, 0, -1 }, { 0, 0, -1, 0 }, { 0, 1, 0, 0 }, { 1, 0, 0, 0 } };

static void lin_comb(double C[4][4], double a, const double A[4][4], double b, const double B[4][4])
{
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) C[p][q] = a * A[p][q] + b * B[p][q];
}

void vh_sibc_matrices(const vh_sibc *s, double A[4][4], double B[4][4])
{
  if (s->orient == 1) {
    lin_comb(A, s->cosa, Acp, s->sina, Asp);
    lin_comb(B, s->cosa, Bcp, s->sina, Bsp);
  } else {
    lin_comb(A, s->cosa, Acm, s->sina, Asm);
    lin_comb(B, s->cosa, Bcm, s->sina, Bsm);
  }
}

/* ---- H-correction operation list ---- */

static void hop_push(vh_ctx *c, int comp, int i, int j, int k, int kind, double cc, int s, int f, int slot1,
                     double d1, double n1, int slot2, double d2, double n2)
{
  if (c->num_hops == c->cap_hops) {
    c->cap_hops = c->cap_hops ? 2 * c->cap_hops : 4096;
    c->hops = realloc(c->hops, sizeof(vgpu_sibc_hop) * c->cap_hops);
  }
  vgpu_sibc_hop *h = &c->hops[c->num_hops++];
  memset(h, 0, sizeof *h);
  h->index = vh_idx(c, i, j, k);
  h->comp = comp;
  h->kind = kind;
  h->c = cc;
  h->s1 = s; h->f1 = f; h->slot1 = slot1; h->d1 = d1; h->n1 = n1;
  h->s2 = s; h->f2 = f; h->slot2 = slot2; h->d2 = d2; h->n2 = n2;
}

static double G(const vh_ctx *c, int comp, int i, int j, int k) { return c->coef[6 + comp - HX][vh_idx(c, i, j, k)]; }

/* One single-term edge correction: H += sign * (G*w) * (d*E). */
#define EDGE(comp, i_, j_, k_, sign, w, d, slot) \
  hop_push(c, comp, i_, j_, k_, 1, (sign) * (G(c, comp, i_, j_, k_) * (w)), s, f, slot, d, 0.0, 0, 0.0, 0.0)
/* Two-term parallel correction: H += sign * ((G*0.5)*w) * (nA*(dA*E1) + nB*(dB*E2)). */
#define PAR(comp, i_, j_, k_, sign, w, dA, slotA, nA, dB, slotB, nB)                                    \
  hop_push(c, comp, i_, j_, k_, 2, (sign) * (G(c, comp, i_, j_, k_) * 0.5 * (w)), s, f, slotA, dA, \
           (double)(nA), slotB, dB, (double)(nB))

static void build_hops(vh_ctx *c)
{
  c->num_hops = 0;
  for (int s = 0; s < c->num_sibcs; s++) {
    const vh_sibc *sb = &c->sibcs[s];
    const int *g = sb->gbbox;
    int nj = g[YHI] - g[YLO], nk = g[ZHI] - g[ZLO];
    for (int i = g[XLO], ii = 0; i < g[XHI]; i++, ii++)
      for (int j = g[YLO], jj = 0; j < g[YHI]; j++, jj++)
        for (int k = g[ZLO], kk = 0; k < g[ZHI]; k++, kk++) {
          int f = (ii * nj + jj) * nk + kk;
          const uint8_t *A = &sb->adjA[4 * f], *B = &sb->adjB[4 * f];
          double *idx_ = c->ide[0], *idy_ = c->ide[1], *idz_ = c->ide[2];
          switch (sb->normal) {
            case XDIR: {
              double wyl = 0.5 * (1 + vh_is_pmc_edge(c, ZDIR, k)), wyh = 0.5 * (1 + vh_is_pmc_edge(c, ZDIR, k + 1));
              double wzl = 0.5 * (1 + vh_is_pmc_edge(c, YDIR, j)), wzh = 0.5 * (1 + vh_is_pmc_edge(c, YDIR, j + 1));
              hop_push(c, HX, i, j, k, 0, 0, s, f, 0, 0, 0, 0, 0, 0);
              EDGE(HY, i - 1, j, k, +1, wzl, idx_[i - 1], 2);
              EDGE(HY, i - 1, j + 1, k, +1, wzh, idx_[i - 1], 2);
              EDGE(HY, i, j, k, -1, wzl, idx_[i], 3);
              EDGE(HY, i, j + 1, k, -1, wzh, idx_[i], 3);
              EDGE(HZ, i - 1, j, k, -1, wyl, idx_[i - 1], 0);
              EDGE(HZ, i - 1, j, k + 1, -1, wyh, idx_[i - 1], 0);
              EDGE(HZ, i, j, k, +1, wyl, idx_[i], 1);
              EDGE(HZ, i, j, k + 1, +1, wyh, idx_[i], 1);
              PAR(HX, i, j + 1, k, -1, wzh, idx_[i - 1], 2, !A[0], idx_[i], 3, !B[0]);
              PAR(HX, i, j - 1, k, +1, wzl, idx_[i - 1], 2, !A[1], idx_[i], 3, !B[1]);
              PAR(HX, i, j, k + 1, -1, wyh, idx_[i - 1], 0, !A[2], idx_[i], 1, !B[2]);
              PAR(HX, i, j, k - 1, +1, wyl, idx_[i - 1], 0, !A[3], idx_[i], 1, !B[3]);
              break;
            }
            case YDIR: {
              double wzl = 0.5 * (1 + vh_is_pmc_edge(c, XDIR, i)), wzh = 0.5 * (1 + vh_is_pmc_edge(c, XDIR, i + 1));
              double wxl = 0.5 * (1 + vh_is_pmc_edge(c, ZDIR, k)), wxh = 0.5 * (1 + vh_is_pmc_edge(c, ZDIR, k + 1));
              hop_push(c, HY, i, j, k, 0, 0, s, f, 0, 0, 0, 0, 0, 0);
              EDGE(HZ, i, j - 1, k, +1, wxl, idy_[j - 1], 2);
              EDGE(HZ, i, j - 1, k + 1, +1, wxh, idy_[j - 1], 2);
              EDGE(HZ, i, j, k, -1, wxl, idy_[j], 3);
              EDGE(HZ, i, j, k + 1, -1, wxh, idy_[j], 3);
              EDGE(HX, i, j - 1, k, -1, wzl, idy_[j - 1], 0);
              EDGE(HX, i + 1, j - 1, k, -1, wzh, idy_[j - 1], 0);
              EDGE(HX, i, j, k, +1, wzl, idy_[j], 1);
              EDGE(HX, i + 1, j, k, +1, wzh, idy_[j], 1);
              /* The reference pairs Eza with Exb here (src/sibc.c:697-698). */
              PAR(HY, i, j, k + 1, +1, wzh, idy_[j - 1], 0, !A[0], idy_[j], 3, !B[0]);
              PAR(HY, i, j, k - 1, -1, wzl, idy_[j - 1], 0, !A[1], idy_[j], 3, !B[1]);
              PAR(HY, i + 1, j, k, +1, wxh, idy_[j - 1], 2, !A[2], idy_[j], 3, !B[2]);
              PAR(HY, i - 1, j, k, -1, wxl, idy_[j - 1], 2, !A[3], idy_[j], 3, !B[3]);
              break;
            }
            default: {
              double wxl = 0.5 * (1 + vh_is_pmc_edge(c, YDIR, j)), wxh = 0.5 * (1 + vh_is_pmc_edge(c, YDIR, j + 1));
              double wyl = 0.5 * (1 + vh_is_pmc_edge(c, XDIR, i)), wyh = 0.5 * (1 + vh_is_pmc_edge(c, XDIR, i + 1));
              hop_push(c, HZ, i, j, k, 0, 0, s, f, 0, 0, 0, 0, 0, 0);
              EDGE(HX, i, j, k - 1, +1, wyl, idz_[k - 1], 2);
              EDGE(HX, i + 1, j, k - 1, +1, wyh, idz_[k - 1], 2);
              EDGE(HX, i, j, k, -1, wyl, idz_[k], 3);
              EDGE(HX, i + 1, j, k, -1, wyh, idz_[k], 3);
              EDGE(HY, i, j, k - 1, -1, wxl, idz_[k - 1], 0);
              EDGE(HY, i, j + 1, k - 1, -1, wxh, idz_[k - 1], 0);
              EDGE(HY, i, j, k, +1, wxl, idz_[k], 1);
              EDGE(HY, i, j + 1, k, +1, wxh, idz_[k], 1);
              PAR(HZ, i + 1, j, k, +1, wyh, idz_[k - 1], 2, !A[0], idz_[k], 3, !B[0]);
              PAR(HZ, i - 1, j, k, -1, wyl, idz_[k - 1], 2, !A[1], idz_[k], 3, !B[1]);
              PAR(HZ, i, j + 1, k, +1, wxh, idz_[k - 1], 0, !A[2], idz_[k], 1, !B[2]);
              PAR(HZ, i, j - 1, k, -1, wxl, idz_[k - 1], 0, !A[3], idz_[k], 1, !B[3]);
              break;
            }
          }
        }
  }
  /* Final pass zeroing the normal H of every face (src/sibc.c:733-770). */
  for (int s = 0; s < c->num_sibcs; s++) {
    const vh_sibc *sb = &c->sibcs[s];
    const int *g = sb->gbbox;
    int comp = HX + sb->normal;
    for (int i = g[XLO]; i < g[XHI]; i++)
      for (int j = g[YLO]; j < g[YHI]; j++)
        for (int k = g[ZLO]; k < g[ZHI]; k++) hop_push(c, comp, i, j, k, 0, 0, s, 0, 0, 0, 0, 0, 0, 0);
  }
}

/* Sort operations by target, keeping each target's operations in the
 * reference's order: each op is tagged with its position so qsort cannot
 * reorder equal targets. */
typedef struct {
  vgpu_sibc_hop h;
  int64_t pos;
} tagged_hop;

static int tagged_hop_cmp(const void *a, const void *b)
{
  const tagged_hop *x = a, *y = b;
  if (x->h.comp != y->h.comp) return x->h.comp - y->h.comp;
  if (x->h.index != y->h.index) return x->h.index < y->h.index ? -1 : 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

static void stable_sort_hops(vh_ctx *c)
{
  int64_t n = c->num_hops;
  tagged_hop *t = malloc(sizeof(tagged_hop) * (n ? n : 1));
  for (int64_t q = 0; q < n; q++) {
    t[q].h = c->hops[q];
    t[q].pos = q;
  }
  qsort(t, n, sizeof(tagged_hop), tagged_hop_cmp);
  for (int64_t q = 0; q < n; q++) c->hops[q] = t[q].h;
  free(t);
}

int vh_init_sibc_surfaces(vh_ctx *c)
{
  if (c->num_sibcs == 0) return 0;
  vh_log(c, 0, "\nInitialising SIBC surfaces...\n\n");
  c->sibcs = calloc(c->num_sibcs, sizeof(vh_sibc));
  int64_t vol = (int64_t)c->n[0] * c->n[1] * c->n[2];
  /* Face-use flags; entries outside the outer box read as false. */
  uint8_t *face = calloc((size_t)vol * 3, 1);
#define FACE(i, j, k, d) face[(vh_idx(c, (i), (j), (k))) * 3 + (d)]
  int s = 0;
  for (int q = 0; q < c->num_surfs; q++) {
    vh_surface *sf = &c->surfs[q];
    if (c->bnds[sf->boundary].type != BT_SIBC) continue;
    vh_sibc *sb = &c->sibcs[s];
    sb->model = c->bnds[sf->boundary].sibc_model;
    sb->orient = sf->orient;
    sb->normal = vh_bbox_direction(sf->mbbox);
    sb->cosa = cos(c->pi * sf->angle / 180.0);
    sb->sina = sin(c->pi * sf->angle / 180.0);
    vh_bbox_offset(sb->gbbox, sf->mbbox, c->gibox);
    sb->gbbox[2 * sb->normal + 1] += 1;
    for (int a = 0; a < 3; a++) sb->nfaces[a] = sb->gbbox[2 * a + 1] - sb->gbbox[2 * a];
    int nf = sb->nfaces[0] * sb->nfaces[1] * sb->nfaces[2];
    sb->adjA = calloc(4 * (size_t)(nf ? nf : 1), 1);
    sb->adjB = calloc(4 * (size_t)(nf ? nf : 1), 1);
    for (int i = sb->gbbox[XLO]; i < sb->gbbox[XHI]; i++)
      for (int j = sb->gbbox[YLO]; j < sb->gbbox[YHI]; j++)
        for (int k = sb->gbbox[ZLO]; k < sb->gbbox[ZHI]; k++) FACE(i, j, k, sb->normal) = 1;
    s++;
  }
  for (s = 0; s < c->num_sibcs; s++) {
    vh_sibc *sb = &c->sibcs[s];
    const int *g = sb->gbbox;
    int nj = sb->nfaces[1], nk = sb->nfaces[2];
    for (int i = g[XLO], ii = 0; i < g[XHI]; i++, ii++)
      for (int j = g[YLO], jj = 0; j < g[YHI]; j++, jj++)
        for (int k = g[ZLO], kk = 0; k < g[ZHI]; k++, kk++) {
          uint8_t *A = &sb->adjA[4 * ((ii * nj + jj) * nk + kk)], *B = &sb->adjB[4 * ((ii * nj + jj) * nk + kk)];
          switch (sb->normal) {
            case XDIR:
              A[0] = FACE(i - 1, j, k, YDIR); A[1] = FACE(i - 1, j + 1, k, YDIR);
              A[2] = FACE(i - 1, j, k, ZDIR); A[3] = FACE(i - 1, j, k + 1, ZDIR);
              B[0] = FACE(i, j, k, YDIR); B[1] = FACE(i, j + 1, k, YDIR);
              B[2] = FACE(i, j, k, ZDIR); B[3] = FACE(i, j + 1, k + 1, ZDIR);
              break;
            case YDIR:
              A[0] = FACE(i, j - 1, k, ZDIR); A[1] = FACE(i, j - 1, k + 1, ZDIR);
              A[2] = FACE(i, j - 1, k, XDIR); A[3] = FACE(i + 1, j - 1, k, XDIR);
              B[0] = FACE(i, j, k, ZDIR); B[1] = FACE(i, j, k + 1, ZDIR);
              B[2] = FACE(i, j, k, XDIR); B[3] = FACE(i + 1, j, k + 1, XDIR);
              break;
            default:
              A[0] = FACE(i, j, k - 1, XDIR); A[1] = FACE(i + 1, j, k - 1, XDIR);
              A[2] = FACE(i, j, k - 1, YDIR); A[3] = FACE(i, j + 1, k - 1, YDIR);
              B[0] = FACE(i, j, k, XDIR); B[1] = FACE(i + 1, j, k, XDIR);
              B[2] = FACE(i, j, k, YDIR); B[3] = FACE(i + 1, j + 1, k, YDIR);
              break;
          }
        }
  }
#undef FACE
  free(face);
  build_rc_models(c);
  build_hops(c);
  stable_sort_hops(c);
  return 0;
}
