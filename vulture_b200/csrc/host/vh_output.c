/*
 * vh_output.c -- observer files and the command line.
 *
 * Writes the reference's text outputs: eh_<name>_td.asc
 * (src/observer.c:726-798), eh_<name>_fd.asc with the DFT normalised by the
 * reference waveform's DFT (src/observer.c:819-995), and the per-waveform
 * wf_<name>_td.asc / wf_<name>_fd.asc the reference adds for every waveform
 * (src/observer.c:449-457).  Waveform observers depend only on the waveform,
 * so they are computed here on the host with the same formulas.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vh.h"

void vh_set_tls_error(const char *msg);

static const char *EH_TD_HEAD = "# %6s %16s %16s %16s %16s %16s %16s %16s\n";
static const char *EH_FD_HEAD = "# %14s %16s %16s %16s %16s %16s %16s %16s %16s %16s %16s %16s %16s\n";

int vh_write_observers(vh_ctx *c, const double *td, uint64_t td_steps, const double *re, const double *im,
                       int full)
{
  const char *F = full ? "%23.16e " : "%16.8e ";
  const char *F2 = full ? "%23.16e %23.16e " : "%16.8e %16.8e ";
  uint64_t nt = c->num_steps;
  unsigned long nf = c->num_freq;
  char fname[VH_PATH + 16];

  /* Waveform DFTs over every step (src/observer.c:632-634, 857-899). */
  double *wf_re = calloc((size_t)(c->num_wfs ? c->num_wfs : 1) * (nf ? nf : 1), sizeof(double));
  double *wf_im = calloc((size_t)(c->num_wfs ? c->num_wfs : 1) * (nf ? nf : 1), sizeof(double));
  for (int w = 0; w < c->num_wfs; w++) {
    snprintf(fname, sizeof fname, "wf_%s_td.asc", c->wfs[w].name);
    FILE *fp = fopen(fname, "w");
    if (!fp) { free(wf_re); free(wf_im); return vh_fail(c, "Failed to open time domain output file %s", fname); }
    fprintf(fp, "# Waveform# %lu\n", (unsigned long)w);
    fprintf(fp, "# %6s %16s %16s\n", "ts (-)", "t (s)", "wf (-)");
    double *r = wf_re + (size_t)w * nf, *q = wf_im + (size_t)w * nf;
    for (uint64_t n = 0; n < nt; n++) {
      double t = n * c->dt;
      double v = vh_waveform_value(c, t, w, 0.0);
      fprintf(fp, "%8lu ", (unsigned long)n);
      fprintf(fp, F, t);
      fprintf(fp, F, v);
      fprintf(fp, "\n");
      for (unsigned long f = 0; f < nf; f++) {
        double wt = c->omega[f] * t;
        r[f] += v * cos(wt);
        q[f] -= v * sin(wt);
      }
    }
    fclose(fp);
    snprintf(fname, sizeof fname, "wf_%s_fd.asc", c->wfs[w].name);
    fp = fopen(fname, "w");
    if (!fp) { free(wf_re); free(wf_im); return vh_fail(c, "Failed to open frequency domain output file %s", fname); }
    fprintf(fp, "# Waveform# %lu\n", (unsigned long)w);
    fprintf(fp, "# %14s %16s %16s\n", "f (Hz)", "Re(wf) (-)", "Im(wf) (-)");
    for (unsigned long f = 0; f < nf; f++) {
      fprintf(fp, F, c->start_freq + f * c->step_freq);
      fprintf(fp, F2, r[f], q[f]);
      fprintf(fp, "\n");
    }
    fclose(fp);
  }

  for (int o = 0; o < c->num_obs; o++) {
    vh_observer *ob = &c->obs[o];
    if (ob->kind == OBS_TD_BINARY) continue;
    bool fd = ob->kind == OBS_FD_ASCII;
    snprintf(fname, sizeof fname, fd ? "eh_%s_fd.asc" : "eh_%s_td.asc", ob->name);
    FILE *fp = fopen(fname, "w");
    if (!fp) { free(wf_re); free(wf_im); return vh_fail(c, "Failed to open output file %s", fname); }
    fprintf(fp, "# (%d,%d,%d)->(%g,%g,%g)\n", ob->mbbox[XLO], ob->mbbox[YLO], ob->mbbox[ZLO],
            c->lines[0][ob->mbbox[XLO]], c->lines[1][ob->mbbox[YLO]], c->lines[2][ob->mbbox[ZLO]]);
    if (!fd) {
      fprintf(fp, EH_TD_HEAD, "ts (-)", "t (s)", "Ex (V/m)", "Ey (V/m)", "Ez (V/m)", "Hx (A/m)", "Hy (A/m)",
              "Hz (A/m)");
      for (uint64_t s = 0; s < td_steps; s++) {
        uint64_t n = c->out_start + s;
        fprintf(fp, "%8lu ", (unsigned long)n);
        fprintf(fp, F, n * c->dt);
        const double *v = td + (s * c->num_td + ob->slot) * 6;
        for (int q = 0; q < 6; q++) fprintf(fp, F, v[q]);
        fprintf(fp, "\n");
      }
    } else {
      fprintf(fp, EH_FD_HEAD, "f (Hz)", "Re(Ex) (V/m)", "Im(Ex) (V/m)", "Re(Ey) (V/m)", "Im(Ey) (V/m)",
              "Re(Ez) (V/m)", "Im(Ez) (V/m)", "Re(Hx) (V/m)", "Im(Hx) (V/m)", "Re(Hy) (V/m)", "Im(Hy) (V/m)",
              "Re(Hz) (V/m)", "Im(Hz) (V/m)");
      const double *wr = wf_re + (size_t)ob->wf * nf, *wi = wf_im + (size_t)ob->wf * nf;
      for (unsigned long f = 0; f < nf; f++) {
        double a = wr[f], b = wi[f];
        double den = a * a + b * b;
        fprintf(fp, F, c->start_freq + f * c->step_freq);
        for (int q = 0; q < 6; q++) {
          double cr = re[((size_t)ob->slot * 6 + q) * nf + f];
          double ci = im[((size_t)ob->slot * 6 + q) * nf + f];
          fprintf(fp, F2, (cr * a + ci * b) / den, (ci * a - cr * b) / den);
        }
        fprintf(fp, "\n");
      }
    }
    fclose(fp);
  }
  free(wf_re);
  free(wf_im);
  return 0;
}

int vhost_write_outputs(vhost *h, const double *td, uint64_t td_steps, const double *dft_re, const double *dft_im,
                        int32_t full_precision)
{
  if (!h) { vh_set_tls_error("null host handle"); return VGPU_EINVAL; }
  if (vh_write_observers(h, td, td_steps, dft_re, dft_im, full_precision)) {
    vh_set_tls_error(h->err);
    return VGPU_EINVAL;
  }
  return 0;
}

/* ---- binary observers (src/observer.c:1016-1212) ---- */

int64_t vhost_num_bin(const vhost *h);

/* Mesh lines, as initGrid() leaves them in the working directory
 * (src/grid.c:942-944, 1164-1178). */
int vhost_write_lines(vhost *h)
{
  if (!h) { vh_set_tls_error("null host handle"); return VGPU_EINVAL; }
  static const char *names[3] = { "xlines.dat", "ylines.dat", "zlines.dat" };
  for (int a = 0; a < 3; a++) {
    FILE *fp = fopen(names[a], "w");
    if (!fp) {
      vh_fail(h, "*** Error: Failed to open %s file.", names[a]);
      vh_set_tls_error(h->err);
      return VGPU_EINVAL;
    }
    for (int i = 0; i < h->num_lines[a]; i++) fprintf(fp, "%d %e\n", i, h->lines[a][i]);
    fclose(fp);
  }
  return 0;
}

static int bin_fail(vhost *h, const char *what)
{
  vh_fail(h, "*** Error: Failed to open %s file", what);
  vh_set_tls_error(h->err);
  return VGPU_EINVAL;
}

/* impulse.dat header, excite.dat and process.dat (src/observer.c:1031-1162). */
int vhost_bin_begin(vhost *h, int32_t full_precision)
{
  if (!h) { vh_set_tls_error("null host handle"); return VGPU_EINVAL; }
  int nbin_obs = 0;
  vh_observer *first = NULL;
  for (int o = 0; o < h->num_obs; o++)
    if (h->obs[o].kind == OBS_TD_BINARY) {
      if (!first) first = &h->obs[o];
      nbin_obs++;
    }
  if (!nbin_obs) return 0;
  if (h->impulse) fclose(h->impulse);
  h->impulse_failed = 0;

  /* impulse.dat: the output step count as a 4-byte int and dt as a float.
   * The reference writes sizeof(float) bytes of its `real` dt; with
   * real=float (the shipped build) that is the float written here. */
  h->impulse = fopen("impulse.dat", "wb");
  if (!h->impulse) return bin_fail(h, "impulse.dat");
  int32_t nout = (int32_t)(uint32_t)(h->out_stop - h->out_start + 1UL);
  float dtf = (float)h->dt;
  if (fwrite(&nout, sizeof nout, 1, h->impulse) != 1 || fwrite(&dtf, sizeof dtf, 1, h->impulse) != 1)
    h->impulse_failed = 1;

  /* excite.dat: waveform 0 at every step's E time. */
  FILE *fp = fopen("excite.dat", "w");
  if (!fp) return bin_fail(h, "excite.dat");
  fprintf(fp, " %d\n", 8);
  for (unsigned long n = 0; n < h->num_steps; n++)
    fprintf(fp, full_precision ? "%23.16e\n" : "%16.8e\n", vh_waveform_value(h, n * h->dt, 0, 0.0));
  fclose(fp);

  /* process.dat. */
  fp = fopen("process.dat", "w");
  if (!fp) return bin_fail(h, "process.dat");
  double mesh_size = h->dt * (2.0 * h->c0);
  double fstart = 0.0;
  double fstep = 1.0 / (h->num_steps * h->dt);
  double fstop = h->num_steps * fstep;
  char comment[70] = "";
  snprintf(comment, sizeof comment - 1, "%s", h->comment);
  fprintf(fp, "CE %s\n", comment);
  fprintf(fp, "%lu\n", (unsigned long)nbin_obs);
  for (int o = 0; o < h->num_obs; o++) {
    vh_observer *ob = &h->obs[o];
    if (ob->kind != OBS_TD_BINARY) continue;
    for (int a = 0; a < 3; a++)
      fprintf(fp, " %d %d %d", ob->gbbox[2 * a] - h->gibox[2 * a], ob->gbbox[2 * a + 1] - h->gibox[2 * a],
              ob->step[a]);
    fprintf(fp, "\n");
  }
  fprintf(fp, "%lu %lu\n", h->out_start + 1, h->out_stop + 1);
  fprintf(fp, "%g %g %g\n", fstart, fstop, fstep);
  fprintf(fp, "%g\n", mesh_size);
  for (int a = 0; a < 3; a++)
    fprintf(fp, " %d %d", first->gbbox[2 * a] - h->gibox[2 * a], first->gbbox[2 * a + 1] - h->gibox[2 * a]);
  fprintf(fp, " %d\n", 1);
  fclose(fp);
  return 0;
}

/* A vgpu_bin_sink: one record per node and row -- i, j, k relative to the
 * inner box as int, then Ex..Hz as float (src/observer.c:1164-1198). */
void vhost_bin_sink(void *user, uint64_t first_row, uint32_t num_rows, int64_t num_points, const float *rows)
{
  vhost *h = user;
  (void)first_row;
  if (!h || !h->impulse || num_points != h->num_bin) {
    if (h) h->impulse_failed = 1;
    return;
  }
  enum { REC = 3 * 4 + 6 * 4 };
  unsigned char *buf = malloc((size_t)num_points * REC);
  if (!buf) { h->impulse_failed = 1; return; }
  for (uint32_t r = 0; r < num_rows; r++) {
    const float *row = rows + (size_t)r * num_points * 6;
    for (int64_t q = 0; q < num_points; q++) {
      int32_t ijk[3] = { h->bin_points[3 * q] - h->gibox[XLO], h->bin_points[3 * q + 1] - h->gibox[YLO],
                         h->bin_points[3 * q + 2] - h->gibox[ZLO] };
      memcpy(buf + q * REC, ijk, sizeof ijk);
      memcpy(buf + q * REC + sizeof ijk, row + q * 6, 6 * sizeof(float));
    }
    if (fwrite(buf, REC, (size_t)num_points, h->impulse) != (size_t)num_points) h->impulse_failed = 1;
  }
  free(buf);
}

/* Close impulse.dat (src/observer.c:1201-1212). */
int vhost_bin_end(vhost *h)
{
  if (!h) { vh_set_tls_error("null host handle"); return VGPU_EINVAL; }
  int failed = h->impulse_failed;
  if (h->impulse && fclose(h->impulse) != 0) failed = 1;
  h->impulse = NULL;
  h->impulse_failed = 0;
  if (failed) {
    vh_fail(h, "*** Error: writing impulse.dat failed");
    vh_set_tls_error(h->err);
    return VGPU_EINVAL;
  }
  return 0;
}
