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
