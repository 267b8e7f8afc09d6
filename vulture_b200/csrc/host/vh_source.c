/*
 * vh_source.c -- waveforms, sources, plane waves and observers set-up.
 *
 * Restates initWaveforms (src/waveform.c:256-347), getWaveformValue and the
 * waveform kernels (src/waveform.c:412-638), the external-waveform spline
 * (src/waveform.c:511-805), initSources (src/source.c:469-599),
 * initPlaneWaves/calcIncidentFieldVectors/initAuxGrid
 * (src/planewave.c:277-554, 1226-1300) and initObservers
 * (src/observer.c:399-519).  Arithmetic is double in the reference's order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vh.h"

/* ---- waveform kernels (src/waveform.c:412-508) ---- */

static double gaussian_pulse(double t, double w) { return exp(-0.5 * (pow(t / w, 2.0))); }
static double diff_gaussian_pulse(double t, double w) { return -t / w * exp(-0.5 * (pow(t / w, 2.0))); }
static double ricker_wavelet(double t, double w)
{
  return (1.0 - pow(t / w, 2)) * exp(-0.5 * (pow(t / w, 2.0)));
}
static double mod_gaussian_pulse(const vh_ctx *c, double t, double w, double f)
{
  return exp(-0.5 * (pow(t / w, 2.0))) * sin(2.0 * c->pi * f * t);
}
static double compact_pulse(const vh_ctx *c, double t, double w)
{
  if (t <= 0.0) return 0.0;
  if (t < 2.0 * w)
    return 1.0 / 32.0 *
           (10.0 - 15.0 * cos(c->pi / w * t) + 6.0 * cos(2.0 * c->pi / w * t) - cos(3.0 * c->pi / w * t));
  return 0.0;
}
static double diff_compact_pulse(const vh_ctx *c, double t, double w)
{
  if (t <= 0.0) return 0.0;
  if (t < 2.0 * w)
    return 1.0 / 32.0 *
           (15.0 * sin(c->pi / w * t) - 12.0 * sin(2.0 * c->pi / w * t) + 3.0 * sin(3.0 * c->pi / w * t));
  return 0.0;
}
static double mod_compact_pulse(const vh_ctx *c, double t, double w, double f)
{
  double env;
  if (t <= 0.0) env = 0.0;
  else if (t < 2.0 * w)
    env = 1.0 / 32.0 *
          (10.0 - 15.0 * cos(c->pi / w * t) + 6.0 * cos(2.0 * c->pi / w * t) - cos(3.0 * c->pi / w * t));
  else env = 0.0;
  return env * sin(2.0 * c->pi * f * t);
}
static double ramped_sinusoid(const vh_ctx *c, double t, double w, double f)
{
  double ramp;
  if (t <= 0.0) ramp = 0.0;
  else if (t < 1.0 * w)
    ramp = 1.0 / 32.0 *
           (10.0 - 15.0 * cos(c->pi / w * t) + 6.0 * cos(2.0 * c->pi / w * t) - cos(3.0 * c->pi / w * t));
  else ramp = 1.0;
  return ramp * sin(2.0 * c->pi * f * t);
}

/* Cubic spline of an external waveform table (src/waveform.c:759-805). */
static double eval_spline(vh_waveform *w, double t)
{
  double(*tab)[3] = (double(*)[3])w->table;
  unsigned long n = (unsigned long)w->table_size;
  unsigned long klo = w->last_idx, khi = klo + 1UL, k;
  if (klo >= n - 1UL) klo = 0;
  if ((tab[klo][0] > t) || (tab[klo + 1][0] < t)) {
    klo = 0;
    khi = n - 1UL;
    while (khi - klo > 1UL) {
      k = (khi + klo) >> 1;
      if (tab[k][0] > t) khi = k;
      else klo = k;
    }
  }
  w->last_idx = klo;
  double h = tab[khi][0] - tab[klo][0];
  double a = (tab[khi][0] - t) / h;
  double b = (t - tab[klo][0]) / h;
  return a * tab[klo][1] + b * tab[khi][1] +
         ((a * a * a - a) * tab[klo][2] + (b * b * b - b) * tab[khi][2]) * (h * h) / 6.0;
}

static double external_waveform(vh_waveform *w, double t)
{
  double(*tab)[3] = (double(*)[3])w->table;
  if (t < tab[0][0] || t > tab[w->table_size - 1][0]) return 0.0;
  return eval_spline(w, t);
}

/* src/waveform.c:590-638 */
double vh_waveform_value(vh_ctx *c, double t, int wf, double delay)
{
  vh_waveform *w = &c->wfs[wf];
  double x = t - delay - w->delay;
  switch (w->type) {
    case VGPU_WF_GAUSSIAN_PULSE:
    case VGPU_WF_NARROW_GAUSSIAN_PULSE: return w->size * gaussian_pulse(x, w->width);
    case VGPU_WF_DIFF_GAUSSIAN_PULSE: return w->size * diff_gaussian_pulse(x, w->width);
    case VGPU_WF_RICKER_WAVELET: return w->size * ricker_wavelet(x, w->width);
    case VGPU_WF_MOD_GAUSSIAN_PULSE: return w->size * mod_gaussian_pulse(c, x, w->width, w->frequency);
    case VGPU_WF_COMPACT_PULSE: return w->size * compact_pulse(c, x, w->width);
    case VGPU_WF_DIFF_COMPACT_PULSE: return w->size * diff_compact_pulse(c, x, w->width);
    case VGPU_WF_MOD_COMPACT_PULSE: return w->size * mod_compact_pulse(c, x, w->width, w->frequency);
    case VGPU_WF_RAMPED_SINUSOID: return w->size * ramped_sinusoid(c, x, w->width, w->frequency);
    case VGPU_WF_EXTERNAL: return w->size * external_waveform(w, x);
    default: return 0.0;
  }
}

/* Second derivatives of the external table (src/waveform.c:640-757). */
static int create_splines(vh_ctx *c, vh_waveform *w, double del_t)
{
  double(*tab)[3] = (double(*)[3])w->table;
  unsigned long n = (unsigned long)w->table_size;
  if (n < 2UL) return vh_fail(c, "Insufficient points for spline evaluation in file %s.", w->file);
  double maxd = 0.0;
  for (unsigned long i = 1; i < n; i++) {
    double d = tab[i][0] - tab[i - 1][0];
    if (d <= 0.0) return vh_fail(c, "Time data in %s is not monotonically increasing.", w->file);
    if (d > maxd) maxd = d;
  }
  double ratio = maxd / del_t;
  if (ratio < 1.5) vh_log(c, 0, "  External waveform in %s is well sampled (ratio %e).\n", w->file, ratio);
  else vh_log(c, 0, "  *** External waveform in %s may be undersampled (ratio %e)!\n", w->file, ratio);
  double *u = calloc(n, sizeof(double));
  const double d1 = 0.0, d2 = 0.0;
  tab[0][2] = -0.5;
  u[0] = (3.0 / (tab[1][0] - tab[0][0])) * ((tab[1][1] - tab[0][1]) / (tab[1][0] - tab[0][0]) - d1);
  for (unsigned long i = 1; i + 2 <= n; i++) {
    double sig = (tab[i][0] - tab[i - 1][0]) / (tab[i + 1][0] - tab[i - 1][0]);
    double p = sig * tab[i - 1][2] + 2.0;
    tab[i][2] = (sig - 1.0) / p;
    u[i] = (tab[i + 1][1] - tab[i][1]) / (tab[i + 1][0] - tab[i][0]) -
           (tab[i][1] - tab[i - 1][1]) / (tab[i][0] - tab[i - 1][0]);
    u[i] = (6.0 * u[i] / (tab[i + 1][0] - tab[i - 1][0]) - sig * u[i - 1]) / p;
  }
  double qn = 0.5;
  double un = (3.0 / (tab[n - 1][0] - tab[n - 2][0])) *
              (d2 - (tab[n - 1][1] - tab[n - 2][1]) / (tab[n - 1][0] - tab[n - 2][0]));
  tab[n - 1][2] = (un - qn * u[n - 2]) / (qn * tab[n - 2][2] + 1.0);
  for (unsigned long k = n - 1UL; k-- > 0;) tab[k][2] = tab[k][2] * tab[k + 1][2] + u[k];
  free(u);
  return 0;
}

static int load_external_waveform(vh_ctx *c, vh_waveform *w)
{
  FILE *fp = fopen(w->file, "r");
  if (!fp) return vh_fail(c, "Cannot open external waveform file %s", w->file);
  double a, b;
  int cap = 1024, n = 0;
  double *tab = malloc(sizeof(double) * 3 * cap);
  for (;;) {
    int r = fscanf(fp, "%lf %lf", &a, &b);
    if (r == 2) {
      if (n == cap) { cap *= 2; tab = realloc(tab, sizeof(double) * 3 * cap); }
      tab[3 * n] = a;
      tab[3 * n + 1] = b;
      tab[3 * n + 2] = 0.0;
      n++;
    } else if (r == EOF || feof(fp)) {
      break;
    } else {
      fclose(fp);
      free(tab);
      return vh_fail(c, "Error reading from %s", w->file);
    }
  }
  fclose(fp);
  w->table = tab;
  w->table_size = n;
  w->last_idx = 0;
  return 0;
}

int vh_init_waveforms(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising waveforms...\n\n");
  double dt = c->dt;
  for (int i = 0; i < c->num_wfs; i++) {
    vh_waveform *w = &c->wfs[i];
    if (w->size < 0) w->size = 1.0;
    switch (w->type) {
      case VGPU_WF_GAUSSIAN_PULSE:
      case VGPU_WF_DIFF_GAUSSIAN_PULSE:
      case VGPU_WF_RICKER_WAVELET:
        if (w->width < 0) w->width = 5.0 * sqrt(2.0) * dt;
        if (w->delay < 0) w->delay = 40.0 * dt;
        w->frequency = 0.0;
        break;
      case VGPU_WF_NARROW_GAUSSIAN_PULSE:
        if (w->width < 0) w->width = 8.0 * dt;
        if (w->delay < 0) w->delay = 12.0 * dt;
        w->frequency = 0.0;
        break;
      case VGPU_WF_MOD_GAUSSIAN_PULSE:
        if (w->width < 0) w->width = 20.0 * sqrt(2.0) * dt;
        if (w->delay < 0) w->delay = 120.0 * dt;
        if (w->frequency < 0) w->frequency = 0.05 / dt;
        break;
      case VGPU_WF_COMPACT_PULSE:
      case VGPU_WF_DIFF_COMPACT_PULSE:
        if (w->width < 0) w->width = 20.0 * dt;
        if (w->delay < 0) w->delay = 0.0;
        w->frequency = 0.0;
        break;
      case VGPU_WF_MOD_COMPACT_PULSE:
        if (w->width < 0) w->width = 80.0 * dt;
        if (w->delay < 0) w->delay = 0.0;
        if (w->frequency < 0) w->frequency = 0.05 / dt;
        break;
      case VGPU_WF_RAMPED_SINUSOID:
        if (w->width < 0) w->width = 20.0 * dt;
        if (w->delay < 0) w->delay = 0.0;
        if (w->frequency < 0) w->frequency = 0.05 / dt;
        break;
      case VGPU_WF_EXTERNAL:
        if (w->delay < 0) w->delay = 0.0;
        if (load_external_waveform(c, w)) return -1;
        vh_log(c, 0, "  Read %d entries from external waveform table in file %s\n", w->table_size, w->file);
        if (create_splines(c, w, dt)) return -1;
        break;
    }
  }
  return 0;
}

/* ---- sources (src/source.c:469-599) ---- */

static void electric_source_size(const vh_ctx *c, const int g[6], int dir, double *len, double *area,
                                 double side[3])
{
  *len = 0.0;
  *area = 0.0;
  side[0] = side[1] = side[2] = 0.0;
  for (int a = 0; a < 3; a++) {
    if (a == dir)
      for (int i = g[2 * a]; i <= g[2 * a + 1] - 1; i++) *len += c->de[a][i];
    else
      for (int i = g[2 * a]; i <= g[2 * a + 1]; i++) side[a] += c->dh[a][i];
  }
  if (dir == XDIR) *area = side[YDIR] * side[ZDIR];
  else if (dir == YDIR) *area = side[ZDIR] * side[XDIR];
  else *area = side[XDIR] * side[YDIR];
}

static void magnetic_source_size(const vh_ctx *c, const int g[6], int dir, double *len, double *area,
                                 double side[3])
{
  *len = 0.0;
  *area = 0.0;
  side[0] = side[1] = side[2] = 0.0;
  for (int a = 0; a < 3; a++) {
    if (a == dir)
      for (int i = g[2 * a]; i <= g[2 * a + 1]; i++) *len += c->dh[a][i];
    else
      for (int i = g[2 * a]; i <= g[2 * a + 1] - 1; i++) side[a] += c->de[a][i];
  }
  if (dir == XDIR) *area = side[YDIR] * side[ZDIR];
  else if (dir == YDIR) *area = side[ZDIR] * side[XDIR];
  else *area = side[XDIR] * side[YDIR];
}

int vh_init_sources(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising sources...\n\n");
  const bool all[6] = { true, true, true, true, true, true };
  for (int s = 0; s < c->num_srcs; s++) {
    vh_source *it = &c->srcs[s];
    double len, area, side[3];
    vh_bbox_offset(it->gbbox, it->mbbox, c->gibox);
    vh_set_field_limits(it->gbbox, it->flim, all);
    switch (it->type) {
      case ST_ELEC_SURF_CURR_DENSITY:
        electric_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / side[it->norm];
        it->type = ST_ELEC_CURR_DENSITY;
        break;
      case ST_MAGN_SURF_CURR_DENSITY:
        magnetic_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / side[it->norm];
        it->type = ST_MAGN_CURR_DENSITY;
        break;
      case ST_ELEC_CURRENT:
        electric_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / area;
        it->type = ST_ELEC_CURR_DENSITY;
        break;
      case ST_MAGN_CURRENT:
        magnetic_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / area;
        it->type = ST_MAGN_CURR_DENSITY;
        break;
      case ST_ELEC_CURRENT_MOMENT:
        electric_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / area / len;
        it->type = ST_ELEC_CURR_DENSITY;
        break;
      case ST_MAGN_CURRENT_MOMENT:
        magnetic_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = it->size / area / len;
        it->type = ST_MAGN_CURR_DENSITY;
        break;
      case ST_VOLTAGE:
        electric_source_size(c, it->gbbox, it->pol, &len, &area, side);
        it->size = -it->size / len;
        it->type = ST_EFIELD;
        break;
      case ST_THEVENIN_VOLTAGE:
      case ST_NORTON_CURRENT: {
        if (it->type == ST_NORTON_CURRENT) {
          it->size = it->resistance * it->size;
          it->type = ST_THEVENIN_VOLTAGE;
        }
        char rname[VH_TAG];
        snprintf(rname, VH_TAG, "__VR_RS_%d__", s + 1);
        int ri = vh_find_medium(c, rname);
        if (ri < 0) return vh_fail(c, "Internal error: lumped source medium %s missing", rname);
        electric_source_size(c, it->gbbox, it->pol, &len, &area, side);
        if (it->resistance > 1e-2) {
          it->size = it->size / area / it->resistance;
          double sigma = len / (area * it->resistance);
          vh_medium *m = &c->media[ri];
          m->eps_r = 1.0;
          m->sigma = sigma;
          m->mu_r = 1.0;
          vh_calc_coeff(c, m);
          vh_set_medium_on_grid(c, it->gbbox, ri, VH_FACE_MASK_ALL);
          it->type = ST_ELEC_CURR_DENSITY;
        } else {
          it->size = -0.5 * it->size / len;
          vh_set_medium_on_grid(c, it->gbbox, MT_PEC, VH_FACE_MASK_ALL);
          it->type = ST_EFIELD;
        }
        break;
      }
      default:
        break;
    }
  }
  return 0;
}

/* ---- plane waves (src/planewave.c:277-554, 1226-1300) ---- */

static void calc_incident_vectors(vh_ctx *c, vh_planewave *p)
{
  double th = c->pi / 180.0 * p->theta, ph = c->pi / 180.0 * p->phi, et = c->pi / 180.0 * p->eta;
  double size = p->size;
  p->kinc[0] = sin(th) * cos(ph);
  p->kinc[1] = sin(th) * sin(ph);
  p->kinc[2] = cos(th);
  p->finc[EX] = size * (cos(et) * sin(ph) - sin(et) * cos(th) * cos(ph));
  p->finc[EY] = size * (-cos(et) * cos(ph) - sin(et) * cos(th) * sin(ph));
  p->finc[EZ] = size * (sin(et) * sin(th));
  p->finc[HX] = size / c->eta0 * (sin(et) * sin(ph) + cos(et) * cos(th) * cos(ph));
  p->finc[HY] = size / c->eta0 * (-sin(et) * cos(ph) + cos(et) * cos(th) * sin(ph));
  p->finc[HZ] = size / c->eta0 * (-cos(et) * sin(th));
  /* Origin corner (Taflove eqns. 5.61/5.62 as src/planewave.c:476-551). */
  const int *g = p->gbbox;
  double theta = p->theta, phi = p->phi;
  int xs, ys;
  if (phi >= 0 && phi <= 90) { xs = XLO; ys = YLO; }
  else if (phi > 90 && phi <= 180) { xs = XHI; ys = YLO; }
  else if (phi > 180 && phi <= 270) { xs = XHI; ys = YHI; }
  else { xs = XLO; ys = YHI; }
  p->ijk0[0] = g[xs];
  p->ijk0[1] = g[ys];
  p->ijk0[2] = (theta >= 0 && theta <= 90) ? g[ZLO] : g[ZHI];
}

static void init_aux_grid(vh_ctx *c, vh_planewave *p)
{
  const int npml = 10;
  double dt = c->dt, d0 = c->duni[0];
  double rel = vh_numerical_phase_velocity(c, 0.0, 0.0) /
               vh_numerical_phase_velocity(c, c->pi * p->theta / 180.0, c->pi * p->phi / 180.0);
  p->beta_eyi = dt / (c->eps0 * d0) / rel;
  p->gamma_hzi = dt / (c->mu0 * d0) / rel;
  int dx = p->gbbox[XHI] - p->gbbox[XLO], dy = p->gbbox[YHI] - p->gbbox[YLO], dz = p->gbbox[ZHI] - p->gbbox[ZLO];
  p->nx = (int)(6 + npml + sqrt(dx * dx + dy * dy + dz * dz));
  p->xb = p->nx - npml;
  for (int i = 0; i < npml; i++) {
    double depth = abs(i) / (double)npml;
    double sprof = 0.5 * dt / c->eps0 * pow(depth, 3.77) * 4.0 / c->eta0 / d0;
    p->bdx[i] = 1.0 / (1.0 + sprof);
    p->adx[i] = (1.0 - sprof) / (1.0 + sprof);
    depth = (abs(i) + 0.5) / (double)(npml);
    sprof = 0.5 * dt / c->eps0 * pow(depth, 3.77) * 4.0 / c->eta0 / d0;
    p->bhx[i] = 1.0 / (1.0 + sprof);
    p->ahx[i] = (1.0 - sprof) / (1.0 + sprof);
  }
}

int vh_init_planewaves(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising plane waves...\n\n");
  for (int n = 0; n < c->num_pws; n++) {
    vh_planewave *p = &c->pws[n];
    vh_bbox_offset(p->gbbox, p->mbbox, c->gibox);
    calc_incident_vectors(c, p);
    for (int a = 0; a < 3; a++) {
      int ig = (int)p->ijk0[a];
      p->r0[a] = c->lines[a][ig - c->gibox[2 * a]];
    }
    switch (c->grid_type) {
      case GT_CUBIC: init_aux_grid(c, p); p->phase_velocity = c->c0; break;
      case GT_UNIFORM:
        p->phase_velocity = vh_numerical_phase_velocity(c, c->pi / 180.0 * p->theta, c->pi / 180.0 * p->phi);
        break;
      default: p->phase_velocity = c->c0; break;
    }
    bool edge[6];
    for (int f = 0; f < 6; f++) {
      edge[f] = p->active[f];
      int t = vh_outer_type(c, f);
      if (p->gbbox[f] == c->gibox[f] && (t == BT_PMC || t == BT_PERIODIC)) edge[f] = true;
    }
    /* Field limits of the six one-cell-thick correction slabs (src/planewave.c:357-411). */
    for (int f = 0; f < 6; f++) {
      int a = f / 2;
      int bb[6];
      bool incl[6];
      memcpy(bb, p->gbbox, sizeof bb);
      for (int g = 0; g < 6; g++) incl[g] = edge[g];
      if (f % 2 == 0) {
        bb[2 * a] = p->gbbox[f] - 1;
        bb[2 * a + 1] = p->gbbox[f];
        incl[2 * a] = false;
        incl[2 * a + 1] = true;
      } else {
        bb[2 * a] = p->gbbox[f];
        bb[2 * a + 1] = p->gbbox[f] + 1;
        incl[2 * a] = true;
        incl[2 * a + 1] = false;
      }
      vh_set_field_limits(bb, p->flim[f], incl);
    }
  }
  return 0;
}

/* ---- observers (src/observer.c:399-519) ---- */

int vh_init_observers(vh_ctx *c)
{
  vh_log(c, 0, "\nInitialising observers...\n\n");
  unsigned long nt = c->num_steps;
  if (!c->has_ot) {
    c->out_start = 0UL;
    c->out_stop = nt - 1UL;
  } else {
    c->out_start = c->ot_start;
    c->out_stop = c->ot_stop;
  }
  if (!c->has_of) {
    c->start_freq = 0.0;
    c->num_freq = (unsigned long)fmax(nt / 10, 1);
    c->step_freq = 1.0 / (nt * c->dt);
    c->stop_freq = c->start_freq + (c->num_freq - 1) * c->step_freq;
  } else {
    c->start_freq = c->of_start;
    c->stop_freq = c->of_stop;
    c->num_freq = c->of_num;
    c->step_freq = (c->stop_freq - c->start_freq) / (c->num_freq - 1);
  }
  vh_log(c, 0, "  Observer freqs: fstart=%g MHz, fstop=%g MHz, fstep=%g MHz, fnumber=%lu\n",
         c->start_freq / 1e6, c->stop_freq / 1e6, c->step_freq / 1e6, c->num_freq);
  int ntd = 0, nfd = 0;
  for (int o = 0; o < c->num_obs; o++) {
    vh_observer *ob = &c->obs[o];
    vh_bbox_offset(ob->gbbox, ob->mbbox, c->gibox);
    if (ob->kind == OBS_TD_ASCII) ob->slot = ntd++;
    else if (ob->kind == OBS_FD_ASCII) ob->slot = nfd++;
    else ob->slot = -1;
  }
  c->num_td = ntd;
  c->num_fd = nfd;
  c->td_points = calloc(3 * (ntd ? ntd : 1), sizeof(int32_t));
  c->fd_points = calloc(3 * (nfd ? nfd : 1), sizeof(int32_t));
  for (int o = 0; o < c->num_obs; o++) {
    vh_observer *ob = &c->obs[o];
    int32_t *dst = ob->kind == OBS_TD_ASCII ? c->td_points : ob->kind == OBS_FD_ASCII ? c->fd_points : NULL;
    if (!dst) continue;
    dst[3 * ob->slot] = ob->gbbox[XLO];
    dst[3 * ob->slot + 1] = ob->gbbox[YLO];
    dst[3 * ob->slot + 2] = ob->gbbox[ZLO];
  }
  c->omega = calloc(c->num_freq ? c->num_freq : 1, sizeof(double));
  for (unsigned long f = 0; f < c->num_freq; f++)
    c->omega[f] = 2.0 * c->pi * (c->start_freq + (int)f * c->step_freq);

  /* Binary observers: their nodes in impulse.dat order, k outermost, then j,
   * then i (src/observer.c:1172-1174).  A zero step never advances the
   * reference's loop; it is refused here. */
  int64_t nbin = 0;
  for (int o = 0; o < c->num_obs; o++) {
    vh_observer *ob = &c->obs[o];
    if (ob->kind != OBS_TD_BINARY) continue;
    for (int a = 0; a < 3; a++)
      if (ob->step[a] <= 0)
        return vh_fail(c, "*** Error: binary observer %s has a zero step along %c", ob->name, "xyz"[a]);
    nbin += (int64_t)(1 + (ob->gbbox[ZHI] - ob->gbbox[ZLO]) / ob->step[2]) *
            (1 + (ob->gbbox[YHI] - ob->gbbox[YLO]) / ob->step[1]) * (1 + (ob->gbbox[XHI] - ob->gbbox[XLO]) / ob->step[0]);
  }
  c->num_bin = nbin;
  c->bin_points = calloc(3 * (size_t)(nbin ? nbin : 1), sizeof(int32_t));
  if (!c->bin_points) return vh_fail(c, "*** Error: out of memory for binary observers");
  int64_t q = 0;
  for (int o = 0; o < c->num_obs; o++) {
    vh_observer *ob = &c->obs[o];
    if (ob->kind != OBS_TD_BINARY) continue;
    for (int k = ob->gbbox[ZLO]; k <= ob->gbbox[ZHI]; k += ob->step[2])
      for (int j = ob->gbbox[YLO]; j <= ob->gbbox[YHI]; j += ob->step[1])
        for (int i = ob->gbbox[XLO]; i <= ob->gbbox[XHI]; i += ob->step[0]) {
          c->bin_points[3 * q] = i;
          c->bin_points[3 * q + 1] = j;
          c->bin_points[3 * q + 2] = k;
          q++;
        }
  }
  return 0;
}
