/*
 * vgpu.h -- C ABI of the B200 FDTD time-stepping engine.
 *
 * The engine replaces the time loop of the Vulture solver: the function
 * propagate() (reference src/simulation.c:136-231, declared in
 * src/simulation.h:41 and called from src/vulture.c:173) together with every
 * update routine it calls.  Everything the reference sets up before that call
 * (grid, media, PML/Mur/Debye/SIBC state, sources, plane waves, observers) is
 * passed in as plain C data in a vgpu_problem.  No torch or CUDA type appears
 * in this header.
 *
 * Conventions
 *   - Face order XLO, XHI, YLO, YHI, ZLO, ZHI = 0..5 and field order
 *     EX, EY, EZ, HX, HY, HZ = 0..5, as the reference's MeshFace and
 *     FieldComponent enums (src/fdtd_types.h:86-110).
 *   - A "limit" int32_t lim[6] is the inclusive index range
 *     [lim[0]..lim[1]] x [lim[2]..lim[3]] x [lim[4]..lim[5]], as the
 *     reference's field-limit arrays (src/grid.c:390-454).
 *   - Volumes are n[0]*n[1]*n[2] values, index (i*n[1]+j)*n[2]+k with k
 *     fastest: the reference's [i][j][k] arrays (src/alloc_array.c:54-141).
 *     n[] counts the ghost cells (src/grid.c:380-383).
 *   - All host inputs are double.  In VGPU_FP32 mode the engine rounds fields
 *     and coefficients to float on upload; the DFT accumulators, Debye
 *     recursion and waveform phase stay double.
 *   - Every function returns 0 on success and a negative VGPU_E* code on
 *     failure; vgpu_last_error() gives the message.  Nothing calls exit().
 *   - The engine copies every input at vgpu_create(); the caller keeps
 *     ownership of its arrays and may free them afterwards.
 */
#ifndef VGPU_H
#define VGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGPU_ABI_VERSION 3

/* Status codes. */
#define VGPU_OK            0
#define VGPU_EINVAL       -1   /* invalid problem description or argument */
#define VGPU_ENOMEM       -2   /* device or host allocation failed */
#define VGPU_ECUDA        -3   /* CUDA runtime error */
#define VGPU_ENODEV       -4   /* no usable sm_100 device */
#define VGPU_ENONFINITE   -5   /* a field became NaN/Inf (finiteness check) */
#define VGPU_ETIMEOUT     -6   /* a bounded device wait ran out */
#define VGPU_ECANCELLED   -7   /* request cancelled (serving API) */

typedef enum { VGPU_FP64 = 0, VGPU_FP32 = 1 } vgpu_precision;

/* Treatment of the ghost layer on an external face (src/surface.c:569-812). */
enum { VGPU_GHOST_NONE = 0, VGPU_GHOST_PEC = 1, VGPU_GHOST_PMC = 2, VGPU_GHOST_PERIODIC = 3 };

/* Source kinds after the reference's init-time conversions (src/source.c:602-753). */
enum {
  VGPU_SRC_FIELD = 0,    /* F = soft*F + v                 (ST_EFIELD / ST_HFIELD) */
  VGPU_SRC_CURRENT = 1   /* F = soft*F - coef(i,j,k)*v      (ST_ELEC/MAGN_CURR_DENSITY) */
};

/* Waveform types (src/waveform.h:44-57). */
enum {
  VGPU_WF_GAUSSIAN_PULSE = 0, VGPU_WF_NARROW_GAUSSIAN_PULSE, VGPU_WF_DIFF_GAUSSIAN_PULSE,
  VGPU_WF_RICKER_WAVELET, VGPU_WF_MOD_GAUSSIAN_PULSE, VGPU_WF_COMPACT_PULSE,
  VGPU_WF_DIFF_COMPACT_PULSE, VGPU_WF_MOD_COMPACT_PULSE, VGPU_WF_RAMPED_SINUSOID,
  VGPU_WF_EXTERNAL
};

/* A waveform, evaluated on the device for the analytic plane-wave incident
 * field (src/waveform.c:590-638).  table holds table_size rows of
 * (t, value, second-derivative) for VGPU_WF_EXTERNAL (src/waveform.c:511-805). */
typedef struct {
  int32_t type;
  int32_t table_size;
  double size, delay, width, frequency;
  const double *table;
} vgpu_waveform;

/* One source after init (src/source.c:469-599).  values[n] is the source
 * amplitude size*wf(t) at the field's time of step n: n*dt for E components,
 * (n+0.5)*dt for H components. */
typedef struct {
  int32_t field;       /* VGPU field index 0..5 */
  int32_t kind;        /* VGPU_SRC_FIELD / VGPU_SRC_CURRENT */
  int32_t soft;        /* 1 = soft (adds), 0 = hard (replaces) */
  int32_t flim[6];
  const double *values;
} vgpu_source;

/* A dispersive block of the Debye medium (src/debye.c:44-55).
 * dalpha/dbeta hold num_poles complex values as (re, im) pairs. */
typedef struct {
  int32_t flim[3][6];  /* limits of Ex, Ey, Ez */
  int32_t num_poles;
  const double *dalpha;
  const double *dbeta;
} vgpu_debye;

/* A total-field/scattered-field plane wave (src/planewave.c:47-93). */
typedef struct {
  int32_t active[6];          /* which Huygens faces correct fields */
  int32_t flim[6][6][6];      /* [face][field][lim] correction limits */
  int32_t waveform;           /* index into vgpu_problem.waveforms */
  int32_t use_aux_grid;       /* 1: cubic grid, 1-D auxiliary grid (planewave.c:1226-1419) */
  double delay;
  double kinc[3];
  double finc[6];
  double r0[3];               /* origin, physical units */
  double ijk0[3];             /* origin, grid indices */
  double phase_velocity;
  /* Auxiliary grid (use_aux_grid == 1). */
  int32_t aux_nx, aux_xb, aux_npml;
  double aux_beta, aux_gamma;
  const double *aux_adx, *aux_bdx, *aux_ahx, *aux_bhx;   /* aux_npml each */
  const double *aux_source;   /* num_steps: wf(n*dt) driving Eyi[0] */
} vgpu_planewave;

/* SIBC boundary model: 4x4 recursive-convolution filters (src/filter.h:40-73).
 * For row p, column q: num_poles[p][q] poles starting at pole_offset[p][q] in
 * q0/q1/q2 (complex, stored as re,im pairs), constant term asymp[p][q]. */
typedef struct {
  int32_t num_poles[4][4];
  int32_t pole_offset[4][4];
  double asymp[4][4];
  const double *q0, *q1, *q2;
} vgpu_sibc_model;

/* An SIBC surface (src/sibc.c:43-58).  gbbox is extended by one in the
 * normal direction as the reference does (src/sibc.c:236-251); its faces are
 * the cells of gbbox, numbered (ii*nj + jj)*nk + kk.  A and B are the pre- and
 * post-filter axis transforms for its orientation and angle. */
typedef struct {
  int32_t normal;
  int32_t model;
  int32_t gbbox[6];
  double A[4][4], B[4][4];
  const uint8_t *adjA;        /* [faces][4] */
  const uint8_t *adjB;        /* [faces][4] */
} vgpu_sibc_surface;

/* One operation of the SIBC magnetic correction (src/sibc.c:616-776),
 * applied to H component `comp` at volume index `index`, in list order:
 *   kind 0: H = 0
 *   kind 1: H = H + c * (d1 * E1)
 *   kind 2: H = H + c * (n1 * (d1 * E1) + n2 * (d2 * E2))
 * E1/E2 are tangential E values of face (surface s, face f, slot 0..3). */
typedef struct {
  int64_t index;
  int32_t comp;
  int32_t kind;
  int32_t s1, f1, slot1;
  int32_t s2, f2, slot2;
  double c, d1, d2, n1, n2;
} vgpu_sibc_hop;

typedef struct {
  int32_t abi_version;        /* VGPU_ABI_VERSION */
  int32_t precision;          /* vgpu_precision */

  /* Grid (src/grid.c:326-454, 583-679). */
  int32_t n[3];
  int32_t gibox[6];
  int32_t gobox[6];
  int32_t gfilim[6][6];       /* bulk update limits per field */
  uint64_t num_steps;
  double dt;
  const double *ide[3];       /* inverse primary edge lengths, n[axis] each */
  const double *idh[3];       /* inverse secondary edge lengths */
  const double *coef[9];      /* alphaEx..z, betaEx..z, gammaHx..z volumes */

  /* External faces. */
  int32_t ghost[6];           /* VGPU_GHOST_* per face */

  /* UPML (src/pml.c:44-84). */
  int32_t pml_present[6];
  int32_t pml_flim[6][6][6];  /* [region][field][lim] */
  const double *pml_ad[3], *pml_bd[3], *pml_ah[3], *pml_bh[3], *pml_ibd[3], *pml_ibh[3];

  /* First-order Mur (src/mur.c:46-52). */
  int32_t mur_present[6];
  int32_t mur_flim[6][6][6];
  double mur_zeta[6];

  /* Debye blocks. */
  int32_t num_debye;
  const vgpu_debye *debye;

  /* SIBC surfaces. */
  int32_t num_sibc_models;
  const vgpu_sibc_model *sibc_models;
  int32_t num_sibc;
  const vgpu_sibc_surface *sibc;
  int64_t num_sibc_hops;
  const vgpu_sibc_hop *sibc_hops;

  /* Sources, in mesh order. */
  int32_t num_sources;
  const vgpu_source *sources;

  /* Plane waves, waveforms and the field-position tables used by the
   * analytic incident field (src/grid.c:1429-1476): pos_node[a][i] is the
   * mesh-line coordinate of grid index i on axis a, pos_half[a][i] the
   * mid-edge coordinate. */
  int32_t num_planewaves;
  const vgpu_planewave *planewaves;
  int32_t num_waveforms;
  const vgpu_waveform *waveforms;
  const double *pos_node[3];
  const double *pos_half[3];

  /* Point observers (src/observer.c:622-650).  All six components are
   * sampled at the top of step n, before any update, when
   * out_start <= n <= out_stop. */
  uint64_t out_start, out_stop;
  int32_t num_td;             /* time-domain points */
  const int32_t *td_points;   /* [num_td][3] grid indices */
  int32_t num_fd;             /* frequency-domain (running DFT) points */
  const int32_t *fd_points;   /* [num_fd][3] */
  int32_t num_freq;
  const double *omega;        /* angular frequencies, num_freq */

  /* Binary (TDOM_BINARY) observers (src/observer.c:1164-1198): every node of
   * every binary observer, in the order the reference writes them to
   * impulse.dat -- observers in mesh order, and within one observer k
   * outermost, then j, then i, each advancing by the observer's step.
   * Sampled with the point observers and delivered as float rows through a
   * vgpu_bin_sink. */
  int64_t num_bin;
  const int32_t *bin_points;  /* [num_bin][3] grid indices */

  /* Optional medium tags, the reference's USE_INDEXED_MEDIA idea
   * (src/grid.h:108-136) kept beside the volumes.  coef_tag[f] holds one byte
   * per cell for component f (Ex, Ey, Ez, Hx, Hy, Hz): 0 where the
   * component's coefficients are zero, t > 0 where they are tag_coef[t - 1]'s
   * -- alpha and beta (coef[f], coef[3 + f]) for an E component, gamma
   * (coef[3 + f]) for an H one.  When set they must describe coef[] exactly;
   * vgpu_create then finds the distinct coefficient tuples from three bytes
   * per cell for E and three for H instead of the nine double volumes.  All
   * NULL (or num_tags 0): it scans coef[].  A tag above num_tags makes
   * vgpu_create return VGPU_EINVAL. */
  const uint8_t *coef_tag[6];
  int32_t num_tags;           /* at most 255 */
  const double *tag_coef;     /* [num_tags][3]: alpha, beta, gamma */
} vgpu_problem;

typedef struct vgpu_engine vgpu_engine;

/* Timing of the last vgpu_run, measured with CUDA events on the engine's
 * stream. */
typedef struct {
  double run_ms;              /* device time of the last vgpu_run */
  uint64_t steps;             /* steps in that run */
  uint64_t kernel_launches;   /* engine kernels launched in that run */
  uint64_t device_bytes;      /* device memory held by the engine */
  uint64_t h2d_bytes;         /* bytes copied host->device since creation (problem upload, writes) */
  /* Stability check, no counterpart in the reference (whose only guard is
   * the Courant check, src/simulation.c:64-84): FP64 sums of squares of the
   * E and of the H components over every stored point, computed on the
   * device at every 64-step boundary and at the problem's last step, as of
   * energy_step (0: not yet computed).  Not the physical energy (no
   * permittivity, permeability or cell-volume weights); it grows without
   * bound when the update is unstable.  vgpu_run and vgpu_synchronize return
   * VGPU_ENONFINITE when it is not finite. */
  double energy_e, energy_h;
  uint64_t energy_step;
  /* Side launches the engine merged for this problem: bit 0, the Debye
   * update and the plane wave's E corrections run as one kernel; bit 1, the
   * plane wave's H corrections and the next step's observer samples do.  Set
   * only where the merged parts touch disjoint points. */
  uint32_t merged_parts;
  uint32_t reserved;
} vgpu_stats;

/* Create an engine on the current CUDA device (cuda:0 unless the caller set
 * another) and upload the problem.  Replaces the state the reference builds
 * in src/vulture.c:95-148 before propagate().  An engine may be driven from
 * any host thread: each entry point that takes it makes its device current
 * on the calling thread first.  Calls on one engine must not overlap. */
int vgpu_create(const vgpu_problem *problem, vgpu_engine **engine);

/* No counterpart in the reference.  Checks on the host, without a device,
 * how the engine would tile the problem's E and H sweeps: every point of each swept component's bulk and
 * UPML update boxes must be claimed by exactly one tile and no other point by
 * any, and every tile must keep the sweep kernel's limits.  *violations
 * receives the number of failures (0 for a sound plan), *tiles the number of
 * tiles of both sweeps.  precision selects the storage word (VGPU_FP32 or
 * VGPU_FP64), which sets the halo alignment. */
int vgpu_check_sweep_plan(const vgpu_problem *problem, int32_t precision, int64_t *violations, int64_t *tiles);

/* No counterpart in the reference.  The calling thread's current CUDA
 * device, for hosts without the CUDA runtime of their own (worker threads
 * that create engines for a device). */
int vgpu_set_device(int32_t device);
int vgpu_get_device(int32_t *device);

/* Advance nsteps time steps (the loop body of src/simulation.c:156-222),
 * continuing from the engine's current step.  Returns once the device has
 * finished. */
int vgpu_run(vgpu_engine *engine, uint64_t nsteps);

/* Receives binary-observer rows of consecutive output steps:
 * rows[(r*num_points + q)*6 + c] is component c (Ex..Hz) of node q at output
 * row first_row + r, rows counting from the window start out_start.  The
 * values are float, as the reference writes them (src/observer.c:1168-1196).
 * `rows` is valid only during the call.  Calls come from the thread running
 * vgpu_run, in row order, while the device computes later steps; the last
 * rows of a run arrive before vgpu_run returns. */
typedef void (*vgpu_bin_sink)(void *user, uint64_t first_row, uint32_t num_rows, int64_t num_points,
                              const float *rows);

/* Install (or, with sink = NULL, remove) the binary-observer sink.  Replaces
 * the per-step fwrite loop of updateImpulseDat (src/observer.c:1164-1198):
 * the device gathers each step's nodes into a ring of 2 x 64 rows and copies
 * every 64-step block to pinned host memory on a second stream. */
int vgpu_set_bin_sink(vgpu_engine *engine, vgpu_bin_sink sink, void *user);

/* Asynchronous stepping, for callers that keep several engines busy on one
 * device (batches, services); the reference runs one mesh per process and
 * has no counterpart.  vgpu_enqueue queues at most max_steps more steps --
 * up to the next 64-step boundary, never past the problem's last step,
 * replayed from captured step graphs of 16, 8, 4, 2 and 1 steps -- on the
 * engine's stream and returns without waiting; *queued receives the count (0 once the problem is
 * done).  Observer folding and binary-row delivery happen as in vgpu_run.
 * vgpu_query returns 1 when the queued work has finished, 0 if it has
 * not, and VGPU_ECUDA when the engine's stream reports a device error;
 * vgpu_synchronize waits for the work and reports any device-side failure. */
int vgpu_enqueue(vgpu_engine *engine, uint64_t max_steps, uint64_t *queued);
int vgpu_query(vgpu_engine *engine);
int vgpu_synchronize(vgpu_engine *engine);

/* Advance n engines of one device by steps[i] each: their blocks are queued
 * round-robin on the engines' own streams, so the device runs them side by
 * side; returns when all have finished.  The batched form of vgpu_run; each
 * engine's results are the ones vgpu_run would give it alone.  If queueing
 * fails for one engine, no further blocks are queued, every engine's queued
 * work is still waited for, and the first error is returned. */
int vgpu_run_batch(vgpu_engine *const *engines, int32_t n, const uint64_t *steps);

/* Grouped stepping: vgpu_run_batch's contract, with the engines that allow
 * it stepped as one group per precision.  Each half step of a group is one
 * sweep launch (per sweep kernel) over the tiles of every member mesh, and
 * one launch each for all members' observer samples, E sources and H
 * sources, replayed from captured step graphs; a member leaves the group
 * when its steps are done (members are ordered by steps left, so a member
 * leaves by shortening the launches' lists).  An engine joins its precision's group when
 * vgpu_groupable says so, it sits at a 64-step boundary and it is on the
 * first engine's device; the others are stepped as vgpu_run_batch steps
 * them, beside the groups.  Every engine's results are the ones vgpu_run
 * gives it alone.  `report` (may be NULL) receives the call's counts. */
typedef struct {
  uint64_t launches;   /* kernels the call launched, grouped and per engine */
  int32_t grouped;     /* engines stepped in groups */
  int32_t rebuilds;    /* changes of a group's membership (members finishing) */
  int64_t tiles;       /* sweep tiles (E + H) of the groups as they started */
  double group_ms;     /* device time of the longest group's work */
} vgpu_group_report;
int vgpu_run_grouped(vgpu_engine *const *engines, int32_t n, const uint64_t *steps, vgpu_group_report *report);

/* 1 if the engine can step in a group: its steps hold only the sweeps,
 * point sources and point observers (no Mur, Debye, SIBC, plane wave,
 * ghost layer or binary observer), and its coefficients are indexed with at
 * most 64 distinct tuples; 0 if not; a negative status on error. */
int vgpu_groupable(const vgpu_engine *engine);

/* Page-locked host memory for read-backs, from blocks the library caches
 * for the process (pinning costs milliseconds per megabyte).  A DFT read
 * (vgpu_read_dft) into such memory goes straight from the device at the
 * link's speed; one into pageable memory is staged and copied on the host,
 * where the copy into freshly allocated pages costs more than the transfer.
 * vgpu_host_alloc returns NULL when no block can be had; vgpu_host_free
 * returns a block to the cache (at most 2 GB are kept). */
void *vgpu_host_alloc(uint64_t bytes);
void vgpu_host_free(void *ptr);

/* Sweep tuning for the engines the calling thread creates afterwards and
 * the groups it runs: march_depth planes per tile (1..32; 0 restores the
 * built-in rule of about 16 tiles per SM), at most blocks_per_sm resident
 * sweep blocks per SM (0: as many as fit) and group_chunk, the tiles a
 * grouped sweep block takes from its launch's counter at a time (1..4096;
 * 0: 4).  Results do not depend on it; vulture_b200/autotune.py chooses it
 * by timing. */
int vgpu_set_sweep_tuning(int32_t march_depth, int32_t blocks_per_sm, int32_t group_chunk);

/* Copy time-domain samples to the host: out[(s*num_td + p)*6 + c] for the
 * first `steps` steps of the output window. */
int vgpu_read_td(vgpu_engine *engine, double *out, uint64_t steps);

/* Copy the running DFTs: re/im[(p*6 + c)*num_freq + f] (src/observer.c:857-899). */
int vgpu_read_dft(vgpu_engine *engine, double *re, double *im);

/* Copy one field component volume (0..5) to the host in the volume layout. */
int vgpu_read_field(vgpu_engine *engine, int32_t component, double *out);

/* Overwrite one field component volume (used to plant host-prepared state). */
int vgpu_write_field(vgpu_engine *engine, int32_t component, const double *in);

/* Scan all fields for NaN/Inf on the device; returns VGPU_ENONFINITE if any. */
int vgpu_check_finite(vgpu_engine *engine);

uint64_t vgpu_current_step(const vgpu_engine *engine);

/* Sweep launches of one time step, for vgpu_time_kernel and
 * vgpu_sweep_points.  Without UPML regions the bulk kernel's launch takes
 * every tile of a half step.  With them the UPML kernel's launch does (bulk
 * tiles, the X and Y regions' tiles, and the bulk-footprint tiles whose rows
 * reach into a Z region), and the bulk kernel's launch is empty: its point
 * counts are 0 and timing it is an error. */
enum { VGPU_K_BULK_E = 0, VGPU_K_BULK_H = 1, VGPU_K_PML_E = 2, VGPU_K_PML_H = 3 };

/* The other parts of a time step, in their order within the step
 * (src/simulation.c:156-222), and the DFT fold of one 64-step block
 * (src/observer.c:857-899), for vgpu_time_kernel.  Each part is the launch
 * (or launches: one per source or plane wave) of that update as the step
 * makes it: where vgpu_stats.merged_parts shows a merge, VGPU_K_DEBYE also
 * applies the E corrections and VGPU_K_TFSF_H also takes the next step's
 * samples, and VGPU_K_OBSERVE (or VGPU_K_TFSF_E without an auxiliary grid)
 * launches nothing.  Timing a part with no launch is an error. */
enum {
  VGPU_K_OBSERVE = 4, VGPU_K_BIN_OBSERVE = 5, VGPU_K_MUR_E = 6, VGPU_K_DEBYE = 7, VGPU_K_SIBC_E = 8,
  VGPU_K_SOURCES_E = 9, VGPU_K_TFSF_E = 10, VGPU_K_GHOST_E = 11, VGPU_K_MUR_H = 12, VGPU_K_SIBC_H = 13,
  VGPU_K_SOURCES_H = 14, VGPU_K_TFSF_H = 15, VGPU_K_GHOST_H = 16, VGPU_K_DFT_BLOCK = 17,
  /* Timing only, never part of a step: the same 64-row DFT fold by the
   * scalar kernel (one thread per point-component and frequency) that the
   * engine's tensor-core fold replaced, for comparison. */
  VGPU_K_DFT_BLOCK_SCALAR = 18
};

/* Field points one sweep kernel updates per launch with the bulk formula
 * and with the UPML formula. */
int vgpu_sweep_points(const vgpu_engine *engine, int32_t kernel, uint64_t *bulk_points, uint64_t *pml_points);

/* Profiling hook: launch one of the step's kernels (VGPU_K_*) `iters`
 * times on the engine's stream (after `warmup` untimed launches) and report
 * the mean device time per launch from CUDA events, plus the number of field
 * points a sweep updates per launch (0 for the other parts).  It advances
 * the state it updates, so call it only when the run's results are no
 * longer needed. */
int vgpu_time_kernel(vgpu_engine *engine, int32_t kernel, int32_t warmup, int32_t iters, double *ms_per_launch,
                     uint64_t *points);
int vgpu_get_stats(const vgpu_engine *engine, vgpu_stats *stats);
void vgpu_destroy(vgpu_engine *engine);

/* Allocation-free running DFT.  No counterpart in the reference; it serves
 * callers that cannot allocate device memory themselves (a host framework
 * that owns every allocation, or code running where cudaMalloc is not
 * allowed).  It adds num_rows rows of samples to running DFT sums:
 *   re[s*num_freq + f] += x * cos(omega[f] * t_r)
 *   im[s*num_freq + f] -= x * sin(omega[f] * t_r)
 * for x = samples[r*num_series + s] and t_r = (first_step + r) * dt, in row
 * order -- the observer DFT of src/observer.c:857-899.  All pointers are
 * device pointers owned by the caller.  It calls no cudaMalloc or cudaFree:
 * its twiddle table is a file-scope __device__ array of
 * VGPU_STATIC_DFT_MAX_ENTRIES double2 (1 MiB), held on every GPU that loads
 * the library until exit, and rows * freqs beyond that, more than
 * VGPU_STATIC_DFT_MAX_ROWS rows or more than VGPU_STATIC_DFT_MAX_SERIES
 * series (8 series per block row of the launch grid, at most 65535 rows) are
 * rejected with VGPU_EINVAL.  The first
 * call on a device looks up the table's device address; make that call
 * before any stream capture.  Calls share the one table, so calls that
 * overlap on the GPU race; each call runs on the default stream and returns
 * after it has finished. */
#define VGPU_STATIC_DFT_MAX_ENTRIES 65536
#define VGPU_STATIC_DFT_MAX_ROWS 256
#define VGPU_STATIC_DFT_MAX_SERIES (65535 * 8)
int vgpu_dft_accumulate_static(const double *samples, int32_t num_series, int32_t num_rows, const double *omega,
                               int32_t num_freq, double dt, uint64_t first_step, double *re, double *im);

/* No counterpart in the reference.  Test hook for the failure path of the
 * sweeps: the number of polls a sweep's compute warps make on a stage's data
 * barrier before they give up (0: give up at once; a negative value restores
 * the default bound of about a second).  A sweep whose wait runs out records
 * it, its blocks wait for their loads in flight and leave, later sweep
 * launches of the engine skip their work, and vgpu_run returns
 * VGPU_ETIMEOUT.  The setting belongs to the current device and holds for
 * every engine on it; change it only while none of them is stepping. */
int vgpu_set_sweep_wait_limit(int64_t polls);

/* Message of the last error on this thread. */
const char *vgpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* VGPU_H */
