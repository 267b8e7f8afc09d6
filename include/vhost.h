/*
 * vhost.h -- C ABI of the vulture_b200 host side: reading a Vulture .mesh
 * file, the solver set-up, and writing the observer files.
 *
 * Together with vgpu.h this is a drop-in for the reference's solver path:
 *   vhost_load()            replaces src/vulture.c:77-148 (parse + init*),
 *   vgpu_create/vgpu_run    replace propagate() (src/simulation.c:136-231),
 *   vhost_write_outputs()   replaces deallocObservers() (src/observer.c:653-700)
 *                           and the per-step text writes of updateObservers()
 *                           (src/observer.c:622-650, 760-798).
 * vhost_main() is the whole command line (src/vulture.c:200-281).
 *
 * Errors are returned as negative codes with a message from
 * vhost_last_error(); nothing here calls exit().
 */
#ifndef VHOST_H
#define VHOST_H

#include <stdint.h>
#include "vgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vhost vhost;

/* Parse a mesh file and run the reference's set-up sequence.  log_path may be
 * NULL (no log) or a file name such as "vulture.log".  verbose selects the
 * reference's -v debug lines. */
int vhost_load(const char *mesh_path, const char *log_path, int verbose, vhost **out);

/* The engine input for this mesh.  The pointer and all arrays it references
 * stay valid until vhost_free(). */
int vhost_problem(vhost *h, int32_t precision, const vgpu_problem **out);

/* Sizes of the output buffers the problem needs. */
uint64_t vhost_num_steps(const vhost *h);
uint64_t vhost_num_output_steps(const vhost *h);
int32_t vhost_num_td(const vhost *h);
int32_t vhost_num_fd(const vhost *h);
int32_t vhost_num_freq(const vhost *h);
double vhost_dt(const vhost *h);
/* Outer-box cell count, the reference's spi/cell denominator (src/timer.c:95). */
uint64_t vhost_num_cells(const vhost *h);

/* No counterpart in the reference.  The set-up paints a one-byte medium tag
 * per cell and component beside the coefficient volumes and hands both to
 * the engine (vgpu_problem.coef_tag).  use = 0 leaves the tags out of the
 * problem, so that the engine finds the coefficient tuples by scanning the
 * volumes; use = 1 puts them back.  The engine's results are the same either
 * way. */
int vhost_use_tags(vhost *h, int32_t use);

/* No counterpart in the reference.  The number of (cell, component) pairs
 * whose tag does not give the coefficient volumes' values bit for bit; -1
 * when the set-up keeps no tags (more than 255 distinct coefficient
 * triples). */
int64_t vhost_check_tags(const vhost *h);

/* Write eh_<name>_td.asc / eh_<name>_fd.asc / wf_<name>_td.asc /
 * wf_<name>_fd.asc into the current directory from the engine's samples
 * (td: [steps][num_td][6]) and DFTs (re/im: [num_fd][6][num_freq]).
 * full_precision=1 prints 17 significant digits instead of the reference's
 * %16.8e so results can be compared at 1e-12. */
int vhost_write_outputs(vhost *h, const double *td, uint64_t td_steps, const double *dft_re,
                        const double *dft_im, int32_t full_precision);

/* Binary (TDOM_BINARY) observers (src/observer.c:1016-1212).  Nodes over
 * all binary observers; 0 when there are none. */
int64_t vhost_num_bin(const vhost *h);

/* Write impulse.dat's header, excite.dat and process.dat into the current
 * directory (initBinaryObservers, src/observer.c:1031-1151) and keep
 * impulse.dat open for vhost_bin_sink.  A no-op without binary observers. */
int vhost_bin_begin(vhost *h, int32_t full_precision);

/* A vgpu_bin_sink (pass the vhost as `user`): appends the rows to impulse.dat
 * in the reference's record layout (updateImpulseDat,
 * src/observer.c:1164-1198). */
void vhost_bin_sink(void *user, uint64_t first_row, uint32_t num_rows, int64_t num_points, const float *rows);

/* Close impulse.dat; an error if any record failed to write. */
int vhost_bin_end(vhost *h);

/* xlines.dat, ylines.dat, zlines.dat: the mesh lines that the reference's
 * grid set-up writes (src/grid.c:942-944). */
int vhost_write_lines(vhost *h);

/* Name of observer slot p of the time- (fd=0) or frequency-domain (fd=1) list. */
const char *vhost_observer_name(const vhost *h, int32_t fd, int32_t p);

void vhost_free(vhost *h);
const char *vhost_last_error(void);

/* The vulture command line: vulture [-v] [-m] [-p] [-g] [-n N] mesh, plus
 * --fp32 (FP32 storage) and --full-precision (17-digit text).  Returns the
 * process exit status the reference would use (0, 1 or 6). */
int vhost_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif

#endif
