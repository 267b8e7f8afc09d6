/*
 * vgpu_on_oracle.c -- ORACLE (test infrastructure): the five vgpu entry
 * points propagate_gpu.c calls (vgpu_create, vgpu_run, vgpu_read_td,
 * vgpu_destroy, vgpu_last_error), implemented on the CPU oracle
 * (oracle/vcpu.c, FP64) instead of the GPU engine.  Linked into the
 * variant vulture_ref_oracle_shim, it lets the CPU test suite check, with no
 * GPU, that propagate_gpu.c hands the engine the state the reference built:
 * that variant's observer files must equal the reference's own byte for byte.
 */
#include <stdint.h>
#include <stdlib.h>

#include "vgpu.h"

void *vcpu64_create(const vgpu_problem *p);
void vcpu64_destroy(void *h);
int vcpu64_run(void *h, uint64_t nsteps);
int vcpu64_read_td(void *h, double *out, uint64_t steps);

struct vgpu_engine {
  void *h;
};

int vgpu_create(const vgpu_problem *problem, vgpu_engine **engine)
{
  vgpu_engine *e = malloc(sizeof *e);
  if (!e) return VGPU_ENOMEM;
  e->h = vcpu64_create(problem);
  if (!e->h) {
    free(e);
    return VGPU_EINVAL;
  }
  *engine = e;
  return VGPU_OK;
}

int vgpu_run(vgpu_engine *engine, uint64_t nsteps) { return vcpu64_run(engine->h, nsteps); }

int vgpu_read_td(vgpu_engine *engine, double *out, uint64_t steps) { return vcpu64_read_td(engine->h, out, steps); }

void vgpu_destroy(vgpu_engine *engine)
{
  if (!engine) return;
  vcpu64_destroy(engine->h);
  free(engine);
}

const char *vgpu_last_error(void) { return "oracle engine"; }
