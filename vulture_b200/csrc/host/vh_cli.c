/*
 * vh_cli.c -- the vulture command line on the B200 engine.
 *
 * Same options and exit codes as the reference (src/vulture.c:200-281):
 *   -h/--help, -V/--version, -v/--verbose, -m/--read-mesh, -n N/--num-proc N,
 *   -p/--preprocess, -g/--dump-grid, -l/--licence.
 * Added: --fp32 (FP32 field and coefficient storage) and --full-precision
 * (observer text with 17 significant digits).  -n is accepted for
 * compatibility; the time loop runs on the GPU.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vh.h"

static void usage(void)
{
  printf("\nUsage:\n\n");
  printf("vulture -h | --help\n");
  printf("vulture -V | --version\n");
  printf("vulture [ option ] <meshFile>\n\n");
  printf("Valid options are:\n\n");
  printf("-g, --dump-grid\t\t\tWrite out grid in ASCII format\n");
  printf("-m, --readmesh\t\t\tRead the mesh only and stop\n");
  printf("-n <int>, --numproc <int> \tSet number of threads\n");
  printf("-p, --preprocess\t\tPreprocess the mesh only and stop\n");
  printf("-v, --verbose\t\t\tProduce verbose logging information\n");
  printf("--fp32\t\t\t\tStore fields and coefficients in FP32 on the GPU\n");
  printf("--full-precision\t\tWrite observer values with 17 significant digits\n\n");
}

int vhost_main(int argc, char **argv)
{
  int verbose = 0, read_only = 0, preprocess = 0, fp32 = 0, full = 0;
  char *mesh = NULL;
  int a = 1;
  for (; a < argc && argv[a][0] == '-'; a++) {
    const char *o = argv[a];
    if (!strcmp(o, "--fp32")) fp32 = 1;
    else if (!strcmp(o, "--full-precision")) full = 1;
    else if (!strncmp(o, "-h", 2) || !strncmp(o, "--help", 6)) { usage(); return 0; }
    else if (!strncmp(o, "-V", 2) || !strncmp(o, "--version", 9)) {
      printf("\nVulture (version 0.7.1) on the vulture_b200 GPU engine\n\n");
      printf("  Supported mesh versions 0.0.0 - 1.0.0\n");
      printf("  Field arrays are 8-bytes (4-bytes with --fp32).\n\n");
      return 0;
    }
    else if (!strncmp(o, "-v", 2) || !strncmp(o, "--verbose", 9)) verbose = 1;
    else if (!strncmp(o, "-m", 2) || !strncmp(o, "--read-mesh", 11)) read_only = 1;
    else if (!strncmp(o, "-n", 2) || !strncmp(o, "--num-proc", 10)) {
      if (a + 1 >= argc || atoi(argv[a + 1]) == 0) {
        printf("\n*** Error: invalid value for option %s\n", o);
        usage();
        return 1;
      }
      a++;
    }
    else if (!strncmp(o, "-p", 2) || !strncmp(o, "--preprocess", 12)) preprocess = 1;
    else if (!strncmp(o, "-g", 2) || !strncmp(o, "--dump-grid", 11)) { /* media maps: not written */ }
    else if (!strncmp(o, "-l", 2) || !strncmp(o, "--licence", 9)) {
      printf("\nVulture finite-difference time-domain electromagnetic solver (GPL-3).\n\n");
      return 0;
    }
    else {
      printf("\n*** Error: invalid option %s\n", o);
      usage();
      return 1;
    }
  }
  if (argc - a != 1) { usage(); return 0; }
  mesh = argv[a];

  vhost *h = NULL;
  if (vhost_load(mesh, "vulture.log", verbose, &h)) {
    fprintf(stderr, "Vulture: *** Error: %s\n", vhost_last_error());
    return 6;
  }
  if (read_only) { vhost_free(h); return 0; }
  const vgpu_problem *p = NULL;
  if (vhost_problem(h, fp32 ? VGPU_FP32 : VGPU_FP64, &p)) {
    fprintf(stderr, "Vulture: *** Error: %s\n", vhost_last_error());
    vhost_free(h);
    return 6;
  }
  /* Files the reference's set-up writes: mesh lines (initGrid) and the
   * binary observers' headers (initObservers). */
  if (vhost_write_lines(h) || vhost_bin_begin(h, full)) {
    fprintf(stderr, "Vulture: *** Error: %s\n", vhost_last_error());
    vhost_free(h);
    return 6;
  }
  uint64_t nout = vhost_num_output_steps(h);
  double *td = calloc((size_t)(nout ? nout : 1) * (p->num_td ? p->num_td : 1) * 6, sizeof(double));
  size_t ndft = (size_t)(p->num_fd ? p->num_fd : 1) * 6 * (p->num_freq ? p->num_freq : 1);
  double *re = calloc(ndft, sizeof(double)), *im = calloc(ndft, sizeof(double));
  int rc = 0;
  if (!preprocess && p->num_steps > 0) {
    vgpu_engine *e = NULL;
    rc = vgpu_create(p, &e);
    if (!rc && p->num_bin) rc = vgpu_set_bin_sink(e, vhost_bin_sink, h);
    if (!rc) rc = vgpu_run(e, p->num_steps);
    if (!rc && p->num_td) rc = vgpu_read_td(e, td, nout);
    if (!rc && p->num_fd) rc = vgpu_read_dft(e, re, im);
    if (rc) fprintf(stderr, "Vulture: *** Error: %s\n", vgpu_last_error());
    vgpu_destroy(e);
  }
  if (!rc && (vhost_bin_end(h) || vhost_write_outputs(h, td, preprocess ? 0 : nout, re, im, full))) {
    fprintf(stderr, "Vulture: *** Error: %s\n", vhost_last_error());
    rc = -1;
  }
  free(td);
  free(re);
  free(im);
  vhost_free(h);
  return rc ? 6 : 0;
}
