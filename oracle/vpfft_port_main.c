/*
 * vpfft_port_main.c -- command-line driver of the plain-C restatement with the
 * same input file and output files as ref_harness.cpp (see oracle/refio.py),
 * so tests can run either oracle interchangeably.  TEST ORACLE ONLY.
 *
 * Usage: vpfft_port <input.bin> <outdir> [--dump-iter K]... [--dump-increments] [--quiet]
 */
#define _POSIX_C_SOURCE 199309L
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "vpfft_oracle.h"

static void die(const char *m) {
  fprintf(stderr, "vpfft_port: %s\n", m);
  exit(2);
}

static void rd(FILE *f, void *p, size_t sz, size_t n) {
  if (fread(p, sz, n, f) != n) die("truncated input");
}

static void wr(const char *dir, const char *name, const double *p, size_t n) {
  char path[4096];
  snprintf(path, sizeof(path), "%s/%s", dir, name);
  FILE *f = fopen(path, "wb");
  if (!f) die("cannot write output");
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct {
  oracle_grid *g;
  size_t n;
  const char *outdir;
  int increment;
  int ndump;
  int dump[64];
  double *allreduce;
  size_t nar, cap;
  double *fwd_times, *fwd_inc;
  size_t nfwd, capfwd;
} ctx_t;

static void push(ctx_t *c, double v) {
  if (c->nar == c->cap) {
    c->cap = c->cap ? 2 * c->cap : 4096;
    c->allreduce = (double *)realloc(c->allreduce, sizeof(double) * c->cap);
  }
  c->allreduce[c->nar++] = v;
}

static void push_fwd(ctx_t *c) {
  if (c->nfwd == c->capfwd) {
    c->capfwd = c->capfwd ? 2 * c->capfwd : 256;
    c->fwd_times = (double *)realloc(c->fwd_times, sizeof(double) * c->capfwd);
    c->fwd_inc = (double *)realloc(c->fwd_inc, sizeof(double) * c->capfwd);
  }
  c->fwd_times[c->nfwd] = now_s();
  c->fwd_inc[c->nfwd] = c->increment;
  c->nfwd++;
}

static void dump_state(ctx_t *c, int iter) {
  double *buf = (double *)malloc(sizeof(double) * 5 * c->n);
  const char *names[4] = {"P", "dtilde", "sigma", "lambda"};
  for (int k = 0; k < 4; ++k) {
    char fn[64];
    snprintf(fn, sizeof(fn), "it%d_%s.bin", iter, names[k]);
    oracle_grid_get(c->g, names[k], buf);
    wr(c->outdir, fn, buf, 5 * c->n);
  }
  free(buf);
}

static int wants(ctx_t *c, int iter) {
  for (int i = 0; i < c->ndump; ++i)
    if (c->dump[i] == iter) return 1;
  return 0;
}

static void on_iter(int iter, const double sums[12], void *user) {
  ctx_t *c = (ctx_t *)user;
  if (!sums) { /* initialisation done, before the first fixed-point iteration */
    if (c->increment == 0 && wants(c, 0)) dump_state(c, 0);
    return;
  }
  for (int i = 0; i < 12; ++i) push(c, sums[i]);
  push_fwd(c); /* the next forward FFT would start here */
  if (c->increment == 0 && wants(c, iter + 1)) dump_state(c, iter + 1);
}

int main(int argc, char **argv) {
  if (argc < 3) die("usage: vpfft_port <input.bin> <outdir> [--dump-iter K]... [--quiet]");
  ctx_t c;
  memset(&c, 0, sizeof(c));
  c.outdir = argv[2];
  int dump_increments = 0;
  for (int a = 3; a < argc; ++a) {
    if (!strcmp(argv[a], "--dump-iter") && a + 1 < argc && c.ndump < 64)
      c.dump[c.ndump++] = atoi(argv[++a]);
    else if (!strcmp(argv[a], "--dump-increments"))
      dump_increments = 1;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) die("cannot open input");
  char magic[8];
  rd(f, magic, 1, 8);
  if (memcmp(magic, "VPFFTIN1", 8)) die("bad magic");
  int32_t hdr[8];
  rd(f, hdr, 4, 8);
  int nx = hdr[0], ny = hdr[1], nz = hdr[2], nsteps = hdr[3], max_iter = hdr[4],
      per_voxel = hdr[5], edot_per_increment = hdr[6];
  double dt, eps, edot[5], h[3];
  rd(f, &dt, 8, 1);
  rd(f, &eps, 8, 1);
  rd(f, edot, 8, 5);
  rd(f, h, 8, 3);
  oracle_material mat;
  int32_t ne[12];
  rd(f, mat.gamma_dot_base, 8, 12);
  rd(f, ne, 4, 12);
  for (int i = 0; i < 12; ++i) mat.rate_sensitivity[i] = ne[i];
  rd(f, mat.tau0, 8, 12);
  rd(f, mat.tau1, 8, 12);
  rd(f, mat.theta0, 8, 12);
  rd(f, mat.theta1, 8, 12);
  rd(f, mat.hardening, 8, 144);
  size_t n = (size_t)nx * ny * nz;
  double *R = (double *)malloc(sizeof(double) * 9 * n);
  double *sig = (double *)malloc(sizeof(double) * 5 * n);
  size_t ncrss = per_voxel ? 12 * n : 12;
  double *crss = (double *)malloc(sizeof(double) * ncrss);
  rd(f, R, 8, 9 * n);
  rd(f, sig, 8, 5 * n);
  rd(f, crss, 8, ncrss);
  double *edot_steps = NULL;
  if (edot_per_increment) {
    edot_steps = (double *)malloc(sizeof(double) * 5 * (size_t)nsteps);
    rd(f, edot_steps, 8, 5 * (size_t)nsteps);
  }
  fclose(f);

  oracle_grid *g = oracle_grid_create(nx, ny, nz, &mat);
  oracle_grid_set(g, R, sig, crss, per_voxel, h);
  c.g = g;
  c.n = n;
  oracle_grid_set_iter_hook(g, on_iter, &c);

  double *steps = (double *)malloc(sizeof(double) * 6 * (size_t)nsteps);
  double *counts = (double *)malloc(sizeof(double) * (size_t)nsteps);
  double *secs = (double *)malloc(sizeof(double) * (size_t)nsteps);
  for (int s = 0; s < nsteps; ++s) {
    c.increment = s;
    size_t ar0 = c.nar;
    double t0 = now_s();
    /* the increment's first 25 reduced values are L0; they are known only
     * after the call, so reserve them and fill in afterwards */
    for (int i = 0; i < 25; ++i) push(&c, 0.0);
    double avg[5];
    push_fwd(&c);
    if (edot_steps) memcpy(edot, edot_steps + 5 * (size_t)s, sizeof(edot));
    int it = oracle_grid_run_increment(g, edot, max_iter, dt, eps, avg);
    double t1 = now_s();
    if (it < 0) die("MaxRSS < 1e-10 during initialisation");
    double sums[25];
    oracle_grid_get(g, "L0_sums", sums);
    memcpy(c.allreduce + ar0, sums, sizeof(sums));
    steps[6 * s] = it;
    memcpy(steps + 6 * s + 1, avg, sizeof(avg));
    counts[s] = (double)(c.nar - ar0);
    secs[s] = t1 - t0;
    if (dump_increments) {
      const char *names[4] = {"sigma", "lambda", "R", "crss"};
      const size_t widths[4] = {5, 5, 9, 12};
      double *buf = (double *)malloc(sizeof(double) * 12 * n);
      for (int k = 0; k < 4; ++k) {
        char fn[64];
        snprintf(fn, sizeof(fn), "inc%d_%s.bin", s, names[k]);
        oracle_grid_get(g, names[k], buf);
        wr(c.outdir, fn, buf, widths[k] * n);
      }
      free(buf);
    }
  }
  const char *od = c.outdir;
  wr(od, "steps.bin", steps, 6 * (size_t)nsteps);
  wr(od, "allreduce.bin", c.allreduce, c.nar);
  wr(od, "allreduce_counts.bin", counts, (size_t)nsteps);
  wr(od, "step_seconds.bin", secs, (size_t)nsteps);
  wr(od, "fwd_times.bin", c.fwd_times, c.nfwd);
  wr(od, "fwd_increment.bin", c.fwd_inc, c.nfwd);
  double *buf = (double *)malloc(sizeof(double) * 60 * n);
  struct {
    const char *name, *file;
    size_t w;
  } outs[] = {{"sigma", "sigma.bin", 5},       {"lambda", "lambda.bin", 5},
              {"R", "R.bin", 9},               {"crss", "crss.bin", 12},
              {"accshear", "accshear.bin", 1}, {"P", "P_last.bin", 5},
              {"dtilde", "dtilde_last.bin", 5}, {"schmid", "schmid.bin", 60}};
  for (size_t k = 0; k < sizeof(outs) / sizeof(outs[0]); ++k) {
    oracle_grid_get(g, outs[k].name, buf);
    wr(od, outs[k].file, buf, outs[k].w * n);
  }
  double hv[3];
  oracle_grid_get(g, "voxlen", hv);
  wr(od, "voxlen.bin", hv, 3);
  printf("{\"increments\": %d, \"iters\": [", nsteps);
  for (int s = 0; s < nsteps; ++s) printf("%s%d", s ? ", " : "", (int)steps[6 * s]);
  printf("], \"seconds\": [");
  for (int s = 0; s < nsteps; ++s) printf("%s%.6f", s ? ", " : "", secs[s]);
  printf("]}\n");
  oracle_grid_free(g);
  return 0;
}
