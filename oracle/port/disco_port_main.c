/*
 * Command-line driver of the C restatement (oracle; test infrastructure only).
 * Same modes, options and dump formats as oracle/ref_driver.c, so the tests
 * and the CPU baseline run either oracle interchangeably:
 *   disco_port run <par> <nsteps> <out.bin> [--load in.bin] [--faces f.bin]
 *                  [--dtlog log.txt] [--warmup W]
 *   disco_port stage <par> <phase> <out.bin> [--load in.bin]   (phase 0-15)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "disco_port.h"

static void wr(FILE *f, const void *p, size_t sz, size_t n) {
  if (fwrite(p, sz, n, f) != n) {
    fprintf(stderr, "write failed\n");
    exit(2);
  }
}
static void rd(FILE *f, void *p, size_t sz, size_t n) {
  if (fread(p, sz, n, f) != n) {
    fprintf(stderr, "read failed\n");
    exit(2);
  }
}

static void dump_state(const char *path, const Port *p, int ext) {
  FILE *f = fopen(path, "wb");
  int hdr[5] = {p->NR, 1, p->NQ, p->N, ext}, i, n, q;
  double td[2] = {p->t, p->dt}, g[12];
  if (!f) exit(2);
  wr(f, "DSTATE1", 1, 8);
  wr(f, hdr, sizeof(int), 5);
  wr(f, td, sizeof(double), 2);
  for (i = 0; i < 2; ++i) {
    g[6 * i + 0] = p->gr[i]; g[6 * i + 1] = p->gphi[i]; g[6 * i + 2] = p->gM[i];
    g[6 * i + 3] = p->gom[i]; g[6 * i + 4] = p->mdot[i]; g[6 * i + 5] = p->macc[i];
  }
  wr(f, g, sizeof(double), 12);
  wr(f, p->N_p, sizeof(int), (size_t)p->NR);
  wr(f, p->rf, sizeof(double), (size_t)p->NR + 1);
  for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) wr(f, &p->prim[q][n], sizeof(double), 1);
  for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) wr(f, &p->cons[q][n], sizeof(double), 1);
  wr(f, p->tiph, sizeof(double), (size_t)p->N);
  wr(f, p->dphi, sizeof(double), (size_t)p->N);
  if (ext) {
    for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) wr(f, &p->grad[q][n], sizeof(double), 1);
    for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) wr(f, &p->gradp[q][n], sizeof(double), 1);
    wr(f, p->wiph, sizeof(double), (size_t)p->N);
    for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) wr(f, &p->rkcons[q][n], sizeof(double), 1);
    wr(f, p->rktiph, sizeof(double), (size_t)p->N);
  }
  fclose(f);
}

static void load_state(const char *path, Port *p) {
  FILE *f = fopen(path, "rb");
  char magic[8];
  int hdr[5], n, q;
  double skip[14], *buf;
  if (!f) exit(2);
  rd(f, magic, 1, 8);
  rd(f, hdr, sizeof(int), 5);
  if (memcmp(magic, "DSTATE1", 8) != 0 || hdr[0] != p->NR || hdr[2] != p->NQ || hdr[3] != p->N) {
    fprintf(stderr, "state file %s does not match the parfile grid\n", path);
    exit(2);
  }
  rd(f, skip, sizeof(double), 14);
  buf = malloc(sizeof(double) * ((size_t)p->NR + 1 + (size_t)p->N * p->NQ));
  rd(f, buf, sizeof(int), (size_t)p->NR);
  rd(f, buf, sizeof(double), (size_t)p->NR + 1);
  for (n = 0; n < p->N; ++n) for (q = 0; q < p->NQ; ++q) rd(f, &p->prim[q][n], sizeof(double), 1);
  rd(f, buf, sizeof(double), (size_t)p->N * p->NQ);
  rd(f, p->tiph, sizeof(double), (size_t)p->N);
  rd(f, p->dphi, sizeof(double), (size_t)p->N);
  free(buf);
  fclose(f);
  port_calc_cons(p);
}

static void dump_faces(const char *path, Port *p) {
  FILE *f = fopen(path, "wb");
  int n;
  if (!f) exit(2);
  port_build_faces(p);
  wr(f, "DFACES1", 1, 8);
  wr(f, &p->NR, sizeof(int), 1);
  wr(f, &p->nf, sizeof(int), 1);
  wr(f, p->nri, sizeof(int), (size_t)p->NR);
  wr(f, p->fL, sizeof(int), (size_t)p->nf);
  wr(f, p->fR, sizeof(int), (size_t)p->nf);
  wr(f, p->fr, sizeof(double), (size_t)p->nf);
  wr(f, p->fdphi, sizeof(double), (size_t)p->nf);
  wr(f, p->fdA, sizeof(double), (size_t)p->nf);
  wr(f, p->fdl, sizeof(double), (size_t)p->nf);
  wr(f, p->fdr, sizeof(double), (size_t)p->nf);
  wr(f, p->fcm, sizeof(double), (size_t)p->nf);
  (void)n;
  fclose(f);
}

int main(int argc, char **argv) {
  const char *mode, *par, *out, *load = NULL, *faces = NULL, *dtlog = NULL;
  int n, a, s, warmup = 0;
  Port P;
  if (argc < 5) {
    fprintf(stderr, "usage: disco_port run|stage <parfile> <nsteps|phase> <out.bin> [options]\n");
    return 2;
  }
  mode = argv[1];
  par = argv[2];
  n = atoi(argv[3]);
  out = argv[4];
  for (a = 5; a < argc; ++a) {
    if (!strcmp(argv[a], "--load") && a + 1 < argc) load = argv[++a];
    else if (!strcmp(argv[a], "--faces") && a + 1 < argc) faces = argv[++a];
    else if (!strcmp(argv[a], "--dtlog") && a + 1 < argc) dtlog = argv[++a];
    else if (!strcmp(argv[a], "--warmup") && a + 1 < argc) warmup = atoi(argv[++a]);
    else {
      fprintf(stderr, "unknown option %s\n", argv[a]);
      return 2;
    }
  }
  memset(&P, 0, sizeof(P));
  if (port_read_parfile(&P, par) || port_setup(&P)) return 3;
  if (load) load_state(load, &P);
  if (!strcmp(mode, "run")) {
    FILE *flog = dtlog ? fopen(dtlog, "w") : NULL;
    struct timespec t0, t1;
    if (faces) dump_faces(faces, &P);
    for (s = 0; s < warmup; ++s) port_step_rk2(&P);
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (s = 0; s < n; ++s) {
      port_step_rk2(&P);
      if (flog) fprintf(flog, "%.17g %.17g\n", P.t, P.dt);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    fprintf(stderr, "steps_wall_s %.9f\n", (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec));
    if (flog) fclose(flog);
    dump_state(out, &P, 0);
  } else if (!strcmp(mode, "stage")) {
    port_stage(&P, n);
    dump_state(out, &P, 1);
  } else {
    return 2;
  }
  port_free(&P);
  return 0;
}
