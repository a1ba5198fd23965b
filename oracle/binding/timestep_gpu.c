/*
 * timestep_rk2 on the B200 library with the reference's own signature
 * (src/TimeStep/timestep_algorithm.c:11-41), so that the loop of
 * src/main.c:124-141 keeps its shape: only the called function's name
 * changes.  Compiled with the reference's headers, on the Disco2 side.
 *
 * The disk's state lives in one library context.  The first call uploads the
 * reference's cells (cell_pack), GravMasses and t; every call then runs
 * dgpu_step_rk2 and, unless lazy, brings the new state back into the
 * reference's structures, so that whatever runs between two steps
 * (diagnostics_set, io_setbuf) reads what timestep_rk2 would have left.
 */
#define CELL_PRIVATE_DEFS
#define PLANET_PRIVATE_DEFS
#define TIMESTEP_PRIVATE_DEFS
#include <stdio.h>
#include <stdlib.h>

#include "Headers/Cell.h"
#include "Headers/GravMass.h"
#include "Headers/MPIsetup.h"
#include "Headers/Sim.h"
#include "Headers/TimeStep.h"
#include "Headers/header.h"
#include "cell_pack.h"
#include "disco_gpu.h"
#include "timestep_gpu.h"

static struct {
  dgpu_sim *sim;
  dgpu_ctx *ctx;
  int uploaded, lazy, N, NQ;
  double *prim, *cons, *tiph, *dphi;
} G;

static void die(const char *what, const char *msg) {
  fprintf(stderr, "%s: %s\n", what, msg ? msg : "");
  exit(1);
}

int timestep_gpu_open(const char *parfile, int device, int fused) {
  int rc = dgpu_sim_from_parfile(parfile, &G.sim);
  if (rc != DGPU_OK) {
    fprintf(stderr, "dgpu_sim_from_parfile: %s\n", dgpu_last_error(NULL));
    return rc;
  }
  rc = dgpu_create((const dgpu_sim *const *)&G.sim, 1, device, NULL, &G.ctx);
  if (rc != DGPU_OK) {
    fprintf(stderr, "dgpu_create: %s\n", dgpu_last_error(NULL));
    return rc;
  }
  if (fused && (rc = dgpu_set_fused(G.ctx, 1)) != DGPU_OK) {
    fprintf(stderr, "dgpu_set_fused: %s\n", dgpu_last_error(G.ctx));
    return rc;
  }
  G.uploaded = 0;
  return DGPU_OK;
}

static void upload(struct TimeStep *ts, struct Sim *s, struct Cell ***cells, struct GravMass *gm) {
  double g6[12];
  int p;
  if (!G.prim) {
    G.N = cell_pack_count(s);
    G.NQ = sim_NUM_Q(s);
    if (dgpu_sim_num_cells(G.sim) != G.N) die("timestep_rk2_gpu", "the library's grid differs from the reference's");
    G.prim = (double *)malloc(sizeof(double) * (size_t)G.N * (size_t)G.NQ);
    G.cons = (double *)malloc(sizeof(double) * (size_t)G.N * (size_t)G.NQ);
    G.tiph = (double *)malloc(sizeof(double) * (size_t)G.N);
    G.dphi = (double *)malloc(sizeof(double) * (size_t)G.N);
    if (!G.prim || !G.cons || !G.tiph || !G.dphi) die("timestep_rk2_gpu", "out of host memory");
  }
  cell_pack(cells, s, G.prim, G.tiph, G.dphi);
  for (p = 0; p < 2; ++p) {
    g6[6 * p + 0] = gm[p].r;
    g6[6 * p + 1] = gm[p].phi;
    g6[6 * p + 2] = gm[p].M;
    g6[6 * p + 3] = gm[p].omega;
    g6[6 * p + 4] = gm[p].Mdot;
    g6[6 * p + 5] = gm[p].Macc;
  }
  if (dgpu_set_state(G.ctx, 0, G.prim, G.tiph, G.dphi) != DGPU_OK || dgpu_set_gravmass(G.ctx, 0, g6) != DGPU_OK ||
      dgpu_set_time(G.ctx, 0, timestep_get_t(ts)) != DGPU_OK)
    die("timestep_rk2_gpu: state upload", dgpu_last_error(G.ctx));
  G.uploaded = 1;
}

void timestep_gpu_sync(struct Sim *s, struct Cell ***cells, struct GravMass *gm) {
  double g6[12];
  int p;
  if (!G.uploaded) return;
  if (dgpu_get_state(G.ctx, 0, G.prim, G.cons, G.tiph, G.dphi) != DGPU_OK ||
      dgpu_get_gravmass(G.ctx, 0, g6) != DGPU_OK)
    die("timestep_rk2_gpu: state download", dgpu_last_error(G.ctx));
  cell_unpack(cells, s, G.prim, G.cons, G.tiph, G.dphi);
  for (p = 0; p < 2; ++p) {
    gm[p].r = g6[6 * p + 0];
    gm[p].phi = g6[6 * p + 1];
    gm[p].M = g6[6 * p + 2];
    gm[p].omega = g6[6 * p + 3];
    gm[p].Mdot = g6[6 * p + 4];
    gm[p].Macc = g6[6 * p + 5];
  }
}

void timestep_rk2_gpu(struct TimeStep *ts, struct Sim *s, struct Cell ***cells, struct GravMass *gm,
                      struct MPIsetup *mpi) {
  double t0 = timestep_get_t(ts), t, dt;
  if (!G.ctx) die("timestep_rk2_gpu", "timestep_gpu_open was not called");
  if (!G.uploaded) upload(ts, s, cells, gm);
  if (dgpu_step_rk2(G.ctx, 1) != DGPU_OK || dgpu_get_time(G.ctx, 0, &t, &dt) != DGPU_OK)
    die("timestep_rk2_gpu", dgpu_last_error(G.ctx));
  /* timestep_algorithm.c:17-19, printed after the step here (dt is known then) */
  if (mpisetup_MyProc(mpi) == 0) printf("t: %e, dt: %e\n", t0, dt);
  ts->t = t;
  ts->dt = dt;
  if (!G.lazy) timestep_gpu_sync(s, cells, gm);
}

void timestep_gpu_lazy(int lazy) { G.lazy = lazy; }

void timestep_gpu_reload(void) { G.uploaded = 0; }

void timestep_gpu_close(void) {
  dgpu_destroy(G.ctx);
  dgpu_sim_destroy(G.sim);
  free(G.prim);
  free(G.cons);
  free(G.tiph);
  free(G.dphi);
  G.ctx = NULL;
  G.sim = NULL;
  G.prim = G.cons = G.tiph = G.dphi = NULL;
  G.uploaded = 0;
}
