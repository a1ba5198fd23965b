/*
 * Oracle driver: runs the reference's own hot path (compiled unmodified from
 * its src/ tree, see oracle/Makefile) on a parfile and writes binary dumps.
 * Test infrastructure only; it replaces src/main.c and is never linked into
 * the product.
 *
 * Set-up follows src/main.c:56-123 (MPIsetup, Sim from the parfile, GravMass,
 * cell_create with its srand(666) phi offsets, clean_pi, syncs, initial data,
 * calc_cons) without IO or Diagnostics.  Then:
 *
 *   disco_ref run <par> <nsteps> <out.bin> [--load in.bin] [--faces f.bin]
 *                 [--dtlog log.txt] [--warmup W]
 *       loops timestep_rk2 (src/TimeStep/timestep_algorithm.c:11-41) nsteps
 *       times and dumps the final state.  --load replaces prim/tiph/dphi after
 *       the initial data (then calc_cons); --faces dumps the r-face list
 *       (face_create, src/Face/face_create_destroy.c:130-193) of the initial
 *       state, --zfaces the z-face list of a 3-D disk in the same format (its
 *       offsets are nzk); --dtlog writes "t dt" per step.  The wall time of the step
 *       loop alone goes to stderr as "steps_wall_s <seconds>"; --warmup runs W
 *       untimed steps first (not dumped).
 *
 *   disco_ref objective <par> <nsteps> <out.txt> [--load in.bin] [--dtfile dt.txt]
 *       runs nsteps steps and writes "n t dt torque mdot" after each: the
 *       binary torque -sum r rho dV F_phi over non-ghost cells (F_phi from the
 *       reference's gravMassForce, src/Cell/cell_source.c:49-71) and the
 *       accretion rate -sum rho v_r r dphi dz over the innermost non-ghost
 *       annulus.  --dtfile freezes the dt schedule: each step runs the calls of
 *       timestep_rk2 (src/TimeStep/timestep_algorithm.c:13-39) in its order
 *       with timestep_set_dt replaced by the next dt of the file.
 *
 *   disco_ref diag <par> <nsteps> <out.bin> [--load in.bin]
 *       creates the reference's Diagnostics at t = 0, runs nsteps steps and
 *       calls diagnostics_set (src/Diagnostics/diagnostics_set.c:13-298) once
 *       (its measuring time is moved to now); it appends to DiagMdot.dat in
 *       the working directory.  Dump: "DDIAG1\0\0", int32 nr neq, double t,
 *       VectorDiag[nr][17], ScalarDiag[16], EquatDiag[neq][18].
 *
 *   disco_ref checkpoint <par> <nsteps> <out.bin> [--load in.bin] [--restart ck.bin]
 *       runs nsteps steps and dumps the reference's checkpoint buffer
 *       (io_allocbuf + io_setbuf, src/IO/io_buffer.c:10-58): "DCKPT1\0\0",
 *       int32 nrows ncols, double t, GravMassBuffer[2][4], buffer[nrows][ncols].
 *
 *   --restart ck.bin (run and checkpoint modes) replaces the initial data by
 *       the restart branch of src/main.c:95-102, with io_hdf5_in replaced by
 *       reading a buffer file in the checkpoint dump format above: T, the
 *       GravMass buffer and the cell buffer, then io_readbuf.  gravMass_create
 *       mallocs the GravMasses, so Mdot and Macc, which the checkpoint does
 *       not hold, would be whatever malloc returned; they are zeroed first.
 *
 *   disco_ref stage <par> <phase> <out.bin> [--load in.bin]
 *       runs the prologue of timestep_rk2 and then the body of
 *       timestep_substep (src/TimeStep/timestep_routines.c:16-113), calling
 *       the same reference functions in the same order, and stops after
 *       <phase> (0: faces+clean_pi+set_w+RK blend, 1: PLM, 2: phi fluxes,
 *       3: r fluxes, 4: sources, 5: mesh motion+cons2prim, 6: BC+damping,
 *       7: calc_cons), dumping the extended cell data.  Phases 8-15: the
 *       whole first substep (timestep_substep, then gravMass_move and
 *       timestep_set_RK(0.5) as timestep_rk2 does), then the second substep
 *       stopped after <phase> - 8.
 *
 * State file (little endian): "DSTATE1\0", int32 NR NZ NUM_Q Ncells ext,
 * double t dt, double gm[2][6] (r phi M omega Mdot Macc), int32 N_p[NR],
 * double r_faces[NR+1], double prim[Ncells][NUM_Q], cons[Ncells][NUM_Q],
 * tiph[Ncells], dphi[Ncells]; if ext: grad, gradp ([Ncells][NUM_Q]),
 * wiph[Ncells], RKcons[Ncells][NUM_Q], RKtiph[Ncells].
 * Face file: "DFACES1\0", int32 NR Nf, int32 nri[NR], int32 L[Nf] R[Nf]
 * (cell numbers in (k,i,j) order), double r dphi dA deltaL deltaR cm [Nf].
 */
#define CELL_PRIVATE_DEFS
#define FACE_PRIVATE_DEFS
#define TIMESTEP_PRIVATE_DEFS
#define PLANET_PRIVATE_DEFS
#define DIAGNOSTICS_PRIVATE_DEFS
#define IO_PRIVATE_DEFS
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "Headers/Cell.h"
#include "Headers/Diagnostics.h"
#include "Headers/Face.h"
#include "Headers/GravMass.h"
#include "Headers/IO.h"
#include "Headers/MPIsetup.h"
#include "Headers/Riemann.h"
#include "Headers/Sim.h"
#include "Headers/TimeStep.h"
#include "Headers/header.h"
#include "ref_newic.h"

int readvar(char *filename, char *varname, int vartype, void *ptr);

static struct Cell *cell_base(struct Cell ***c) { return c[0][0]; }

static int count_cells(struct Sim *s) {
  int n = 0, i;
  for (i = 0; i < sim_N(s, R_DIR); ++i) n += sim_N_p(s, i) * sim_N(s, Z_DIR);
  return n;
}

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

static void dump_state(const char *path, struct Sim *s, struct Cell ***cells, struct GravMass *gm,
                       struct TimeStep *ts, int ext) {
  FILE *f = fopen(path, "wb");
  int NR = sim_N(s, R_DIR), NZ = sim_N(s, Z_DIR), NQ = sim_NUM_Q(s), N = count_cells(s);
  int hdr[5];
  double td[2];
  double g[12];
  int i, n, p;
  struct Cell *c = cell_base(cells);
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  wr(f, "DSTATE1", 1, 8);
  hdr[0] = NR; hdr[1] = NZ; hdr[2] = NQ; hdr[3] = N; hdr[4] = ext;
  wr(f, hdr, sizeof(int), 5);
  td[0] = ts->t; td[1] = ts->dt;
  wr(f, td, sizeof(double), 2);
  for (p = 0; p < 2; ++p) {
    g[6 * p + 0] = gm[p].r; g[6 * p + 1] = gm[p].phi; g[6 * p + 2] = gm[p].M;
    g[6 * p + 3] = gm[p].omega; g[6 * p + 4] = gm[p].Mdot; g[6 * p + 5] = gm[p].Macc;
  }
  wr(f, g, sizeof(double), 12);
  for (i = 0; i < NR; ++i) { int np = sim_N_p(s, i); wr(f, &np, sizeof(int), 1); }
  for (i = -1; i < NR; ++i) { double rf = sim_FacePos(s, i, R_DIR); wr(f, &rf, sizeof(double), 1); }
  for (n = 0; n < N; ++n) wr(f, c[n].prim, sizeof(double), NQ);
  for (n = 0; n < N; ++n) wr(f, c[n].cons, sizeof(double), NQ);
  for (n = 0; n < N; ++n) wr(f, &c[n].tiph, sizeof(double), 1);
  for (n = 0; n < N; ++n) wr(f, &c[n].dphi, sizeof(double), 1);
  if (ext) {
    for (n = 0; n < N; ++n) wr(f, c[n].grad, sizeof(double), NQ);
    for (n = 0; n < N; ++n) wr(f, c[n].gradp, sizeof(double), NQ);
    for (n = 0; n < N; ++n) wr(f, &c[n].wiph, sizeof(double), 1);
    for (n = 0; n < N; ++n) wr(f, c[n].RKcons, sizeof(double), NQ);
    for (n = 0; n < N; ++n) wr(f, &c[n].RKtiph, sizeof(double), 1);
  }
  fclose(f);
}

static void load_state(const char *path, struct Sim *s, struct Cell ***cells) {
  FILE *f = fopen(path, "rb");
  int NR = sim_N(s, R_DIR), NQ = sim_NUM_Q(s), N = count_cells(s);
  char magic[8];
  int hdr[5], n;
  double skip[14];
  struct Cell *c = cell_base(cells);
  double *buf;
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  rd(f, magic, 1, 8);
  rd(f, hdr, sizeof(int), 5);
  if (memcmp(magic, "DSTATE1", 8) != 0 || hdr[0] != NR || hdr[2] != NQ || hdr[3] != N) {
    fprintf(stderr, "state file %s does not match the parfile grid\n", path);
    exit(2);
  }
  rd(f, skip, sizeof(double), 14);
  buf = malloc(sizeof(double) * (size_t)(NR + 1) * 2 + sizeof(double) * (size_t)N * NQ);
  rd(f, buf, sizeof(int), NR);
  rd(f, buf, sizeof(double), NR + 1);
  for (n = 0; n < N; ++n) rd(f, c[n].prim, sizeof(double), NQ);
  rd(f, buf, sizeof(double), (size_t)N * NQ); /* cons: recomputed by calc_cons */
  for (n = 0; n < N; ++n) rd(f, &c[n].tiph, sizeof(double), 1);
  for (n = 0; n < N; ++n) rd(f, &c[n].dphi, sizeof(double), 1);
  free(buf);
  fclose(f);
}

/* the r faces (dir 0: face_create's nri offsets) or the z faces (dir 1: nzk) */
static void dump_faces(const char *path, struct Sim *s, struct Cell ***cells, struct TimeStep *ts, int dir) {
  struct Face *F = face_create(cells, s, ts, dir);
  int NR = dir ? sim_N(s, Z_DIR) : sim_N(s, R_DIR);
  int *off = dir ? ts->nzk : ts->nri;
  int Nf = off[NR - 1];
  struct Cell *c0 = cell_base(cells);
  FILE *f = fopen(path, "wb");
  int n;
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  wr(f, "DFACES1", 1, 8);
  wr(f, &NR, sizeof(int), 1);
  wr(f, &Nf, sizeof(int), 1);
  wr(f, off, sizeof(int), NR);
  for (n = 0; n < Nf; ++n) { int x = (int)(F[n].L - c0); wr(f, &x, sizeof(int), 1); }
  for (n = 0; n < Nf; ++n) { int x = (int)(F[n].R - c0); wr(f, &x, sizeof(int), 1); }
  for (n = 0; n < Nf; ++n) wr(f, &F[n].r, sizeof(double), 1);
  for (n = 0; n < Nf; ++n) wr(f, &F[n].dphi, sizeof(double), 1);
  for (n = 0; n < Nf; ++n) wr(f, &F[n].dA, sizeof(double), 1);
  for (n = 0; n < Nf; ++n) wr(f, &F[n].deltaL, sizeof(double), 1);
  for (n = 0; n < Nf; ++n) wr(f, &F[n].deltaR, sizeof(double), 1);
  for (n = 0; n < Nf; ++n) wr(f, &F[n].cm, sizeof(double), 1);
  fclose(f);
  face_destroy(F);
}

/* The body of timestep_substep (src/TimeStep/timestep_routines.c:16-113) as
 * the same sequence of reference calls, stopping after phase `stop`. */
static void substep_phases(struct TimeStep *ts, struct Cell ***cells, struct Sim *s,
                           struct GravMass *gm, struct MPIsetup *mpi, double fac, int stop) {
  double dt = fac * ts->dt;
  struct Face *Fr = face_create(cells, s, ts, 0);
  int i, j, k, n;
  cell_clean_pi(cells, s);
  gravMass_clean_pi(gm, s);
  cell_clear_w(cells, s);
  cell_set_w(cells, s);
  cell_adjust_RK_cons(cells, s, ts->RK);
  if (stop == 0) goto out;
  cell_plm_p(cells, s);
  cell_plm_rz(cells, s, Fr, ts, mpi, R_DIR);
  if (stop == 1) goto out;
  for (k = 0; k < sim_N(s, Z_DIR); ++k)
    for (i = 0; i < sim_N(s, R_DIR); ++i)
      for (j = 0; j < sim_N_p(s, i); ++j) {
        struct Riemann *R = riemann_create(s);
        riemann_setup_p(R, cells, s, i, j, k, PDIRECTION);
        riemann_AddFlux(R, s, gm, dt);
        riemann_destroy(R);
      }
  if (stop == 2) goto out;
  for (n = 0; n < timestep_n(ts, sim_N(s, R_DIR) - 1, R_DIR); ++n) {
    struct Riemann *R = riemann_create(s);
    riemann_setup_rz(R, Fr, s, n, RDIRECTION);
    riemann_AddFlux(R, s, gm, dt);
    riemann_destroy(R);
  }
  if (stop == 3) goto out;
  cell_add_src(cells, s, gm, dt);
  if (sim_EXPLICIT_VISCOSITY(s) > 0.0) cell_add_visc_src(cells, s, gm, dt);
  cell_add_split_fictitious(cells, s, gm, dt);
  if (stop == 4) goto out;
  cell_update_phi(cells, s, gm, ts->RK, dt);
  cell_update_dphi(cells, s);
  gravMass_update_RK(gm, s, ts->RK);
  cell_calc_prim(cells, s);
  if (stop == 5) goto out;
  if (sim_BoundTypeR(s) == BOUND_OUTFLOW) {
    cell_boundary_outflow_r(cells, Fr, s, mpi, ts);
  } else if (sim_BoundTypeR(s) == BOUND_FIXED) {
    cell_boundary_fixed_r(cells, s, gm, mpi, (*cell_single_init_ptr(s)));
  }
  if (sim_DAMP_TIME(s) > 0.0) cell_bc_damp(cells, s, gm, dt, (*cell_single_init_ptr(s)));
  if (stop == 6) goto out;
  cell_calc_cons(cells, s);
out:
  face_destroy(Fr);
}

void gravMassForce(struct GravMass *theGravMasses, struct Sim *theSim, int p, double r, double phi, double *fr,
                   double *fp);

/* timestep_rk2 (src/TimeStep/timestep_algorithm.c:13-39) with a given dt in
 * place of timestep_set_dt: the same reference calls in the same order. */
static void rk2_frozen_dt(struct TimeStep *ts, struct Sim *s, struct Cell ***cells, struct GravMass *gm,
                          struct MPIsetup *mpi, double dt) {
  int p;
  cell_clear_w(cells, s);
  cell_set_w(cells, s);
  ts->dt = dt;
  cell_copy(cells, s);
  gravMass_copy(gm, s);
  timestep_set_RK(ts, 0.0);
  timestep_substep(ts, cells, s, gm, mpi, 1.0);
  gravMass_move(s, gm, timestep_get_t(ts), 1.0 * timestep_dt(ts));
  timestep_set_RK(ts, 0.5);
  timestep_substep(ts, cells, s, gm, mpi, 0.5);
  gravMass_move(s, gm, timestep_get_t(ts), 0.5 * timestep_dt(ts));
  timestep_update_t(ts);
  for (p = 0; p < sim_NumGravMass(s); ++p)
    gravMass_set_Macc(gm, gravMass_Macc(gm, p) + gravMass_Mdot(gm, p) * timestep_dt(ts), p);
}

/* The two objectives of the differentiated runs on the current state. */
static void objectives(struct Sim *s, struct Cell ***cells, struct GravMass *gm, double *torque, double *mdot) {
  int i, j, p, NR = sim_N(s, R_DIR), n = 0;
  int i0 = sim_Nghost_min(s, R_DIR), i1 = NR - sim_Nghost_max(s, R_DIR);
  double dz = sim_FacePos(s, 0, Z_DIR) - sim_FacePos(s, -1, Z_DIR);
  struct Cell *c = cell_base(cells);
  double T = 0.0, M = 0.0;
  for (i = 0; i < NR; ++i) {
    double rm = sim_FacePos(s, i - 1, R_DIR), rp = sim_FacePos(s, i, R_DIR);
    double r = .5 * (rm + rp);
    for (j = 0; j < sim_N_p(s, i); ++j, ++n) {
      double dphi = c[n].dphi, phi = c[n].tiph - .5 * dphi, rho = c[n].prim[RHO];
      if (i >= i0 && i < i1) {
        double dV = dphi * .5 * (rp * rp - rm * rm) * dz, Fp = 0.0;
        for (p = 0; p < 2; ++p) {
          double fr, fp;
          gravMassForce(gm, s, p, r, phi, &fr, &fp);
          Fp += fp;
        }
        T += -(r * rho * dV * Fp);
      }
      if (i == i0) M += -(rho * c[n].prim[URR] * r * dphi * dz);
    }
  }
  *torque = T;
  *mdot = M;
}

/* the checkpoint buffer of io_setbuf, dumped */
static void dump_ckpt(const char *path, struct Sim *s, struct Cell ***cells, struct GravMass *gm,
                      struct TimeStep *ts) {
  struct IO *io = io_create(s);
  int nrows = sim_Ncells(s), ncols = sim_NUM_Q(s) + 3;
  FILE *f;
  io_allocbuf(io, s);
  io_setbuf(io, cells, s, gm);
  f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  wr(f, "DCKPT1\0", 1, 8);
  wr(f, &nrows, sizeof(int), 1);
  wr(f, &ncols, sizeof(int), 1);
  wr(f, &ts->t, sizeof(double), 1);
  wr(f, io->GravMassBuffer, sizeof(double), 8);
  wr(f, io->buffer[0], sizeof(double), (size_t)nrows * (size_t)ncols);
  fclose(f);
  io_deallocbuf(io);
  io_destroy(io);
}

/* the restart branch of main.c:95-102 with io_hdf5_in replaced by a read of
 * the dump format of dump_ckpt */
static void restart_from(const char *path, struct Sim *s, struct Cell ***cells, struct GravMass *gm,
                         struct TimeStep *ts) {
  struct IO *io = io_create(s);
  int nrows, ncols;
  char magic[8];
  double t;
  FILE *f = fopen(path, "rb");
  if (!f || fread(magic, 1, 8, f) != 8 || memcmp(magic, "DCKPT1\0", 8) || fread(&nrows, sizeof(int), 1, f) != 1 ||
      fread(&ncols, sizeof(int), 1, f) != 1 || nrows != sim_Ncells(s) || ncols != sim_NUM_Q(s) + 3) {
    fprintf(stderr, "bad checkpoint buffer %s\n", path);
    exit(2);
  }
  io_allocbuf(io, s);
  if (fread(&t, sizeof(double), 1, f) != 1 || fread(io->GravMassBuffer, sizeof(double), 8, f) != 8 ||
      fread(io->buffer[0], sizeof(double), (size_t)nrows * (size_t)ncols, f) != (size_t)nrows * (size_t)ncols) {
    fprintf(stderr, "short checkpoint buffer %s\n", path);
    exit(2);
  }
  fclose(f);
  timestep_set_t(ts, t);
  memset(gm, 0, sizeof(struct GravMass) * (size_t)sim_NumGravMass(s));
  io_readbuf(io, cells, s, gm);
  io_deallocbuf(io);
  io_destroy(io);
}

int main(int argc, char **argv) {
  const char *mode, *par, *out, *load = NULL, *faces = NULL, *zfaces = NULL, *dtlog = NULL, *dtfile = NULL,
             *restart = NULL;
  int nsteps, a, step, warmup = 0;
  char parbuf[1024];
  struct MPIsetup *mpi;
  struct Sim *s;
  struct GravMass *gm;
  struct Cell ***cells;
  struct TimeStep *ts;
  FILE *flog = NULL;
  if (argc < 5) {
    fprintf(stderr, "usage: disco_ref run|stage <parfile> <nsteps|phase> <out.bin> [options]\n");
    return 2;
  }
  mode = argv[1];
  par = argv[2];
  nsteps = atoi(argv[3]);
  out = argv[4];
  for (a = 5; a < argc; ++a) {
    if (!strcmp(argv[a], "--load") && a + 1 < argc) load = argv[++a];
    else if (!strcmp(argv[a], "--faces") && a + 1 < argc) faces = argv[++a];
    else if (!strcmp(argv[a], "--zfaces") && a + 1 < argc) zfaces = argv[++a];
    else if (!strcmp(argv[a], "--dtlog") && a + 1 < argc) dtlog = argv[++a];
    else if (!strcmp(argv[a], "--warmup") && a + 1 < argc) warmup = atoi(argv[++a]);
    else if (!strcmp(argv[a], "--dtfile") && a + 1 < argc) dtfile = argv[++a];
    else if (!strcmp(argv[a], "--restart") && a + 1 < argc) restart = argv[++a];
    else {
      fprintf(stderr, "unknown option %s\n", argv[a]);
      return 2;
    }
  }
  strncpy(parbuf, par, sizeof(parbuf) - 1);
  parbuf[sizeof(parbuf) - 1] = 0;

  /* the reference prints its per-step "t: dt:" line and read notices on stdout */
  if (!freopen("/dev/null", "w", stdout)) return 2;

  mpi = mpisetup_create(argc, argv);
  mpisetup_setprocs(mpi, parbuf);
  mpisetup_cart_create(mpi);
  mpisetup_left_right(mpi);
  s = sim_create(mpi);
  if (sim_read_par_file(s, mpi, parbuf) != 0) {
    fprintf(stderr, "parfile read failed: %s\n", par);
    return 3;
  }
  readvar(parbuf, "IC_HoR", VAR_DOUB, &oracle_ic_hor);
  readvar(parbuf, "IC_Noise", VAR_DOUB, &oracle_ic_noise);
  readvar(parbuf, "IC_Seed", VAR_INT, &oracle_ic_seed);
  sim_alloc_arr(s, mpi);
  sim_set_rz(s, mpi);
  sim_set_N_p(s);
  sim_set_misc(s, mpi);
  gm = gravMass_create(sim_NumGravMass(s));
  cells = cell_create(s, mpi);
  cell_clean_pi(cells, s);
  cell_syncproc_r(cells, s, mpi);
  cell_syncproc_z(cells, s, mpi);
  ts = timestep_create(s);
  ts->dt = 0.0;
  if (restart) {
    restart_from(restart, s, cells, gm, ts);
  } else {
    (*gravMass_init_ptr(s))(gm, s);
    (*cell_init_ptr(s))(cells, s, gm, mpi);
  }
  gravMass_clean_pi(gm, s);
  if (load) load_state(load, s, cells);
  cell_syncproc_r(cells, s, mpi);
  cell_syncproc_z(cells, s, mpi);
  cell_calc_cons(cells, s);

  if (!strcmp(mode, "run")) {
    if (faces) dump_faces(faces, s, cells, ts, 0);
    if (zfaces && sim_N_global(s, Z_DIR) > 1) dump_faces(zfaces, s, cells, ts, 1);
    struct timespec t0, t1;
    if (dtlog) flog = fopen(dtlog, "w");
    for (step = 0; step < warmup; ++step) timestep_rk2(ts, s, cells, gm, mpi);
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (step = 0; step < nsteps; ++step) {
      timestep_rk2(ts, s, cells, gm, mpi);
      if (flog) fprintf(flog, "%.17g %.17g\n", ts->t, ts->dt);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    fprintf(stderr, "steps_wall_s %.9f\n", (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec));
    if (flog) fclose(flog);
    dump_state(out, s, cells, gm, ts, 0);
  } else if (!strcmp(mode, "checkpoint")) {
    for (step = 0; step < nsteps; ++step) timestep_rk2(ts, s, cells, gm, mpi);
    dump_ckpt(out, s, cells, gm, ts);
  } else if (!strcmp(mode, "objective")) {
    FILE *fo = fopen(out, "w"), *fd = dtfile ? fopen(dtfile, "r") : NULL;
    if (!fo || (dtfile && !fd)) {
      fprintf(stderr, "cannot open %s\n", fo ? dtfile : out);
      return 2;
    }
    for (step = 0; step < nsteps; ++step) {
      double T, M;
      if (fd) {
        double dt;
        if (fscanf(fd, "%lf", &dt) != 1) {
          fprintf(stderr, "dt file has fewer than %d values\n", nsteps);
          return 2;
        }
        rk2_frozen_dt(ts, s, cells, gm, mpi, dt);
      } else {
        timestep_rk2(ts, s, cells, gm, mpi);
      }
      objectives(s, cells, gm, &T, &M);
      fprintf(fo, "%d %.17g %.17g %.17g %.17g\n", step + 1, ts->t, ts->dt, T, M);
    }
    fclose(fo);
    if (fd) fclose(fd);
  } else if (!strcmp(mode, "diag")) {
    struct Diagnostics *D = diagnostics_create(s, ts, mpi);
    FILE *f;
    int nr = sim_N_global(s, R_DIR), n;
    for (step = 0; step < nsteps; ++step) timestep_rk2(ts, s, cells, gm, mpi);
    D->tdiag_measure = -1.0;
    diagnostics_set(D, cells, s, ts, mpi, gm);
    f = fopen(out, "wb");
    if (!f) {
      fprintf(stderr, "cannot open %s\n", out);
      return 2;
    }
    wr(f, "DDIAG1\0", 1, 8);
    wr(f, &nr, sizeof(int), 1);
    wr(f, &D->N_eq_cells, sizeof(int), 1);
    wr(f, &ts->t, sizeof(double), 1);
    for (n = 0; n < nr; ++n) wr(f, D->VectorDiag[n], sizeof(double), 17);
    wr(f, D->ScalarDiag, sizeof(double), 16);
    for (n = 0; n < D->N_eq_cells; ++n) wr(f, D->EquatDiag[n], sizeof(double), 18);
    fclose(f);
  } else if (!strcmp(mode, "stage")) {
    /* prologue of timestep_rk2 (timestep_algorithm.c:13-24), then one substep */
    cell_clear_w(cells, s);
    cell_set_w(cells, s);
    timestep_set_dt(ts, cells, s, gm);
    cell_copy(cells, s);
    gravMass_copy(gm, s);
    timestep_set_RK(ts, 0.0);
    if (nsteps >= 8) {
      /* timestep_algorithm.c:23-29 */
      timestep_substep(ts, cells, s, gm, mpi, 1.0);
      gravMass_move(s, gm, timestep_get_t(ts), 1.0 * timestep_dt(ts));
      timestep_set_RK(ts, 0.5);
      substep_phases(ts, cells, s, gm, mpi, 0.5, nsteps - 8);
    } else {
      substep_phases(ts, cells, s, gm, mpi, 1.0, nsteps);
    }
    dump_state(out, s, cells, gm, ts, 1);
  } else {
    fprintf(stderr, "unknown mode %s\n", mode);
    return 2;
  }
  return 0;
}
