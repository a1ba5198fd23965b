/*
 * The reference's own main loop with timestep_rk2 handed to the B200 library:
 * the Disco2-side binding a maintainer would add, compiled from the reference's
 * objects (oracle/Makefile, target `binding`) and linked against
 * libdisco_gpu.so.
 *
 * Set-up is the reference's (src/main.c:56-123: MPIsetup, Sim from the
 * parfile, GravMass, cell_create with its srand(666) phi offsets, clean_pi,
 * syncs, initial data, calc_cons).  Then the state crosses to the GPU once
 * (cell_pack -> dgpu_set_state, the GravMass and t), the loop of
 * src/main.c:124-141 calls dgpu_step_rk2 in place of timestep_rk2, and the
 * state comes back (dgpu_get_state -> cell_unpack, the GravMass, t and dt)
 * into the reference's own structures, which are dumped in the oracle
 * driver's state format.
 *
 *   disco_gpu_main <par> <nsteps> <out.bin> [--fused] [--lazy]
 *
 * The loop is the reference's own (src/main.c:124-141) with timestep_rk2
 * replaced by timestep_rk2_gpu (timestep_gpu.c: the same signature, the
 * state kept on the GPU), for at most nsteps steps.  --fused steps with the
 * fused substep (k_prep + k_sweep) instead of the eight kernels; --lazy
 * leaves the state on the GPU between steps and brings it back only for the
 * checkpoints and the final dump.
 *
 * Checkpoints follow the reference too: with Restart 1 the state comes from
 * input.h5 (main.c:95-102), and after a step that passes the next checkpoint
 * time the state is written to checkpoint_%04d.h5 (main.c:132-139), both in
 * the working directory.  The reference's io_setbuf / io_readbuf fill and
 * read its checkpoint buffer; io_hdf5_out and io_hdf5_in, the two functions
 * that need an HDF5 library, become dgpu_hdf5_out and dgpu_hdf5_in.  Each
 * checkpoint written is reported on stderr as "checkpoint <file> step <n>".
 * Test infrastructure: the parity test compares its dump with the reference
 * build's own run of the same parfile (disco_ref run).
 */
#define CELL_PRIVATE_DEFS
#define PLANET_PRIVATE_DEFS
#define TIMESTEP_PRIVATE_DEFS
#define IO_PRIVATE_DEFS
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Headers/Cell.h"
#include "Headers/GravMass.h"
#include "Headers/IO.h"
#include "Headers/MPIsetup.h"
#include "Headers/Sim.h"
#include "Headers/TimeStep.h"
#include "Headers/header.h"
#include "cell_pack.h"
#include "disco_gpu.h"
#include "ref_newic.h"
#include "timestep_gpu.h"

int readvar(char *filename, char *varname, int vartype, void *ptr);

static int die(const char *what, const char *msg) {
  fprintf(stderr, "%s: %s\n", what, msg ? msg : "");
  return 1;
}

static void wr(FILE *f, const void *p, size_t sz, size_t n) {
  if (fwrite(p, sz, n, f) != n) {
    fprintf(stderr, "write failed\n");
    exit(2);
  }
}

/* the reference's cells, GravMass and clock in the driver's DSTATE1 format */
static int dump(const char *path, struct Sim *s, struct Cell ***cells, struct GravMass *gm, struct TimeStep *ts) {
  FILE *f = fopen(path, "wb");
  int NR = sim_N(s, R_DIR), NZ = sim_N(s, Z_DIR), NQ = sim_NUM_Q(s), N = cell_pack_count(s);
  int hdr[5] = {NR, NZ, NQ, N, 0}, i, n, p;
  double td[2] = {ts->t, ts->dt}, g[12];
  struct Cell *c = cells[0][0];
  if (!f) return die("cannot open", path);
  wr(f, "DSTATE1", 1, 8);
  wr(f, hdr, sizeof(int), 5);
  wr(f, td, sizeof(double), 2);
  for (p = 0; p < 2; ++p) {
    g[6 * p + 0] = gm[p].r;
    g[6 * p + 1] = gm[p].phi;
    g[6 * p + 2] = gm[p].M;
    g[6 * p + 3] = gm[p].omega;
    g[6 * p + 4] = gm[p].Mdot;
    g[6 * p + 5] = gm[p].Macc;
  }
  wr(f, g, sizeof(double), 12);
  for (i = 0; i < NR; ++i) {
    int np = sim_N_p(s, i);
    wr(f, &np, sizeof(int), 1);
  }
  for (i = -1; i < NR; ++i) {
    double rf = sim_FacePos(s, i, R_DIR);
    wr(f, &rf, sizeof(double), 1);
  }
  for (n = 0; n < N; ++n) wr(f, c[n].prim, sizeof(double), NQ);
  for (n = 0; n < N; ++n) wr(f, c[n].cons, sizeof(double), NQ);
  for (n = 0; n < N; ++n) wr(f, &c[n].tiph, sizeof(double), 1);
  for (n = 0; n < N; ++n) wr(f, &c[n].dphi, sizeof(double), 1);
  fclose(f);
  return 0;
}

int main(int argc, char **argv) {
  char parbuf[1024];
  int nsteps, step = 0, a, fused = 0, lazy = 0;
  struct MPIsetup *mpi;
  struct Sim *s;
  struct GravMass *gm;
  struct Cell ***cells;
  struct TimeStep *ts;
  struct IO *io;
  if (argc < 4) {
    fprintf(stderr, "usage: disco_gpu_main <parfile> <nsteps> <out.bin> [--fused] [--lazy]\n");
    return 2;
  }
  strncpy(parbuf, argv[1], sizeof(parbuf) - 1);
  parbuf[sizeof(parbuf) - 1] = 0;
  nsteps = atoi(argv[2]);
  for (a = 4; a < argc; ++a) {
    if (!strcmp(argv[a], "--fused")) fused = 1;
    else if (!strcmp(argv[a], "--lazy")) lazy = 1;
    else return die("unknown option", argv[a]);
  }
  /* the reference prints read notices and its per-step line on stdout */
  if (!freopen("/dev/null", "w", stdout)) return 2;

  /* src/main.c:56-119 */
  mpi = mpisetup_create(argc, argv);
  mpisetup_setprocs(mpi, parbuf);
  mpisetup_cart_create(mpi);
  mpisetup_left_right(mpi);
  s = sim_create(mpi);
  if (sim_read_par_file(s, mpi, parbuf) != 0) return die("parfile read failed", parbuf);
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
  io = io_create(s);
  if (sim_Restart(s) == 1) {
    /* main.c:95-102 with io_hdf5_in -> dgpu_hdf5_in; Mdot and Macc, which the
     * file does not hold, are zeroed rather than left as malloc returned them */
    double tr;
    memset(gm, 0, sizeof(struct GravMass) * (size_t)sim_NumGravMass(s));
    io_allocbuf(io, s);
    if (dgpu_hdf5_in("input.h5", sim_offset(s), sim_Ncells(s), sim_NUM_Q(s) + 3, &tr, &io->GravMassBuffer[0][0],
                     io->buffer[0]) != DGPU_OK)
      return die("dgpu_hdf5_in", dgpu_last_error(NULL));
    timestep_set_t(ts, tr);
    io_readbuf(io, cells, s, gm);
    io_deallocbuf(io);
  } else {
    (*gravMass_init_ptr(s))(gm, s);
    (*cell_init_ptr(s))(cells, s, gm, mpi);
  }
  gravMass_clean_pi(gm, s);
  io_setup(io, s, ts);
  cell_syncproc_r(cells, s, mpi);
  cell_syncproc_z(cells, s, mpi);
  cell_calc_cons(cells, s);

  if (timestep_gpu_open(parbuf, 0, fused) != DGPU_OK) return 1;
  timestep_gpu_lazy(lazy);

  /* src/main.c:124-141 */
  while (timestep_get_t(ts) < sim_get_T_MAX(s) && step < nsteps) {
    timestep_rk2_gpu(ts, s, cells, gm, mpi);
    ++step;
    if (timestep_get_t(ts) > io_tcheck(io)) {
      /* main.c:132-139 with io_hdf5_out -> dgpu_hdf5_out, and the bookkeeping
       * of io_hdf5.c:152-155 */
      if (lazy) timestep_gpu_sync(s, cells, gm);
      io_allocbuf(io, s);
      io_setbuf(io, cells, s, gm);
      if (dgpu_hdf5_out(io->filename, timestep_get_t(ts), &io->GravMassBuffer[0][0], io->buffer[0], sim_Ncells(s),
                        sim_NUM_Q(s) + 3) != DGPU_OK)
        return die("dgpu_hdf5_out", dgpu_last_error(NULL));
      io_deallocbuf(io);
      fprintf(stderr, "checkpoint %s step %d\n", io->filename, step);
      io->tcheck += io->dtcheck;
      ++io->nfile;
      sprintf(io->filename, "checkpoint_%04d.h5", io_nfile(io));
    }
  }
  if (lazy) timestep_gpu_sync(s, cells, gm);
  if (dump(argv[3], s, cells, gm, ts)) return 2;
  timestep_gpu_close();
  io_destroy(io);
  return 0;
}
