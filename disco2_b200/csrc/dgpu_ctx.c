/*
 * Host orchestration of the B200 step (C99 over the CUDA runtime API).
 *
 * A context owns the device copy of one or more disks: the annulus-major
 * structure-of-arrays state, the per-annulus tables, the r-face slabs and the
 * per-disk GravMass/time state.  One RK2 step (timestep_rk2,
 * src/TimeStep/timestep_algorithm.c:11-41) is eight kernel launches, captured
 * once into a CUDA graph and replayed; no host synchronisation happens inside
 * a step (dt, t and the GravMass orbit live on the device).
 */
#define _DEFAULT_SOURCE
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dgpu_ctx.h"

static __thread char g_err[512];

int dctx_fail(struct dgpu_ctx *c, int code, const char *fmt, ...) {
  va_list ap;
  char *dst = c ? c->err : g_err;
  va_start(ap, fmt);
  vsnprintf(dst, 512, fmt, ap);
  va_end(ap);
  return code;
}
#define fail dctx_fail

/* ---------------- Sim ---------------- */

int dgpu_sim_from_text(const char *text, dgpu_sim **out) {
  struct dgpu_sim *s;
  int rc;
  if (!text || !out) return fail(NULL, DGPU_ERR_ARG, "null argument");
  s = (struct dgpu_sim *)calloc(1, sizeof(*s));
  if (!s) return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
  rc = dsim_parse(text, s, g_err, sizeof(g_err));
  if (rc == DGPU_OK) rc = dsim_build_grid(s, g_err, sizeof(g_err));
  if (rc != DGPU_OK) {
    dsim_free(s);
    return rc;
  }
  *out = s;
  return DGPU_OK;
}

int dgpu_sim_from_parfile(const char *path, dgpu_sim **out) {
  FILE *f;
  long n;
  char *buf;
  int rc;
  if (!path) return fail(NULL, DGPU_ERR_ARG, "null path");
  f = fopen(path, "rb");
  if (!f) return fail(NULL, DGPU_ERR_PARFILE, "cannot open parfile %s", path);
  fseek(f, 0, SEEK_END);
  n = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf = (char *)malloc((size_t)n + 1);
  if (!buf) {
    fclose(f);
    return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
  }
  if (fread(buf, 1, (size_t)n, f) != (size_t)n) {
    fclose(f);
    free(buf);
    return fail(NULL, DGPU_ERR_PARFILE, "cannot read parfile %s", path);
  }
  fclose(f);
  buf[n] = 0;
  rc = dgpu_sim_from_text(buf, out);
  free(buf);
  return rc;
}

void dgpu_sim_destroy(dgpu_sim *sim) { dsim_free(sim); }
int dgpu_sim_num_annuli(const dgpu_sim *sim) { return sim ? sim->NR : DGPU_ERR_ARG; }
int dgpu_sim_num_cells(const dgpu_sim *sim) { return sim ? sim->Ncells : DGPU_ERR_ARG; }

int dgpu_sim_grid(const dgpu_sim *sim, int *N_p, double *r_faces) {
  if (!sim) return DGPU_ERR_ARG;
  if (N_p) memcpy(N_p, sim->N_p, sizeof(int) * (size_t)sim->NR);
  if (r_faces) memcpy(r_faces, sim->r_faces, sizeof(double) * (size_t)(sim->NR + 1));
  return DGPU_OK;
}

int dgpu_sim_param(const dgpu_sim *sim, const char *key, double *value) {
#define P_I(n, f) if (!strcmp(key, n)) { *value = (double)sim->f; return DGPU_OK; }
#define P_D(n, f) if (!strcmp(key, n)) { *value = sim->f; return DGPU_OK; }
  if (!sim || !key || !value) return DGPU_ERR_ARG;
  P_I("Restart", Restart) P_I("InitialDataType", InitialDataType) P_I("GravMassType", GravMassType)
  P_D("MassRatio", MassRatio) P_D("OrbShrinkTscale", OrbShrinkTscale) P_D("OrbShrinkT0", OrbShrinkT0)
  P_I("BoundTypeR", BoundTypeR) P_I("BoundTypeZ", BoundTypeZ) P_I("NoInnerBC", NoInnerBC)
  P_I("NumR", NumR) P_I("NumZ", NumZ) P_I("ng", ng) P_D("R_Min", R_Min) P_D("R_Max", R_Max)
  P_D("Z_Min", Z_Min) P_D("Z_Max", Z_Max) P_I("NP_CONST", NP_CONST) P_I("NPCAP", NPCAP)
  P_D("aspect", aspect) P_I("NUM_C", NUM_C) P_I("NUM_N", NUM_N) P_D("Time_Max", Time_Max)
  P_I("w_numeric_type", w_numeric_type) P_I("RiemannSolver", RiemannSolver)
  P_D("Adiabatic_Index", Adiabatic_Index) P_I("Cooling", Cooling)
  P_D("Explicit_Viscosity", Explicit_Viscosity) P_I("ViscConst", ViscConst) P_D("PoRho_r1", PoRho_r1)
  P_D("CFL", CFL) P_D("PLM", PLM) P_I("Grav_2D", Grav_2D) P_D("G_EPS", G_EPS)
  P_I("RhoSinkOn", RhoSinkOn) P_I("PHI_ORDER", PHI_ORDER) P_D("Rho_Floor", Rho_Floor)
  P_D("Cs_Floor", Cs_Floor) P_D("Cs_Cap", Cs_Cap) P_D("Vel_Cap", Vel_Cap) P_D("DAMP_TIME", DAMP_TIME)
  P_D("RDAMP_INNER", RDAMP_INNER) P_D("RDAMP_OUTER", RDAMP_OUTER) P_D("RLogScale", RLogScale)
  P_D("ZLogScale", ZLogScale) P_D("HiResSigma", HiResSigma) P_D("HiResR0a", HiResR0a)
  P_D("HiResR0b", HiResR0b) P_D("HiResFac", HiResFac) P_I("w_analytic_type", w_analytic_type)
  P_D("IC_HoR", IC_HoR) P_D("IC_Noise", IC_Noise) P_I("IC_Seed", IC_Seed)
  P_I("NR", NR) P_I("NZ", NZ) P_I("Ncells", Ncells)
#undef P_I
#undef P_D
  return DGPU_ERR_ARG;
}

int dgpu_sim_initial_state(const dgpu_sim *s, double *prim, double *tiph, double *dphi, double *gm) {
  double *t = tiph, *d = dphi, g[12];
  long idx = 0;
  int i, j, rc;
  if (!s) return fail(NULL, DGPU_ERR_ARG, "null sim");
  if (!t) t = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  if (!d) d = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  if (!t || !d) {
    if (t != tiph) free(t);
    if (d != dphi) free(d);
    return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
  }
  dsim_initial_tiph(s, t, d);
  /* the reference sets the GravMasses up before the gas (main.c:95-96); the
   * initialisers leave every phi in [0, 2pi], so gravMass_clean_pi after the
   * gas changes nothing the gas could have read */
  rc = dsim_initial_gravmass(s, g);
  if (rc != DGPU_OK) rc = fail(NULL, rc, "bad GravMassType");
  else if (gm) memcpy(gm, g, sizeof(g));
  if (rc == DGPU_OK && prim) {
    /* cell_init_torus re-seeds rand() with srand(666 + rank) */
    struct random_data rd;
    char state[128];
    memset(&rd, 0, sizeof(rd));
    memset(state, 0, sizeof(state));
    initstate_r(666, state, sizeof(state), &rd);
    int k;
    for (k = 0; k < s->NZ && rc == DGPU_OK; ++k)
      for (i = 0; i < s->NR && rc == DGPU_OK; ++i)
        for (j = 0; j < s->N_p[i]; ++j, ++idx)
          if (dsim_grid_init(s, k, i, idx, t[idx], d[idx], g, &rd, prim + (size_t)s->NQ * idx) != 0) {
            rc = fail(NULL, DGPU_ERR_UNSUPPORTED, "InitialDataType %d has no whole-grid initialiser here", s->InitialDataType);
            break;
          }
  }
  /* main.c:66-67,111-112: the syncs after cell_create and after the initial
   * data */
  if (rc == DGPU_OK) dsim_host_zsync(s, t, prim);
  if (t != tiph) free(t);
  if (d != dphi) free(d);
  return rc;
}

/* ---------------- Context ---------------- */

static int check_supported(const struct dgpu_sim *s, int k, char *err, int n) {
  int i;
  if (s->NumZ != 1) {
    /* 3-D: z faces, z slopes and fluxes, and the single-rank periodic z copy
     * (cell_syncproc_z) */
    if (s->BoundTypeZ != DB_PERIODIC)
      return snprintf(err, (size_t)n, "disk %d: NumZ > 1 needs BoundTypeZ 2 (periodic): on one rank the reference's z copy is periodic whatever the boundary type", k), DGPU_ERR_UNSUPPORTED;
    if (s->InitialDataType != DI_TORUS)
      return snprintf(err, (size_t)n, "disk %d: NumZ > 1 is implemented for the torus initial data (InitialDataType 3)", k), DGPU_ERR_UNSUPPORTED;
    if (s->NUM_N > 0)
      return snprintf(err, (size_t)n, "disk %d: passive scalars with NumZ > 1 are not implemented", k), DGPU_ERR_UNSUPPORTED;
    if (s->NumZ < s->ng)
      return snprintf(err, (size_t)n, "disk %d: the periodic z copy needs NumZ >= ng", k), DGPU_ERR_UNSUPPORTED;
  }
  if (s->NUM_C != 5 || s->NUM_N < 0 || s->NUM_N > DGPU_MAX_PASSIVE)
    return snprintf(err, (size_t)n, "disk %d: only NUM_C = 5 with NUM_N <= %d is implemented", k, DGPU_MAX_PASSIVE), DGPU_ERR_UNSUPPORTED;
  if (s->NUM_N > 0 && s->DAMP_TIME > 0.0)
    return snprintf(err, (size_t)n, "disk %d: passive scalars in a damping zone (the reference relaxes them toward an uninitialised value, cell_misc.c:119-124)", k), DGPU_ERR_UNSUPPORTED;
  if (s->NR < 3) return snprintf(err, (size_t)n, "disk %d: need at least 3 annuli", k), DGPU_ERR_UNSUPPORTED;
  for (i = 0; i < s->NR; ++i)
    if (s->N_p[i] < 2) return snprintf(err, (size_t)n, "disk %d: annulus %d has fewer than 2 cells", k, i), DGPU_ERR_UNSUPPORTED;
  if (s->w_numeric_type == DC_WCELL || s->w_numeric_type < 0 || s->w_numeric_type > DC_POWERLAW)
    return snprintf(err, (size_t)n, "disk %d: w_numeric_type %d is not usable (the reference exits on C_WCELL)", k, s->w_numeric_type), DGPU_ERR_UNSUPPORTED;
  if (s->w_analytic_type < 0 || s->w_analytic_type > DA_POWERLAW)
    return snprintf(err, (size_t)n, "disk %d: bad w_analytic_type", k), DGPU_ERR_PARFILE;
  if (s->RiemannSolver != DR_HLLC && s->RiemannSolver != DR_HLL)
    return snprintf(err, (size_t)n, "disk %d: bad RiemannSolver", k), DGPU_ERR_PARFILE;
  if (s->GravMassType < 0 || s->GravMassType > 2)
    return snprintf(err, (size_t)n, "disk %d: bad GravMassType", k), DGPU_ERR_PARFILE;
  if (s->BoundTypeR == DB_FIXED || s->DAMP_TIME > 0.0) {
    double prim[DGPU_NQ];
    if (dsim_single_init(s, 0, prim) < 0)
      return snprintf(err, (size_t)n, "disk %d: InitialDataType %d has no axisymmetric single-cell form for the fixed boundary/damping", k, s->InitialDataType), DGPU_ERR_UNSUPPORTED;
  }
  return DGPU_OK;
}

static void *dmalloc(size_t bytes, int *ok) {
  void *p = NULL;
  if (bytes == 0) bytes = 8;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    *ok = 0;
    return NULL;
  }
  cudaMemset(p, 0, bytes);
  return p;
}

void dgpu_destroy(dgpu_ctx *c) {
  int k;
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->have_graph) cudaGraphExecDestroy(c->graph);
  dctx_diff_free(c);
  if (c->d_diag) cudaFree(c->d_diag);
  {
    void *ps[] = {c->d_par, c->d_ist, c->d_ann, c->d_cell_ann, c->d_slot_ann, c->d.prim, c->d.cons,
                  c->d.rkcons, c->d.grad, c->d.gradp, c->d.tiph0, c->d.tiph1, c->d.tiphw, c->d.rktiph,
                  c->d.dphi, c->d.w_ann, c->d.fphi, c->d.frf, c->d.fS, c->d.fdp, c->d.ann_c, c->d.src, c->d.rr, c->d.fstart, c->d.fL, c->d.fR, c->d.fdphi,
                  c->d.fcm, c->d.pair_nf, c->d.pair_jpmin, c->d.pair_T, c->d.pair_seq, c->d.runs,
                  c->d.mdot_part, c->d.counters, c->d.err, c->d.obuf, c->d_stage, c->d_torque,
                  c->d.cfl_ann, c->d.sweep_flag, c->d_zslot_ann, c->d.zfL, c->d.zfR, c->d.zfdphi, c->d.zfcm,
                  c->d.zfstart, c->d.zrr, c->d.zruns, c->d.zpair_nf, c->d.zpair_jpmin, c->d.zpair_T,
                  c->d.zpair_seq, c->d.zfS, c->d.zfdp, c->d.zfrf, c->d.gradz};
    for (k = 0; k < (int)(sizeof(ps) / sizeof(ps[0])); ++k)
      if (ps[k]) cudaFree(ps[k]);
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->side) cudaStreamDestroy(c->side);
  for (k = 0; k < 4; ++k)
    if (c->fork[k]) cudaEventDestroy(c->fork[k]);
  if (c->sims) {
    for (k = 0; k < c->n_inst; ++k) dsim_free(c->sims[k]);
    free(c->sims);
  }
  free(c->h_par);
  free(c->h_ann);
  free(c);
}

int dgpu_create(const dgpu_sim *const *sims, int n, int device, void *stream, dgpu_ctx **out) {
  struct dgpu_ctx *c;
  int k, i, kz, rc, ok = 1;
  int ann = 0, cells = 0, slots = 0, runs = 0, zslots = 0, zruns = 0, maxcells = 0, n_ob = 0, n_pass = 0;
  int has_z = 0;
  int *h_cell_ann, *h_slot_ann, *h_zslot_ann;
  if (!sims || n < 1 || !out) return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_create");
  for (k = 0; k < n; ++k) {
    if (!sims[k]) return fail(NULL, DGPU_ERR_ARG, "sim %d is null", k);
    rc = check_supported(sims[k], k, g_err, sizeof(g_err));
    if (rc != DGPU_OK) return rc;
  }
  c = (struct dgpu_ctx *)calloc(1, sizeof(*c));
  if (!c) return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
  c->device = device;
  c->n_inst = n;
  c->sims = (struct dgpu_sim **)calloc((size_t)n, sizeof(*c->sims));
  c->h_par = (DiskParams *)calloc((size_t)n, sizeof(DiskParams));
  for (k = 0; k < n; ++k) {
    c->sims[k] = dsim_clone(sims[k]);
    if (!c->sims[k]) {
      dgpu_destroy(c);
      return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
    }
    ann += sims[k]->NR * sims[k]->NZ;
    cells += sims[k]->Ncells;
    if (sims[k]->NZ > 1) has_z = 1;
    if (sims[k]->NUM_N > n_pass) n_pass = sims[k]->NUM_N;
    if (sims[k]->Ncells > maxcells) maxcells = sims[k]->Ncells;
  }
  c->n_ann = ann;
  c->n_cells = cells;
  c->h_ann = (Annulus *)calloc((size_t)ann, sizeof(Annulus));
  h_cell_ann = (int *)malloc(sizeof(int) * (size_t)cells);
  /* tables */
  ann = 0;
  cells = 0;
  for (k = 0; k < n; ++k) {
    const struct dgpu_sim *s = c->sims[k];
    DiskParams *p = &c->h_par[k];
    dsim_fill_params(s, p);
    p->ann_base = ann;
    p->cell_base = cells;
    /* rings k-major, in the reference's (k, i, j) cell order */
    for (kz = 0; kz < s->NZ; ++kz) {
      for (i = 0; i < s->NR; ++i) {
        Annulus *a = &c->h_ann[ann + kz * s->NR + i];
        int j;
        dsim_fill_annulus(s, kz, i, a);
        a->inst = k;
        a->cell_off = cells;
        /* the outflow boundary reads annuli 1 and NR-3 and writes 0, NR-2 and NR-1 */
        if (s->BoundTypeR == DB_OUTFLOW && (i >= s->NR - 3 || (s->NoInnerBC != 1 && i <= 1))) {
          a->ob_off = n_ob;
          n_ob += s->N_p[i];
        } else {
          a->ob_off = -1;
        }
        for (j = 0; j < s->N_p[i]; ++j) h_cell_ann[cells + j] = ann + kz * s->NR + i;
        cells += s->N_p[i];
        a->face_base = slots;
        a->run_base = runs;
        a->face_cap = a->run_cap = 0;
        if (i < s->NR - 1) {
          a->face_cap = s->N_p[i] + s->N_p[i + 1] + DGPU_FACE_SLACK;
          slots += a->face_cap;
          a->run_cap = s->N_p[i + 1] + DGPU_RUN_SLACK;
          runs += a->run_cap;
        }
        /* z pair (k, k+1) of annulus i: both rings hold N_p[i] cells */
        a->zface_base = zslots;
        a->zrun_base = zruns;
        a->zface_cap = a->zrun_cap = 0;
        if (s->NZ > 1 && kz < s->NZ - 1) {
          a->zface_cap = 2 * s->N_p[i] + DGPU_FACE_SLACK;
          zslots += a->zface_cap;
          a->zrun_cap = s->N_p[i] + DGPU_RUN_SLACK;
          zruns += a->zrun_cap;
        }
      }
    }
    ann += s->NR * s->NZ;
  }
  c->n_slots = slots;
  c->n_runs = runs;
  c->n_ob = n_ob;
  h_slot_ann = (int *)malloc(sizeof(int) * (size_t)(slots > 0 ? slots : 1));
  h_zslot_ann = (int *)malloc(sizeof(int) * (size_t)(zslots > 0 ? zslots : 1));
  h_zslot_ann[0] = -1;
  for (i = 0; i < c->n_ann; ++i) {
    int f;
    for (f = 0; f < c->h_ann[i].face_cap; ++f) h_slot_ann[c->h_ann[i].face_base + f] = i;
    for (f = 0; f < c->h_ann[i].zface_cap; ++f) h_zslot_ann[c->h_ann[i].zface_base + f] = i;
  }
  c->d.n_zslots = zslots;
  c->d.n_zruns = zruns;
  c->d.has_z = has_z;
  c->d.max_nz = 1;
  for (k = 0; k < n; ++k)
    if (c->sims[k]->NZ > c->d.max_nz) c->d.max_nz = c->sims[k]->NZ;
  /* one 3-D disk: its ghost layers are the first and last cells, and the
   * periodic z copy launches over those alone */
  c->d.zghost = 0;
  if (n == 1 && has_z && c->sims[0]->NZ >= 2 * c->sims[0]->ng_min[1])
    c->d.zghost = c->sims[0]->ng_min[1] * (c->sims[0]->Ncells / c->sims[0]->NZ);
  c->n_upd_blocks = dgk_update_blocks(c->n_cells);

  if (cudaSetDevice(device) != cudaSuccess) {
    free(h_cell_ann);
    free(h_slot_ann);
    free(h_zslot_ann);
    dgpu_destroy(c);
    return fail(NULL, DGPU_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  }
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      free(h_cell_ann);
      free(h_slot_ann);
      free(h_zslot_ann);
      dgpu_destroy(c);
      return fail(NULL, DGPU_ERR_CUDA, "cudaStreamCreate failed");
    }
    c->own_stream = 1;
  }
  {
    int k, bad = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess;
    for (k = 0; k < 4 && !bad; ++k)
      bad = cudaEventCreateWithFlags(&c->fork[k], cudaEventDisableTiming) != cudaSuccess;
    if (bad) {
      free(h_cell_ann);
      free(h_slot_ann);
      free(h_zslot_ann);
      dgpu_destroy(c);
      return fail(NULL, DGPU_ERR_CUDA, "stream/event creation failed");
    }
  }
  c->n_pass = n_pass;
  {
    size_t N = (size_t)c->n_cells, S = (size_t)c->n_slots, A = (size_t)c->n_ann;
    const size_t NQ = 5 + (size_t)n_pass, NF = 8 + (size_t)n_pass;
    c->d_par = (DiskParams *)dmalloc(sizeof(DiskParams) * (size_t)n, &ok);
    c->d_ist = (InstState *)dmalloc(sizeof(InstState) * (size_t)n, &ok);
    c->d_ann = (Annulus *)dmalloc(sizeof(Annulus) * A, &ok);
    c->d_cell_ann = (int *)dmalloc(sizeof(int) * N, &ok);
    c->d_slot_ann = (int *)dmalloc(sizeof(int) * (S ? S : 1), &ok);
    c->d.prim = (double *)dmalloc(sizeof(double) * NQ * N, &ok);
    c->d.cons = (double *)dmalloc(sizeof(double) * NQ * N, &ok);
    c->d.rkcons = (double *)dmalloc(sizeof(double) * NQ * N, &ok);
    c->d.grad = (double *)dmalloc(sizeof(double) * NQ * N, &ok);
    c->d.gradp = (double *)dmalloc(sizeof(double) * NQ * N, &ok);
    c->d.tiph0 = (double *)dmalloc(sizeof(double) * N, &ok);
    c->d.tiph1 = (double *)dmalloc(sizeof(double) * N, &ok);
    c->d.tiphw = (double *)dmalloc(sizeof(double) * N, &ok);
    c->d.rktiph = (double *)dmalloc(sizeof(double) * N, &ok);
    c->d.dphi = (double *)dmalloc(sizeof(double) * N, &ok);
    c->d.w_ann = (double *)dmalloc(sizeof(double) * A, &ok);
    c->d.fphi = (double *)dmalloc(sizeof(double) * NF * N, &ok);
    c->d.frf = (double *)dmalloc(sizeof(double) * NF * (S ? S : 1), &ok);
    c->d.fS = (double *)dmalloc(sizeof(double) * NQ * (S ? S : 1), &ok);
    c->d.src = (double *)dmalloc(sizeof(double) * 8 * N, &ok);
    c->d.fdp = (double *)dmalloc(sizeof(double) * 2 * (S ? S : 1), &ok);
    c->d.ann_c = (double *)dmalloc(sizeof(double) * 4 * A, &ok);
    c->d.fstart = (int *)dmalloc(sizeof(int) * N, &ok);
    c->d.rr = (int *)dmalloc(sizeof(int) * 4 * N, &ok);
    c->d.fL = (int *)dmalloc(sizeof(int) * (S ? S : 1), &ok);
    c->d.fR = (int *)dmalloc(sizeof(int) * (S ? S : 1), &ok);
    c->d.fdphi = (double *)dmalloc(sizeof(double) * (S ? S : 1), &ok);
    c->d.fcm = (double *)dmalloc(sizeof(double) * (S ? S : 1), &ok);
    c->d.pair_nf = (int *)dmalloc(sizeof(int) * A, &ok);
    c->d.pair_jpmin = (int *)dmalloc(sizeof(int) * A, &ok);
    c->d.pair_T = (int *)dmalloc(sizeof(int) * A, &ok);
    c->d.pair_seq = (int *)dmalloc(sizeof(int) * A, &ok);
    c->d.runs = (int *)dmalloc(sizeof(int) * (size_t)(c->n_runs ? c->n_runs : 1), &ok);
    c->d.mdot_part = (double *)dmalloc(sizeof(double) * 2 * (size_t)c->n_upd_blocks, &ok);
    c->d.counters = (unsigned int *)dmalloc(sizeof(unsigned int) * 8, &ok);
    c->d.cfl_ann = (unsigned long long *)dmalloc(sizeof(unsigned long long) * A, &ok);
    c->d.sweep_flag = (int *)dmalloc(sizeof(int) * A, &ok);
    if (has_z) {
      const size_t ZS = (size_t)(zslots > 0 ? zslots : 1);
      c->d_zslot_ann = (int *)dmalloc(sizeof(int) * ZS, &ok);
      c->d.zfL = (int *)dmalloc(sizeof(int) * ZS, &ok);
      c->d.zfR = (int *)dmalloc(sizeof(int) * ZS, &ok);
      c->d.zfdphi = (double *)dmalloc(sizeof(double) * ZS, &ok);
      c->d.zfcm = (double *)dmalloc(sizeof(double) * ZS, &ok);
      c->d.zfstart = (int *)dmalloc(sizeof(int) * N, &ok);
      c->d.zrr = (int *)dmalloc(sizeof(int) * 4 * N, &ok);
      c->d.zruns = (int *)dmalloc(sizeof(int) * (size_t)(zruns > 0 ? zruns : 1), &ok);
      c->d.zpair_nf = (int *)dmalloc(sizeof(int) * A, &ok);
      c->d.zpair_jpmin = (int *)dmalloc(sizeof(int) * A, &ok);
      c->d.zpair_T = (int *)dmalloc(sizeof(int) * A, &ok);
      c->d.zpair_seq = (int *)dmalloc(sizeof(int) * A, &ok);
      c->d.zfS = (double *)dmalloc(sizeof(double) * 5 * ZS, &ok);
      c->d.zfdp = (double *)dmalloc(sizeof(double) * 2 * ZS, &ok);
      c->d.zfrf = (double *)dmalloc(sizeof(double) * 5 * ZS, &ok);
      c->d.gradz = (double *)dmalloc(sizeof(double) * 5 * N, &ok);
    }
    c->d.err = (int *)dmalloc(sizeof(int), &ok);
    if (n_ob > 0) c->d.obuf = (double *)dmalloc(sizeof(double) * NQ * (size_t)n_ob, &ok);
    c->d_stage = (double *)dmalloc(sizeof(double) * NQ * (size_t)maxcells, &ok);
    c->d_torque = (double *)dmalloc(sizeof(double) * ((size_t)maxcells / dgk_block_size() + 8), &ok);
  }
  if (!ok) {
    free(h_cell_ann);
    free(h_slot_ann);
    free(h_zslot_ann);
    dgpu_destroy(c);
    return fail(NULL, DGPU_ERR_NOMEM, "device allocation failed");
  }
  {
    /* k_merge stages the phi edges and widths of its annulus pair, and
     * builds the pair's runs, in shared memory */
    int a, mx = 0;
    for (a = 0; a < c->n_ann; ++a) {
      const Annulus *A = &c->h_ann[a];
      int m = 2 * (int)sizeof(double) * (A->np + (A->face_cap > 0 ? c->h_ann[a + 1].np : 0)) +
              (int)sizeof(int) * A->run_cap;
      /* a z pair stages two rings of N_p cells and the upper ring's runs */
      int mz = A->zface_cap > 0 ? 2 * (int)sizeof(double) * 2 * A->np + (int)sizeof(int) * A->zrun_cap : 0;
      if (m > mx) mx = m;
      if (mz > mx) mx = mz;
    }
    c->d.smem_face = mx <= 48 * 1024 ? mx : 0;
  }
  {
    /* threads per merge block: 256, or fewer when every annulus is small, so
     * that more pairs are resident per SM (a torus ring of 20 cells leaves
     * most of 256 threads idle); at least a warp, and about two inner cells
     * per thread at most */
    int a, mnp = 0, nt = 32;
    for (a = 0; a < c->n_ann; ++a)
      if (c->h_ann[a].np > mnp) mnp = c->h_ann[a].np;
    while (nt < 256 && 2 * nt < mnp) nt *= 2;
    c->d.merge_nt = nt;
  }
  /* the fused substep covers the forward step of disks without passive
   * scalars, outflow radial boundary or sink; it is opt-in (dgpu_set_fused):
   * on B200 the eight-kernel graph is faster (0.375 against 0.55 ms per step
   * on the 258k-cell circumbinary disk) */
  c->fused_ok = c->n_pass == 0 && c->n_ob == 0 && !has_z;
  for (k = 0; k < n; ++k)
    if (c->h_par[k].rho_sink_on == 1) c->fused_ok = 0;
  c->fused = 0;
  c->d.n_inst = n;
  c->d.n_ann = c->n_ann;
  c->d.n_cells = c->n_cells;
  c->d.n_slots = c->n_slots;
  c->d.n_runs = c->n_runs;
  c->d.n_ob = c->n_ob;
  c->d.n_pass = c->n_pass;
  c->d.par = c->d_par;
  c->d.ist = c->d_ist;
  c->d.ann = c->d_ann;
  c->d.cell_ann = c->d_cell_ann;
  c->d.slot_ann = c->d_slot_ann;
  c->d.zslot_ann = c->d_zslot_ann;
  if (cudaMemcpy(c->d_par, c->h_par, sizeof(DiskParams) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_ann, c->h_ann, sizeof(Annulus) * (size_t)c->n_ann, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_cell_ann, h_cell_ann, sizeof(int) * (size_t)c->n_cells, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_slot_ann, h_slot_ann, sizeof(int) * (size_t)(c->n_slots ? c->n_slots : 1),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      (has_z && cudaMemcpy(c->d_zslot_ann, h_zslot_ann, sizeof(int) * (size_t)(zslots ? zslots : 1),
                           cudaMemcpyHostToDevice) != cudaSuccess)) {
    free(h_cell_ann);
    free(h_slot_ann);
    free(h_zslot_ann);
    dgpu_destroy(c);
    return fail(NULL, DGPU_ERR_CUDA, "table upload failed");
  }
  free(h_cell_ann);
  free(h_slot_ann);
  free(h_zslot_ann);
  *out = c;
  return DGPU_OK;
}

const char *dgpu_last_error(const dgpu_ctx *c) { return c ? c->err : g_err; }
int dgpu_num_instances(const dgpu_ctx *c) { return c ? c->n_inst : DGPU_ERR_ARG; }

static int check_inst(struct dgpu_ctx *c, int inst) {
  if (!c) return DGPU_ERR_ARG;
  if (inst < 0 || inst >= c->n_inst) return fail(c, DGPU_ERR_ARG, "instance %d out of range", inst);
  cudaSetDevice(c->device);
  return DGPU_OK;
}

int dctx_read_err(struct dgpu_ctx *c) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, c->d.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  /* a flag is reported once; the caller reloads a valid state to continue */
  if (e) CK(cudaMemsetAsync(c->d.err, 0, sizeof(int), c->stream));
  if (e & (DGPU_EF_FACE_OVERFLOW | DGPU_EF_RUN_OVERFLOW))
    return fail(c, DGPU_ERR_FACE_OVERFLOW, "face list overflowed its buffer (flags 0x%x)", e);
  if (e & DGPU_EF_WRAP_LIMIT)
    return fail(c, DGPU_ERR_NUMERIC, "a phi wrap loop did not terminate (non-finite phi edge; flags 0x%x)", e);
  if (e & DGPU_EF_NONFINITE)
    return fail(c, DGPU_ERR_NUMERIC, "non-finite state: a non-ghost cell's CFL time step is NaN (flags 0x%x)", e);
  if (e & DGPU_EF_SWEEP_WAIT)
    return fail(c, DGPU_ERR_CUDA, "a k_sweep block gave up waiting for the previous annulus (flags 0x%x)", e);
  if (e & DGPU_EF_VISC_VZ)
    return fail(c, DGPU_ERR_NUMERIC, "viscosity with nonzero v_z (the reference exits here, Riemann_routines.c:271-274)");
  return DGPU_OK;
}

int dgpu_synchronize(dgpu_ctx *c) {
  if (!c) return DGPU_ERR_ARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return dctx_read_err(c);
}

/* state upload of one disk: prim AoS [N][5], tiph, dphi (host) */
static int upload_disk(struct dgpu_ctx *c, int inst, const double *prim, const double *tiph, const double *dphi) {
  const DiskParams *p = &c->h_par[inst];
  int n = p->n_cells, base = p->cell_base;
  if (prim) {
    const int nq = 5 + p->num_n;
    CK(cudaMemcpyAsync(c->d_stage, prim, sizeof(double) * nq * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    CKK(dgk_aos_to_soa(c->d.prim, nq, c->n_cells, base, c->d_stage, n, c->stream));
  }
  if (tiph) CK(cudaMemcpyAsync(c->d.tiph0 + base, tiph, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  if (dphi) CK(cudaMemcpyAsync(c->d.dphi + base, dphi, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  CKK(dgk_calc_cons(&c->d, NULL, c->stream));
  return DGPU_OK;
}

int dgpu_set_state(dgpu_ctx *c, int inst, const double *prim, const double *tiph, const double *dphi) {
  int rc = check_inst(c, inst);
  if (rc) return rc;
  rc = upload_disk(c, inst, prim, tiph, dphi);
  if (rc) return rc;
  return DGPU_OK;
}

int dgpu_get_state(dgpu_ctx *c, int inst, double *prim, double *cons, double *tiph, double *dphi) {
  const DiskParams *p;
  int n, base, rc = check_inst(c, inst);
  if (rc) return rc;
  p = &c->h_par[inst];
  n = p->n_cells;
  base = p->cell_base;
  if (prim) {
    CKK(dgk_soa_to_aos(c->d_stage, 5 + p->num_n, c->n_cells, base, c->d.prim, n, c->stream));
    CK(cudaMemcpyAsync(prim, c->d_stage, sizeof(double) * (5 + p->num_n) * (size_t)n, cudaMemcpyDeviceToHost,
                       c->stream));
    if (cons) CK(cudaStreamSynchronize(c->stream));
  }
  if (cons) {
    CKK(dgk_soa_to_aos(c->d_stage, 5 + p->num_n, c->n_cells, base, c->d.cons, n, c->stream));
    CK(cudaMemcpyAsync(cons, c->d_stage, sizeof(double) * (5 + p->num_n) * (size_t)n, cudaMemcpyDeviceToHost,
                       c->stream));
  }
  if (tiph) CK(cudaMemcpyAsync(tiph, c->d.tiph0 + base, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  if (dphi) CK(cudaMemcpyAsync(dphi, c->d.dphi + base, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  return dgpu_synchronize(c);
}

int dgpu_get_stage_data(dgpu_ctx *c, int inst, double *grad, double *gradp, double *wiph, double *rkcons,
                        double *rktiph) {
  const DiskParams *p;
  int n, base, rc = check_inst(c, inst);
  if (rc) return rc;
  p = &c->h_par[inst];
  n = p->n_cells;
  base = p->cell_base;
  {
    double *srcs[3] = {c->d.grad, c->d.gradp, c->d.rkcons};
    double *dsts[3] = {grad, gradp, rkcons};
    int k;
    for (k = 0; k < 3; ++k) {
      if (!dsts[k]) continue;
      CKK(dgk_soa_to_aos(c->d_stage, 5 + p->num_n, c->n_cells, base, srcs[k], n, c->stream));
      CK(cudaMemcpyAsync(dsts[k], c->d_stage, sizeof(double) * (5 + p->num_n) * (size_t)n, cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  }
  if (rktiph) CK(cudaMemcpyAsync(rktiph, c->d.rktiph + base, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  if (wiph) {
    /* wiph is one value per annulus */
    const struct dgpu_sim *s = c->sims[inst];
    double *w = (double *)malloc(sizeof(double) * (size_t)s->NR);
    int i, j, m = 0;
    if (!w) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
    if (cudaMemcpyAsync(w, c->d.w_ann + p->ann_base, sizeof(double) * (size_t)s->NR, cudaMemcpyDeviceToHost,
                        c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
      free(w);
      return fail(c, DGPU_ERR_CUDA, "wiph download failed");
    }
    for (i = 0; i < s->NR; ++i)
      for (j = 0; j < s->N_p[i]; ++j) wiph[m++] = w[i];
    free(w);
  }
  return dgpu_synchronize(c);
}

static int get_ist(struct dgpu_ctx *c, int inst, InstState *st) {
  CK(cudaMemcpyAsync(st, c->d_ist + inst, sizeof(InstState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DGPU_OK;
}
static int put_ist(struct dgpu_ctx *c, int inst, const InstState *st) {
  CK(cudaMemcpyAsync(c->d_ist + inst, st, sizeof(InstState), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DGPU_OK;
}

int dgpu_set_gravmass(dgpu_ctx *c, int inst, const double *gm) {
  InstState st;
  int p, rc = check_inst(c, inst);
  if (rc) return rc;
  if (!gm) return fail(c, DGPU_ERR_ARG, "null gm");
  if ((rc = get_ist(c, inst, &st))) return rc;
  for (p = 0; p < 2; ++p) {
    st.gr[p] = gm[6 * p + 0];
    st.gphi[p] = gm[6 * p + 1];
    st.gM[p] = gm[6 * p + 2];
    st.gom[p] = gm[6 * p + 3];
    st.mdot[p] = gm[6 * p + 4];
    st.macc[p] = gm[6 * p + 5];
  }
  return put_ist(c, inst, &st);
}

int dgpu_get_gravmass(dgpu_ctx *c, int inst, double *gm) {
  InstState st;
  int p, rc = check_inst(c, inst);
  if (rc) return rc;
  if ((rc = get_ist(c, inst, &st))) return rc;
  for (p = 0; p < 2; ++p) {
    gm[6 * p + 0] = st.gr[p];
    gm[6 * p + 1] = st.gphi[p];
    gm[6 * p + 2] = st.gM[p];
    gm[6 * p + 3] = st.gom[p];
    gm[6 * p + 4] = st.mdot[p];
    gm[6 * p + 5] = st.macc[p];
  }
  return DGPU_OK;
}

int dgpu_get_time(dgpu_ctx *c, int inst, double *t, double *dt) {
  InstState st;
  int rc = check_inst(c, inst);
  if (rc) return rc;
  if ((rc = get_ist(c, inst, &st))) return rc;
  if (t) *t = st.t;
  if (dt) *dt = st.dt;
  return DGPU_OK;
}

int dgpu_set_time(dgpu_ctx *c, int inst, double t) {
  InstState st;
  int rc = check_inst(c, inst);
  if (rc) return rc;
  if ((rc = get_ist(c, inst, &st))) return rc;
  st.t = t;
  return put_ist(c, inst, &st);
}

int dgpu_init_state(dgpu_ctx *c, int inst) {
  const struct dgpu_sim *s;
  double *prim, *tiph, *dphi, gm[12];
  int rc = check_inst(c, inst);
  if (rc) return rc;
  s = c->sims[inst];
  prim = (double *)malloc(sizeof(double) * (size_t)s->NQ * (size_t)s->Ncells);
  tiph = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  dphi = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  if (!prim || !tiph || !dphi) {
    free(prim); free(tiph); free(dphi);
    return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  rc = dgpu_sim_initial_state(s, prim, tiph, dphi, gm);
  if (rc != DGPU_OK) {
    free(prim); free(tiph); free(dphi);
    return fail(c, rc, "%s", g_err);
  }
  rc = upload_disk(c, inst, prim, tiph, dphi);
  if (rc == DGPU_OK) rc = dgpu_synchronize(c);
  free(prim); free(tiph); free(dphi);
  if (rc) return rc;
  {
    InstState st;
    int p;
    memset(&st, 0, sizeof(st));
    for (p = 0; p < 2; ++p) {
      st.gr[p] = gm[6 * p + 0];
      st.gphi[p] = gm[6 * p + 1];
      st.gM[p] = gm[6 * p + 2];
      st.gom[p] = gm[6 * p + 3];
    }
    rc = put_ist(c, inst, &st);
  }
  return rc;
}

int dctx_substep(struct dgpu_ctx *c, const TanPtrs *t, int sub, int mode, double *rec, const int *rec_idx) {
  /* the layout of the step graph: merge beside cellprep, source and the phi
   * faces beside the r faces */
  CK(cudaEventRecord(c->fork[0], c->stream));
  CK(cudaStreamWaitEvent(c->side, c->fork[0], 0));
  CKK(dgk_merge(&c->d, sub, c->side));
  CKK(dgk_cellprep(&c->d, t, sub, c->stream));
  CK(cudaEventRecord(c->fork[1], c->side));
  CK(cudaStreamWaitEvent(c->stream, c->fork[1], 0));
  CKK(dgk_rslope(&c->d, t, c->stream));
  CKK(dgk_plm_r(&c->d, t, sub, c->stream));
  if (mode == DCTX_ADJPREP) {
    CKK(dgk_ann_consts(&c->d, sub, c->stream));
    return DGPU_OK;
  }
  CK(cudaEventRecord(c->fork[2], c->stream));
  CK(cudaStreamWaitEvent(c->side, c->fork[2], 0));
  CKK(dgk_source(&c->d, t, sub, c->side));
  CKK(dgk_flux_phi(&c->d, t, sub, c->side));
  CKK(dgk_flux_r(&c->d, t, sub, c->stream));
  CK(cudaEventRecord(c->fork[3], c->side));
  CK(cudaStreamWaitEvent(c->stream, c->fork[3], 0));
  if (mode == DCTX_REC) CKK(dgk_update_rec(&c->d, sub, rec, rec_idx, c->stream));
  else CKK(dgk_update(&c->d, t, sub, 7, c->stream));
  if (c->n_ob > 0) CKK(dgk_outflow(&c->d, 7, c->stream));
  return DGPU_OK;
}

/* One substep of a context holding a 3-D disk: the z faces' increments are
 * added after the r faces' in the update (timestep_routines.c:63-71), the
 * viscous source reads the z slopes, and the periodic z copy closes the
 * substep.  Three branches on the second stream: the r- and z-face lists
 * beside cellprep, the z slopes beside the r slopes, and the sources and phi
 * faces beside the r and z faces; each branch reads only what was written
 * before its fork. */
static int launch_substep_3d(struct dgpu_ctx *c, int sub) {
  CK(cudaEventRecord(c->fork[0], c->stream));
  CK(cudaStreamWaitEvent(c->side, c->fork[0], 0));
  CKK(dgk_merge(&c->d, sub, c->side));
  CKK(dgk_zmerge(&c->d, sub, c->side));
  CKK(dgk_cellprep(&c->d, NULL, sub, c->stream));
  CK(cudaEventRecord(c->fork[1], c->side));
  CK(cudaStreamWaitEvent(c->stream, c->fork[1], 0));
  CK(cudaEventRecord(c->fork[2], c->stream));
  CK(cudaStreamWaitEvent(c->side, c->fork[2], 0));
  CKK(dgk_zslope(&c->d, c->side));
  CKK(dgk_plm_z(&c->d, c->side));
  CKK(dgk_rslope(&c->d, NULL, c->stream));
  CKK(dgk_plm_r(&c->d, NULL, sub, c->stream));
  CK(cudaEventRecord(c->fork[3], c->side));
  CK(cudaStreamWaitEvent(c->stream, c->fork[3], 0));
  CK(cudaEventRecord(c->fork[0], c->stream));
  CK(cudaStreamWaitEvent(c->side, c->fork[0], 0));
  CKK(dgk_source(&c->d, NULL, sub, c->side));
  CKK(dgk_flux_phi(&c->d, NULL, sub, c->side));
  CKK(dgk_flux_r(&c->d, NULL, sub, c->stream));
  CKK(dgk_flux_z(&c->d, sub, c->stream));
  CK(cudaEventRecord(c->fork[1], c->side));
  CK(cudaStreamWaitEvent(c->stream, c->fork[1], 0));
  CKK(dgk_update(&c->d, NULL, sub, 7, c->stream));
  if (c->n_ob > 0) CKK(dgk_outflow(&c->d, 7, c->stream));
  CKK(dgk_zsync(&c->d, sub, c->stream));
  return DGPU_OK;
}

int dctx_launch_step(struct dgpu_ctx *c) {
  int sub;
  if (c->d.has_z) {
    for (sub = 1; sub <= 2; ++sub) {
      int rc = launch_substep_3d(c, sub);
      if (rc) return rc;
    }
    return DGPU_OK;
  }
  if (c->fused) {
    /* per substep: k_prep (face list, phi slopes, CFL minima), then k_sweep */
    for (sub = 1; sub <= 2; ++sub) {
      CKK(dgk_prep(&c->d, sub, c->stream));
      CKK(dgk_sweep(&c->d, sub, c->stream));
    }
    return DGPU_OK;
  }
  for (sub = 1; sub <= 2; ++sub) {
    /* k_merge (per annulus pair) alongside k_cellprep (per cell) */
    CK(cudaEventRecord(c->fork[0], c->stream));
    CK(cudaStreamWaitEvent(c->side, c->fork[0], 0));
    CKK(dgk_merge(&c->d, sub, c->side));
    CKK(dgk_cellprep(&c->d, NULL, sub, c->stream));
    CK(cudaEventRecord(c->fork[1], c->side));
    CK(cudaStreamWaitEvent(c->stream, c->fork[1], 0));
    CKK(dgk_rslope(&c->d, NULL, c->stream));
    CKK(dgk_plm_r(&c->d, NULL, sub, c->stream));
    /* k_source and the phi faces (per cell) alongside the r faces (per face) */
    CK(cudaEventRecord(c->fork[2], c->stream));
    CK(cudaStreamWaitEvent(c->side, c->fork[2], 0));
    CKK(dgk_source(&c->d, NULL, sub, c->side));
    CKK(dgk_flux_phi(&c->d, NULL, sub, c->side));
    CKK(dgk_flux_r(&c->d, NULL, sub, c->stream));
    CK(cudaEventRecord(c->fork[3], c->side));
    CK(cudaStreamWaitEvent(c->stream, c->fork[3], 0));
    CKK(dgk_update(&c->d, NULL, sub, 7, c->stream));
    if (c->n_ob > 0) CKK(dgk_outflow(&c->d, 7, c->stream));
  }
  return DGPU_OK;
}

int dgpu_step_rk2(dgpu_ctx *c, int nsteps) {
  int k;
  if (!c || nsteps < 0) return DGPU_ERR_ARG;
  cudaSetDevice(c->device);
  if (!c->have_graph) {
    cudaGraph_t g;
    int rc;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = dctx_launch_step(c);
    {
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return fail(c, DGPU_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    }
    {
      cudaError_t e = cudaGraphInstantiate(&c->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(c, DGPU_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    }
    c->have_graph = 1;
  }
  for (k = 0; k < nsteps; ++k) CK(cudaGraphLaunch(c->graph, c->stream));
  return DGPU_OK;
}

int dgpu_set_fused(dgpu_ctx *c, int fused) {
  if (!c || fused < 0 || fused > 1) return DGPU_ERR_ARG;
  if (fused && !c->fused_ok)
    return fail(c, DGPU_ERR_UNSUPPORTED, "the fused substep needs disks without passive scalars, outflow radial "
                                         "boundary or sink");
  if (fused != c->fused && c->have_graph) {
    cudaSetDevice(c->device);
    cudaGraphExecDestroy(c->graph);
    c->have_graph = 0;
  }
  c->fused = fused;
  return DGPU_OK;
}

int dgpu_fused(const dgpu_ctx *c) { return c ? c->fused : DGPU_ERR_ARG; }

int dgpu_step_rk2_timed(dgpu_ctx *c, int nsteps, double *kernel_ms) {
  cudaEvent_t ev[DGPU_STEP_KERNELS + 1];
  int k, s, sub, rc = DGPU_OK;
  if (!c || nsteps < 0 || !kernel_ms) return DGPU_ERR_ARG;
  cudaSetDevice(c->device);
  for (k = 0; k <= DGPU_STEP_KERNELS; ++k) CK(cudaEventCreate(&ev[k]));
  if (c->fused) {
    /* kernel_ms[0], [1]: k_prep, k_sweep of substep 1; [8], [9]: of substep 2 */
    for (s = 0; s < nsteps; ++s) {
      for (sub = 1; sub <= 2; ++sub) {
        CK(cudaEventRecord(ev[0], c->stream));
        CKK(dgk_prep(&c->d, sub, c->stream));
        CK(cudaEventRecord(ev[1], c->stream));
        CKK(dgk_sweep(&c->d, sub, c->stream));
        CK(cudaEventRecord(ev[2], c->stream));
        CK(cudaEventSynchronize(ev[2]));
        for (k = 0; k < 2; ++k) {
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
          kernel_ms[8 * (sub - 1) + k] += (double)ms;
        }
      }
    }
    for (k = 0; k <= DGPU_STEP_KERNELS; ++k) cudaEventDestroy(ev[k]);
    return dctx_read_err(c);
  }
  for (s = 0; s < nsteps && rc == DGPU_OK; ++s) {
    int e = 0;
    CK(cudaEventRecord(ev[e++], c->stream));
    for (sub = 1; sub <= 2; ++sub) {
      CKK(dgk_cellprep(&c->d, NULL, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_merge(&c->d, sub, c->stream));
      CKK(dgk_zmerge(&c->d, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_rslope(&c->d, NULL, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_plm_r(&c->d, NULL, sub, c->stream));
      /* 3-D: the z faces, whose slopes the viscous source reads, in the
       * plm_r slot (no-ops for 2-D disks) */
      CKK(dgk_zslope(&c->d, c->stream));
      CKK(dgk_plm_z(&c->d, c->stream));
      CKK(dgk_flux_z(&c->d, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_source(&c->d, NULL, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_flux_phi(&c->d, NULL, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_flux_r(&c->d, NULL, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
      CKK(dgk_update(&c->d, NULL, sub, 7, c->stream));
      if (c->n_ob > 0) CKK(dgk_outflow(&c->d, 7, c->stream));
      CKK(dgk_zsync(&c->d, sub, c->stream));
      CK(cudaEventRecord(ev[e++], c->stream));
    }
    CK(cudaEventSynchronize(ev[DGPU_STEP_KERNELS]));
    for (k = 0; k < DGPU_STEP_KERNELS; ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      kernel_ms[k] += (double)ms;
    }
  }
  for (k = 0; k <= DGPU_STEP_KERNELS; ++k) cudaEventDestroy(ev[k]);
  return dctx_read_err(c);
}

/* The autotuner: a coordinate search over the resident blocks per SM of the
 * five heavy kernels (the register budget the compiler gets), each timed on
 * the context's own disks by dgpu_step_rk2_timed from the same saved state.
 * The instances differ only in register allocation, so the results are
 * bitwise the same whatever is chosen. */
#define TUNE_NCAND 4
static const int tune_cand[TUNE_NCAND] = {2, 3, 4, 5};
/* kernel_ms slot of each tuned kernel in substep 1 (substep 2 is +8) */
static const int tune_slot[DGPU_TUNE_N] = {3, 5, 6, 4, 7, 1};

int dgpu_autotune(dgpu_ctx *c, int steps, int *choice) {
  double *buf = NULL, ms[DGPU_STEP_KERNELS];
  InstState *ist = NULL;
  int k, v, rc = DGPU_OK;
  static const int order[DGPU_TUNE_N - 1] = {DGPU_TUNE_UPDATE, DGPU_TUNE_FLUXR, DGPU_TUNE_FLUXPHI, DGPU_TUNE_SOURCE,
                                             DGPU_TUNE_PLM};
  static const int order_fused[1] = {DGPU_TUNE_SWEEP};
  if (!c || steps < 0) return DGPU_ERR_ARG;
  cudaSetDevice(c->device);
  if (steps == 0) {
    /* apply the given choice */
    if (!choice) return fail(c, DGPU_ERR_ARG, "steps == 0 needs a choice to apply");
    for (k = 0; k < DGPU_TUNE_N; ++k) {
      if (choice[k] != 0 && (choice[k] < 2 || choice[k] > (k == DGPU_TUNE_SWEEP ? 4 : 5)))
        return fail(c, DGPU_ERR_ARG, "blocks per SM must be 0 or 2..5 (sweep 2..4), got %d", choice[k]);
    }
    for (k = 0; k < DGPU_TUNE_N; ++k) c->d.tune[k] = choice[k];
  } else {
    /* save the state, time each candidate from it, restore it */
    if (cudaMalloc((void **)&buf, sizeof(double) * (19 + 3 * (size_t)c->n_pass) * (size_t)c->n_cells) != cudaSuccess ||
        cudaMalloc((void **)&ist, sizeof(InstState) * (size_t)c->n_inst) != cudaSuccess) {
      cudaFree(buf);
      cudaGetLastError();
      return fail(c, DGPU_ERR_NOMEM, "autotune: device allocation failed");
    }
    if (dgk_snap(&c->d, buf, ist, 1, c->stream)) rc = fail(c, DGPU_ERR_CUDA, "autotune: state save failed");
    /* the fused step tunes k_sweep (2..4 blocks per SM), the other the five
     * heavy kernels */
    const int nk = c->fused ? 1 : DGPU_TUNE_N - 1;
    for (k = 0; k < nk && rc == DGPU_OK; ++k) {
      const int kk = c->fused ? order_fused[k] : order[k];
      const int ncand = kk == DGPU_TUNE_SWEEP ? TUNE_NCAND - 1 : TUNE_NCAND;
      double best = 1e300;
      int bestv = c->d.tune[kk];
      for (v = 0; v < ncand && rc == DGPU_OK; ++v) {
        double t;
        c->d.tune[kk] = tune_cand[v];
        if (dgk_snap(&c->d, buf, ist, 0, c->stream)) {
          rc = fail(c, DGPU_ERR_CUDA, "autotune: state restore failed");
          break;
        }
        memset(ms, 0, sizeof(ms));
        if ((rc = dgpu_step_rk2_timed(c, 1, ms))) break; /* warm-up */
        memset(ms, 0, sizeof(ms));
        if ((rc = dgpu_step_rk2_timed(c, steps, ms))) break;
        t = ms[tune_slot[kk]] + ms[tune_slot[kk] + 8];
        if (t < best) {
          best = t;
          bestv = tune_cand[v];
        }
      }
      c->d.tune[kk] = bestv;
    }
    if (rc == DGPU_OK && dgk_snap(&c->d, buf, ist, 0, c->stream))
      rc = fail(c, DGPU_ERR_CUDA, "autotune: state restore failed");
    if (rc == DGPU_OK) rc = dgpu_synchronize(c);
    cudaFree(buf);
    cudaFree(ist);
    if (rc) return rc;
  }
  /* the step graph holds the old launch shapes */
  if (c->have_graph) {
    cudaGraphExecDestroy(c->graph);
    c->have_graph = 0;
  }
  if (choice)
    for (k = 0; k < DGPU_TUNE_N; ++k) choice[k] = c->d.tune[k];
  return DGPU_OK;
}

int dgpu_stage(dgpu_ctx *c, int phase) {
  int sub = phase >= 8 ? 2 : 1, stop = phase & 7;
  if (!c || phase < 0 || phase > 15) return DGPU_ERR_ARG;
  if (c->d.has_z) return fail(c, DGPU_ERR_UNSUPPORTED, "stage parity of 3-D disks (NumZ > 1) is not implemented");
  cudaSetDevice(c->device);
  /* phases 8-15: the whole first substep (its k_update also moves the
   * GravMass, as timestep_rk2 does between the substeps), then the second */
  if (sub == 2) {
    int rc = dctx_substep(c, NULL, 1, DCTX_FULL, NULL, NULL);
    if (rc) return rc;
  }
  CKK(dgk_cellprep(&c->d, NULL, sub, c->stream));
  CKK(dgk_merge(&c->d, sub, c->stream));
  /* the CFL minimum (and dt) come from k_plm_r; PLM results are kept only from phase 1 on */
  CKK(dgk_rslope(&c->d, NULL, c->stream));
  CKK(dgk_plm_r(&c->d, NULL, sub, c->stream));
  CKK(dgk_source(&c->d, NULL, sub, c->stream));
  if (stop >= 2) {
    CKK(dgk_flux_phi(&c->d, NULL, sub, c->stream));
    CKK(dgk_flux_r(&c->d, NULL, sub, c->stream));
  }
  CKK(dgk_update_stage(&c->d, sub, stop, c->stream));
  if (stop >= 6 && c->n_ob > 0) CKK(dgk_outflow(&c->d, stop, c->stream));
  /* from phase 5 of substep 1 on the advanced phi edges live in the substep's
   * output buffer (substep 2 writes them where the state is read) */
  if (sub == 1 && stop >= 5)
    CK(cudaMemcpyAsync(c->d.tiph0, c->d.tiph1, sizeof(double) * (size_t)c->n_cells,
                       cudaMemcpyDeviceToDevice, c->stream));
  return dgpu_synchronize(c);
}

/* The r faces (z = 0) or the z faces (z = 1) of one disk in the reference's
 * face-list order: face_create lists the r faces annulus pair by annulus
 * pair, the layers inside each, and the z faces layer pair by layer pair, the
 * annuli inside each (src/Face/face_create_destroy.c:130-193).  off[] gets
 * the first face of each pair (timestep_n's nri / nzk). */
static int face_list_dir(dgpu_ctx *c, int inst, int z, int cap, int *off, int *L, int *R, double *r,
                         double *dphi, double *dA, double *deltaL, double *deltaR, double *cm, int *nf_out) {
  const struct dgpu_sim *s;
  const DiskParams *p;
  int i, k, total = 0, rc = check_inst(c, inst), nrings, nslots;
  int *nf, *fL, *fR;
  double *fd, *fc;
  if (rc) return rc;
  s = c->sims[inst];
  p = &c->h_par[inst];
  if (z && s->NZ == 1) return fail(c, DGPU_ERR_ARG, "a 2-D disk has no z faces");
  nrings = s->NR * s->NZ;
  nslots = z ? c->d.n_zslots : c->n_slots;
  /* build the list of the current state: one merge pass (substep-1 buffers) */
  if (z) CKK(dgk_zmerge(&c->d, 1, c->stream));
  else CKK(dgk_merge(&c->d, 1, c->stream));
  if ((rc = dgpu_synchronize(c))) return rc;
  nf = (int *)malloc(sizeof(int) * (size_t)nrings);
  fL = (int *)malloc(sizeof(int) * (size_t)(nslots > 0 ? nslots : 1));
  fR = (int *)malloc(sizeof(int) * (size_t)(nslots > 0 ? nslots : 1));
  fd = (double *)malloc(sizeof(double) * (size_t)(nslots > 0 ? nslots : 1));
  fc = (double *)malloc(sizeof(double) * (size_t)(nslots > 0 ? nslots : 1));
  if (!nf || !fL || !fR || !fd || !fc) {
    free(nf); free(fL); free(fR); free(fd); free(fc);
    return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  if (cudaMemcpy(nf, (z ? c->d.zpair_nf : c->d.pair_nf) + p->ann_base, sizeof(int) * (size_t)nrings,
                 cudaMemcpyDeviceToHost) ||
      cudaMemcpy(fL, z ? c->d.zfL : c->d.fL, sizeof(int) * (size_t)nslots, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(fR, z ? c->d.zfR : c->d.fR, sizeof(int) * (size_t)nslots, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(fd, z ? c->d.zfdphi : c->d.fdphi, sizeof(double) * (size_t)nslots, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(fc, z ? c->d.zfcm : c->d.fcm, sizeof(double) * (size_t)nslots, cudaMemcpyDeviceToHost)) {
    free(nf); free(fL); free(fR); free(fd); free(fc);
    return fail(c, DGPU_ERR_CUDA, "face download failed");
  }
  /* pairs: r -- ring (k, i) with i < NR-1; z -- ring (k, i) with k < NZ-1 */
  for (k = 0; k < s->NZ; ++k)
    for (i = 0; i < s->NR; ++i)
      if (z ? k < s->NZ - 1 : i < s->NR - 1) total += nf[k * s->NR + i];
  if (nf_out) *nf_out = total;
  if (total > cap) {
    free(nf); free(fL); free(fR); free(fd); free(fc);
    return fail(c, DGPU_ERR_ARG, "face list has %d faces, capacity %d", total, cap);
  }
  {
    const int nouter = z ? s->NZ - 1 : s->NR - 1, ninner = z ? s->NR : s->NZ;
    int o, n = 0;
    for (o = 0; o < nouter; ++o) {
      if (off) off[o] = n;
      for (i = 0; i < ninner; ++i) {
        const int ring = z ? o * s->NR + i : i * s->NR + o;
        const Annulus *A = &c->h_ann[p->ann_base + ring];
        const int base = z ? A->zface_base : A->face_base;
        const double fr = z ? A->zf_r : A->f_r, fperp = z ? A->zf_dperp : A->f_dperp;
        int f;
        for (f = 0; f < nf[ring]; ++f, ++n) {
          const int slot = base + f;
          if (L) L[n] = fL[slot] - p->cell_base;
          if (R) R[n] = fR[slot] - p->cell_base;
          if (r) r[n] = fr;
          if (dphi) dphi[n] = fd[slot];
          if (dA) dA[n] = fr * fd[slot] * fperp;
          if (deltaL) deltaL[n] = z ? A->zf_dl : A->f_dl;
          if (deltaR) deltaR[n] = z ? A->zf_dr : A->f_dr;
          if (cm) cm[n] = fc[slot];
        }
      }
    }
    if (off) off[nouter] = n;
  }
  free(nf); free(fL); free(fR); free(fd); free(fc);
  return DGPU_OK;
}

int dgpu_face_list(dgpu_ctx *c, int inst, int cap, int *nri, int *L, int *R, double *r, double *dphi,
                   double *dA, double *deltaL, double *deltaR, double *cm, int *nf_out) {
  return face_list_dir(c, inst, 0, cap, nri, L, R, r, dphi, dA, deltaL, deltaR, cm, nf_out);
}

int dgpu_face_list_z(dgpu_ctx *c, int inst, int cap, int *nzk, int *L, int *R, double *r, double *dphi,
                     double *dA, double *deltaL, double *deltaR, double *cm, int *nf_out) {
  return face_list_dir(c, inst, 1, cap, nzk, L, R, r, dphi, dA, deltaL, deltaR, cm, nf_out);
}

int dgpu_diagnostics(dgpu_ctx *c, int inst, double *vector, double *scalar, double *equat, double *extra) {
  const struct dgpu_sim *s;
  const DiskParams *p;
  int nvec, neq, nextra, nrow, i, imin, imax, first = 0, ncell = 0, rc = check_inst(c, inst);
  size_t need, nr;
  double *rows, *dv, *ds, *de, *dx;
  if (rc) return rc;
  if (c->h_par[inst].NZ > 1) return fail(c, DGPU_ERR_UNSUPPORTED, "diagnostics of a 3-D disk (NumZ > 1) are not implemented");
  s = c->sims[inst];
  p = &c->h_par[inst];
  dgk_diag_sizes(&nvec, &neq, &nextra, &nrow);
  imin = s->ng_min[0];
  imax = s->NR - s->ng_max[0];
  for (i = 0; i < s->NR; ++i) {
    if (i < imin) first += s->N_p[i];
    else if (i < imax) ncell += s->N_p[i];
  }
  nr = (size_t)(imax - imin);
  need = (size_t)s->NR * nrow + nr * nvec + 16 + (size_t)ncell * neq + nextra;
  if (c->diag_cap < need) {
    if (c->d_diag) cudaFree(c->d_diag);
    c->d_diag = NULL;
    c->diag_cap = 0;
    CK(cudaMalloc((void **)&c->d_diag, sizeof(double) * need));
    c->diag_cap = need;
  }
  rows = c->d_diag;
  dv = rows + (size_t)s->NR * nrow;
  ds = dv + nr * nvec;
  de = ds + 16;
  dx = de + (size_t)ncell * neq;
  CKK(dgk_diagnostics(&c->d, inst, s->NR, rows, dv, ds, equat ? de : NULL, p->cell_base + first, dx,
                      s->Z_Max - s->Z_Min, s->R_Min, s->R_Max, c->stream));
  if (vector) CK(cudaMemcpyAsync(vector, dv, sizeof(double) * nr * nvec, cudaMemcpyDeviceToHost, c->stream));
  if (scalar) CK(cudaMemcpyAsync(scalar, ds, sizeof(double) * 16, cudaMemcpyDeviceToHost, c->stream));
  if (equat) CK(cudaMemcpyAsync(equat, de, sizeof(double) * (size_t)ncell * neq, cudaMemcpyDeviceToHost, c->stream));
  if (extra) CK(cudaMemcpyAsync(extra, dx, sizeof(double) * nextra, cudaMemcpyDeviceToHost, c->stream));
  return dgpu_synchronize(c);
}

int dgpu_torque(dgpu_ctx *c, int inst, double *torque) {
  const DiskParams *p;
  int rc = check_inst(c, inst), nb;
  if (rc) return rc;
  if (!torque) return fail(c, DGPU_ERR_ARG, "null torque");
  p = &c->h_par[inst];
  if (p->NZ > 1) return fail(c, DGPU_ERR_UNSUPPORTED, "the torque of a 3-D disk (NumZ > 1) is not implemented");
  nb = (p->n_cells + dgk_block_size() - 1) / dgk_block_size();
  CKK(dgk_torque(&c->d, inst, c->d_torque, c->d_torque + nb, p->n_cells, c->stream));
  CK(cudaMemcpyAsync(torque, c->d_torque + nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return dgpu_synchronize(c);
}
