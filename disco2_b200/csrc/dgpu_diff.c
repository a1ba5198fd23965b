/*
 * Objective, forward-mode tangent and reverse-mode adjoint runs of the step
 * (C over the CUDA runtime API).
 *
 * Objectives (neither exists in the reference; both are defined from its
 * quantities): after each step n of a run, the binary torque
 * T_n = -sum over non-ghost cells of r rho dV F_phi (F_phi of gravMassForce,
 * src/Cell/cell_source.c:49-71) and the accretion rate through the innermost
 * non-ghost annulus Mdot_n = -sum rho v_r r dphi dz.  A run of nsteps steps
 * reports their dt-weighted means over the steps window_start+1..nsteps:
 *   J_k = sum_n dt_n X_{k,n} / sum_n dt_n.
 * Differentiation freezes the dt schedule (dt_n is the CFL value of the
 * unperturbed run, a constant of the derivative) and the mesh: the runs accept
 * only state-independent mesh motion (no C_RIGID), so the phi edges, the face
 * list and all geometry are the same in every perturbed run.  The inputs are
 * the mass ratio q (through the binary's masses and orbit radii), alpha
 * (Explicit_Viscosity) and the initial prims.
 *
 * The adjoint stores the state every ckpt_every steps, and replays each
 * segment forward before running it backwards: per step it keeps the state
 * before each substep, rebuilds that substep's intermediates with the
 * forward kernels and runs the substep's adjoint kernels.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dgpu_ctx.h"

#define fail dctx_fail

/* A stored state: every per-cell array a substep reads, and the disk state. */
typedef struct {
  double *buf; /* [19][n_cells]: prim, cons, rkcons (5 each), tiph0, tiph1, rktiph, dphi */
  InstState *ist;
} Snap;

struct dgpu_diff {
  /* tangent */
  TanPtrs t;
  double *t_buf, *t_seed;
  /* adjoint */
  AdjPtrs J;
  double *j_buf, *j_dq;
  /* objective */
  double *o_part, *o_val, *o_dot, *dtlog, *dtin;
  int o_cap;
  /* stored states */
  Snap *snaps;
  int n_snaps;
};

void dctx_diff_free(struct dgpu_ctx *c) {
  struct dgpu_diff *D = c->diff;
  int k;
  if (!D) return;
  cudaFree(D->t_buf);
  cudaFree(D->t_seed);
  cudaFree(D->j_buf);
  cudaFree(D->j_dq);
  cudaFree(D->o_part);
  cudaFree(D->o_val);
  cudaFree(D->o_dot);
  cudaFree(D->dtlog);
  cudaFree(D->dtin);
  for (k = 0; k < D->n_snaps; ++k) {
    cudaFree(D->snaps[k].buf);
    cudaFree(D->snaps[k].ist);
  }
  free(D->snaps);
  free(D);
  c->diff = NULL;
}

static int diff_get(struct dgpu_ctx *c, struct dgpu_diff **out) {
  if (!c->diff) {
    c->diff = (struct dgpu_diff *)calloc(1, sizeof(struct dgpu_diff));
    if (!c->diff) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  *out = c->diff;
  return DGPU_OK;
}

/* The differentiated runs: one disk, state-independent mesh, no cooling or
 * sinks (their clamps and the sink radius make the step non-smooth). */
static int diff_check(struct dgpu_ctx *c) {
  const DiskParams *P = &c->h_par[0];
  if (c->n_inst != 1) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation needs a context with one disk");
  if (P->w_numeric == DC_RIGID)
    return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation needs a state-independent mesh (w_numeric_type != C_RIGID)");
  if (P->cooling) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation with Cooling is not implemented");
  if (P->rho_sink_on) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation with RhoSinkOn is not implemented");
  return DGPU_OK;
}

static int ensure_obj(struct dgpu_ctx *c, struct dgpu_diff *D, int nsteps) {
  if (D->o_cap < nsteps) {
    cudaFree(D->o_val);
    cudaFree(D->o_dot);
    cudaFree(D->dtlog);
    cudaFree(D->dtin);
    D->o_val = D->o_dot = D->dtlog = D->dtin = NULL;
    D->o_cap = 0;
    CK(cudaMalloc((void **)&D->dtin, sizeof(double) * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->o_val, sizeof(double) * 2 * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->o_dot, sizeof(double) * 2 * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->dtlog, sizeof(double) * (size_t)nsteps));
    D->o_cap = nsteps;
  }
  if (!D->o_part) CK(cudaMalloc((void **)&D->o_part, sizeof(double) * 4 * ((size_t)c->n_cells / 256 + 2)));
  return DGPU_OK;
}

static int ensure_tan(struct dgpu_ctx *c, struct dgpu_diff *D) {
  size_t N = (size_t)c->n_cells, S = (size_t)(c->n_slots ? c->n_slots : 1), n;
  double *p;
  if (D->t_buf) return DGPU_OK;
  n = 25 * N + 5 * S + 16 * N + 8 * S;
  CK(cudaMalloc((void **)&D->t_buf, sizeof(double) * n));
  CK(cudaMalloc((void **)&D->t_seed, sizeof(double) * DGPU_TP_N));
  p = D->t_buf;
  D->t.prim = p; p += 5 * N;
  D->t.cons = p; p += 5 * N;
  D->t.rkcons = p; p += 5 * N;
  D->t.grad = p; p += 5 * N;
  D->t.gradp = p; p += 5 * N;
  D->t.fS = p; p += 5 * S;
  D->t.fphi = p; p += 8 * N;
  D->t.src = p; p += 8 * N;
  D->t.frf = p;
  D->t.seed = D->t_seed;
  return DGPU_OK;
}

static int ensure_adj(struct dgpu_ctx *c, struct dgpu_diff *D) {
  size_t N = (size_t)c->n_cells, S = (size_t)(c->n_slots ? c->n_slots : 1), rows, n;
  double *p;
  if (D->j_buf) return DGPU_OK;
  rows = (size_t)dgk_adj_rows(&c->d) + 1;
  n = 35 * N + 30 * N + 30 * S + 10 * S + DGPU_AP_N * rows + 8;
  CK(cudaMalloc((void **)&D->j_buf, sizeof(double) * n));
  CK(cudaMalloc((void **)&D->j_dq, sizeof(double) * 4));
  p = D->j_buf;
  D->J.lW = p; p += 5 * N;
  D->J.lC = p; p += 5 * N;
  D->J.lCrk = p; p += 5 * N;
  D->J.lU = p; p += 5 * N;
  D->J.lWt = p; p += 5 * N;
  D->J.lG = p; p += 5 * N;
  D->J.lGp = p; p += 5 * N;
  D->J.aphiL = p; p += 15 * N;
  D->J.aphiR = p; p += 15 * N;
  D->J.arL = p; p += 15 * S;
  D->J.arR = p; p += 15 * S;
  D->J.fsL = p; p += 5 * S;
  D->J.fsR = p; p += 5 * S;
  D->J.part = p; p += DGPU_AP_N * rows;
  D->J.acc = p;
  D->J.dq = D->j_dq;
  return DGPU_OK;
}

static int ensure_snaps(struct dgpu_ctx *c, struct dgpu_diff *D, int count) {
  int k;
  if (D->n_snaps >= count) return DGPU_OK;
  {
    Snap *s = (Snap *)realloc(D->snaps, sizeof(Snap) * (size_t)count);
    if (!s) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
    D->snaps = s;
  }
  for (k = D->n_snaps; k < count; ++k) {
    D->snaps[k].buf = NULL;
    D->snaps[k].ist = NULL;
    if (cudaMalloc((void **)&D->snaps[k].buf, sizeof(double) * 19 * (size_t)c->n_cells) != cudaSuccess ||
        cudaMalloc((void **)&D->snaps[k].ist, sizeof(InstState) * (size_t)c->n_inst) != cudaSuccess) {
      cudaFree(D->snaps[k].buf);
      D->n_snaps = k;
      cudaGetLastError();
      return fail(c, DGPU_ERR_NOMEM, "device allocation of %d stored states failed", count);
    }
  }
  D->n_snaps = count;
  return DGPU_OK;
}

static int snap_copy(struct dgpu_ctx *c, const Snap *s, int save) {
  size_t N = (size_t)c->n_cells, b = sizeof(double) * N;
  double *arr[7] = {c->d.prim, c->d.cons, c->d.rkcons, c->d.tiph0, c->d.tiph1, c->d.rktiph, c->d.dphi};
  size_t off[7] = {0, 5 * N, 10 * N, 15 * N, 16 * N, 17 * N, 18 * N};
  size_t len[7] = {5 * b, 5 * b, 5 * b, b, b, b, b};
  int k;
  enum cudaMemcpyKind kind = cudaMemcpyDeviceToDevice;
  for (k = 0; k < 7; ++k) {
    if (save) CK(cudaMemcpyAsync(s->buf + off[k], arr[k], len[k], kind, c->stream));
    else CK(cudaMemcpyAsync(arr[k], s->buf + off[k], len[k], kind, c->stream));
  }
  if (save) CK(cudaMemcpyAsync(s->ist, c->d_ist, sizeof(InstState) * (size_t)c->n_inst, kind, c->stream));
  else CK(cudaMemcpyAsync(c->d_ist, s->ist, sizeof(InstState) * (size_t)c->n_inst, kind, c->stream));
  return DGPU_OK;
}

/* d/dq of the binary's masses and orbit radii (gravMass_init_binary,
 * src/GravMass/GravMass_init.c:55-86, and gravMass_move, GravMass_misc.c:31-64:
 * M_0 = 1/(1+q), M_1 = q/(1+q), r_0 = M_1 a / M, r_1 = M_0 a / M). */
static int dq_consts(struct dgpu_ctx *c, double *dq) {
  InstState st;
  const struct dgpu_sim *s = c->sims[0];
  CK(cudaMemcpyAsync(&st, c->d_ist, sizeof(InstState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  memset(dq, 0, 4 * sizeof(double));
  if (s->GravMassType == 2) {
    double q = s->MassRatio;
    double dm1 = 1.0 / ((1.0 + q) * (1.0 + q));
    double a = st.gr[0] + st.gr[1], M = st.gM[0] + st.gM[1];
    dq[0] = -dm1;
    dq[1] = dm1;
    dq[2] = a / M * dm1;
    dq[3] = -a / M * dm1;
  }
  return DGPU_OK;
}

static int step_log(struct dgpu_ctx *c, struct dgpu_diff *D, int n) {
  CK(cudaMemcpyAsync(D->dtlog + n, &c->d_ist[0].dt, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return DGPU_OK;
}

static int window_mean(struct dgpu_ctx *c, struct dgpu_diff *D, int nsteps, int w0, const double *vals,
                       double *out, double *wsum) {
  double *dt = (double *)malloc(sizeof(double) * (size_t)nsteps);
  double *v = (double *)malloc(sizeof(double) * 2 * (size_t)nsteps);
  double s0 = 0.0, s1 = 0.0, W = 0.0;
  int n;
  if (!dt || !v) {
    free(dt);
    free(v);
    return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  if (cudaMemcpy(dt, D->dtlog, sizeof(double) * (size_t)nsteps, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(v, vals, sizeof(double) * 2 * (size_t)nsteps, cudaMemcpyDeviceToHost) != cudaSuccess) {
    free(dt);
    free(v);
    return fail(c, DGPU_ERR_CUDA, "objective download failed");
  }
  for (n = w0; n < nsteps; ++n) {
    s0 += dt[n] * v[2 * n];
    s1 += dt[n] * v[2 * n + 1];
    W += dt[n];
  }
  out[0] = s0 / W;
  out[1] = s1 / W;
  if (wsum) *wsum = W;
  free(dt);
  free(v);
  return DGPU_OK;
}

static int run_args(struct dgpu_ctx *c, int nsteps, int w0) {
  if (!c) return DGPU_ERR_ARG;
  if (nsteps < 1 || w0 < 0 || w0 >= nsteps)
    return fail(c, DGPU_ERR_ARG, "need nsteps >= 1 and 0 <= window_start < nsteps");
  cudaSetDevice(c->device);
  return diff_check(c);
}

/* One step with dt = dt_dev[0] in place of the CFL value (timestep_set_dt,
 * src/TimeStep/timestep_set.c:16-21): the kernels of substep 1 up to the CFL
 * minimum, then the given dt, then the rest. */
static int step_frozen_dt(struct dgpu_ctx *c, const double *dt_dev) {
  CKK(dgk_cellprep(&c->d, NULL, 1, c->stream));
  CKK(dgk_merge(&c->d, 1, c->stream));
  CKK(dgk_rslope(&c->d, NULL, c->stream));
  CKK(dgk_plm_r(&c->d, NULL, 1, c->stream));
  CK(cudaMemcpyAsync(&c->d_ist[0].dt, dt_dev, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CKK(dgk_source(&c->d, NULL, 1, c->stream));
  CKK(dgk_flux_phi(&c->d, NULL, 1, c->stream));
  CKK(dgk_flux_r(&c->d, NULL, 1, c->stream));
  CKK(dgk_update(&c->d, NULL, 1, 7, c->stream));
  return dctx_substep(c, NULL, 2, 1);
}

int dgpu_objective(dgpu_ctx *c, int nsteps, int window_start, const double *dt_in, double *dt_out, double *J) {
  struct dgpu_diff *D = NULL;
  int n, rc = run_args(c, nsteps, window_start);
  if (rc) return rc;
  if (!J) return fail(c, DGPU_ERR_ARG, "null J");
  if ((rc = diff_get(c, &D)) || (rc = ensure_obj(c, D, nsteps))) return rc;
  if (dt_in) CK(cudaMemcpyAsync(D->dtin, dt_in, sizeof(double) * (size_t)nsteps, cudaMemcpyHostToDevice, c->stream));
  for (n = 0; n < nsteps; ++n) {
    rc = dt_in ? step_frozen_dt(c, D->dtin + n) : dgpu_step_rk2(c, 1);
    if (rc || (rc = step_log(c, D, n))) return rc;
    if (n >= window_start) CKK(dgk_objective(&c->d, NULL, D->o_part, D->o_val + 2 * n, NULL, c->stream));
  }
  if ((rc = dgpu_synchronize(c))) return rc;
  if (dt_out) CK(cudaMemcpy(dt_out, D->dtlog, sizeof(double) * (size_t)nsteps, cudaMemcpyDeviceToHost));
  return window_mean(c, D, nsteps, window_start, D->o_val, J, NULL);
}

int dgpu_tangent(dgpu_ctx *c, int nsteps, int window_start, double dq_dir, double dalpha_dir,
                 const double *dprim, double *J, double *dJ) {
  struct dgpu_diff *D = NULL;
  int n, rc = run_args(c, nsteps, window_start);
  double dq[4], seed[DGPU_TP_N];
  if (rc) return rc;
  if (!J || !dJ) return fail(c, DGPU_ERR_ARG, "null J or dJ");
  if ((rc = diff_get(c, &D)) || (rc = ensure_obj(c, D, nsteps)) || (rc = ensure_tan(c, D))) return rc;
  if ((rc = dq_consts(c, dq))) return rc;
  memset(seed, 0, sizeof(seed));
  seed[DGPU_TP_DM0] = dq[0] * dq_dir;
  seed[DGPU_TP_DM1] = dq[1] * dq_dir;
  seed[DGPU_TP_DR0] = dq[2] * dq_dir;
  seed[DGPU_TP_DR1] = dq[3] * dq_dir;
  seed[DGPU_TP_DALPHA] = dalpha_dir;
  CK(cudaMemcpyAsync(D->t_seed, seed, sizeof(seed), cudaMemcpyHostToDevice, c->stream));
  {
    size_t N = (size_t)c->n_cells, S = (size_t)(c->n_slots ? c->n_slots : 1);
    CK(cudaMemsetAsync(D->t_buf, 0, sizeof(double) * (41 * N + 13 * S), c->stream));
  }
  if (dprim) {
    CK(cudaMemcpyAsync(c->d_stage, dprim, sizeof(double) * 5 * (size_t)c->n_cells, cudaMemcpyHostToDevice,
                       c->stream));
    CKK(dgk_aos_to_soa(D->t.prim, 5, c->n_cells, 0, c->d_stage, c->n_cells, c->stream));
  }
  CKK(dgk_calc_cons(&c->d, &D->t, c->stream));
  for (n = 0; n < nsteps; ++n) {
    if ((rc = dctx_substep(c, &D->t, 1, 1)) || (rc = dctx_substep(c, &D->t, 2, 1))) return rc;
    if ((rc = step_log(c, D, n))) return rc;
    if (n >= window_start)
      CKK(dgk_objective(&c->d, &D->t, D->o_part, D->o_val + 2 * n, D->o_dot + 2 * n, c->stream));
  }
  if ((rc = dgpu_synchronize(c))) return rc;
  if ((rc = window_mean(c, D, nsteps, window_start, D->o_val, J, NULL))) return rc;
  return window_mean(c, D, nsteps, window_start, D->o_dot, dJ, NULL);
}

int dgpu_adjoint(dgpu_ctx *c, int nsteps, int window_start, int ckpt_every, const double *weights, double *J,
                 double *dJ_dq, double *dJ_dalpha, double *dJ_dprim) {
  struct dgpu_diff *D = NULL;
  int n, seg, nck, K = ckpt_every, rc = run_args(c, nsteps, window_start);
  double dq[4], W, wts[2], acc[2];
  double *dt = NULL;
  size_t N;
  Snap *ck, *sS, *sM, *fin;
  if (rc) return rc;
  if (K < 1) return fail(c, DGPU_ERR_ARG, "ckpt_every must be >= 1");
  if (!J) return fail(c, DGPU_ERR_ARG, "null J");
  if (K > nsteps) K = nsteps;
  nck = (nsteps + K - 1) / K;
  N = (size_t)c->n_cells;
  wts[0] = weights ? weights[0] : 1.0;
  wts[1] = weights ? weights[1] : 0.0;
  if ((rc = diff_get(c, &D)) || (rc = ensure_obj(c, D, nsteps)) || (rc = ensure_adj(c, D)) ||
      (rc = ensure_snaps(c, D, nck + 2 * K + 2)))
    return rc;
  ck = D->snaps;
  sS = ck + nck;     /* K + 1: state before substep 1 of each step of a segment, and the segment's end */
  sM = sS + K + 1;   /* K: state before substep 2 */
  fin = sM + K;
  if ((rc = dq_consts(c, dq))) return rc;
  CK(cudaMemcpyAsync(D->j_dq, dq, sizeof(dq), cudaMemcpyHostToDevice, c->stream));

  /* forward sweep: checkpoints, dt schedule, objective */
  for (n = 0; n < nsteps; ++n) {
    if (n % K == 0 && (rc = snap_copy(c, &ck[n / K], 1))) return rc;
    if ((rc = dgpu_step_rk2(c, 1)) || (rc = step_log(c, D, n))) return rc;
    if (n >= window_start) CKK(dgk_objective(&c->d, NULL, D->o_part, D->o_val + 2 * n, NULL, c->stream));
  }
  if ((rc = snap_copy(c, fin, 1))) return rc;
  if ((rc = dgpu_synchronize(c))) return rc;
  if ((rc = window_mean(c, D, nsteps, window_start, D->o_val, J, &W))) return rc;
  dt = (double *)malloc(sizeof(double) * (size_t)nsteps);
  if (!dt) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  if (cudaMemcpy(dt, D->dtlog, sizeof(double) * (size_t)nsteps, cudaMemcpyDeviceToHost) != cudaSuccess) {
    free(dt);
    return fail(c, DGPU_ERR_CUDA, "dt download failed");
  }

  /* reverse sweep */
  rc = DGPU_OK;
  if (cudaMemsetAsync(D->J.lW, 0, sizeof(double) * 15 * N, c->stream) != cudaSuccess ||
      cudaMemsetAsync(D->J.acc, 0, sizeof(double) * 8, c->stream) != cudaSuccess)
    rc = fail(c, DGPU_ERR_CUDA, "adjoint reset failed");
  for (seg = nck - 1; seg >= 0 && rc == DGPU_OK; --seg) {
    int n0 = seg * K, n1 = n0 + K < nsteps ? n0 + K : nsteps;
    if ((rc = snap_copy(c, &ck[seg], 0))) break;
    for (n = n0; n < n1 && rc == DGPU_OK; ++n) {
      if (!(rc = snap_copy(c, &sS[n - n0], 1)) && !(rc = dctx_substep(c, NULL, 1, 1)) &&
          !(rc = snap_copy(c, &sM[n - n0], 1)))
        rc = dctx_substep(c, NULL, 2, 1);
    }
    if (rc || (rc = snap_copy(c, &sS[n1 - n0], 1))) break;
    for (n = n1 - 1; n >= n0 && rc == DGPU_OK; --n) {
      if (n >= window_start) {
        double w = dt[n] / W;
        if ((rc = snap_copy(c, &sS[n - n0 + 1], 0))) break;
        if (dgk_adj_objective(&c->d, &D->J, wts[0] * w, wts[1] * w, c->stream)) {
          rc = fail(c, DGPU_ERR_CUDA, "objective adjoint launch failed");
          break;
        }
      }
      if ((rc = snap_copy(c, &sM[n - n0], 0)) || (rc = dctx_substep(c, NULL, 2, 0))) break;
      if (dgk_adj_substep(&c->d, &D->J, 2, c->stream)) {
        rc = fail(c, DGPU_ERR_CUDA, "adjoint launch failed");
        break;
      }
      if ((rc = snap_copy(c, &sS[n - n0], 0)) || (rc = dctx_substep(c, NULL, 1, 0))) break;
      if (dgk_adj_substep(&c->d, &D->J, 1, c->stream)) {
        rc = fail(c, DGPU_ERR_CUDA, "adjoint launch failed");
        break;
      }
    }
  }
  free(dt);
  if (rc) return rc;
  /* the initial cons are cell_calc_cons of the initial prims */
  if ((rc = snap_copy(c, &ck[0], 0))) return rc;
  CKK(dgk_adj_calc_cons(&c->d, &D->J, c->stream));
  if (dJ_dprim) {
    CKK(dgk_soa_to_aos(c->d_stage, 5, c->n_cells, 0, D->J.lW, c->n_cells, c->stream));
    CK(cudaMemcpyAsync(dJ_dprim, c->d_stage, sizeof(double) * 5 * N, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(acc, D->J.acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
  /* leave the context at the end of the run, like the forward */
  if ((rc = snap_copy(c, fin, 0))) return rc;
  if ((rc = dgpu_synchronize(c))) return rc;
  if (dJ_dq) *dJ_dq = acc[0];
  if (dJ_dalpha) *dJ_dalpha = acc[1];
  return DGPU_OK;
}
