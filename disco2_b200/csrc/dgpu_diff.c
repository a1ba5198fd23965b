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
 * forward kernels and runs the substep's adjoint kernels.  The rebuild of a
 * step's intermediates runs one reverse step ahead, on its own stream and
 * buffer sets, beside the adjoint kernels of the step after it.
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

/* step graphs: logged forward step, the same without the objective (steps
 * before the objective window), the same with a frozen dt, tangent step,
 * segment replay step into stored-state set 0 / 1 (shadow buffers, second
 * stream), reverse step from set s with intermediates in buffer parity p
 * (G_REV + 2 s + p), the rebuild of a segment's first reverse step
 * (G_PRIME + 2 s + p) */
enum { G_OBJ, G_STEP, G_OBJ_DT, G_TAN, G_SEG0, G_SEG1, G_REV, G_PRIME = G_REV + 4, G_N = G_PRIME + 4 };

struct dgpu_diff {
  /* tangent */
  TanPtrs t;
  double *t_buf, *t_seed;
  /* adjoint */
  AdjPtrs J;
  double *j_buf, *j_dq;
  /* objective and dt logs, indexed on the device by *d_idx */
  double *o_part, *o_val, *o_dot, *dtlog, *dtin, *wts;
  int o_cap;
  int *d_idx, *d_base, *d_idx2;
  /* stored states: checkpoints, then two sets of a segment's K+1 step starts
   * and K mid-steps (device pointer tables tab_buf / tab_ist per set), then
   * the run's end.  A set is filled by the replay of one segment while the
   * reverse sweep reads the other. */
  Snap *snaps;
  int n_snaps;
  double **tab_buf[2];
  InstState **tab_ist[2];
  double *rec[2]; /* per set [2K][6][n_cells]: conserved sums and new widths of the substeps */
  int tab_K, tab_base;
  /* the replay's own copy of the per-cell and per-face buffers (tables shared) */
  DevPtrs sh;
  void *sh_mem;
  cudaStream_t s2;
  cudaEvent_t e_rep, e_rev;
  /* the reverse step's buffers: rb[p] holds substep 2's intermediates and
   * rb[2 + p] substep 1's, for the reverse steps of parity p; the other
   * parity's are rebuilt (stream s3) while these are reversed */
  DevPtrs rb[4];
  void *rb_mem[4];
  cudaStream_t s3;
  cudaEvent_t e_fork, e_join;
  /* step graphs (G_*), valid for tab_K */
  cudaGraphExec_t g[G_N];
  int have[G_N];
};

static void drop_graphs(struct dgpu_diff *D) {
  int k;
  for (k = 0; k < G_N; ++k)
    if (D->have[k]) {
      cudaGraphExecDestroy(D->g[k]);
      D->have[k] = 0;
    }
}

void dctx_diff_free(struct dgpu_ctx *c) {
  struct dgpu_diff *D = c->diff;
  int k;
  if (!D) return;
  drop_graphs(D);
  cudaFree(D->t_buf);
  cudaFree(D->t_seed);
  cudaFree(D->j_buf);
  cudaFree(D->j_dq);
  cudaFree(D->o_part);
  cudaFree(D->o_val);
  cudaFree(D->o_dot);
  cudaFree(D->dtlog);
  cudaFree(D->dtin);
  cudaFree(D->wts);
  cudaFree(D->d_idx);
  cudaFree(D->d_base);
  for (k = 0; k < 2; ++k) {
    cudaFree(D->tab_buf[k]);
    cudaFree(D->tab_ist[k]);
    cudaFree(D->rec[k]);
  }
  cudaFree(D->d_idx2);
  cudaFree(D->sh_mem);
  if (D->s2) cudaStreamDestroy(D->s2);
  if (D->e_rep) cudaEventDestroy(D->e_rep);
  if (D->e_rev) cudaEventDestroy(D->e_rev);
  for (k = 0; k < 4; ++k) cudaFree(D->rb_mem[k]);
  if (D->s3) cudaStreamDestroy(D->s3);
  if (D->e_fork) cudaEventDestroy(D->e_fork);
  if (D->e_join) cudaEventDestroy(D->e_join);
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
  if (P->outflow) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation with the outflow radial boundary is not implemented");
  if (P->NZ > 1) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation of a 3-D disk (NumZ > 1) is not implemented");
  if (P->num_n) return fail(c, DGPU_ERR_UNSUPPORTED, "differentiation with passive scalars is not implemented");
  return DGPU_OK;
}

static int ensure_obj(struct dgpu_ctx *c, struct dgpu_diff *D, int nsteps) {
  if (!D->d_idx) {
    CK(cudaMalloc((void **)&D->d_idx, sizeof(int)));
    CK(cudaMalloc((void **)&D->d_base, sizeof(int)));
  }
  if (D->o_cap < nsteps) {
    /* the log buffers move: graphs that write them are rebuilt */
    drop_graphs(D);
    cudaFree(D->o_val);
    cudaFree(D->o_dot);
    cudaFree(D->dtlog);
    cudaFree(D->dtin);
    cudaFree(D->wts);
    D->o_val = D->o_dot = D->dtlog = D->dtin = D->wts = NULL;
    D->o_cap = 0;
    CK(cudaMalloc((void **)&D->dtin, sizeof(double) * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->o_val, sizeof(double) * 2 * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->o_dot, sizeof(double) * 2 * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->dtlog, sizeof(double) * (size_t)nsteps));
    CK(cudaMalloc((void **)&D->wts, sizeof(double) * 2 * (size_t)nsteps));
    D->o_cap = nsteps;
  }
  if (!D->o_part)
    CK(cudaMalloc((void **)&D->o_part, sizeof(double) * 4 * ((size_t)c->n_cells / dgk_block_size() + 2)));
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

/* nck checkpoints, two sets of 2K+1 segment states (with their device
 * pointer tables S[0..K], M[0..K-1]), the run's end: nck + 4K + 3 states */
static int ensure_snaps(struct dgpu_ctx *c, struct dgpu_diff *D, int nck, int K) {
  const int count = nck + 4 * K + 3;
  int k, set;
  if (D->n_snaps < count) {
    Snap *sn = (Snap *)realloc(D->snaps, sizeof(Snap) * (size_t)count);
    if (!sn) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
    D->snaps = sn;
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
    D->tab_K = 0;
  }
  if (D->tab_K != K || D->tab_base != nck) {
    double **hb = (double **)malloc(sizeof(double *) * (size_t)(2 * K + 1));
    InstState **hi = (InstState **)malloc(sizeof(InstState *) * (size_t)(2 * K + 1));
    if (!hb || !hi) {
      free(hb);
      free(hi);
      return fail(c, DGPU_ERR_NOMEM, "out of host memory");
    }
    drop_graphs(D);
    for (set = 0; set < 2; ++set) {
      const int base = nck + set * (2 * K + 1);
      for (k = 0; k < 2 * K + 1; ++k) {
        hb[k] = D->snaps[base + k].buf;
        hi[k] = D->snaps[base + k].ist;
      }
      cudaFree(D->tab_buf[set]);
      cudaFree(D->tab_ist[set]);
      cudaFree(D->rec[set]);
      D->tab_buf[set] = NULL;
      D->tab_ist[set] = NULL;
      D->rec[set] = NULL;
      if (cudaMalloc((void **)&D->rec[set], sizeof(double) * 12 * (size_t)K * (size_t)c->n_cells) != cudaSuccess ||
          cudaMalloc((void **)&D->tab_buf[set], sizeof(double *) * (size_t)(2 * K + 1)) != cudaSuccess ||
          cudaMalloc((void **)&D->tab_ist[set], sizeof(InstState *) * (size_t)(2 * K + 1)) != cudaSuccess ||
          cudaMemcpy(D->tab_buf[set], hb, sizeof(double *) * (size_t)(2 * K + 1), cudaMemcpyHostToDevice) !=
              cudaSuccess ||
          cudaMemcpy(D->tab_ist[set], hi, sizeof(InstState *) * (size_t)(2 * K + 1), cudaMemcpyHostToDevice) !=
              cudaSuccess) {
        free(hb);
        free(hi);
        cudaGetLastError();
        D->tab_K = 0;
        return fail(c, DGPU_ERR_NOMEM, "device allocation of the segment states failed");
      }
    }
    free(hb);
    free(hi);
    D->tab_K = K;
    D->tab_base = nck;
  }
  return DGPU_OK;
}

/* The replay's buffers: every per-cell, per-face and per-annulus array the
 * step writes, and its own disk state and counters; the read-only tables and
 * the error flags are shared with the context. */
/* Lays out in fresh device memory (*mem) a copy of every per-cell, per-face
 * and per-disk buffer the step writes, in *h; the tables stay shared. */
static int alloc_shadow(struct dgpu_ctx *c, DevPtrs *h, void **mem) {
  const size_t N = (size_t)c->n_cells, S = (size_t)(c->n_slots ? c->n_slots : 1), A = (size_t)c->n_ann;
  const size_t R = (size_t)(c->n_runs ? c->n_runs : 1), B = (size_t)c->n_upd_blocks;
  size_t sz[32], off[33], k = 0, n;
  char *m;
#define SZ(bytes) sz[k++] = ((bytes) + 255) / 256 * 256
  SZ(8 * 25 * N);              /* 0: prim cons rkcons grad gradp */
  SZ(8 * 5 * N);               /* 1: tiph0 tiph1 tiphw rktiph dphi */
  SZ(8 * A);                   /* 2: w_ann */
  SZ(8 * 16 * N);              /* 3: fphi src */
  SZ(8 * 8 * S);               /* 4: frf */
  SZ(8 * 5 * S);               /* 5: fS */
  SZ(8 * 2 * S);               /* 6: fdp */
  SZ(8 * 4 * A);               /* 7: ann_c */
  SZ(4 * N);                   /* 8: fstart */
  SZ(4 * 4 * N);               /* 9: rr */
  SZ(4 * 2 * S);               /* 10: fL fR */
  SZ(8 * 2 * S);               /* 11: fdphi fcm */
  SZ(4 * 4 * A);               /* 12: pair_nf pair_jpmin pair_T pair_seq */
  SZ(4 * R);                   /* 13: runs */
  SZ(8 * 2 * B);               /* 14: mdot_part */
  SZ(4 * 8);                   /* 15: counters */
  SZ(sizeof(InstState) * (size_t)c->n_inst); /* 16: ist */
#undef SZ
  off[0] = 0;
  for (n = 0; n < k; ++n) off[n + 1] = off[n] + sz[n];
  CK(cudaMalloc(mem, off[k]));
  CK(cudaMemset(*mem, 0, off[k]));
  m = (char *)*mem;
  *h = c->d;
  h->prim = (double *)(m + off[0]);
  h->cons = h->prim + 5 * N;
  h->rkcons = h->cons + 5 * N;
  h->grad = h->rkcons + 5 * N;
  h->gradp = h->grad + 5 * N;
  h->tiph0 = (double *)(m + off[1]);
  h->tiph1 = h->tiph0 + N;
  h->tiphw = h->tiph1 + N;
  h->rktiph = h->tiphw + N;
  h->dphi = h->rktiph + N;
  h->w_ann = (double *)(m + off[2]);
  h->fphi = (double *)(m + off[3]);
  h->src = h->fphi + 8 * N;
  h->frf = (double *)(m + off[4]);
  h->fS = (double *)(m + off[5]);
  h->fdp = (double *)(m + off[6]);
  h->ann_c = (double *)(m + off[7]);
  h->fstart = (int *)(m + off[8]);
  h->rr = (int *)(m + off[9]);
  h->fL = (int *)(m + off[10]);
  h->fR = h->fL + S;
  h->fdphi = (double *)(m + off[11]);
  h->fcm = h->fdphi + S;
  h->pair_nf = (int *)(m + off[12]);
  h->pair_jpmin = h->pair_nf + A;
  h->pair_T = h->pair_jpmin + A;
  h->pair_seq = h->pair_T + A;
  h->runs = (int *)(m + off[13]);
  h->mdot_part = (double *)(m + off[14]);
  h->counters = (unsigned int *)(m + off[15]);
  h->ist = (InstState *)(m + off[16]);
  return DGPU_OK;
}

static int ensure_shadow(struct dgpu_ctx *c, struct dgpu_diff *D) {
  if (D->sh_mem) return DGPU_OK;
  int k;
  if (alloc_shadow(c, &D->sh, &D->sh_mem)) return DGPU_ERR_CUDA;
  for (k = 0; k < 4; ++k)
    if (alloc_shadow(c, &D->rb[k], &D->rb_mem[k])) return DGPU_ERR_CUDA;
  CK(cudaMalloc((void **)&D->d_idx2, sizeof(int)));
  CK(cudaStreamCreateWithFlags(&D->s2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&D->e_rep, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&D->e_rev, cudaEventDisableTiming));
  CK(cudaStreamCreateWithFlags(&D->s3, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&D->e_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&D->e_join, cudaEventDisableTiming));
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

/* ---- step graphs -------------------------------------------------------- */
/* One substep of the replay on the shadow buffers (stream s): the eight
 * kernels in order, k_update recording into rec slot 2 * (*idx) + sub - 1. */
static int shadow_substep(struct dgpu_ctx *c, DevPtrs *h, cudaStream_t s, int sub, double *rec, const int *idx) {
  CKK(dgk_cellprep(h, NULL, sub, s));
  CKK(dgk_merge(h, sub, s));
  CKK(dgk_rslope(h, NULL, s));
  CKK(dgk_plm_r(h, NULL, sub, s));
  CKK(dgk_source(h, NULL, sub, s));
  CKK(dgk_flux_phi(h, NULL, sub, s));
  CKK(dgk_flux_r(h, NULL, sub, s));
  CKK(dgk_update_rec(h, sub, rec, idx, s));
  return DGPU_OK;
}

/* The forward intermediates the reverse of a substep reads (cellprep, merge,
 * face and cell r slopes, per-annulus constants) on buffers h, stream s. */
static int prep_substep(struct dgpu_ctx *c, DevPtrs *h, cudaStream_t s, int sub) {
  CKK(dgk_cellprep(h, NULL, sub, s));
  CKK(dgk_merge(h, sub, s));
  CKK(dgk_rslope(h, NULL, s));
  CKK(dgk_plm_r(h, NULL, sub, s));
  CKK(dgk_ann_consts(h, sub, s));
  return DGPU_OK;
}

static int record_graph(struct dgpu_ctx *c, struct dgpu_diff *D, int which) {
  struct dgpu_diff *Dd = D;
  const int nbK = D->tab_K;
  const int set = which == G_SEG1 ? 1 : which >= G_REV ? ((which - G_REV) / 2) & 1 : 0;
  const int par = which >= G_REV ? (which - G_REV) & 1 : 0;
  double *const *tabS = (double *const *)D->tab_buf[set];
  InstState *const *istS = (InstState *const *)D->tab_ist[set];
  double *const *tabM = (double *const *)(D->tab_buf[set] + nbK + 1);
  InstState *const *istM = (InstState *const *)(D->tab_ist[set] + nbK + 1);
  switch (which) {
    case G_OBJ: /* one step, its objective and dt into slot *idx, ++*idx */
      if (dctx_launch_step(c)) return -1;
      if (dgk_objective(&c->d, NULL, Dd->o_part, Dd->o_val, NULL, Dd->d_idx, c->stream)) return -1;
      return dgk_step_end(&c->d, Dd->dtlog, Dd->d_idx, c->stream);
    case G_STEP: /* one step and its dt into slot *idx, ++*idx */
      if (dctx_launch_step(c)) return -1;
      return dgk_step_end(&c->d, Dd->dtlog, Dd->d_idx, c->stream);
    case G_OBJ_DT: /* the same with dt = dtin[*idx] */
      if (dgk_cellprep(&c->d, NULL, 1, c->stream) || dgk_merge(&c->d, 1, c->stream) ||
          dgk_rslope(&c->d, NULL, c->stream) || dgk_plm_r(&c->d, NULL, 1, c->stream) ||
          dgk_set_dt(&c->d, Dd->dtin, Dd->d_idx, c->stream) || dgk_source(&c->d, NULL, 1, c->stream) ||
          dgk_flux_phi(&c->d, NULL, 1, c->stream) || dgk_flux_r(&c->d, NULL, 1, c->stream) ||
          dgk_update(&c->d, NULL, 1, 7, c->stream) || dctx_substep(c, NULL, 2, DCTX_FULL, NULL, NULL))
        return -1;
      if (dgk_objective(&c->d, NULL, Dd->o_part, Dd->o_val, NULL, Dd->d_idx, c->stream)) return -1;
      return dgk_step_end(&c->d, Dd->dtlog, Dd->d_idx, c->stream);
    case G_TAN: /* one tangent step */
      if (dctx_substep(c, &Dd->t, 1, DCTX_FULL, NULL, NULL) || dctx_substep(c, &Dd->t, 2, DCTX_FULL, NULL, NULL))
        return -1;
      if (dgk_objective(&c->d, &Dd->t, Dd->o_part, Dd->o_val, Dd->o_dot, Dd->d_idx, c->stream)) return -1;
      return dgk_step_end(&c->d, Dd->dtlog, Dd->d_idx, c->stream);
    case G_SEG0:
    case G_SEG1: /* replay one step of a segment on the shadow buffers (stream s2),
                    storing its substep inputs in slot *idx2 of the set */
      if (dgk_snap_tab(&Dd->sh, tabS, istS, Dd->d_idx2, 0, 1, Dd->s2) ||
          shadow_substep(c, &Dd->sh, Dd->s2, 1, Dd->rec[set], Dd->d_idx2) ||
          dgk_snap_tab(&Dd->sh, tabM, istM, Dd->d_idx2, 0, 1, Dd->s2) ||
          shadow_substep(c, &Dd->sh, Dd->s2, 2, Dd->rec[set], Dd->d_idx2))
        return -1;
      return dgk_add_int(Dd->d_idx2, 1, Dd->s2);
    case G_REV:
    case G_REV + 1:
    case G_REV + 2:
    case G_REV + 3: { /* reverse step *idx of the segment (step n = *base + *idx)
                         on the intermediates of buffers rb[par], rb[2 + par],
                         while step *idx - 1's are rebuilt in the other parity's
                         (stream s3; at *idx = 0 the slot is clamped to 0 and the
                         rebuild goes unused) */
      DevPtrs *b2 = &Dd->rb[par], *b1 = &Dd->rb[2 + par], *n2 = &Dd->rb[1 - par], *n1 = &Dd->rb[3 - par];
      if (dgk_adj_objective(&c->d, &Dd->J, tabS, istS, Dd->d_idx, 1, Dd->wts, Dd->d_base, c->stream)) return -1;
      if (cudaEventRecord(Dd->e_fork, c->stream) != cudaSuccess ||
          cudaStreamWaitEvent(Dd->s3, Dd->e_fork, 0) != cudaSuccess)
        return -1;
      if (dgk_snap_tab(n2, tabM, istM, Dd->d_idx, -1, 0, Dd->s3) || prep_substep(c, n2, Dd->s3, 2) ||
          dgk_snap_tab(n1, tabS, istS, Dd->d_idx, -1, 0, Dd->s3) || prep_substep(c, n1, Dd->s3, 1))
        return -1;
      if (dgk_adj_substep(b2, &Dd->J, 2, Dd->rec[set], Dd->d_idx, c->stream, c->side, c->fork[0], c->fork[1]) ||
          dgk_adj_substep(b1, &Dd->J, 1, Dd->rec[set], Dd->d_idx, c->stream, c->side, c->fork[0], c->fork[1]))
        return -1;
      if (cudaEventRecord(Dd->e_join, Dd->s3) != cudaSuccess ||
          cudaStreamWaitEvent(c->stream, Dd->e_join, 0) != cudaSuccess)
        return -1;
      return dgk_add_int(Dd->d_idx, -1, c->stream);
    }
    case G_PRIME:
    case G_PRIME + 1:
    case G_PRIME + 2:
    case G_PRIME + 3: { /* the intermediates of reverse step *idx in rb[par], rb[2 + par] */
      const int pr = (which - G_PRIME) & 1;
      const int st = ((which - G_PRIME) / 2) & 1;
      double *const *tS = (double *const *)D->tab_buf[st];
      InstState *const *iS = (InstState *const *)D->tab_ist[st];
      double *const *tM = (double *const *)(D->tab_buf[st] + nbK + 1);
      InstState *const *iM = (InstState *const *)(D->tab_ist[st] + nbK + 1);
      if (dgk_snap_tab(&Dd->rb[pr], tM, iM, Dd->d_idx, 0, 0, c->stream) || prep_substep(c, &Dd->rb[pr], c->stream, 2) ||
          dgk_snap_tab(&Dd->rb[2 + pr], tS, iS, Dd->d_idx, 0, 0, c->stream) ||
          prep_substep(c, &Dd->rb[2 + pr], c->stream, 1))
        return -1;
      return DGPU_OK;
    }
  }
  return -1;
}

/* Captures graph `which` on its stream the first time, then launches it. */
static int launch_graph(struct dgpu_ctx *c, struct dgpu_diff *D, int which) {
  cudaStream_t s = (which == G_SEG0 || which == G_SEG1) ? D->s2 : c->stream;
  if (!D->have[which]) {
    cudaGraph_t g;
    int rc;
    cudaError_t e;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    rc = record_graph(c, D, which);
    e = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return fail(c, DGPU_ERR_CUDA, "differentiation step capture failed (%d)", which);
    }
    if (e != cudaSuccess) return fail(c, DGPU_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&D->g[which], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(c, DGPU_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    D->have[which] = 1;
  }
  CK(cudaGraphLaunch(D->g[which], s));
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

int dgpu_objective(dgpu_ctx *c, int nsteps, int window_start, const double *dt_in, double *dt_out, double *J) {
  struct dgpu_diff *D = NULL;
  int n, rc = run_args(c, nsteps, window_start);
  if (rc) return rc;
  if (!J) return fail(c, DGPU_ERR_ARG, "null J");
  if ((rc = diff_get(c, &D)) || (rc = ensure_obj(c, D, nsteps))) return rc;
  if (dt_in) CK(cudaMemcpyAsync(D->dtin, dt_in, sizeof(double) * (size_t)nsteps, cudaMemcpyHostToDevice, c->stream));
  CKK(dgk_set_int(D->d_idx, 0, c->stream));
  for (n = 0; n < nsteps; ++n)
    if ((rc = launch_graph(c, D, dt_in ? G_OBJ_DT : n >= window_start ? G_OBJ : G_STEP))) return rc;
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
  CKK(dgk_set_int(D->d_idx, 0, c->stream));
  for (n = 0; n < nsteps; ++n)
    if ((rc = launch_graph(c, D, G_TAN))) return rc;
  if ((rc = dgpu_synchronize(c))) return rc;
  if ((rc = window_mean(c, D, nsteps, window_start, D->o_val, J, NULL))) return rc;
  return window_mean(c, D, nsteps, window_start, D->o_dot, dJ, NULL);
}

int dgpu_adjoint(dgpu_ctx *c, int nsteps, int window_start, int ckpt_every, const double *weights, double *J,
                 double *dJ_dq, double *dJ_dalpha, double *dJ_dprim) {
  struct dgpu_diff *D = NULL;
  int n, seg, nck, K = ckpt_every, rc = run_args(c, nsteps, window_start);
  double dq[4], W, wts[2], acc[2];
  double *w = NULL;
  size_t N;
  Snap *ck, *fin;
  if (rc) return rc;
  if (K < 1) return fail(c, DGPU_ERR_ARG, "ckpt_every must be >= 1");
  if (!J) return fail(c, DGPU_ERR_ARG, "null J");
  if (K > nsteps) K = nsteps;
  nck = (nsteps + K - 1) / K;
  N = (size_t)c->n_cells;
  wts[0] = weights ? weights[0] : 1.0;
  wts[1] = weights ? weights[1] : 0.0;
  if ((rc = diff_get(c, &D)) || (rc = ensure_obj(c, D, nsteps)) || (rc = ensure_adj(c, D)) ||
      (rc = ensure_snaps(c, D, nck, K)) || (rc = ensure_shadow(c, D)))
    return rc;
  ck = D->snaps;
  fin = D->snaps + nck + 4 * K + 2;
  if ((rc = dq_consts(c, dq))) return rc;
  CK(cudaMemcpyAsync(D->j_dq, dq, sizeof(dq), cudaMemcpyHostToDevice, c->stream));

  /* forward sweep: checkpoints, dt schedule, objective */
  CKK(dgk_set_int(D->d_idx, 0, c->stream));
  for (n = 0; n < nsteps; ++n) {
    if (n % K == 0) CKK(dgk_snap(&c->d, ck[n / K].buf, ck[n / K].ist, 1, c->stream));
    /* the objective only inside its window */
    if ((rc = launch_graph(c, D, n >= window_start ? G_OBJ : G_STEP))) return rc;
  }
  CKK(dgk_snap(&c->d, fin->buf, fin->ist, 1, c->stream));
  if ((rc = dgpu_synchronize(c))) return rc;
  if ((rc = window_mean(c, D, nsteps, window_start, D->o_val, J, &W))) return rc;

  /* objective weights of each step: w_k dt_n / sum dt over the window */
  w = (double *)malloc(sizeof(double) * 3 * (size_t)nsteps);
  if (!w) return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  if (cudaMemcpy(w + 2 * nsteps, D->dtlog, sizeof(double) * (size_t)nsteps, cudaMemcpyDeviceToHost) != cudaSuccess) {
    free(w);
    return fail(c, DGPU_ERR_CUDA, "dt download failed");
  }
  for (n = 0; n < nsteps; ++n) {
    double f = n >= window_start ? w[2 * nsteps + n] / W : 0.0;
    w[2 * n] = wts[0] * f;
    w[2 * n + 1] = wts[1] * f;
  }
  rc = cudaMemcpy(D->wts, w, sizeof(double) * 2 * (size_t)nsteps, cudaMemcpyHostToDevice) != cudaSuccess
           ? fail(c, DGPU_ERR_CUDA, "weight upload failed")
           : DGPU_OK;
  free(w);
  if (rc) return rc;

  /* reverse sweep, segment by segment: the replay of segment seg - 1 (shadow
   * buffers, stream s2, stored-state set (seg - 1) % 2) runs while segment seg
   * is reversed (context buffers, the context's stream, set seg % 2) */
  CK(cudaMemsetAsync(D->J.lW, 0, sizeof(double) * 15 * N, c->stream));
  CK(cudaMemsetAsync(D->J.acc, 0, sizeof(double) * 8, c->stream));
  CK(cudaEventRecord(D->e_rev, c->stream));
  for (seg = nck; seg >= 0; --seg) {
    /* replay segment seg - 1 once the reverse of seg + 1 (same set) is done */
    if (seg - 1 >= 0) {
      const int rs = seg - 1, n0 = rs * K, n1 = n0 + K < nsteps ? n0 + K : nsteps, set = rs & 1;
      CK(cudaStreamWaitEvent(D->s2, D->e_rev, 0));
      CKK(dgk_snap(&D->sh, ck[rs].buf, ck[rs].ist, 0, D->s2));
      CKK(dgk_set_int(D->d_idx2, 0, D->s2));
      for (n = n0; n < n1; ++n)
        if ((rc = launch_graph(c, D, set ? G_SEG1 : G_SEG0))) return rc;
      /* the segment's end state in slot n1 - n0 */
      CKK(dgk_snap_tab(&D->sh, (double *const *)D->tab_buf[set], (InstState *const *)D->tab_ist[set], D->d_idx2, 0,
                       1, D->s2));
    }
    /* reverse segment seg, replayed in the previous iteration */
    if (seg < nck) {
      const int n0 = seg * K, n1 = n0 + K < nsteps ? n0 + K : nsteps, set = seg & 1;
      CK(cudaStreamWaitEvent(c->stream, D->e_rep, 0));
      CKK(dgk_set_int(D->d_idx, n1 - n0 - 1, c->stream));
      CKK(dgk_set_int(D->d_base, n0, c->stream));
      if ((rc = launch_graph(c, D, G_PRIME + 2 * set + ((n1 - 1 - n0) & 1)))) return rc;
      for (n = n1 - 1; n >= n0; --n)
        if ((rc = launch_graph(c, D, G_REV + 2 * set + ((n - n0) & 1)))) return rc;
      CK(cudaEventRecord(D->e_rev, c->stream));
    }
    if (seg - 1 >= 0) CK(cudaEventRecord(D->e_rep, D->s2));
  }
  /* the initial cons are cell_calc_cons of the initial prims */
  CKK(dgk_snap(&c->d, ck[0].buf, ck[0].ist, 0, c->stream));
  CKK(dgk_adj_calc_cons(&c->d, &D->J, c->stream));
  if (dJ_dprim) {
    CKK(dgk_soa_to_aos(c->d_stage, 5, c->n_cells, 0, D->J.lW, c->n_cells, c->stream));
    CK(cudaMemcpyAsync(dJ_dprim, c->d_stage, sizeof(double) * 5 * N, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(acc, D->J.acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
  /* leave the context at the end of the run, like the forward */
  CKK(dgk_snap(&c->d, fin->buf, fin->ist, 0, c->stream));
  if ((rc = dgpu_synchronize(c))) return rc;
  if (dJ_dq) *dJ_dq = acc[0];
  if (dJ_dalpha) *dJ_dalpha = acc[1];
  return DGPU_OK;
}
