/*
 * The device context, private to the host layer (dgpu_ctx.c: state and the
 * step; dgpu_diff.c: objective, tangent and adjoint runs).
 */
#ifndef DGPU_CTX_H
#define DGPU_CTX_H

#include <cuda_runtime.h>

#include "../../include/disco_gpu.h"
#include "dgpu_internal.h"
#include "dgpu_sim.h"

struct dgpu_diff; /* differentiation buffers (dgpu_diff.c), allocated on first use */

struct dgpu_ctx {
  int device;
  cudaStream_t stream;
  int own_stream;
  cudaStream_t side;        /* second stream: concurrent branches inside the step graph */
  cudaEvent_t fork[4];
  int n_inst;
  struct dgpu_sim **sims;
  DiskParams *h_par;
  Annulus *h_ann;
  int n_ann, n_cells, n_slots, n_runs, n_upd_blocks;
  int n_ob;              /* cells in d.obuf (0: no disk has an outflow radial boundary) */
  int n_pass;            /* passive-scalar planes (largest NUM_N) */
  DevPtrs d;          /* device pointers */
  DiskParams *d_par;
  InstState *d_ist;
  Annulus *d_ann;
  int *d_cell_ann, *d_slot_ann, *d_zslot_ann;
  double *d_stage;    /* AoS staging buffer: max cells of a disk x NQ */
  double *d_torque;   /* partial sums + result */
  cudaGraphExec_t graph;
  int have_graph;
  int fused_ok;       /* every disk can take the fused substep (k_prep + k_sweep) */
  int fused;          /* the step uses it */
  struct dgpu_diff *diff;
  double *d_diag;     /* diagnostics buffers (allocated on first use) */
  size_t diag_cap;    /* their size in doubles */
  char err[512];
};

/* Records a failure message on the context (or the thread's create error when
 * c is NULL) and returns code. */
int dctx_fail(struct dgpu_ctx *c, int code, const char *fmt, ...);
/* Reads and clears the device error flags; DGPU_OK or the matching error. */
int dctx_read_err(struct dgpu_ctx *c);
/* Launches one substep on the context's stream, forward (t == NULL) or
 * tangent: DCTX_FULL the eight kernels; DCTX_REC the same with k_update
 * recording into rec slot 2 * (*rec_idx) + substep - 1 (forward only);
 * DCTX_ADJPREP only what the substep's adjoint reads (phi slopes, face list,
 * face slopes, r slopes, annulus constants). */
enum { DCTX_FULL, DCTX_REC, DCTX_ADJPREP };
int dctx_substep(struct dgpu_ctx *c, const TanPtrs *t, int substep, int mode, double *rec, const int *rec_idx);
/* Launches one RK2 step (the sequence the step graph captures) on the
 * context's stream. */
int dctx_launch_step(struct dgpu_ctx *c);
/* Frees the differentiation buffers (dgpu_diff.c). */
void dctx_diff_free(struct dgpu_ctx *c);

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return dctx_fail(c, DGPU_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                           \
  } while (0)
#define CKK(call)                                                                         \
  do {                                                                                    \
    int e_ = (call);                                                                      \
    if (e_ != 0)                                                                          \
      return dctx_fail(c, DGPU_ERR_CUDA, "%s: %s (%s:%d)", #call,                     \
                           cudaGetErrorString((cudaError_t)e_), __FILE__, __LINE__);      \
  } while (0)

#endif
