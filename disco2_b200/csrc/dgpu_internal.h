/*
 * Internal data layout shared by the C host layer and the CUDA kernels.
 *
 * Cells of every disk in a context are numbered globally, disk after disk,
 * each disk in the reference's (k, i, j) order (annulus-major: annulus i holds
 * N_p[i] consecutive cells).  Per-cell variables are structure-of-arrays:
 * variable q of cell g lives at X[q * n_cells + g].  Annulus-level constants
 * (radii, frame terms, boundary profile) live in an Annulus table; the r-faces
 * of the annulus pair (i, i+1) of a disk live in a slab of capacity
 * N_p[i] + N_p[i+1] + DGPU_FACE_SLACK starting at Annulus.face_base.
 */
#ifndef DGPU_INTERNAL_H
#define DGPU_INTERNAL_H

#include <stdint.h>

#define DGPU_NQ 5
#define DGPU_MAX_PASSIVE 3  /* NUM_N at most */
#define DGPU_FACE_SLACK 8
#define DGPU_RUN_SLACK 8
#define DGPU_WRAP_LIMIT 64
#define DGPU_STEP_KERNELS 16 /* launches per RK2 step: 8 per substep */

/* enums of src/Headers/header.h:1-13 */
enum { D_RHO, D_PPP, D_URR, D_UPP, D_UZZ };
enum { D_DDD, D_TAU, D_SRR, D_LLL, D_SZZ };
enum { DC_FIXED, DC_WCELL, DC_RIGID, DC_KEPLER, DC_OMEGA20, DC_MILOS, DC_POWERLAW };
enum { DA_FIXED, DA_KEPLER, DA_OMEGA20, DA_MILOS, DA_POWERLAW };
enum { DS_LEFT, DS_LEFTSTAR, DS_RIGHTSTAR, DS_RIGHT };
enum { DB_FIXED, DB_OUTFLOW, DB_PERIODIC };
enum { DI_SHEAR, DI_VORTEX, DI_SSTEST, DI_TORUS, DI_MILOS_MACFADYEN, DI_RAD_DOM, DI_MIDDLE,
       DI_GRESHO, DI_KEPLER_RING, DI_CIRCUMBINARY };
enum { DR_HLLC, DR_HLL };

/* device error flags (bitwise) */
#define DGPU_EF_FACE_OVERFLOW 1
#define DGPU_EF_WRAP_LIMIT 2
#define DGPU_EF_VISC_VZ 4
#define DGPU_EF_RUN_OVERFLOW 8
#define DGPU_EF_NONFINITE 16   /* a non-ghost cell's CFL step is not a number (its state holds a NaN) */
#define DGPU_EF_SWEEP_WAIT 32  /* a k_sweep block gave up waiting for the block of the previous annulus */

/* annulus kind bits */
#define DGPU_AK_CFL 1        /* non-ghost: enters the CFL minimum (cell_mindt.c:38-42) */
#define DGPU_AK_BC_FIXED 2   /* ghost annulus reset by the fixed radial boundary */
#define DGPU_AK_DAMP 4       /* inside a damping zone (cell_misc.c:98-132) */
#define DGPU_AK_SINK_SUM 8   /* counted in the Mdot sum (cell_source.c:80-88,181) */
#define DGPU_AK_IC 16        /* boundary profile ic[] is defined for this annulus */
#define DGPU_AK_MDOT 32      /* innermost non-ghost annulus: the accretion-rate objective */
#define DGPU_AK_OUT_DST 64   /* rewritten by the outflow radial boundary (cell_boundary.c:14-139):
                                k_outflow applies its damping and cell_calc_cons */

/* Per-disk parameters (constant during a run). */
typedef struct {
  int NR;           /* annuli incl. ghosts, sim_N(R_DIR) */
  int ann_base;     /* global index of annulus 0 */
  int cell_base;    /* global index of cell 0 */
  int n_cells;
  int riemann;      /* DR_HLLC / DR_HLL */
  int visc_const;
  int has_visc;     /* EXPLICIT_VISCOSITY > 0 */
  int w_numeric;
  int w_analytic;
  int grav2d;
  int phi_order;
  int rho_sink_on;
  int cooling;
  int init_type;
  int has_damp;     /* DAMP_TIME > 0 */
  int num_sinks;    /* GravMassType (cell_source.c:177) */
  int outflow;      /* bit 0: outflow radial boundary; bit 1: also the inner annulus (NoInnerBC != 1) */
  int num_n;        /* passive scalars (NUM_N): planes 5.. of prim, cons, rkcons, grad, gradp */
  int NZ;           /* layers incl. ghosts, sim_N(Z_DIR); a disk's rings (k, i) are numbered k * NR + i */
  int ngz;          /* ghost layers at each z end (0 for NumZ = 1) */
  double gamma, plm, cfl, visc, g_eps;
  double rho_floor, cs_floor, cs_cap, vel_cap;
  double t_max, poro_r1, orb_tscale, orb_t0;
  double dz, z;     /* z-extent and centre of layer 0 (the single layer of a 2-D disk) */
} DiskParams;

/* Per-ring constants (host-computed with the host libm, like the reference).
 * A ring is annulus i of layer k; a 2-D disk has one layer, so its rings are
 * its annuli.  The rings of a disk are numbered k * NR + i, so the r-face pair
 * of ring a is (a, a+1) and its z-face pair (a, a+NR). */
typedef struct {
  int inst;         /* owning disk */
  int i;            /* annulus index within the disk */
  int k;            /* layer index within the disk */
  int np;           /* N_p */
  int cell_off;     /* global cell index of j = 0 */
  int kind;         /* DGPU_AK_* bits */
  int face_base;    /* r-faces of pair (i, i+1): slab start, capacity */
  int face_cap;
  int run_base;     /* run starts of pair (i, i+1): slab start, capacity */
  int run_cap;
  int ob_off;       /* first cell of this annulus in DevPtrs.obuf; -1: the outflow boundary
                       neither reads nor writes it */
  double rm, rp, r; /* FacePos(i-1), FacePos(i), 0.5*(rp+rm) */
  double dr;        /* rp - rm */
  double dv_half;   /* .5*(rp*rp-rm*rm)   (cell_calc_cons dV factor) */
  double dv_diff;   /* rp*rp-rm*rm          (cell_add_src dV factor)  */
  double rom, rdrom, dtom; /* sim_rOm_a, sim_rdrOm_a, sim_dtOm_a at r (a = 1 tables; MILOS: device) */
  double wnum;      /* wiph for the non-rigid w_numeric_type choices (cell_set_w.c:158-201) */
  double ic[DGPU_NQ];/* single-cell initial data (boundary + damping target) */
  double damp_rate; /* rate of cell_bc_damp (0 outside the zones) */
  /* pair (i, i+1) constants (build_jloop, face_create_destroy.c:27-35) */
  double f_r, f_dl, f_dr, f_dperp;
  double f_rdrom;   /* sim_rdrOm_a at the face radius (riemann_visc_flux) */
  double z, dz;     /* centre and extent of layer k */
  /* z pair (ring a, ring a+NR) (build_jloop with zDir, face_create_destroy.c:37-46):
     slab of z faces and their runs, r = the ring's centre, deltaL/deltaR the
     half heights of layers k and k+1, deltaPerp = dr */
  int zface_base, zface_cap, zrun_base, zrun_cap;
  double zf_r, zf_dl, zf_dr, zf_dperp;
} Annulus;

/* Per-disk dynamic state (device-resident, updated by the kernels). */
typedef struct {
  double t, dt;     /* time, dt of the current step */
  double gr[2], gphi[2], gM[2], gom[2];         /* GravMass r, phi, M, omega */
  double grk_r[2], grk_phi[2], grk_M[2], grk_om[2]; /* GravMass RK copies */
  double mdot[2], macc[2];
  unsigned long long dtkey;                      /* CFL minimum (bit pattern of a positive double) */
  int pad[2];
  /* per-substep GravMass trigonometry, computed once per disk:
     gx = r cos(phi), gy = r sin(phi) of the current positions (after clean_pi),
     rkx/rky the same for the step-start copies (the CFL reads those) */
  double gx[2], gy[2], gc[2], gs[2], rkx[2], rky[2];
} InstState;

/* Kernels whose launch shape the autotuner chooses (DevPtrs.tune). */
#define DGPU_TUNE_PLM 0
#define DGPU_TUNE_FLUXPHI 1
#define DGPU_TUNE_FLUXR 2
#define DGPU_TUNE_SOURCE 3
#define DGPU_TUNE_UPDATE 4
#define DGPU_TUNE_SWEEP 5
#define DGPU_TUNE_N 6

/* Device pointers and sizes handed to every kernel. */
typedef struct {
  int n_inst, n_ann, n_cells, n_slots, n_runs;
  const DiskParams *par;
  InstState *ist;
  const Annulus *ann;
  const int *cell_ann;    /* cell -> global annulus */
  const int *slot_ann;    /* face slot -> global annulus of its pair (or -1) */
  double *prim, *cons, *rkcons, *grad, *gradp;
  double *tiph0, *tiph1;  /* ping-pong raw phi edges */
  double *tiphw;          /* phi edges wrapped into [0, 2pi] (cell_clean_pi) */
  double *rktiph, *dphi;
  double *w_ann;          /* wiph per annulus */
  double *fphi;           /* [8][n_cells] phi-face increments, face (j, j+1) at cell j */
  double *frf;            /* [8][n_slots] r-face increments */
  double *src;            /* [8][n_cells] source increments of the substep (k_source) */
  double *fS;             /* [5][n_slots] r-face slopes (WR - WL)/(deltaR + deltaL) */
  double *fdp;            /* [2][n_slots] r-face offsets dpL, dpR (wrapped to [-pi, pi]) */
  double *ann_c;          /* [4][n_ann] per substep: kappa, cos(kappa dt), sin(kappa dt), 1-exp(-rate dt) */
  int smem_face;          /* dynamic shared bytes of k_merge (0: merge reads global memory) */
  int merge_nt;           /* threads per k_merge / k_zmerge block (32..256) */
  int zghost;             /* cells of the ng lowest layers of the context's one 3-D disk, which
                             with the ng highest are the first and last cells (0: several disks) */
  int *fstart;            /* first r-face (within the pair slab) of each inner cell */
  int *rr;                /* [n_cells][4] r-face ranges (within the slab of pair i-1) of each outer cell:
                             [x, y) and [z, w) for its two runs; z = INT_MIN: more runs */
  int *fL, *fR;           /* r-face cells (global cell numbers); fL = -1 past the list of a pair */
  double *fdphi, *fcm;    /* r-face dphi and cm */
  int *pair_nf, *pair_jpmin, *pair_T, *pair_seq; /* per annulus (pair i, i+1) */
  int *runs;              /* run starts */
  double *mdot_part;      /* [n_blocks_update][2] per-block sink sums */
  unsigned int *counters; /* last-block counters */
  int *err;               /* error flags */
  double *obuf;           /* [5 + n_pass][n_ob] prims, before damping, of the annuli the outflow
                             boundary reads or writes (k_update writes them, k_outflow finishes them) */
  int n_ob;
  int n_pass;             /* passive-scalar planes (largest NUM_N of the disks): prim, cons, rkcons,
                             grad and gradp hold 5 + n_pass planes, fS 5 + n_pass, fphi and frf
                             8 + n_pass (the passive increments after the viscous ones) */
  int tune[DGPU_TUNE_N];  /* host-side launch choice of the tuned kernels: resident blocks per SM (0: built-in) */
  /* the fused substep (k_prep, k_sweep) */
  unsigned long long *cfl_ann; /* [n_ann] CFL minimum of each annulus (bit pattern; ~0: none) */
  int *sweep_flag;             /* [n_ann] last k_sweep phase done for each annulus */
  /* z faces of 3-D disks (NZ > 1): the same structures as the r faces, per
     z pair (ring a, ring a+NR) of each ring a with k < NZ-1 */
  int n_zslots, n_zruns, has_z;
  int max_nz;             /* largest NZ of the disks */
  const int *zslot_ann;   /* z-face slot -> ring of its pair (the lower ring) */
  int *zfL, *zfR;         /* z-face cells (global); zfL = -1 past the list of a pair */
  double *zfdphi, *zfcm;
  int *zfstart;           /* first z face (within the slab) of each lower-ring cell */
  int *zrr;               /* [n_cells][4] z-face ranges of each upper-ring cell (as rr) */
  int *zruns;
  int *zpair_nf, *zpair_jpmin, *zpair_T, *zpair_seq;
  double *zfS;            /* [5][n_zslots] z-face slopes */
  double *zfdp;           /* [2][n_zslots] z-face offsets dpL, dpR */
  double *zfrf;           /* [5][n_zslots] z-face increments dt*dA*F */
  double *gradz;          /* [5][n_cells] z slopes (cell_plm_rz with Z_DIR, which overwrites grad) */
} DevPtrs;

/* Forward-mode tangent: d/de of the state and of the substep intermediates
 * along one direction e, in the layouts of the matching DevPtrs arrays.
 * Only the arrays that depend on the state, on the mass ratio q or on alpha
 * have tangents: the mesh (phi edges, face list, geometry), the frozen dt and
 * the GravMass orbit phases do not. */
#define DGPU_TP_DM0 0   /* dM_0/de  */
#define DGPU_TP_DM1 1   /* dM_1/de  */
#define DGPU_TP_DR0 2   /* dr_0/de (orbit radius of mass 0) */
#define DGPU_TP_DR1 3   /* dr_1/de  */
#define DGPU_TP_DALPHA 4/* dalpha/de */
#define DGPU_TP_N 8     /* per-disk stride of TanPtrs.seed */
typedef struct {
  double *prim, *cons, *rkcons, *grad, *gradp; /* [5][n_cells] */
  double *fS;                                  /* [5][n_slots] */
  double *fphi, *src;                          /* [8][n_cells] */
  double *frf;                                 /* [8][n_slots] */
  const double *seed;                          /* [n_inst][DGPU_TP_N] */
} TanPtrs;

/* Reverse mode (one disk per context): adjoints of the state and of the
 * substep intermediates, and per-block partial adjoints of the binary and of
 * alpha.  Columns of part: DGPU_AP_* below. */
#define DGPU_AP_M0 0
#define DGPU_AP_M1 1
#define DGPU_AP_R0 2
#define DGPU_AP_R1 3
#define DGPU_AP_ALPHA 4
#define DGPU_AP_N 8
typedef struct {
  double *lW;          /* [5][n_cells] adjoint of prim */
  double *lC;          /* [5][n_cells] adjoint of cons */
  double *lCrk;        /* [5][n_cells] adjoint of rkcons (substep 2 -> substep 1) */
  double *lU;          /* [5][n_cells] adjoint of the conserved sum before cons2prim */
  double *lWt;         /* [5][n_cells] partial adjoint of prim within a substep */
  double *lG, *lGp;    /* [5][n_cells] adjoints of grad and gradp */
  double *aphiL, *aphiR; /* [15][n_cells] phi face (j, j+1): adjoints of (prim, gradp, grad) of cell j / j+1 */
  double *arL, *arR;   /* [15][n_slots] r face: the same for its inner / outer cell */
  double *fsL, *fsR;   /* [5][n_slots] adjoint of the face slope from the inner / outer cell's limiter */
  double *part;        /* [rows][DGPU_AP_N] per-block partial adjoints */
  double *acc;         /* [8]: dJ/dq, dJ/dalpha accumulated */
  const double *dq;    /* [4]: dM_0/dq, dM_1/dq, dr_0/dq, dr_1/dq */
} AdjPtrs;

#ifdef __cplusplus
extern "C" {
#endif
/* kernel launchers (dgpu_kernels.cu); return cudaError_t as int.  t = NULL
 * launches the forward kernels, t != NULL their tangent instances. */
int dgk_cellprep(const DevPtrs *d, const TanPtrs *t, int substep, void *stream);
int dgk_merge(const DevPtrs *d, int substep, void *stream);
int dgk_source(const DevPtrs *d, const TanPtrs *t, int substep, void *stream);
int dgk_rslope(const DevPtrs *d, const TanPtrs *t, void *stream);
int dgk_plm_r(const DevPtrs *d, const TanPtrs *t, int substep, void *stream);
int dgk_flux_phi(const DevPtrs *d, const TanPtrs *t, int substep, void *stream);
int dgk_flux_r(const DevPtrs *d, const TanPtrs *t, int substep, void *stream);
int dgk_update(const DevPtrs *d, const TanPtrs *t, int substep, int stop, void *stream);
int dgk_update_stage(const DevPtrs *d, int substep, int stop, void *stream);
/* the outflow radial boundary, its damping and cell_calc_cons on the annuli
 * it rewrites (one block per disk); after k_update, for stop >= 6 */
int dgk_outflow(const DevPtrs *d, int stop, void *stream);
/* 3-D disks: the z-face list (zmerge), z-face slopes, z slopes (cell_plm_rz
 * with Z_DIR), z-face fluxes, and the single-rank periodic z copy of
 * cell_syncproc_z with the cell_calc_cons of the copied cells */
int dgk_zmerge(const DevPtrs *d, int substep, void *stream);
int dgk_zslope(const DevPtrs *d, void *stream);
int dgk_plm_z(const DevPtrs *d, void *stream);
int dgk_flux_z(const DevPtrs *d, int substep, void *stream);
int dgk_zsync(const DevPtrs *d, int substep, void *stream);
/* the fused substep: k_prep (face list, phi slopes, CFL minima) then k_sweep
 * (the wavefront over the annuli); forward, no passive scalar, no outflow
 * boundary, no sink */
int dgk_prep(const DevPtrs *d, int substep, void *stream);
int dgk_sweep(const DevPtrs *d, int substep, void *stream);
/* k_update recording the conserved sum and new widths into rec (adjoint replay) */
int dgk_update_rec(const DevPtrs *d, int substep, double *rec, const int *rec_idx, void *stream);
/* the per-annulus constants of k_source only (ann_c) */
int dgk_ann_consts(const DevPtrs *d, int substep, void *stream);
int dgk_calc_cons(const DevPtrs *d, const TanPtrs *t, void *stream);
/* differentiation (dgpu_adjoint.cu) */
int dgk_objective(const DevPtrs *d, const TanPtrs *t, double *part, double *out, double *out_d, const int *idx,
                  void *stream);
int dgk_step_end(const DevPtrs *d, double *dtlog, int *idx, void *stream);
int dgk_set_dt(const DevPtrs *d, const double *dtin, const int *idx, void *stream);
int dgk_set_int(int *p, int v, void *stream);
int dgk_add_int(int *p, int dv, void *stream);
int dgk_snap(const DevPtrs *d, double *buf, InstState *ist, int save, void *stream);
int dgk_snap_tab(const DevPtrs *d, double *const *bufs, InstState *const *ists, const int *idx, int off, int save,
                 void *stream);
int dgk_adj_rows(const DevPtrs *d);
int dgk_adj_objective(const DevPtrs *d, const AdjPtrs *J, double *const *bufs, InstState *const *ists,
                      const int *idx, int off, const double *wts, const int *base, void *stream);
int dgk_adj_substep(const DevPtrs *d, const AdjPtrs *J, int substep, const double *rec, const int *idx,
                    void *stream, void *side, void *ev_fork, void *ev_join);
int dgk_adj_calc_cons(const DevPtrs *d, const AdjPtrs *J, void *stream);
/* diagnostics (dgpu_diag.cu) */
int dgk_diag_sizes(int *nvec, int *neq, int *nextra, int *nrow);
int dgk_diagnostics(const DevPtrs *d, int inst, int n_ann_disk, double *rows, double *vector, double *scalar,
                    double *equat, int eq_first, double *extra, double zspan, double rmin, double rmax, void *stream);
int dgk_torque(const DevPtrs *d, int inst, double *part, double *out, int n_inst_cells, void *stream);
int dgk_update_blocks(int n_cells);
int dgk_block_size(void);
int dgk_aos_to_soa(double *soa, int nq, int stride, int base, const double *aos, int n, void *stream);
int dgk_soa_to_aos(double *aos, int nq, int stride, int base, const double *soa, int n, void *stream);
#ifdef __cplusplus
}
#endif

#endif
