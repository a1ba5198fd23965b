/*
 * disco_gpu.h -- C ABI of the B200 moving-mesh finite-volume step.
 *
 * The library replaces the per-step hot path of Disco2: timestep_rk2 and
 * everything below it (src/Headers/TimeStep.h:21-32, Face.h:22, Riemann.h:37-42,
 * Cell.h:25-91, GravMass.h:24-46).  Host code is C; all per-cell and per-face
 * work runs in hand-written sm_100a kernels on one GPU.  Plain C types only:
 * pointers, sizes, doubles, ints.  No CUDA or torch types appear here; the
 * optional stream is passed as `void *` (a cudaStream_t, or NULL for the
 * library's own stream).
 *
 * Conventions
 *   - Every function that can fail returns int: 0 (DGPU_OK) or a negative
 *     DGPU_ERR_* code; dgpu_last_error() returns the message.  The reference
 *     printf()s and exit()s instead (19 sites, e.g. Riemann_routines.c:168,
 *     Riemann_routines.c:271-274, cell_set_w.c:15-16).
 *   - Ownership: the caller owns every host buffer; a context owns all device
 *     memory it allocates.  No global state except the last-error string.
 *   - Cell order at the boundary is the reference's (k, i, j) order of the
 *     contiguous cell array built by cell_create (src/Cell/cell_create_destroy.c:
 *     37-48), ghost annuli included; per-cell variables are NUM_Q-wide rows,
 *     prim = (rho, P, v_r, omega, v_z), cons = (D, tau, S_r, L, S_z) x dV
 *     (src/Headers/header.h:1-2).
 *   - Threading: one host thread per context at a time.
 *   - A context holds one or more independent disks ("instances"); the plain
 *     method is a context with one instance, the batched sweep one with many.
 */
#ifndef DISCO_GPU_H
#define DISCO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define DGPU_OK 0
#define DGPU_ERR_ARG (-1)          /* bad argument or index */
#define DGPU_ERR_PARFILE (-2)      /* parfile missing, unreadable or missing a key */
#define DGPU_ERR_UNSUPPORTED (-3)  /* option outside the implemented path (e.g. NumZ > 1
                                      without a periodic z boundary) */
#define DGPU_ERR_CUDA (-4)         /* a CUDA runtime call failed */
#define DGPU_ERR_FACE_OVERFLOW (-5)/* face list exceeded its buffer (device flag) */
#define DGPU_ERR_NUMERIC (-6)      /* device-detected condition the reference exit()s on or
                                      loops forever on, or a NaN in a non-ghost cell's state */
#define DGPU_ERR_NOMEM (-7)        /* host or device allocation failed */
#define DGPU_ERR_IO (-8)           /* checkpoint file unreadable, unwritable or not in the
                                      layout of the reference's checkpoints */

typedef struct dgpu_sim dgpu_sim; /* host-side Sim: parameters + grid */
typedef struct dgpu_ctx dgpu_ctx; /* device context: state of one or more disks */

/* ---- Sim (host) -------------------------------------------------------
 * Replaces sim_create + sim_read_par_file + sim_alloc_arr + sim_set_rz +
 * sim_set_N_p + sim_set_misc (src/Sim/sim_readpar.c:48-122,
 * src/Sim/sim_alloc_arr.c:9-46, src/Sim/sim_set.c:10-177): same 52 keys, same
 * key matching and value parsing, same grid and N_p rules.  Unlike the
 * reference, a missing key is an error (the reference prints "cant find" and
 * leaves the field uninitialised, src/Sim/sim_readpar.c:25-28). */
int dgpu_sim_from_parfile(const char *path, dgpu_sim **out);
int dgpu_sim_from_text(const char *text, dgpu_sim **out);
void dgpu_sim_destroy(dgpu_sim *sim);
/* Numbers of annuli (sim_N(R_DIR), ghosts included) and cells. */
int dgpu_sim_num_annuli(const dgpu_sim *sim);
int dgpu_sim_num_cells(const dgpu_sim *sim);
/* N_p[NR] (sim_N_p) and r_faces[NR+1] (r_faces[i+1] = sim_FacePos(i, R_DIR)). */
int dgpu_sim_grid(const dgpu_sim *sim, int *N_p, double *r_faces);
/* Value of a parfile key as read (ints are returned as doubles). */
int dgpu_sim_param(const dgpu_sim *sim, const char *key, double *value);
/* Host-only: the initial state dgpu_init_state uploads -- prim[N][NUM_Q],
 * tiph[N], dphi[N] and gm[2][6] -- computed on the CPU (any pointer may be
 * NULL).  Same set-up sequence as src/main.c:74-117 (see dgpu_init_state). */
int dgpu_sim_initial_state(const dgpu_sim *sim, double *prim, double *tiph, double *dphi, double *gm);

/* ---- Context ---------------------------------------------------------- */
/* Allocates device state for n disks on `device`; stream may be NULL.
 * The sims are copied; the caller may destroy them afterwards. */
int dgpu_create(const dgpu_sim *const *sims, int n, int device, void *stream, dgpu_ctx **out);
void dgpu_destroy(dgpu_ctx *ctx);
/* Message of the last failure on this context (ctx may be NULL: last failure
 * of a create call on this thread). */
const char *dgpu_last_error(const dgpu_ctx *ctx);
int dgpu_num_instances(const dgpu_ctx *ctx);

/* ---- State --------------------------------------------------------------
 * dgpu_init_state repeats the reference set-up of src/main.c:74-119 for one
 * disk: cell_create's phi offsets (srand(666); tiph_0 = 2pi*rand()/RAND_MAX
 * per annulus, src/Cell/cell_create_destroy.c:64-91), cell_clean_pi, the
 * GravMass initialiser of GravMassType (src/GravMass/GravMass_init.c:9-84),
 * the initial data of InitialDataType, gravMass_clean_pi and cell_calc_cons.
 * t is set to 0. */
int dgpu_init_state(dgpu_ctx *ctx, int inst);
/* Replace prim[N][NUM_Q], tiph[N], dphi[N] of a disk (host buffers), then
 * recompute cons as cell_calc_cons does (src/Cell/cell_conversion.c:35-55). */
int dgpu_set_state(dgpu_ctx *ctx, int inst, const double *prim, const double *tiph,
                   const double *dphi);
/* Copy a disk's state to host buffers; any pointer may be NULL. */
int dgpu_get_state(dgpu_ctx *ctx, int inst, double *prim, double *cons, double *tiph,
                   double *dphi);
/* GravMass state gm[2][6] = (r, phi, M, omega, Mdot, Macc) per mass
 * (src/Headers/GravMass.h:7-20). */
int dgpu_set_gravmass(dgpu_ctx *ctx, int inst, const double *gm);
int dgpu_get_gravmass(dgpu_ctx *ctx, int inst, double *gm);
/* Simulation time t and the dt of the last step (timestep_get_t, timestep_dt). */
int dgpu_get_time(dgpu_ctx *ctx, int inst, double *t, double *dt);
int dgpu_set_time(dgpu_ctx *ctx, int inst, double t);

/* ---- Stepping --------------------------------------------------------------
 * dgpu_step_rk2 advances every disk of the context by nsteps calls of
 * timestep_rk2 (src/TimeStep/timestep_algorithm.c:11-41), each disk with its
 * own CFL dt.  The first call captures one step into a CUDA graph; later calls
 * replay it.  Asynchronous: returns once the work is queued; device errors
 * surface at the next dgpu_synchronize (or any dgpu_get_*). */
int dgpu_step_rk2(dgpu_ctx *ctx, int nsteps);
int dgpu_synchronize(dgpu_ctx *ctx);
/* Which kernels make up a substep (no counterpart in the reference; the
 * results are bitwise the same either way).  The fused substep is two
 * launches: k_prep (one block per annulus: the face list, cell_clean_pi,
 * cell_plm_p and, in substep 1, the CFL minimum) and k_sweep (one wavefront
 * over the annuli: face slopes, r slopes, the r- and phi-face fluxes, the
 * sources and the update).  The other form is eight kernels per substep
 * (cellprep, merge, rslope, plm_r, source, flux_phi, flux_r, update), the
 * default, which is the faster on B200.  dgpu_set_fused(ctx, 1) selects the
 * fused form where every disk of the context allows it (no passive scalar, no
 * outflow radial boundary, no sink; else DGPU_ERR_UNSUPPORTED),
 * dgpu_set_fused(ctx, 0) the eight kernels.  dgpu_fused returns 1 when the
 * step uses the fused form.  The tangent, adjoint and stage runs always use
 * the eight kernels. */
int dgpu_set_fused(dgpu_ctx *ctx, int fused);
int dgpu_fused(const dgpu_ctx *ctx);
/* The same steps launched one kernel at a time with CUDA events between the
 * kernels on the context's stream (no graph); adds each kernel's device time in
 * milliseconds to kernel_ms[16]: for the eight-kernel substep cellprep,
 * merge, rslope, plm_r, source, flux_phi, flux_r, update of substep 1, then of
 * substep 2; for the fused one k_prep, k_sweep of substep 1 in [0], [1] and of
 * substep 2 in [8], [9].  Synchronous.  For measurement only: inside the step
 * graph of the eight kernels merge runs beside cellprep, and source and
 * flux_phi beside flux_r. */
int dgpu_step_rk2_timed(dgpu_ctx *ctx, int nsteps, double *kernel_ms);
/* Autotuner (no counterpart in the reference): chooses how many blocks of 256
 * threads each SM should hold for the heavy step kernels (the register budget
 * per thread), by timing every choice on this context's own disks from its
 * current state with dgpu_step_rk2_timed (1 warm-up + `steps` steps per
 * choice), one kernel after the other: for the eight-kernel substep plm_r,
 * flux_phi, flux_r, source and update (2..5 each), for the fused one k_sweep
 * (2..4).  The state, t and the GravMass are restored afterwards, and results
 * are bitwise the same under every choice.  choice[6] (may be NULL) receives
 * the chosen values in the order plm_r, flux_phi, flux_r, source, update,
 * sweep; with steps == 0 the given choice[6] is applied instead (0 = the
 * built-in value).  The next dgpu_step_rk2 captures a new step graph.
 * Synchronous. */
int dgpu_autotune(dgpu_ctx *ctx, int steps, int *choice);
/* Stage parity: the prologue of timestep_rk2 and the first substep
 * (src/TimeStep/timestep_routines.c:16-113) stopped after `phase`
 * (0 faces/clean_pi/set_w/RK blend, 1 PLM, 2 phi fluxes, 3 r fluxes,
 * 4 sources, 5 mesh motion + cons2prim, 6 boundary + damping, 7 calc_cons);
 * phases 8-15: the whole first substep and gravMass_move
 * (src/TimeStep/timestep_algorithm.c:23-28), then the second substep stopped
 * after phase - 8 (its RKtiph is not stored: only the first substep's is).
 * Leaves the context mid-step; reload the state before stepping again. */
int dgpu_stage(dgpu_ctx *ctx, int phase);
/* Per-cell intermediates after dgpu_stage: grad, gradp ([N][NUM_Q]), wiph[N],
 * RKcons[N][NUM_Q], RKtiph[N]; any pointer may be NULL. */
int dgpu_get_stage_data(dgpu_ctx *ctx, int inst, double *grad, double *gradp, double *wiph,
                        double *rkcons, double *rktiph);

/* ---- Face list ---------------------------------------------------------------
 * The r-face list of the current state, as face_create(..., 0) builds it
 * (src/Face/face_create_destroy.c:130-193) and in its order: nri[NR] offsets
 * (timestep_n(..., R_DIR)), L/R cell numbers in (k, i, j) order, r, dphi,
 * dA, deltaL, deltaR, cm (src/Headers/Face.h:9-18).  cap = capacity of the
 * per-face arrays; *nf receives the face count (also when cap is too small,
 * which returns DGPU_ERR_ARG). */
int dgpu_face_list(dgpu_ctx *ctx, int inst, int cap, int *nri, int *L, int *R, double *r,
                   double *dphi, double *dA, double *deltaL, double *deltaR, double *cm,
                   int *nf);
/* The z-face list of a 3-D disk (NumZ > 1), as face_create(..., 1) builds it
 * (src/Face/face_create_destroy.c:165-191) and in its order: layer pair
 * (k, k+1) after layer pair, the annuli inside each; nzk[NZ] offsets
 * (timestep_n(..., Z_DIR)), r = the annulus centre, dA = r dphi dr, deltaL and
 * deltaR the half heights of the two layers.  Arguments as for
 * dgpu_face_list; DGPU_ERR_ARG for a 2-D disk. */
int dgpu_face_list_z(dgpu_ctx *ctx, int inst, int cap, int *nzk, int *L, int *R, double *r,
                     double *dphi, double *dA, double *deltaL, double *deltaR, double *cm,
                     int *nf);

/* ---- Face list without allocation ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running inside another framework's memory pool or a
 * pre-sized arena, or a service that must not grow its footprint after start-up
 * -- this builds the same r-face list as dgpu_face_list for one disk, reading
 * the phi edges tiph[N] and widths dphi[N] from the caller's device memory and
 * writing nri[NR], L, R, dphi, dA, cm (cap entries each) to the caller's device
 * memory.  Cell numbers are in the disk's (k, i, j) order.  It calls no
 * cudaMalloc/cudaFree or other allocating routine: its working memory is one
 * static device array of DGPU_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library keeps until the process exits, sized for at most
 * DGPU_NOALLOC_MAX_ANNULI annuli (any number of cells); larger grids return
 * DGPU_ERR_ARG, as does a face count above cap (*nf then holds the count).
 * Every call looks up that array's device address in the calling thread's
 * current device and context; every pointer argument must be memory of that
 * device.  Every call reuses the same array, so calls that overlap on the GPU
 * (other streams or threads) race; serialise them.  Synchronous: returns after
 * the list is complete. */
#define DGPU_NOALLOC_MAX_ANNULI 4096
#define DGPU_NOALLOC_SCRATCH_BYTES (128 * 1024)
int dgpu_face_list_noalloc(const dgpu_sim *sim, const double *tiph, const double *dphi, int cap,
                           int *nri, int *L, int *R, double *dphi_out, double *dA, double *cm,
                           int *nf, void *stream);

/* ---- Objective -----------------------------------------------------------------
 * Gravitational torque on the binary from the gas, T = sum over non-ghost cells
 * of r * rho * dV * F_phi(r, phi) with F_phi the azimuthal point-mass force of
 * gravMassForce (src/Cell/cell_source.c:49-71), evaluated on the current
 * state (it has no counterpart in the reference, which has no torque
 * diagnostic). */
int dgpu_torque(dgpu_ctx *ctx, int inst, double *torque);

/* ---- Diagnostics -----------------------------------------------------------------
 * The reductions of diagnostics_set (src/Diagnostics/diagnostics_set.c:13-298)
 * on the current state of a disk, before the reference's weighting by the time
 * since the last measurement (dtout), which the caller applies when it
 * accumulates time averages.  Any pointer may be NULL.
 *   vector[nr][17]: per non-ghost annulus (nr = NumR), the phi average times
 *     dz/(Z_Max - Z_Min) of r, rho, P, v_r, v_phi (frame included), v_z,
 *     v_phi - w, Cool, passive scalar, E_hydro, KE, rho e, 0, 0, 0, 0, 0
 *     (VectorDiag / dtout; Cool and the passive scalar are 0 here: no cooling,
 *     NUM_Q = 5);
 *   scalar[16]: sum over annuli of vector[i][n+1] (rp^2 - rm^2) divided by
 *     (R_Max^2 - R_Min^2) (ScalarDiag / dtout);
 *   equat[cells][18]: the equatorial row of every non-ghost cell, in (k, i, j)
 *     order (EquatDiag);
 *   extra[14]: the DiagMdot line after t (Mdot_near_req1, r_near_req1,
 *     mass_inside_1, mass_inner_wedge, Mdot_0, Mdot_1, Macc_0, Macc_1, mass
 *     within 0.2 of mass 0 and 1, within 0.4 of mass 0 and 1), then the masses
 *     within 0.1 of mass 0 and 1.  The reference's quirks are kept: its
 *     Mdot_near_req1 is built from the v_z column, and its inner wedge sums the
 *     first N_p(outer ghost) cells of the disk with the radii of annulus 0. */
int dgpu_diagnostics(dgpu_ctx *ctx, int inst, double *vector, double *scalar, double *equat, double *extra);

/* ---- Differentiation (a context holding one disk) ------------------------------
 * No counterpart in the reference.  A run advances the context's disk by
 * nsteps RK2 steps from its current state (leaving it at the final state,
 * like dgpu_step_rk2) and evaluates, after each step n, the binary torque T_n
 * (as dgpu_torque) and the accretion rate through the innermost non-ghost
 * annulus Mdot_n = -sum rho v_r r dphi dz; J[0] and J[1] are their
 * dt-weighted means over steps window_start+1 .. nsteps.
 * Derivatives are taken with the dt schedule of the run frozen and are with
 * respect to the mass ratio q (MassRatio, through the binary's masses and
 * orbit radii), alpha (Explicit_Viscosity) and the initial prims.  Refused
 * (DGPU_ERR_UNSUPPORTED) for contexts with several disks, C_RIGID meshes
 * (state-dependent mesh motion), Cooling and RhoSinkOn. */
/* dt_in (nsteps values, or NULL for the CFL dt) replaces the CFL dt of each
 * step: the frozen schedule under which finite differences match the
 * derivatives below; dt_out (nsteps, may be NULL) receives the dt used. */
int dgpu_objective(dgpu_ctx *ctx, int nsteps, int window_start, const double *dt_in, double *dt_out, double *J);
/* Forward-mode tangent: dJ[k] = dJ_k/de along dq/de = dq, dalpha/de = dalpha,
 * d prim_0/de = dprim ([N][NUM_Q] in the cell order of dgpu_set_state, or
 * NULL for zero). */
int dgpu_tangent(dgpu_ctx *ctx, int nsteps, int window_start, double dq, double dalpha, const double *dprim,
                 double *J, double *dJ);
/* Reverse mode: the gradient of weights[0] J[0] + weights[1] J[1] (weights
 * NULL: J[0]) with respect to q, alpha and the initial prims (dJ_dprim
 * [N][NUM_Q], may be NULL).  Stores the state every ckpt_every steps and
 * recomputes the steps in between (device memory grows with
 * nsteps / ckpt_every + 2 ckpt_every stored states of 19 doubles per cell). */
int dgpu_adjoint(dgpu_ctx *ctx, int nsteps, int window_start, int ckpt_every, const double *weights, double *J,
                 double *dJ_dq, double *dJ_dalpha, double *dJ_dprim);

/* ---- Checkpoint and restart ------------------------------------------------
 * The reference's checkpoint files (src/IO/io_hdf5.c:15-266) without an HDF5
 * library: datasets T [1], GravMass [2][4] (r, phi, M, omega per mass) and
 * Data [rows][NUM_Q+3] of 64-bit floats in the root group of an HDF5 file
 * (superblock 0, symbol-table root group, version-1 object headers,
 * contiguous storage: the structures the HDF5 library writes by default).
 * Host-only; every pointer is a host pointer.
 *
 * dgpu_hdf5_out replaces io_hdf5_out for one rank: writes a new file (it
 * does not advance the reference's tcheck/nfile, which the caller keeps, as
 * io_hdf5_out does at :152-155). */
int dgpu_hdf5_out(const char *path, double t, const double *gravmass, const double *data, long long nrows, int ncols);
/* One dataset of 64-bit floats (rank 0-2) in the root group of any HDF5
 * file in the formats above: rank, dims[2] (1 past the rank) and, when data
 * is not NULL, its values in row-major order. */
int dgpu_hdf5_dataset(const char *path, const char *name, int *rank, long long *dims, double *data);
/* Row and column counts of a checkpoint's Data. */
int dgpu_hdf5_dims(const char *path, long long *nrows, int *ncols);
/* Replaces io_hdf5_in (:161-266): T, GravMass (either pointer may be NULL)
 * and rows [row0, row0 + nrows) of Data (the hyperslab at sim_offset of
 * Ncells rows).  Unlike the reference, which ignores every HDF5 status, a
 * missing dataset, a shape other than [rows][ncols] or rows outside Data is
 * DGPU_ERR_IO. */
int dgpu_hdf5_in(const char *path, long long row0, long long nrows, int ncols, double *t, double *gravmass,
                 double *data);
/* Host-only restart state: the restart branch of src/main.c:74-117 --
 * cell_create's phi widths (dphi = 2pi/N_p; the file holds no dphi), tiph and
 * prim from the file with prim[UZZ] = 0 when NumZ is 1 (io_readbuf,
 * src/IO/io_buffer.c:60-81), the GravMass (r, phi, M, omega) from the file
 * then gravMass_clean_pi, and the periodic z copy.  gm[2][6] as
 * dgpu_get_gravmass (Mdot = Macc = 0: the reference leaves them
 * uninitialised), t the file's T.  Any output pointer may be NULL. */
int dgpu_sim_restart_state(const dgpu_sim *sim, const char *path, double *prim, double *tiph, double *dphi,
                           double *gm, double *t);
/* io_setbuf + io_hdf5_out for one disk of the context: Data rows in (k, i, j)
 * order over all cells, ghosts included: tiph, annulus centre r, layer centre
 * z, prim[NUM_Q] (src/IO/io_buffer.c:26-58). */
int dgpu_checkpoint_out(dgpu_ctx *ctx, int inst, const char *path);
/* Restart of one disk from a checkpoint: dgpu_sim_restart_state, then the
 * state, GravMass and t uploaded and cons recomputed (cell_calc_cons,
 * main.c:115).  The next dgpu_step_rk2 continues from there. */
int dgpu_checkpoint_in(dgpu_ctx *ctx, int inst, const char *path);

#ifdef __cplusplus
}
#endif
#endif
