/*
 * Host-side Sim: parfile parameters and the radial/vertical grid.
 * Mirrors struct Sim (src/Headers/Sim.h:8-71) for a single process (no MPI
 * domain split: the whole disk is one "rank 0" with N0 = 0).
 */
#ifndef DGPU_SIM_H
#define DGPU_SIM_H

#include "../../include/disco_gpu.h"
#include "dgpu_internal.h"

struct dgpu_sim {
  /* the 52 keys of src/Sim/sim_readpar.c:55-106 */
  int Restart, InitialDataType, GravMassType;
  double MassRatio, OrbShrinkTscale, OrbShrinkT0;
  int BoundTypeR, BoundTypeZ, NoInnerBC, NumR, NumZ, ng;
  double R_Min, R_Max, Z_Min, Z_Max;
  int NP_CONST, NPCAP;
  double aspect;
  int NUM_C, NUM_N;
  double Time_Max;
  int Num_Checkpoints, Num_Diag_Dump, Num_Diag_Measure, w_numeric_type, RiemannSolver;
  double Adiabatic_Index;
  int Cooling;
  double Explicit_Viscosity;
  int ViscConst;
  double PoRho_r1, CFL, PLM;
  int Grav_2D;
  double G_EPS;
  int RhoSinkOn, PHI_ORDER;
  double Rho_Floor, Cs_Floor, Cs_Cap, Vel_Cap, DAMP_TIME, RDAMP_INNER, RDAMP_OUTER;
  double RLogScale, ZLogScale, HiResSigma, HiResR0a, HiResR0b, HiResFac;
  int w_analytic_type;
  /* initial-data keys the reference reader never asks for (optional) */
  double IC_HoR, IC_Noise;
  int IC_Seed;
  /* grid (sim_alloc_arr / sim_set_rz / sim_set_N_p / sim_set_misc) */
  int NR, NZ, NQ, Ncells;
  int ng_min[2], ng_max[2];
  int *N_p;
  double *r_faces; /* NR+1: r_faces[i+1] = sim_FacePos(i, R_DIR) */
  double *z_faces; /* NZ+1 */
};

/* sim_FacePos(i, R_DIR) */
static inline double dsim_rface(const struct dgpu_sim *s, int i) { return s->r_faces[i + 1]; }
static inline double dsim_zface(const struct dgpu_sim *s, int k) { return s->z_faces[k + 1]; }

int dsim_parse(const char *text, struct dgpu_sim *s, char *err, int errlen);
int dsim_build_grid(struct dgpu_sim *s, char *err, int errlen);
struct dgpu_sim *dsim_clone(const struct dgpu_sim *s);
void dsim_free(struct dgpu_sim *s);

/* Frame rotation sim_rOm_a / sim_rdrOm_a / sim_dtOm_a (src/Sim/sim_w_a.c:8-72). */
double dsim_rOm_a(const struct dgpu_sim *s, double r, double a);
double dsim_rdrOm_a(const struct dgpu_sim *s, double r, double a);
double dsim_dtOm_a(const struct dgpu_sim *s, double r, double a);

/* Single-cell initial data of annulus i (the profile that the fixed boundary
 * and the damping zone relax to).  Returns 1 when it sets prim[0..4], 0 when
 * the reference routine leaves the cell unchanged at this radius, -1 when the
 * initial data type has no axisymmetric single-cell form here. */
int dsim_single_init(const struct dgpu_sim *s, int i, double *prim);

/* Whole-grid initial data (cell_init_*) for cell j of annulus i with global
 * (k,i,j) cell number idx (noise included), NQ = 5 + NUM_N values.  tiph, dphi: the cell's phi edge
 * and width after cell_create and cell_clean_pi; gm: the GravMass state
 * (dsim_initial_gravmass); rnd: the generator of cell_init_torus, seeded like
 * srand(666), drawn once per cell for that type only.  Returns 0 or -1
 * (unsupported type). */
struct random_data;
int dsim_grid_init(const struct dgpu_sim *s, int k, int i, long idx, double tiph, double dphi, const double *gm,
                   struct random_data *rnd, double *prim);

/* Fill the per-annulus table entries that depend only on the Sim. */
void dsim_fill_annulus(const struct dgpu_sim *s, int k, int i, Annulus *a);
void dsim_fill_params(const struct dgpu_sim *s, DiskParams *p);

/* Initial phi edges of cell_create: srand(666), one rand() per annulus. */
void dsim_initial_tiph(const struct dgpu_sim *s, double *tiph, double *dphi);
/* The periodic z copy of the single-rank cell_syncproc_z on host arrays in
 * (k, i, j) order: tiph[Ncells] and prim[Ncells][NQ] (either may be NULL).
 * Nothing for NZ 1. */
void dsim_host_zsync(const struct dgpu_sim *s, double *tiph, double *prim);

/* GravMass initialisers (src/GravMass/GravMass_init.c:9-84) + gravMass_clean_pi;
 * gm[2][6] = r, phi, M, omega, Mdot, Macc. */
int dsim_initial_gravmass(const struct dgpu_sim *s, double *gm);

#endif
