/*
 * C restatement of Disco2's per-step hot path (test infrastructure only: the
 * oracle's portable half, used where the reference build is absent and as a
 * cross-check of it).  Sequential, structure-of-arrays, same FP64 expressions
 * and operation order as the reference, so with the same libm and
 * -ffp-contract=off it reproduces the reference bit for bit.
 *
 * Scope: 2-D (NumZ = 1), single process, fixed or outflow radial boundaries,
 * NUM_C = 5 with up to PORT_MAXQ - 5 passive scalars, every initial-data type.
 */
#ifndef DISCO_PORT_H
#define DISCO_PORT_H

#define PORT_MAXQ 8 /* NUM_Q = NUM_C + NUM_N at most */

typedef struct {
  /* parfile keys (src/Sim/sim_readpar.c:55-106) + the initial-data keys */
  int Restart, InitialDataType, GravMassType;
  double MassRatio, OrbShrinkTscale, OrbShrinkT0;
  int BoundTypeR, BoundTypeZ, NoInnerBC, NumR, NumZ, ng;
  double R_Min, R_Max, Z_Min, Z_Max;
  int NP_CONST, NPCAP;
  double aspect;
  int NUM_C, NUM_N;
  double Time_Max;
  int w_numeric_type, RiemannSolver;
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
  double IC_HoR, IC_Noise;
  int IC_Seed;

  /* grid */
  int NR, N, ng_min, ng_max, NQ;
  int *N_p, *off;        /* cells per annulus, first cell of each annulus */
  double *rf;            /* NR+1 radial faces: rf[i+1] = FacePos(i) */
  double zf[2];          /* the single z layer */

  /* cells (structure of arrays, (k,i,j) order) */
  double *prim[PORT_MAXQ], *cons[PORT_MAXQ], *rkcons[PORT_MAXQ], *grad[PORT_MAXQ], *gradp[PORT_MAXQ];
  double *tiph, *rktiph, *dphi, *wiph;

  /* GravMass */
  double gr[2], gphi[2], gM[2], gom[2], grk_r[2], grk_phi[2], grk_M[2], grk_om[2];
  double mdot[2], macc[2];

  /* TimeStep */
  double t, dt, RK;
  int *nri;

  /* r faces */
  int nf, fcap;
  int *fL, *fR;
  double *fr, *fdphi, *fdA, *fdl, *fdr, *fcm;
} Port;

int port_read_parfile(Port *p, const char *path);
int port_setup(Port *p);               /* grid, cells, phi offsets, GravMass, initial data, calc_cons */
void port_free(Port *p);
void port_calc_cons(Port *p);
void port_build_faces(Port *p);        /* face_create(..., 0) */
void port_step_rk2(Port *p);           /* timestep_rk2 */
void port_prologue(Port *p);           /* timestep_rk2 up to the first substep */
void port_substep(Port *p, double fac, int stop);  /* timestep_substep, stopped after a phase */
/* the prologue of timestep_rk2, then phase 0-7 of substep 1, or (8-15) all of
 * substep 1, gravMass_move, and phase - 8 of substep 2 */
void port_stage(Port *p, int phase);

#endif
