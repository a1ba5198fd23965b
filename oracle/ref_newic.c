/*
 * Oracle replacement for the reference's initial-data selector
 * (src/Cell/cell_init_function_ptr.c:6-46), plus three axisymmetric initial
 * conditions the reference lacks.  Test infrastructure only: it is compiled
 * with the unmodified reference sources into oracle/_ref and never linked into
 * the product.
 *
 * Selector: InitialDataType 0..6 return exactly the reference's routines
 * (same order as cell_init_function_ptr.c:7-20); 7..9 return the routines
 * below.  The single-cell variants are what the reference's fixed radial
 * boundary (src/Cell/cell_boundary.c:208-231) and damping zone
 * (src/Cell/cell_misc.c:98-132) evaluate every substep, so they give the
 * noise-free profile; the whole-grid variants add the seeded density noise.
 *
 * Profiles (r = cell-centre radius 0.5*(r_{i-1/2}+r_{i+1/2}), as every
 * reference initial-data routine uses, e.g. cell_init_vortex.c:66-68):
 *   GRESHO        rho=1; v_phi = 5r | 2-5r | 0 on r<0.2 | r<0.4 | else;
 *                 P = 5+12.5r^2 | 9+12.5r^2-20r+4ln(5r) | 3+4ln2.
 *   KEPLER_RING   Sigma = exp(-(r-2)^2/(2*0.1^2)) + 1e-4; c_s^2 = (h/r)^2/r;
 *                 P = Sigma c_s^2/gamma; v_phi^2 = 1/r + r (dP/dr)/Sigma.
 *   CIRCUMBINARY  Sigma = r^-1/2 exp(-(2/r)^12) + 1e-5; c_s^2 = (h/r)^2/r;
 *                 P = Sigma c_s^2/gamma; v_phi = r^-1/2.
 * prim[UPP] is the angular velocity relative to the analytic frame,
 * v_phi/r - rOm_a(r)/r, as in cell_init_SStest.c:37.
 * Noise: Sigma (or rho) *= 1 + IC_Noise*U, U = oracle_ic_noise_u(seed, idx);
 * for the disks the pressure uses the perturbed Sigma (isothermal noise).
 */
#define CELL_PRIVATE_DEFS
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include "Headers/Cell.h"
#include "Headers/GravMass.h"
#include "Headers/Sim.h"
#include "Headers/header.h"
#include "ref_newic.h"

double oracle_ic_hor = 0.05;
double oracle_ic_noise = 0.0;
int oracle_ic_seed = 0;

double oracle_ic_noise_u(int seed, long idx) {
  uint64_t z = ((uint64_t)(uint32_t)seed << 40) ^ (uint64_t)idx;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

/* Noise-free profile at annulus i; fills prim[0..4]. */
static void newic_profile(struct Sim *theSim, int type, int i, double *prim) {
  double rm = sim_FacePos(theSim, i - 1, R_DIR);
  double rp = sim_FacePos(theSim, i, R_DIR);
  double r = 0.5 * (rm + rp);
  double gam = sim_GAMMALAW(theSim);
  double hor = oracle_ic_hor;
  double rho = 1.0, P = 1.0, vphi = 0.0;
  if (type == IC_GRESHO) {
    rho = 1.0;
    if (r < 0.2) {
      vphi = 5. * r;
      P = 5. + 12.5 * r * r;
    } else if (r < 0.4) {
      vphi = 2. - 5. * r;
      P = 9. + 12.5 * r * r - 20. * r + 4. * log(5. * r);
    } else {
      vphi = 0.0;
      P = 3. + 4. * log(2.);
    }
  } else if (type == IC_KEPLER_RING) {
    double w = 0.1;
    double x = r - 2.;
    double s0 = exp(-(x * x) / (2. * w * w));
    double sig = s0 + 1.e-4;
    double cs2 = hor * hor / r;
    double dsig = -x / (w * w) * s0;
    double dP = hor * hor / gam * (dsig / r - sig / (r * r));
    rho = sig;
    P = sig * cs2 / gam;
    vphi = sqrt(1. / r + r * dP / sig);
  } else if (type == IC_CIRCUMBINARY) {
    double s0 = pow(r, -0.5) * exp(-pow(2. / r, 12.));
    double sig = s0 + 1.e-5;
    double cs2 = hor * hor / r;
    rho = sig;
    P = sig * cs2 / gam;
    vphi = pow(r, -0.5);
  } else {
    printf("ERROR, unknown oracle initial data %d\n", type);
    exit(1);
  }
  prim[RHO] = rho;
  prim[PPP] = P;
  prim[URR] = 0.0;
  prim[UPP] = vphi / r - sim_rOm_a(theSim, r, 1.) / r;
  prim[UZZ] = 0.0;
}

static void newic_single(struct Cell *c, struct Sim *theSim, int i) {
  double prim[5];
  int q;
  newic_profile(theSim, sim_InitialDataType(theSim), i, prim);
  for (q = 0; q < 5; ++q) c->prim[q] = prim[q];
  for (q = 5; q < sim_NUM_Q(theSim); ++q) c->prim[q] = 0.0;
}

static void newic_grid(struct Cell ***theCells, struct Sim *theSim) {
  int type = sim_InitialDataType(theSim);
  double gam = sim_GAMMALAW(theSim);
  long idx = 0;
  int i, j, k, q;
  for (k = 0; k < sim_N(theSim, Z_DIR); ++k) {
    for (i = 0; i < sim_N(theSim, R_DIR); ++i) {
      double prim[5];
      double rm = sim_FacePos(theSim, i - 1, R_DIR);
      double rp = sim_FacePos(theSim, i, R_DIR);
      double r = 0.5 * (rm + rp);
      newic_profile(theSim, type, i, prim);
      for (j = 0; j < sim_N_p(theSim, i); ++j, ++idx) {
        struct Cell *c = &theCells[k][i][j];
        double f = 1. + oracle_ic_noise * oracle_ic_noise_u(oracle_ic_seed, idx);
        for (q = 0; q < 5; ++q) c->prim[q] = prim[q];
        for (q = 5; q < sim_NUM_Q(theSim); ++q) c->prim[q] = 0.0;
        c->prim[RHO] = prim[RHO] * f;
        if (type != IC_GRESHO) c->prim[PPP] = c->prim[RHO] * (oracle_ic_hor * oracle_ic_hor / r) / gam;
      }
    }
  }
}

static void cell_init_gresho(struct Cell ***c, struct Sim *s, struct GravMass *g, struct MPIsetup *m) {
  (void)g; (void)m;
  newic_grid(c, s);
}
static void cell_single_init_newic(struct Cell *c, struct Sim *s, struct GravMass *g, int i, int j, int k) {
  (void)g; (void)j; (void)k;
  newic_single(c, s, i);
}

void (*cell_init_ptr(struct Sim *theSim))(struct Cell ***, struct Sim *, struct GravMass *, struct MPIsetup *) {
  switch (sim_InitialDataType(theSim)) {
    case SHEAR: return &cell_init_shear;
    case VORTEX: return &cell_init_vortex;
    case TORUS: return &cell_init_torus;
    case MILOS_MACFADYEN: return &cell_init_milos_macfadyen;
    case RAD_DOM: return &cell_init_rad_dom;
    case MIDDLE: return &cell_init_middle;
    case SSTEST: return &cell_init_SStest;
    case IC_GRESHO:
    case IC_KEPLER_RING:
    case IC_CIRCUMBINARY: return &cell_init_gresho;
    default:
      printf("ERROR, not a valid global initial data routine choice\n");
      exit(0);
  }
}

void (*cell_single_init_ptr(struct Sim *theSim))(struct Cell *, struct Sim *, struct GravMass *, int, int, int) {
  switch (sim_InitialDataType(theSim)) {
    case SHEAR: return &cell_single_init_shear;
    case VORTEX: return &cell_single_init_vortex;
    case TORUS: return &cell_single_init_torus;
    case MILOS_MACFADYEN: return &cell_single_init_milos_macfadyen;
    case RAD_DOM: return &cell_single_init_rad_dom;
    case MIDDLE: return &cell_single_init_middle;
    case SSTEST: return &cell_single_init_SStest;
    case IC_GRESHO:
    case IC_KEPLER_RING:
    case IC_CIRCUMBINARY: return &cell_single_init_newic;
    default:
      printf("ERROR, not a valid single point initial data routine choice\n");
      exit(0);
  }
}
