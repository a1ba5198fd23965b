/*
 * Host-side Sim: parfile reader, grid, frame terms, initial data and the
 * per-annulus tables handed to the kernels.  Plain C99, compiled with
 * -ffp-contract=off so that every expression rounds exactly as the reference's
 * C does; expressions keep the reference's operation order.
 */
#define _DEFAULT_SOURCE
#include "dgpu_sim.h"

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PHIMAX (2.0 * M_PI)

enum { VT_INT, VT_DOUB };
typedef struct {
  const char *name;
  int type;
  size_t off;
  int optional;
} KeyDef;

#define KI(n, f) {n, VT_INT, offsetof(struct dgpu_sim, f), 0}
#define KD(n, f) {n, VT_DOUB, offsetof(struct dgpu_sim, f), 0}
/* src/Sim/sim_readpar.c:55-106, in that order */
static const KeyDef KEYS[] = {
    KI("Restart", Restart), KI("InitialDataType", InitialDataType),
    KI("GravMassType", GravMassType), KD("MassRatio", MassRatio),
    KD("OrbShrinkTscale", OrbShrinkTscale), KD("OrbShrinkT0", OrbShrinkT0),
    KI("BoundTypeR", BoundTypeR), KI("BoundTypeZ", BoundTypeZ), KI("NoInnerBC", NoInnerBC),
    KI("NumR", NumR), KI("NumZ", NumZ), KI("ng", ng), KD("R_Min", R_Min), KD("R_Max", R_Max),
    KD("Z_Min", Z_Min), KD("Z_Max", Z_Max), KI("NP_CONST", NP_CONST), KI("NPCAP", NPCAP),
    KD("aspect", aspect), KI("NUM_C", NUM_C), KI("NUM_N", NUM_N), KD("Time_Max", Time_Max),
    KI("Num_Checkpoints", Num_Checkpoints), KI("Num_Diag_Dump", Num_Diag_Dump),
    KI("Num_Diag_Measure", Num_Diag_Measure), KI("w_numeric_type", w_numeric_type),
    KI("RiemannSolver", RiemannSolver), KD("Adiabatic_Index", Adiabatic_Index),
    KI("Cooling", Cooling), KD("Explicit_Viscosity", Explicit_Viscosity),
    KI("ViscConst", ViscConst), KD("PoRho_r1", PoRho_r1), KD("CFL", CFL), KD("PLM", PLM),
    KI("Grav_2D", Grav_2D), KD("G_EPS", G_EPS), KI("RhoSinkOn", RhoSinkOn),
    KI("PHI_ORDER", PHI_ORDER), KD("Rho_Floor", Rho_Floor), KD("Cs_Floor", Cs_Floor),
    KD("Cs_Cap", Cs_Cap), KD("Vel_Cap", Vel_Cap), KD("DAMP_TIME", DAMP_TIME),
    KD("RDAMP_INNER", RDAMP_INNER), KD("RDAMP_OUTER", RDAMP_OUTER), KD("RLogScale", RLogScale),
    KD("ZLogScale", ZLogScale), KD("HiResSigma", HiResSigma), KD("HiResR0a", HiResR0a),
    KD("HiResR0b", HiResR0b), KD("HiResFac", HiResFac), KI("w_analytic_type", w_analytic_type),
    {"IC_HoR", VT_DOUB, offsetof(struct dgpu_sim, IC_HoR), 1},
    {"IC_Noise", VT_DOUB, offsetof(struct dgpu_sim, IC_Noise), 1},
    {"IC_Seed", VT_INT, offsetof(struct dgpu_sim, IC_Seed), 1},
};
#define NKEYS ((int)(sizeof(KEYS) / sizeof(KEYS[0])))

/* readvar (src/Sim/sim_readpar.c:10-46) over an in-memory parfile: lines as
 * fgets(s,512) yields them; the first line whose first token equals the key
 * wins; the value starts after the key and any of "\t :=>_". */
static int readvar_text(const char *text, const char *name, double *out) {
  const char *p = text;
  char s[512], nm[512];
  nm[0] = 0;
  while (*p) {
    size_t n = 0;
    while (p[n] && p[n] != '\n' && n < sizeof(s) - 2) ++n;
    if (p[n] == '\n') ++n; /* fgets keeps the newline */
    memcpy(s, p, n);
    s[n] = 0;
    p += n;
    sscanf(s, "%511s ", nm);
    if (strcmp(nm, name) == 0) {
      const char *s2 = s + strlen(nm);
      double temp;
      s2 += strspn(s2, "\t :=>_");
      if (sscanf(s2, "%lf", &temp) != 1) return 2;
      *out = temp;
      return 0;
    }
  }
  return 1;
}

int dsim_parse(const char *text, struct dgpu_sim *s, char *err, int errlen) {
  int k;
  memset(s, 0, sizeof(*s));
  s->IC_HoR = 0.05;
  s->IC_Noise = 0.0;
  s->IC_Seed = 0;
  for (k = 0; k < NKEYS; ++k) {
    double v = 0.0;
    int rc = readvar_text(text, KEYS[k].name, &v);
    if (rc != 0) {
      if (KEYS[k].optional && rc == 1) continue;
      snprintf(err, (size_t)errlen, "parfile: %s key %s", rc == 1 ? "missing" : "unparsable",
               KEYS[k].name);
      return DGPU_ERR_PARFILE;
    }
    if (KEYS[k].type == VT_INT)
      *(int *)((char *)s + KEYS[k].off) = (int)v;
    else
      *(double *)((char *)s + KEYS[k].off) = v;
  }
  return DGPU_OK;
}

/* r_func / sgn / get_r: src/Sim/sim_set.c:36-71 */
static double r_func(double r, double r2, double fac, double sigma, double r0a, double r0b) {
  double F = r + fac * sigma * sqrt(M_PI / 4.0) * (erf((r - r0a) / sigma) + 1.0) +
             fac * sigma * sqrt(M_PI / 4.0) * (erf((r - r0b) / sigma) + 1.0) - r2;
  return F;
}
static int sgn(double x) {
  if (x > 0) return 1;
  if (x < 0) return -1;
  return 0;
}
static double get_r(double r2, double RMIN, double RMAX, double r0a, double r0b, double sigma,
                    double fac) {
  double r = 0.0;
  int n = 1;
  int NMAX = 1000;
  double a = RMIN;
  double b = RMAX;
  double TOL = 1.0e-12;
  while (n <= NMAX) {
    double c = (a + b) / 2.;
    if ((r_func(c, r2, fac, sigma, r0a, r0b) == 0.0) || ((b - a) / 2. < TOL)) {
      r = c;
      break;
    }
    n = n + 1;
    if (sgn(r_func(c, r2, fac, sigma, r0a, r0b)) == sgn(r_func(a, r2, fac, sigma, r0a, r0b))) {
      a = c;
    } else {
      b = c;
    }
  }
  return r;
}

int dsim_build_grid(struct dgpu_sim *s, char *err, int errlen) {
  int i, k;
  if (s->NumR < 1 || s->NumZ < 1 || s->ng < 1) {
    snprintf(err, (size_t)errlen, "grid: NumR, NumZ and ng must be positive");
    return DGPU_ERR_PARFILE;
  }
  /* every annulus holds at least one cell, so NumR x NumZ bounds the cell
   * count from below: refuse what cannot fit before laying out the grid */
  if ((long)s->NumR * (long)s->NumZ > 0x7fffffffL / 16 || s->ng > 1024) {
    snprintf(err, (size_t)errlen, "grid: NumR %d x NumZ %d (ng %d) is too large", s->NumR, s->NumZ, s->ng);
    return DGPU_ERR_ARG;
  }
  /* sim_alloc_arr (src/Sim/sim_alloc_arr.c:9-46) for the only rank */
  s->ng_min[0] = 1;
  s->ng_max[0] = s->ng;
  if (s->NumZ == 1) {
    s->ng_min[1] = 0;
    s->ng_max[1] = 0;
  } else {
    s->ng_min[1] = s->ng;
    s->ng_max[1] = s->ng;
  }
  s->NR = s->NumR + s->ng_min[0] + s->ng_max[0];
  s->NZ = s->NumZ + s->ng_min[1] + s->ng_max[1];
  s->NQ = s->NUM_C + s->NUM_N;
  s->N_p = (int *)malloc(sizeof(int) * (size_t)s->NR);
  s->r_faces = (double *)malloc(sizeof(double) * (size_t)(s->NR + 1));
  s->z_faces = (double *)malloc(sizeof(double) * (size_t)(s->NZ + 1));
  if (!s->N_p || !s->r_faces || !s->z_faces) {
    snprintf(err, (size_t)errlen, "grid: out of host memory");
    return DGPU_ERR_NOMEM;
  }
  {
    /* sim_set_rz (src/Sim/sim_set.c:73-143) with N0 = 0 */
    double RMIN = s->R_Min, RMAX = s->R_Max, ZMIN = s->Z_Min, ZMAX = s->Z_Max;
    double Rscale = s->RLogScale, sigma = s->HiResSigma, r0a = s->HiResR0a, r0b = s->HiResR0b;
    double fac = s->HiResFac;
    double r2_max = RMAX + fac * sigma * sqrt(M_PI / 4.0) * (erf((RMAX - r0a) / sigma) + 1.0) +
                    fac * sigma * sqrt(M_PI / 4.0) * (erf((RMAX - r0b) / sigma) + 1.0);
    double r2_min = RMIN + fac * sigma * sqrt(M_PI / 4.0) * (erf((RMIN - r0a) / sigma) + 1.0) +
                    fac * sigma * sqrt(M_PI / 4.0) * (erf((RMIN - r0b) / sigma) + 1.0);
    double r1_max = Rscale * log(1.0 + r2_max / Rscale);
    double r1_min = Rscale * log(1.0 + r2_min / Rscale);
    double Zscale, z1_max, z1_min;
    for (i = 0; i < s->NR + 1; i++) {
      int ig = i - s->ng_min[0];
      double delta = (r1_max - r1_min) / (double)s->NumR;
      double r1 = r1_min + (double)ig * delta;
      double r2 = Rscale * (exp(r1 / Rscale) - 1.0);
      s->r_faces[i] = get_r(r2, 0., 2. * RMAX, r0a, r0b, sigma, fac);
    }
    if (s->NoInnerBC == 1) s->r_faces[0] = 0.0;
    Zscale = s->ZLogScale;
    z1_max = sgn(ZMAX) * Zscale * log(1.0 + fabs(ZMAX) / Zscale);
    z1_min = sgn(ZMIN) * Zscale * log(1.0 + fabs(ZMIN) / Zscale);
    for (k = 0; k < s->NZ + 1; k++) {
      int kg = k - s->ng_min[1];
      double delta = (z1_max - z1_min) / (double)s->NumZ;
      double z1 = z1_min + (double)kg * delta;
      s->z_faces[k] = sgn(z1) * Zscale * (exp(fabs(z1) / Zscale) - 1.0);
    }
  }
  /* sim_set_N_p (src/Sim/sim_set.c:10-33) */
  for (i = 0; i < s->NR; ++i) {
    if (s->NP_CONST > 0) {
      s->N_p[i] = s->NP_CONST;
    } else {
      double r_cell = 0.5 * (dsim_rface(s, i - 1) + dsim_rface(s, i));
      double dr = dsim_rface(s, i) - dsim_rface(s, i - 1);
      if (r_cell < s->R_Min) {
        double dr_plus = dsim_rface(s, i + 1) - dsim_rface(s, i);
        s->N_p[i] = (int)(PHIMAX * (1. + (r_cell / dr_plus - 1.) / s->aspect));
      } else {
        s->N_p[i] = (int)(PHIMAX * (1. + (r_cell / dr - 1.) / s->aspect));
      }
      if (s->NPCAP > 0) {
        if (s->N_p[i] > s->NPCAP) s->N_p[i] = s->NPCAP;
      }
    }
    if (s->N_p[i] < 1) {
      snprintf(err, (size_t)errlen, "grid: annulus %d has N_p = %d", i, s->N_p[i]);
      return DGPU_ERR_PARFILE;
    }
  }
  /* sim_set_misc cell count */
  {
    long n = 0;
    for (i = 0; i < s->NR; ++i) n += (long)s->N_p[i] * s->NZ;
    if (n > 0x7fffffffL / 16) {
      snprintf(err, (size_t)errlen, "grid: %ld cells is too many", n);
      return DGPU_ERR_ARG;
    }
    s->Ncells = (int)n;
  }
  return DGPU_OK;
}

struct dgpu_sim *dsim_clone(const struct dgpu_sim *s) {
  struct dgpu_sim *c = (struct dgpu_sim *)malloc(sizeof(*c));
  if (!c) return NULL;
  *c = *s;
  c->N_p = (int *)malloc(sizeof(int) * (size_t)s->NR);
  c->r_faces = (double *)malloc(sizeof(double) * (size_t)(s->NR + 1));
  c->z_faces = (double *)malloc(sizeof(double) * (size_t)(s->NZ + 1));
  if (!c->N_p || !c->r_faces || !c->z_faces) {
    dsim_free(c);
    return NULL;
  }
  memcpy(c->N_p, s->N_p, sizeof(int) * (size_t)s->NR);
  memcpy(c->r_faces, s->r_faces, sizeof(double) * (size_t)(s->NR + 1));
  memcpy(c->z_faces, s->z_faces, sizeof(double) * (size_t)(s->NZ + 1));
  return c;
}

void dsim_free(struct dgpu_sim *s) {
  if (!s) return;
  free(s->N_p);
  free(s->r_faces);
  free(s->z_faces);
  free(s);
}

/* src/Sim/sim_w_a.c:8-72 (w_a_milos_index = 8, src/Headers/header.h:25) */
#define W_A_MILOS_INDEX 8
double dsim_rOm_a(const struct dgpu_sim *s, double r, double a) {
  switch (s->w_analytic_type) {
    case DA_FIXED: return 0.0;
    case DA_KEPLER: return pow(r, -0.5);
    case DA_OMEGA20: return r * 20;
    case DA_MILOS:
      return r * (pow(r, W_A_MILOS_INDEX - 1.5) + pow(a, W_A_MILOS_INDEX - 1.5)) /
             (pow(r, W_A_MILOS_INDEX) + pow(a, W_A_MILOS_INDEX));
    case DA_POWERLAW: return pow(r, -1.0);
    default: return 0.0;
  }
}
double dsim_rdrOm_a(const struct dgpu_sim *s, double r, double a) {
  switch (s->w_analytic_type) {
    case DA_FIXED: return 0.0;
    case DA_KEPLER: return -1.5 * pow(r, -1.5);
    case DA_OMEGA20: return 0.0;
    case DA_MILOS: {
      int n = W_A_MILOS_INDEX;
      double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
      double arn = pow(a / r, n);
      return ((-1.5 + n * arn / (1. + arn)) * Omega_a +
              (1.5 - n) * pow(a / r, n - 1.5) / (1. + arn) * pow(r, -1.5));
    }
    case DA_POWERLAW: return -2. * pow(r, -2.0);
    default: return 0.0;
  }
}
double dsim_dtOm_a(const struct dgpu_sim *s, double r, double a) {
  if (s->w_analytic_type == DA_MILOS) {
    double a0 = 1.0;
    double tau = s->OrbShrinkTscale;
    double dta_o_a = -.25 * pow(a / a0, -4) / tau;
    int n = W_A_MILOS_INDEX;
    double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
    double arn = pow(a / r, n);
    if (a > 0.0) {
      return (dta_o_a * (Omega_a * (-1.5 + n / (1. + arn)) + (1.5 - n) * pow(r, -1.5) / (1. + arn)));
    }
    return 0.0;
  }
  return 0.0;
}

/* Profiles of the new initial data types (GRESHO, KEPLER_RING,
 * CIRCUMBINARY); the oracle restates the same formulas independently. */
static void newic_profile(const struct dgpu_sim *s, int i, double *prim) {
  double rm = dsim_rface(s, i - 1);
  double rp = dsim_rface(s, i);
  double r = 0.5 * (rm + rp);
  double gam = s->Adiabatic_Index;
  double hor = s->IC_HoR;
  double rho = 1.0, P = 1.0, vphi = 0.0;
  if (s->InitialDataType == DI_GRESHO) {
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
  } else if (s->InitialDataType == DI_KEPLER_RING) {
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
  } else { /* DI_CIRCUMBINARY */
    double s0 = pow(r, -0.5) * exp(-pow(2. / r, 12.));
    double sig = s0 + 1.e-5;
    double cs2 = hor * hor / r;
    rho = sig;
    P = sig * cs2 / gam;
    vphi = pow(r, -0.5);
  }
  prim[D_RHO] = rho;
  prim[D_PPP] = P;
  prim[D_URR] = 0.0;
  prim[D_UPP] = vphi / r - dsim_rOm_a(s, r, 1.) / r;
  prim[D_UZZ] = 0.0;
}

/* The radiation-dominated disk of cell_init_rad_dom.c:13-76 (single-cell and
 * whole-grid forms give the same values: omega - 1/r^1.5 and
 * omega - sqrt(1)/r^1.5 round alike; the file's global `blah` is 0). */
static void rad_dom_profile(const struct dgpu_sim *s, double r, double *prim) {
  const double blah = 0.0;
  double xi = 0.005, a_o_M = 100;
  double alpha = s->Explicit_Viscosity;
  double gam = s->Adiabatic_Index;
  double rho0 = 2. / (9. * xi * alpha * gam) * sqrt(a_o_M);
  double P0 = 8. * xi / (9. * alpha * gam) * sqrt(a_o_M);
  double rho = rho0 * pow(r, 1.5);
  double P = P0 * pow(r, -1.5);
  double o2 = 1. / r / r / r - 3. / 2. * P / rho / r / r;
  double omega = sqrt(o2);
  double vr = -1.5 * alpha * gam * (P / rho) * sqrt(r) - blah * pow(r, -4.5);
  prim[D_RHO] = rho;
  prim[D_PPP] = P;
  prim[D_URR] = vr;
  prim[D_UPP] = omega - 1. / pow(r, 1.5);
  prim[D_UZZ] = 0.0;
}

/* The disk of cell_init_middle.c:12-91; the whole-grid form (grid = 1) also
 * zeroes v_r inside r = 1. */
static void middle_profile(const struct dgpu_sim *s, double r, int grid, double *prim) {
  const int w_idx = 8; /* w_a_milos_index (header.h) */
  double alpha = s->Explicit_Viscosity;
  double r0 = 2.5;
  int d = 10;
  double rho = pow(r, -3. / 5.) * exp(-pow(r / r0, -d));
  double P = s->PoRho_r1 * pow(r, -3. / 2.) * exp(-pow(r / r0, -d));
  double r_drP_o_P = -1.5 + d * pow(r / r0, -d);
  double o2, omega, a = 1.0, vr;
  if (rho < 1.e-3) rho = 1.e-3;
  if (P < 1.e-6) P = 1.e-6;
  o2 = 1. / r / r / r * pow(1. + 3. / 16. / r / r, 2) + r_drP_o_P * P / rho / r / r;
  omega = sqrt(o2);
  omega = (pow(r, w_idx) * omega + pow(a, w_idx - 1.5)) / (pow(r, w_idx) + pow(a, w_idx));
  vr = -3. * alpha / r / omega * P / rho * (2. + r_drP_o_P);
  if (grid && r < 1.) vr = 0.0;
  prim[D_RHO] = rho;
  prim[D_PPP] = P;
  prim[D_URR] = vr;
  prim[D_UPP] = omega - dsim_rOm_a(s, r, a) / r;
  prim[D_UZZ] = 0.0;
}

int dsim_single_init(const struct dgpu_sim *s, int i, double *prim) {
  double rm = dsim_rface(s, i - 1);
  double rp = dsim_rface(s, i);
  double r = 0.5 * (rm + rp);
  switch (s->InitialDataType) {
    case DI_GRESHO:
    case DI_KEPLER_RING:
    case DI_CIRCUMBINARY:
      newic_profile(s, i, prim);
      return 1;
    case DI_VORTEX: {
      /* cell_single_init_vortex (src/Cell/initial_data/cell_init_vortex.c:11-37) */
      double rho = 1.0, P0 = 1.0, R = 1.0, A = 0.5, g = 3.0;
      double Pp, vp;
      if (r >= R) return 0;
      Pp = P0 * (1. - A * exp(g * (r / R - R / (R - r) + 1.)));
      vp = sqrt(A * g * P0 / rho * (2. * R - r) / R * r * r / pow(R - r, 2.) *
                exp(g * (r / R - R / (R - r) + 1.)));
      prim[D_RHO] = rho;
      prim[D_PPP] = Pp;
      prim[D_URR] = 0.0;
      prim[D_UPP] = vp / r;
      prim[D_UZZ] = 0.0;
      return 1;
    }
    case DI_SSTEST: {
      /* cell_single_init_SStest (src/Cell/initial_data/cell_init_SStest.c:11-45) */
      double r0 = 5.;
      int d = 4;
      double rho = pow(r, -3. / 5.) * exp(-pow(r / r0, -d));
      double P = s->PoRho_r1 * pow(r, -3. / 2.) * exp(-pow(r / r0, -d));
      double a = 1.0;
      if (rho < 1.e-4) rho = 1.e-4;
      if (P < 1.e-7) P = 1.e-7;
      prim[D_RHO] = rho;
      prim[D_PPP] = P;
      prim[D_URR] = 0.0;
      prim[D_UPP] = pow(r, -1.5) - dsim_rOm_a(s, r, a) / r;
      prim[D_UZZ] = 0.0;
      return 1;
    }
    case DI_MILOS_MACFADYEN: {
      /* cell_single_init_milos_macfadyen
       * (src/Cell/initial_data/cell_init_milos_macfadyen.c:11-36) */
      double Mach = 1. / sqrt(s->PoRho_r1);
      double gam = s->Adiabatic_Index;
      double rho0 = 1.0, rs = 10., delta_exp = 3.0, xi_exp = 2.0;
      double rho = rho0 * (pow(rs / r, delta_exp)) * exp(-pow(rs / r, xi_exp));
      double PoRho = 1. / Mach / Mach / gam;
      prim[D_RHO] = rho;
      prim[D_PPP] = PoRho * rho;
      prim[D_URR] = 0.0;
      prim[D_UPP] = 0.0;
      prim[D_UZZ] = 0.0;
      return 1;
    }
    case DI_RAD_DOM:
      /* cell_single_init_rad_dom (src/Cell/initial_data/cell_init_rad_dom.c:13-36) */
      rad_dom_profile(s, r, prim);
      return 1;
    case DI_MIDDLE:
      /* cell_single_init_middle (src/Cell/initial_data/cell_init_middle.c:12-45) */
      middle_profile(s, r, 0, prim);
      return 1;
    default:
      /* SHEAR: the profile depends on the cell's phi; TORUS: the reference
       * exits (cell_init_torus.c:12-15) */
      return -1;
  }
}

/* splitmix64 step on (seed << 40) ^ idx; same definition as the oracle's. */
static double noise_u(int seed, long idx) {
  uint64_t z = ((uint64_t)(uint32_t)seed << 40) ^ (uint64_t)idx;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

/* gravMass_dist (src/GravMass/GravMass_access.c:25-31) on gm[2][6]. */
static double gm_dist(const double *gm, int p, double r, double phi, double z) {
  double xbh = gm[6 * p] * cos(gm[6 * p + 1]);
  double ybh = gm[6 * p] * sin(gm[6 * p + 1]);
  double x = r * cos(phi);
  double y = r * sin(phi);
  return sqrt((x - xbh) * (x - xbh) + (y - ybh) * (y - ybh) + z * z);
}

int dsim_grid_init(const struct dgpu_sim *s, int k, int i, long idx, double tiph, double dphi, const double *gm,
                   struct random_data *rnd, double *prim) {
  double rm = dsim_rface(s, i - 1);
  double rp = dsim_rface(s, i);
  double r = 0.5 * (rm + rp);
  int t = s->InitialDataType, q;
  /* passive scalars: only cell_init_vortex sets one (below); the reference
   * leaves them as cell_create's allocation gives them, zero here */
  for (q = DGPU_NQ; q < s->NQ; ++q) prim[q] = 0.0;
  if (t == DI_SHEAR) {
    /* cell_init_shear (src/Cell/initial_data/cell_init_shear.c:57-116) */
    double rho = 1.0, Pp = 0.01, v0 = 1.0, t0 = 0.25;
    double ph = tiph - .5 * dphi;
    double x = r * cos(ph) - 3.;
    double y = r * sin(ph);
    double nu = s->Explicit_Viscosity > 0.0 ? s->Explicit_Viscosity : 0.05;
    double vy = 0.0, omega;
    if (fabs(y) < 50.) vy = v0 / sqrt(2. * M_PI * nu * t0) * exp(-x * x / (4. * nu * t0));
    omega = vy * cos(ph) / r;
    prim[D_RHO] = rho;
    prim[D_PPP] = Pp;
    prim[D_URR] = vy * sin(ph);
    prim[D_UPP] = omega - dsim_rOm_a(s, r, 1.) / r;
    prim[D_UZZ] = 0.0;
    return 0;
  }
  if (t == DI_TORUS) {
    /* cell_init_torus (src/Cell/initial_data/cell_init_torus.c:17-89): z is
     * the centre of layer k (0 for a single layer); one rand() per cell after
     * srand(666), layer after layer.  The magnetic terms of the file are never
     * stored, and its Pp = rho branch follows a clamp that already holds
     * PoRho >= 1e-5, so neither is here. */
    double gam = s->Adiabatic_Index, M = 1.0, r_inner = 0.7, r_max = 1.0, q = 2.;
    double sx = 2. * q - q;
    double GammaFac = (gam - 1.) / gam;
    double Phi_inner = -1.0 / r_inner, Phi_max = -1.0 / r_max;
    double Rho_norm = pow(GammaFac * (Phi_inner - Phi_max + pow(r_inner, -sx) / sx - pow(1.0, -sx) / sx), 1.0 / (gam - 1.0));
    double z = 0.0;
    if (s->NumZ != 1) z = 0.5 * (dsim_zface(s, k - 1) + dsim_zface(s, k));
    double R = sqrt(r * r + z * z);
    double Phi = -M / R;
    double omega = pow(r, -q);
    double PoRho = GammaFac * (Phi_inner - Phi + pow(r_inner, -sx) / sx - pow(r, -sx) / sx);
    double rho, Pp, delta;
    int32_t v;
    if (PoRho < 1.0e-5) PoRho = 1.0e-5;
    rho = pow(PoRho, 1.0 / (gam - 1.0)) / Rho_norm;
    Pp = pow(PoRho, 1.0 / GammaFac) / Rho_norm;
    random_r(rnd, &v);
    delta = .02 * ((double)v / (double)RAND_MAX - .5);
    prim[D_RHO] = rho;
    prim[D_PPP] = Pp;
    prim[D_URR] = 0.0;
    prim[D_UPP] = omega * (1. + delta) - pow(r, -2.);
    prim[D_UZZ] = 0.0;
    return 0;
  }
  if (t == DI_MILOS_MACFADYEN) {
    /* cell_init_milos_macfadyen (src/Cell/initial_data/cell_init_milos_macfadyen.c:38-151) */
    double rs = 10.0, rho0 = 1.0, Mach = 1. / sqrt(s->PoRho_r1);
    double delta_exp = 3.0, xi_exp = 2.0, gam = s->Adiabatic_Index;
    double cp = 1. / Mach, fac = 0.0001, Mtotal = 1.0, sep = 1.0, massratio = s->MassRatio;
    double M0, M1, r0, r1, eps0, eps1, alpha = s->Explicit_Viscosity;
    double cs, ph, d0, d1, cs0, cs1, PoRho, Pot1, Pot2, rho, omega, O2, vr, Pp;
    int n = s->PHI_ORDER;
    if (fabs(massratio) > 1.e-8) {
      M0 = Mtotal / (1. + massratio);
      M1 = Mtotal / (1. + 1. / massratio);
      r0 = M1 / Mtotal * sep;
      r1 = M0 / Mtotal * sep;
    } else {
      M0 = 1.0;
      M1 = 0.0;
      r0 = 0.0;
      r1 = 0.0;
    }
    eps0 = s->G_EPS * r0;
    eps1 = s->G_EPS * r1;
    cs = r < 1. ? 1. / Mach : sqrt(1. / r) / Mach;
    ph = tiph - 0.5 * dphi;
    d0 = gm_dist(gm, 0, r, ph, 0.);
    d1 = gm_dist(gm, 1, r, ph, 0.);
    cs0 = d0 < 0.5 ? sqrt(1. / .5) / Mach * sqrt(M0) : sqrt(1. / d0) / Mach * sqrt(M0);
    cs1 = d1 < 0.5 ? sqrt(1. / .5) / Mach * sqrt(M1) : sqrt(1. / d1) / Mach * sqrt(M1);
    PoRho = (cs0 * cs0 + cs1 * cs1) / gam;
    Pot1 = M0 / pow(pow(d0, n) + pow(eps0, n), 1. / n);
    Pot2 = M1 / pow(pow(d1, n) + pow(eps1, n), 1. / n);
    rho = rho0 * (pow(rs / r, delta_exp)) * exp(-pow(rs / r, xi_exp));
    omega = sqrt(1.) / pow(r, 1.5);
    omega *= 1. + 3. / 16. / r / r;
    O2 = omega * omega + cs * cs / r / r * (2. * rs * rs / r / r - 3.);
    if (r < 3.0) {
      omega = 1. / pow(r, 1.5);
      vr = 0.0;
    } else {
      omega = sqrt(O2);
      vr = -3.0 / sqrt(r) * alpha * (1.0 / Mach) * (1.0 / Mach) * (1.0 - delta_exp + xi_exp * pow(r / rs, -xi_exp));
    }
    if (rho < (100. * s->Rho_Floor)) rho = 100. * s->Rho_Floor;
    Pp = PoRho * rho;
    prim[D_RHO] = rho * exp(fac * (Pot1 + Pot2) / cp / cp);
    prim[D_PPP] = Pp * exp(fac * (Pot1 + Pot2) / cp / cp);
    prim[D_URR] = vr;
    prim[D_UPP] = omega - sqrt(1.) / pow(r, 1.5);
    prim[D_UZZ] = 0.0;
    return 0;
  }
  if (t == DI_RAD_DOM) {
    rad_dom_profile(s, r, prim);
    return 0;
  }
  if (t == DI_MIDDLE) {
    middle_profile(s, r, 1, prim);
    return 0;
  }
  if (t == DI_GRESHO || t == DI_KEPLER_RING || t == DI_CIRCUMBINARY) {
    double f = 1. + s->IC_Noise * noise_u(s->IC_Seed, idx);
    newic_profile(s, i, prim);
    prim[D_RHO] = prim[D_RHO] * f;
    if (t != DI_GRESHO) prim[D_PPP] = prim[D_RHO] * (s->IC_HoR * s->IC_HoR / r) / s->Adiabatic_Index;
    return 0;
  }
  if (t == DI_VORTEX) {
    /* cell_init_vortex leaves r >= R cells at cell_create's zeros */
    if (dsim_single_init(s, i, prim) == 0) {
      for (q = 0; q < DGPU_NQ; ++q) prim[q] = 0.0;
    } else if (s->NQ > DGPU_NQ) {
      /* the dye: 1 where cos(phi) >= 0 (cell_init_vortex.c:64-68) */
      prim[DGPU_NQ] = cos(tiph - .5 * dphi) < 0.0 ? 0.0 : 1.0;
    }
    return 0;
  }
  if (t == DI_SSTEST) {
    dsim_single_init(s, i, prim);
    return 0;
  }
  return -1;
}

void dsim_fill_params(const struct dgpu_sim *s, DiskParams *p) {
  memset(p, 0, sizeof(*p));
  p->NR = s->NR;
  p->n_cells = s->Ncells;
  p->riemann = s->RiemannSolver;
  p->visc_const = s->ViscConst;
  p->has_visc = s->Explicit_Viscosity > 0.0;
  p->w_numeric = s->w_numeric_type;
  p->w_analytic = s->w_analytic_type;
  p->grav2d = s->Grav_2D;
  p->phi_order = s->PHI_ORDER;
  p->rho_sink_on = s->RhoSinkOn;
  p->cooling = s->Cooling;
  p->init_type = s->InitialDataType;
  p->has_damp = s->DAMP_TIME > 0.0;
  p->num_sinks = s->GravMassType;
  p->outflow = s->BoundTypeR == DB_OUTFLOW ? (1 | (s->NoInnerBC != 1 ? 2 : 0)) : 0;
  p->num_n = s->NUM_N;
  p->gamma = s->Adiabatic_Index;
  p->plm = s->PLM;
  p->cfl = s->CFL;
  p->visc = s->Explicit_Viscosity;
  p->g_eps = s->G_EPS;
  p->rho_floor = s->Rho_Floor;
  p->cs_floor = s->Cs_Floor;
  p->cs_cap = s->Cs_Cap;
  p->vel_cap = s->Vel_Cap;
  p->t_max = s->Time_Max;
  p->poro_r1 = s->PoRho_r1;
  p->orb_tscale = s->OrbShrinkTscale;
  p->orb_t0 = s->OrbShrinkT0;
  {
    double zp = dsim_zface(s, 0), zm = dsim_zface(s, -1);
    p->dz = zp - zm;
    p->z = .5 * (zp + zm);
  }
  p->NZ = s->NZ;
  p->ngz = s->ng_min[1];
}

void dsim_fill_annulus(const struct dgpu_sim *s, int k, int i, Annulus *a) {
  double rm = dsim_rface(s, i - 1), rp = dsim_rface(s, i);
  double r = .5 * (rp + rm);
  double zm = dsim_zface(s, k - 1), zp = dsim_zface(s, k);
  int NR = s->NR, NZ = s->NZ;
  int kreal = k >= s->ng_min[1] && k < NZ - s->ng_max[1];
  a->i = i;
  a->k = k;
  a->dz = zp - zm;
  a->z = .5 * (zp + zm);
  a->np = s->N_p[i];
  a->rm = rm;
  a->rp = rp;
  a->r = r;
  a->dr = rp - rm;
  a->dv_half = .5 * (rp * rp - rm * rm);
  a->dv_diff = rp * rp - rm * rm;
  a->rom = dsim_rOm_a(s, r, 1.0);
  a->rdrom = dsim_rdrOm_a(s, r, 1.0);
  a->dtom = dsim_dtOm_a(s, r, 1.0);
  switch (s->w_numeric_type) {
    case DC_KEPLER: a->wnum = pow(r, -0.5); break;
    case DC_OMEGA20: a->wnum = r * 20.; break;
    case DC_MILOS: a->wnum = (1. - exp(-pow(r, 1.5))) / sqrt(r); break;
    case DC_POWERLAW: a->wnum = pow(r, -1.0); break;
    default: a->wnum = 0.0; break;
  }
  a->kind = 0;
  /* cell_mindt and the Mdot sum skip the ghost layers too (cell_mindt.c:38-42,
   * cell_source.c:86-88) */
  if (i >= s->ng_min[0] && i < NR - s->ng_max[0] && kreal) a->kind |= DGPU_AK_CFL;
  /* the accretion-rate objective is measured on the innermost non-ghost annulus */
  if (i == s->ng_min[0]) a->kind |= DGPU_AK_MDOT;
  {
    int imin = (s->ng_min[0] == 1) ? 0 : s->ng_min[0];
    if (i >= imin && i < NR - s->ng_max[0] && kreal) a->kind |= DGPU_AK_SINK_SUM;
  }
  if (dsim_single_init(s, i, a->ic) == 1) {
    a->kind |= DGPU_AK_IC;
  } else {
    int q;
    for (q = 0; q < DGPU_NQ; ++q) a->ic[q] = 0.0;
  }
  if (s->BoundTypeR == DB_FIXED) {
    if ((s->NoInnerBC != 1 && i < s->ng_min[0]) || (i > NR - s->ng_max[0] - 1))
      a->kind |= DGPU_AK_BC_FIXED;
  }
  /* cell_boundary_outflow_r rewrites annulus 0 (unless NoInnerBC == 1) and
   * the last two annuli, whatever the ghost counts (cell_boundary.c:24-138) */
  if (s->BoundTypeR == DB_OUTFLOW && ((s->NoInnerBC != 1 && i == 0) || i >= NR - 2))
    a->kind |= DGPU_AK_OUT_DST;
  a->damp_rate = 0.0;
  if (s->DAMP_TIME > 0.0) {
    double R0 = 1. / s->DAMP_TIME / 2. / M_PI;
    if (r < s->RDAMP_INNER || r > s->RDAMP_OUTER) {
      double rate = R0 * (r - s->RDAMP_INNER) / (s->R_Min - s->RDAMP_INNER);
      if (r > s->RDAMP_OUTER) rate = R0 * (r - s->RDAMP_OUTER) / (s->R_Max - s->RDAMP_OUTER);
      a->damp_rate = rate;
      a->kind |= DGPU_AK_DAMP;
    }
  }
  /* build_jloop (src/Face/face_create_destroy.c:27-46): the r pair (i, i+1)
   * of layer k, and the z pair (k, k+1) of annulus i */
  if (i < NR - 1) {
    a->f_r = dsim_rface(s, i);
    a->f_dl = .5 * (dsim_rface(s, i) - dsim_rface(s, i - 1));
    a->f_dr = .5 * (dsim_rface(s, i + 1) - dsim_rface(s, i));
    a->f_dperp = zp - zm;
    a->f_rdrom = dsim_rdrOm_a(s, a->f_r, 1.0);
  } else {
    a->f_r = a->f_dl = a->f_dr = a->f_dperp = a->f_rdrom = 0.0;
  }
  if (NZ > 1 && k < NZ - 1) {
    a->zf_dl = .5 * (dsim_zface(s, k) - dsim_zface(s, k - 1));
    a->zf_dr = .5 * (dsim_zface(s, k + 1) - dsim_zface(s, k));
    a->zf_dperp = rp - rm;
    a->zf_r = .5 * (rp + rm);
  } else {
    a->zf_dl = a->zf_dr = a->zf_dperp = a->zf_r = 0.0;
  }
}

void dsim_initial_tiph(const struct dgpu_sim *s, double *tiph, double *dphi) {
  /* cell_create (src/Cell/cell_create_destroy.c:64-91) followed by
   * cell_clean_pi (src/Cell/cell_misc.c:12-26).  glibc's srand/rand are
   * random_r over a TYPE_3 state of 128 bytes, so initstate_r(666) with such a
   * buffer reproduces srand(666+0); rand() without touching the caller's
   * generator. */
  struct random_data rd;
  char state[128];
  long n = 0;
  int i, j, k;
  memset(&rd, 0, sizeof(rd));
  memset(state, 0, sizeof(state));
  initstate_r(666, state, sizeof(state), &rd);
  for (k = 0; k < s->NZ; k++) {
    for (i = 0; i < s->NR; i++) {
      int32_t v;
      double tiph_0, dp;
      random_r(&rd, &v);
      tiph_0 = PHIMAX * (double)v / (double)RAND_MAX;
      dp = PHIMAX / (double)s->N_p[i];
      for (j = 0; j < s->N_p[i]; j++, n++) {
        double phi = tiph_0 + (double)j * dp;
        while (phi > PHIMAX) phi -= PHIMAX;
        while (phi < 0.0) phi += PHIMAX;
        tiph[n] = phi;
        dphi[n] = dp;
      }
    }
  }
}

int dsim_initial_gravmass(const struct dgpu_sim *s, double *gm) {
  int p;
  memset(gm, 0, sizeof(double) * 12);
  if (s->GravMassType == 0) {
    /* gravMass_init_none: all zero */
  } else if (s->GravMassType == 1) {
    gm[0 * 6 + 2] = 1.0; /* M */
    gm[1 * 6 + 0] = 1.0; /* r */
  } else if (s->GravMassType == 2) {
    double Mtotal = 1.0, sep = 1.0, massratio = s->MassRatio;
    double M0 = Mtotal / (1. + massratio);
    double M1 = Mtotal / (1. + 1. / massratio);
    double r0 = M1 / Mtotal * sep;
    double r1 = M0 / Mtotal * sep;
    double om2 = 1. / sep / sep / sep;
    gm[0] = r0; gm[1] = 0.0; gm[2] = M0; gm[3] = sqrt(om2);
    gm[6] = r1; gm[7] = M_PI; gm[8] = M1; gm[9] = sqrt(om2);
  } else {
    return DGPU_ERR_UNSUPPORTED;
  }
  for (p = 0; p < 2; ++p) { /* gravMass_clean_pi (src/GravMass/GravMass_misc.c:9-17) */
    double phi = gm[6 * p + 1];
    while (phi > 2. * M_PI) phi -= 2. * M_PI;
    while (phi < 0.0) phi += 2. * M_PI;
    gm[6 * p + 1] = phi;
  }
  return DGPU_OK;
}

void dsim_host_zsync(const struct dgpu_sim *s, double *tiph, double *prim) {
  /* the single-rank cell_syncproc_z (src/Cell/cell_sync.c:156-205) copies
   * tiph and prim (and RKcons) of layers NZ-2ng .. NZ-ng-1 into the ng lowest
   * layers and of layers ng .. 2ng-1 into the ng highest: a periodic copy */
  const long per = s->NZ > 0 ? (long)s->Ncells / s->NZ : 0;
  const int ng = s->ng_min[1], shift = s->NZ - 2 * ng;
  int k;
  if (s->NZ <= 1) return;
  for (k = 0; k < s->NZ; ++k) {
    int ks;
    long c0;
    if (k < ng) ks = k + shift;
    else if (k >= s->NZ - ng) ks = k - shift;
    else continue;
    for (c0 = 0; c0 < per; ++c0) {
      const long dst = (long)k * per + c0, src = (long)ks * per + c0;
      if (tiph) tiph[dst] = tiph[src];
      if (prim) memcpy(prim + (size_t)s->NQ * dst, prim + (size_t)s->NQ * src, sizeof(double) * (size_t)s->NQ);
    }
  }
}
