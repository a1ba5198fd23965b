/*
 * C restatement of the reference hot path (oracle; test infrastructure only).
 * Each function names the reference routine it restates.  Expressions keep the
 * reference's operation order; with the same libm and -ffp-contract=off the
 * results equal the reference build's bit for bit (tests/test_oracle.py pins
 * this against the reference's golden outputs).
 */
#define _DEFAULT_SOURCE
#include "disco_port.h"

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PHIMAX 2.0 * M_PI /* src/Headers/header.h:20, unparenthesised like the reference */
#define TVISC_FAC 1.0
#define WA_MILOS 8
enum { RHO, PPP, URR, UPP, UZZ };
enum { DDD, TAU, SRR, LLL, SZZ };
enum { C_FIXED, C_WCELL, C_RIGID, C_KEPLER, C_OMEGA20, C_MILOS, C_POWERLAW };
enum { A_FIXED, A_KEPLER, A_OMEGA20, A_MILOS, A_POWERLAW };
enum { LEFT, LEFTSTAR, RIGHTSTAR, RIGHT };
enum { SHEAR, VORTEX, SSTEST, TORUS, MILOS_MACFADYEN, RAD_DOM, MIDDLE, GRESHO, KEPLER_RING, CIRCUMBINARY };
enum { HLLC, HLL };

static double FP(const Port *p, int i) { return p->rf[i + 1]; } /* sim_FacePos(i, R_DIR) */

#ifdef PORT_ULP_NOISE
/* Sensitivity build (tests only, a separate binary): once the first substep
 * starts, every libm result moves one ulp up or down, pseudo-randomly.  The
 * spread this causes is the part of a case's result that any implementation
 * whose transcendentals differ in the last ulp (the GPU's device libm) cannot
 * pin down; the grid and the initial data are left exact. */
static int ulp_on = 0;
static unsigned long long ulp_state = 0x9E3779B97F4A7C15ULL;
static double ulp_noise(double x) {
  if (!ulp_on || !isfinite(x) || x == 0.0) return x;
  ulp_state = ulp_state * 6364136223846793005ULL + 1442695040888963407ULL;
  return (ulp_state >> 63) ? nextafter(x, INFINITY) : nextafter(x, -INFINITY);
}
#define pow(a, b) ulp_noise(pow(a, b))
#define exp(a) ulp_noise(exp(a))
#define log(a) ulp_noise(log(a))
#define sin(a) ulp_noise(sin(a))
#define cos(a) ulp_noise(cos(a))
#define ULP_NOISE_START() (ulp_on = 1)
#else
#define ULP_NOISE_START() ((void)0)
#endif

/* ---------------- parfile (readvar, src/Sim/sim_readpar.c:10-46) ---------------- */
static int readvar(const char *file, const char *name, double *out) {
  FILE *f = fopen(file, "r");
  char s[512], nm[512], s1[512];
  int found = 0;
  if (!f) return 2;
  nm[0] = 0;
  while ((fgets(s, 512, f) != NULL) && found == 0) {
    sscanf(s, "%511s ", nm);
    if (strcmp(nm, name) == 0) {
      strcpy(s1, s);
      found = 1;
    }
  }
  fclose(f);
  if (!found) return 1;
  {
    char *s2 = s1 + strlen(nm) + strspn(s1 + strlen(nm), "\t :=>_");
    double temp;
    if (sscanf(s2, "%lf", &temp) != 1) return 2;
    *out = temp;
  }
  return 0;
}

int port_read_parfile(Port *p, const char *path) {
  struct { const char *k; int is_int; size_t off; int optional; } keys[] = {
#define I(n, f) {n, 1, offsetof(Port, f), 0}
#define D(n, f) {n, 0, offsetof(Port, f), 0}
      I("Restart", Restart), I("InitialDataType", InitialDataType), I("GravMassType", GravMassType),
      D("MassRatio", MassRatio), D("OrbShrinkTscale", OrbShrinkTscale), D("OrbShrinkT0", OrbShrinkT0),
      I("BoundTypeR", BoundTypeR), I("BoundTypeZ", BoundTypeZ), I("NoInnerBC", NoInnerBC),
      I("NumR", NumR), I("NumZ", NumZ), I("ng", ng), D("R_Min", R_Min), D("R_Max", R_Max),
      D("Z_Min", Z_Min), D("Z_Max", Z_Max), I("NP_CONST", NP_CONST), I("NPCAP", NPCAP),
      D("aspect", aspect), I("NUM_C", NUM_C), I("NUM_N", NUM_N), D("Time_Max", Time_Max),
      I("w_numeric_type", w_numeric_type), I("RiemannSolver", RiemannSolver),
      D("Adiabatic_Index", Adiabatic_Index), I("Cooling", Cooling),
      D("Explicit_Viscosity", Explicit_Viscosity), I("ViscConst", ViscConst), D("PoRho_r1", PoRho_r1),
      D("CFL", CFL), D("PLM", PLM), I("Grav_2D", Grav_2D), D("G_EPS", G_EPS), I("RhoSinkOn", RhoSinkOn),
      I("PHI_ORDER", PHI_ORDER), D("Rho_Floor", Rho_Floor), D("Cs_Floor", Cs_Floor), D("Cs_Cap", Cs_Cap),
      D("Vel_Cap", Vel_Cap), D("DAMP_TIME", DAMP_TIME), D("RDAMP_INNER", RDAMP_INNER),
      D("RDAMP_OUTER", RDAMP_OUTER), D("RLogScale", RLogScale), D("ZLogScale", ZLogScale),
      D("HiResSigma", HiResSigma), D("HiResR0a", HiResR0a), D("HiResR0b", HiResR0b),
      D("HiResFac", HiResFac), I("w_analytic_type", w_analytic_type),
      {"IC_HoR", 0, offsetof(Port, IC_HoR), 1}, {"IC_Noise", 0, offsetof(Port, IC_Noise), 1},
      {"IC_Seed", 1, offsetof(Port, IC_Seed), 1},
#undef I
#undef D
  };
  size_t k;
  p->IC_HoR = 0.05;
  for (k = 0; k < sizeof(keys) / sizeof(keys[0]); ++k) {
    double v;
    int rc = readvar(path, keys[k].k, &v);
    if (rc) {
      if (keys[k].optional && rc == 1) continue;
      fprintf(stderr, "parfile: cannot read %s\n", keys[k].k);
      return 1;
    }
    if (keys[k].is_int) *(int *)((char *)p + keys[k].off) = (int)v;
    else *(double *)((char *)p + keys[k].off) = v;
  }
  return 0;
}

/* ---------------- grid (src/Sim/sim_set.c) ---------------- */
static double r_func(double r, double r2, double fac, double sigma, double r0a, double r0b) {
  double F = r + fac * sigma * sqrt(M_PI / 4.0) * (erf((r - r0a) / sigma) + 1.0) +
             fac * sigma * sqrt(M_PI / 4.0) * (erf((r - r0b) / sigma) + 1.0) - r2;
  return (F);
}
static int sgn(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
static double get_r(double r2, double RMIN, double RMAX, double r0a, double r0b, double sigma, double fac) {
  double r = 0.0, a = RMIN, b = RMAX, TOL = 1.0e-12;
  int n = 1, NMAX = 1000;
  while (n <= NMAX) {
    double c = (a + b) / 2.;
    if ((r_func(c, r2, fac, sigma, r0a, r0b) == 0.0) || ((b - a) / 2. < TOL)) {
      r = c;
      break;
    }
    n = n + 1;
    if (sgn(r_func(c, r2, fac, sigma, r0a, r0b)) == sgn(r_func(a, r2, fac, sigma, r0a, r0b))) a = c;
    else b = c;
  }
  return (r);
}

static void set_grid(Port *p) {
  /* sim_alloc_arr + sim_set_rz + sim_set_N_p for one process (N0 = 0) */
  double RMIN = p->R_Min, RMAX = p->R_Max, Rscale = p->RLogScale, sigma = p->HiResSigma;
  double r0a = p->HiResR0a, r0b = p->HiResR0b, fac = p->HiResFac;
  double r2_max = RMAX + fac * sigma * sqrt(M_PI / 4.0) * (erf((RMAX - r0a) / sigma) + 1.0) +
                  fac * sigma * sqrt(M_PI / 4.0) * (erf((RMAX - r0b) / sigma) + 1.0);
  double r2_min = RMIN + fac * sigma * sqrt(M_PI / 4.0) * (erf((RMIN - r0a) / sigma) + 1.0) +
                  fac * sigma * sqrt(M_PI / 4.0) * (erf((RMIN - r0b) / sigma) + 1.0);
  double r1_max = Rscale * log(1.0 + r2_max / Rscale);
  double r1_min = Rscale * log(1.0 + r2_min / Rscale);
  double Zscale = p->ZLogScale;
  double z1_max = sgn(p->Z_Max) * Zscale * log(1.0 + fabs(p->Z_Max) / Zscale);
  double z1_min = sgn(p->Z_Min) * Zscale * log(1.0 + fabs(p->Z_Min) / Zscale);
  int i, k;
  p->ng_min = 1;
  p->ng_max = p->ng;
  p->NR = p->NumR + p->ng_min + p->ng_max;
  p->rf = malloc(sizeof(double) * (size_t)(p->NR + 1));
  p->N_p = malloc(sizeof(int) * (size_t)p->NR);
  p->off = malloc(sizeof(int) * (size_t)(p->NR + 1));
  for (i = 0; i < p->NR + 1; i++) {
    int ig = i - p->ng_min;
    double delta = (r1_max - r1_min) / (double)p->NumR;
    double r1 = r1_min + (double)ig * delta;
    double r2 = Rscale * (exp(r1 / Rscale) - 1.0);
    p->rf[i] = get_r(r2, 0., 2. * RMAX, r0a, r0b, sigma, fac);
  }
  if (p->NoInnerBC == 1) p->rf[0] = 0.0;
  for (k = 0; k < 2; k++) {
    double delta = (z1_max - z1_min) / (double)p->NumZ;
    double z1 = z1_min + (double)k * delta;
    p->zf[k] = sgn(z1) * Zscale * (exp(fabs(z1) / Zscale) - 1.0);
  }
  p->N = 0;
  for (i = 0; i < p->NR; ++i) {
    if (p->NP_CONST > 0) {
      p->N_p[i] = p->NP_CONST;
    } else {
      double r_cell = 0.5 * (FP(p, i - 1) + FP(p, i));
      double dr = FP(p, i) - FP(p, i - 1);
      if (r_cell < p->R_Min) {
        double dr_plus = FP(p, i + 1) - FP(p, i);
        p->N_p[i] = (int)(PHIMAX * (1. + (r_cell / dr_plus - 1.) / p->aspect));
      } else {
        p->N_p[i] = (int)(PHIMAX * (1. + (r_cell / dr - 1.) / p->aspect));
      }
      if (p->NPCAP > 0 && p->N_p[i] > p->NPCAP) p->N_p[i] = p->NPCAP;
    }
    p->off[i] = p->N;
    p->N += p->N_p[i];
  }
  p->off[p->NR] = p->N;
}

/* ---------------- frame (src/Sim/sim_w_a.c:8-72) ---------------- */
static double rOm_a(const Port *p, double r, double a) {
  switch (p->w_analytic_type) {
    case A_FIXED: return (0.0);
    case A_KEPLER: return (pow(r, -0.5));
    case A_OMEGA20: return (r * 20);
    case A_MILOS:
      return (r * (pow(r, WA_MILOS - 1.5) + pow(a, WA_MILOS - 1.5)) / (pow(r, WA_MILOS) + pow(a, WA_MILOS)));
    default: return (pow(r, -1.0));
  }
}
static double rdrOm_a(const Port *p, double r, double a) {
  switch (p->w_analytic_type) {
    case A_FIXED: return (0.0);
    case A_KEPLER: return (-1.5 * pow(r, -1.5));
    case A_OMEGA20: return (0.0);
    case A_MILOS: {
      int n = WA_MILOS;
      double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
      double arn = pow(a / r, n);
      return ((-1.5 + n * arn / (1. + arn)) * Omega_a + (1.5 - n) * pow(a / r, n - 1.5) / (1. + arn) * pow(r, -1.5));
    }
    default: return (-2. * pow(r, -2.0));
  }
}
static double dtOm_a(const Port *p, double r, double a) {
  if (p->w_analytic_type == A_MILOS) {
    double a0 = 1.0, tau = p->OrbShrinkTscale;
    double dta_o_a = -.25 * pow(a / a0, -4) / tau;
    int n = WA_MILOS;
    double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
    double arn = pow(a / r, n);
    if (a > 0.0) return (dta_o_a * (Omega_a * (-1.5 + n / (1. + arn)) + (1.5 - n) * pow(r, -1.5) / (1. + arn)));
    return (0.0);
  }
  return (0.0);
}

/* ---------------- initial data ---------------- */
static double noise_u(int seed, long idx) {
  uint64_t z = ((uint64_t)(uint32_t)seed << 40) ^ (uint64_t)idx;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

/* cell_init_middle.c:12-91; grid != 0: the whole-grid form (v_r = 0 inside r = 1) */
static void middle(const Port *p, double r, int grid, double *prim) {
  double r0 = 2.5, a = 1.0, al = p->Explicit_Viscosity;
  int d = 10;
  double rh = pow(r, -3. / 5.) * exp(-pow(r / r0, -d));
  double Pq = p->PoRho_r1 * pow(r, -3. / 2.) * exp(-pow(r / r0, -d));
  double rdp = -1.5 + d * pow(r / r0, -d), om, vr;
  if (rh < 1.e-3) rh = 1.e-3;
  if (Pq < 1.e-6) Pq = 1.e-6;
  om = sqrt(1. / r / r / r * pow(1. + 3. / 16. / r / r, 2) + rdp * Pq / rh / r / r);
  om = (pow(r, WA_MILOS) * om + pow(a, WA_MILOS - 1.5)) / (pow(r, WA_MILOS) + pow(a, WA_MILOS));
  vr = -3. * al / r / om * Pq / rh * (2. + rdp);
  if (grid && r < 1.) vr = 0.0;
  prim[RHO] = rh; prim[PPP] = Pq; prim[URR] = vr; prim[UPP] = om - rOm_a(p, r, a) / r; prim[UZZ] = 0.0;
}

/* single-cell initial data of annulus i: 1 = set, 0 = left unchanged */
static int single_init(const Port *p, int i, double *prim) {
  double rm = FP(p, i - 1), rp = FP(p, i);
  double r = 0.5 * (rm + rp);
  double gam = p->Adiabatic_Index, hor = p->IC_HoR;
  double rho = 1.0, P = 1.0, vphi = 0.0;
  switch (p->InitialDataType) {
    case VORTEX: { /* cell_single_init_vortex, initial_data/cell_init_vortex.c:11-37 */
      double rh = 1.0, P0 = 1.0, R = 1.0, A = 0.5, g = 3.0, Pp, vp;
      if (r >= R) return 0;
      Pp = P0 * (1. - A * exp(g * (r / R - R / (R - r) + 1.)));
      vp = sqrt(A * g * P0 / rh * (2. * R - r) / R * r * r / pow(R - r, 2.) * exp(g * (r / R - R / (R - r) + 1.)));
      prim[RHO] = rh; prim[PPP] = Pp; prim[URR] = 0.0; prim[UPP] = vp / r; prim[UZZ] = 0.0;
      return 1;
    }
    case SSTEST: { /* cell_single_init_SStest, initial_data/cell_init_SStest.c:11-45 */
      double r0 = 5., a = 1.0;
      int d = 4;
      double rh = pow(r, -3. / 5.) * exp(-pow(r / r0, -d));
      double Pq = p->PoRho_r1 * pow(r, -3. / 2.) * exp(-pow(r / r0, -d));
      if (rh < 1.e-4) rh = 1.e-4;
      if (Pq < 1.e-7) Pq = 1.e-7;
      prim[RHO] = rh; prim[PPP] = Pq; prim[URR] = 0.0;
      prim[UPP] = pow(r, -1.5) - rOm_a(p, r, a) / r; prim[UZZ] = 0.0;
      return 1;
    }
    case MILOS_MACFADYEN: { /* cell_single_init_milos_macfadyen, initial_data/cell_init_milos_macfadyen.c:11-36 */
      double Mach = 1. / sqrt(p->PoRho_r1), rs = 10.;
      double rh = 1.0 * (pow(rs / r, 3.0)) * exp(-pow(rs / r, 2.0));
      prim[RHO] = rh; prim[PPP] = 1. / Mach / Mach / gam * rh; prim[URR] = 0.0; prim[UPP] = 0.0; prim[UZZ] = 0.0;
      return 1;
    }
    case RAD_DOM: { /* cell_single_init_rad_dom, initial_data/cell_init_rad_dom.c:13-36 */
      double xi = 0.005, aM = 100., al = p->Explicit_Viscosity, zero = 0.0;
      double rho0 = 2. / (9. * xi * al * gam) * sqrt(aM), P0 = 8. * xi / (9. * al * gam) * sqrt(aM);
      double rh = rho0 * pow(r, 1.5), Pq = P0 * pow(r, -1.5);
      double om = sqrt(1. / r / r / r - 3. / 2. * Pq / rh / r / r);
      prim[RHO] = rh; prim[PPP] = Pq;
      prim[URR] = -1.5 * al * gam * (Pq / rh) * sqrt(r) - zero * pow(r, -4.5);
      prim[UPP] = om - 1. / pow(r, 1.5); prim[UZZ] = 0.0;
      return 1;
    }
    case MIDDLE: /* cell_single_init_middle, initial_data/cell_init_middle.c:12-45 */
      middle(p, r, 0, prim);
      return 1;
    case GRESHO:
      rho = 1.0;
      if (r < 0.2) { vphi = 5. * r; P = 5. + 12.5 * r * r; }
      else if (r < 0.4) { vphi = 2. - 5. * r; P = 9. + 12.5 * r * r - 20. * r + 4. * log(5. * r); }
      else { vphi = 0.0; P = 3. + 4. * log(2.); }
      break;
    case KEPLER_RING: {
      double w = 0.1, x = r - 2.;
      double s0 = exp(-(x * x) / (2. * w * w));
      double sig = s0 + 1.e-4, cs2 = hor * hor / r;
      double dsig = -x / (w * w) * s0;
      double dP = hor * hor / gam * (dsig / r - sig / (r * r));
      rho = sig; P = sig * cs2 / gam; vphi = sqrt(1. / r + r * dP / sig);
      break;
    }
    case CIRCUMBINARY: {
      double s0 = pow(r, -0.5) * exp(-pow(2. / r, 12.));
      double sig = s0 + 1.e-5, cs2 = hor * hor / r;
      rho = sig; P = sig * cs2 / gam; vphi = pow(r, -0.5);
      break;
    }
    default:
      return -1;
  }
  prim[RHO] = rho; prim[PPP] = P; prim[URR] = 0.0;
  prim[UPP] = vphi / r - rOm_a(p, r, 1.) / r; prim[UZZ] = 0.0;
  return 1;
}

/* gravMass_dist (GravMass/GravMass_access.c:25-31) */
static double bh_dist(const Port *p, int k, double r, double phi) {
  double xb = p->gr[k] * cos(p->gphi[k]), yb = p->gr[k] * sin(p->gphi[k]);
  double x = r * cos(phi), y = r * sin(phi);
  return sqrt((x - xb) * (x - xb) + (y - yb) * (y - yb) + 0. * 0.);
}

/* whole-grid initial data that differs from the single-cell form, for cell g
 * of annulus i: 1 = set here, 0 = use single_init */
static int grid_cell(const Port *p, int i, int g, double *prim) {
  double r = 0.5 * (FP(p, i - 1) + FP(p, i)), gam = p->Adiabatic_Index;
  double ph = p->tiph[g] - .5 * p->dphi[g];
  switch (p->InitialDataType) {
    case SHEAR: { /* cell_init_shear, initial_data/cell_init_shear.c:57-116 */
      double nu = p->Explicit_Viscosity > 0.0 ? p->Explicit_Viscosity : 0.05, t0 = 0.25, vy = 0.0;
      double x = r * cos(ph) - 3., y = r * sin(ph);
      if (fabs(y) < 50.) vy = 1.0 / sqrt(2. * M_PI * nu * t0) * exp(-x * x / (4. * nu * t0));
      prim[RHO] = 1.0; prim[PPP] = 0.01; prim[URR] = vy * sin(ph);
      prim[UPP] = vy * cos(ph) / r - rOm_a(p, r, 1.) / r; prim[UZZ] = 0.0;
      return 1;
    }
    case TORUS: { /* cell_init_torus, initial_data/cell_init_torus.c:17-89, z = 0 */
      double q = 2., sx = 2. * q - q, gf = (gam - 1.) / gam, ri = 0.7;
      double norm = pow(gf * (-1.0 / ri - -1.0 / 1.0 + pow(ri, -sx) / sx - pow(1.0, -sx) / sx), 1.0 / (gam - 1.0));
      double pr = gf * (-1.0 / ri - -1.0 / sqrt(r * r + 0.0 * 0.0) + pow(ri, -sx) / sx - pow(r, -sx) / sx);
      double delta;
      if (pr < 1.0e-5) pr = 1.0e-5;
      delta = .02 * ((double)rand() / (double)RAND_MAX - .5);
      prim[RHO] = pow(pr, 1.0 / (gam - 1.0)) / norm; prim[PPP] = pow(pr, 1.0 / gf) / norm;
      prim[URR] = 0.0; prim[UPP] = pow(r, -q) * (1. + delta) - pow(r, -2.); prim[UZZ] = 0.0;
      return 1;
    }
    case MILOS_MACFADYEN: { /* cell_init_milos_macfadyen, initial_data/cell_init_milos_macfadyen.c:38-151 */
      double rs = 10.0, Mach = 1. / sqrt(p->PoRho_r1), cp = 1. / Mach, mr = p->MassRatio;
      double M0 = 1.0, M1 = 0.0, r0 = 0.0, r1 = 0.0, cs, d0, d1, c0, c1, pot, rh, om, vr;
      int n = p->PHI_ORDER;
      if (fabs(mr) > 1.e-8) {
        M0 = 1.0 / (1. + mr); M1 = 1.0 / (1. + 1. / mr);
        r0 = M1 / 1.0 * 1.0; r1 = M0 / 1.0 * 1.0;
      }
      cs = r < 1. ? 1. / Mach : sqrt(1. / r) / Mach;
      d0 = bh_dist(p, 0, r, ph);
      d1 = bh_dist(p, 1, r, ph);
      c0 = (d0 < 0.5 ? sqrt(1. / .5) : sqrt(1. / d0)) / Mach * sqrt(M0);
      c1 = (d1 < 0.5 ? sqrt(1. / .5) : sqrt(1. / d1)) / Mach * sqrt(M1);
      pot = M0 / pow(pow(d0, n) + pow(p->G_EPS * r0, n), 1. / n) + M1 / pow(pow(d1, n) + pow(p->G_EPS * r1, n), 1. / n);
      rh = 1.0 * (pow(rs / r, 3.0)) * exp(-pow(rs / r, 2.0));
      om = sqrt(1.) / pow(r, 1.5) * (1. + 3. / 16. / r / r);
      if (r < 3.0) {
        om = 1. / pow(r, 1.5);
        vr = 0.0;
      } else {
        om = sqrt(om * om + cs * cs / r / r * (2. * rs * rs / r / r - 3.));
        vr = -3.0 / sqrt(r) * p->Explicit_Viscosity * (1.0 / Mach) * (1.0 / Mach) * (1.0 - 3.0 + 2.0 * pow(r / rs, -2.0));
      }
      if (rh < (100. * p->Rho_Floor)) rh = 100. * p->Rho_Floor;
      prim[RHO] = rh * exp(0.0001 * pot / cp / cp);
      prim[PPP] = (c0 * c0 + c1 * c1) / gam * rh * exp(0.0001 * pot / cp / cp);
      prim[URR] = vr; prim[UPP] = om - sqrt(1.) / pow(r, 1.5); prim[UZZ] = 0.0;
      return 1;
    }
    case MIDDLE:
      middle(p, r, 1, prim);
      return 1;
    default:
      return 0;
  }
}

/* ---------------- conversions (src/Cell/cell_conversion.c) ---------------- */
static void prim2cons(const Port *p, const double *prim, double *cons, double r, double dV) {
  double GAMMALAW = p->Adiabatic_Index;
  double rho = prim[RHO], Pp = prim[PPP], vr = prim[URR], vp = prim[UPP] * r, vz = prim[UZZ];
  double v2 = vr * vr + vp * vp + vz * vz;
  double rhoe = Pp / (GAMMALAW - 1.);
  cons[DDD] = rho * dV;
  cons[SRR] = rho * vr * dV;
  cons[LLL] = r * rho * vp * dV;
  cons[SZZ] = rho * vz * dV;
  cons[TAU] = (.5 * rho * v2 + rhoe) * dV;
  for (int q = 5; q < p->NQ; ++q) cons[q] = prim[q] * cons[DDD]; /* passive scalars */
}
static void cons2prim(const Port *p, const double *cons, double *prim, double r, double dV) {
  double CS_FLOOR = p->Cs_Floor, CS_CAP = p->Cs_Cap, RHO_FLOOR = p->Rho_Floor, VEL_CAP = p->Vel_Cap;
  double GAMMALAW = p->Adiabatic_Index;
  double rho = cons[DDD] / dV;
  double Sr, Sp, Sz, E, vr, vp, vz, KE, v_magnitude, rhoe, Pp;
  if (rho < RHO_FLOOR) rho = RHO_FLOOR;
  Sr = cons[SRR] / dV;
  Sp = cons[LLL] / dV / r;
  Sz = cons[SZZ] / dV;
  E = cons[TAU] / dV;
  vr = Sr / rho;
  vp = Sp / rho;
  vz = Sz / rho;
  KE = .5 * (Sr * vr + Sp * vp + Sz * vz);
  v_magnitude = sqrt(2. * KE / rho);
  rhoe = E - KE;
  Pp = (GAMMALAW - 1.) * rhoe;
  if (Pp < CS_FLOOR * CS_FLOOR * rho / GAMMALAW) Pp = CS_FLOOR * CS_FLOOR * rho / GAMMALAW;
  if (Pp > CS_CAP * CS_CAP * rho / GAMMALAW) Pp = CS_CAP * CS_CAP * rho / GAMMALAW;
  if (v_magnitude > VEL_CAP) {
    vr = vr * VEL_CAP / v_magnitude;
    vp = vp * VEL_CAP / v_magnitude;
    vz = vz * VEL_CAP / v_magnitude;
  }
  prim[RHO] = rho; prim[PPP] = Pp; prim[URR] = vr; prim[UPP] = vp / r; prim[UZZ] = vz;
  for (int q = 5; q < p->NQ; ++q) prim[q] = cons[q] / cons[DDD]; /* passive scalars */
}

void port_calc_cons(Port *p) {
  double dz = p->zf[1] - p->zf[0];
  int i, j, q;
  for (i = 0; i < p->NR; ++i) {
    double rp = FP(p, i), rm = FP(p, i - 1), r = .5 * (rp + rm);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double dV = .5 * (rp * rp - rm * rm) * p->dphi[g] * dz;
      double pr[PORT_MAXQ], c[PORT_MAXQ];
      for (q = 0; q < p->NQ; ++q) pr[q] = p->prim[q][g];
      prim2cons(p, pr, c, r, dV);
      for (q = 0; q < p->NQ; ++q) p->cons[q][g] = c[q];
    }
  }
}

static void calc_prim(Port *p) {
  double dz = p->zf[1] - p->zf[0];
  int i, j, q;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i), r = .5 * (rp + rm);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double dV = .5 * (rp * rp - rm * rm) * p->dphi[g] * dz;
      double c[PORT_MAXQ], pr[PORT_MAXQ];
      for (q = 0; q < p->NQ; ++q) c[q] = p->cons[q][g];
      cons2prim(p, c, pr, r, dV);
      for (q = 0; q < p->NQ; ++q) p->prim[q][g] = pr[q];
    }
  }
}

/* ---------------- set-up (src/main.c:56-119) ---------------- */
int port_setup(Port *p) {
  int i, j, q;
  long idx = 0;
  if (p->NumZ != 1 || p->NUM_C != 5 || p->NUM_N < 0 || 5 + p->NUM_N > PORT_MAXQ) {
    fprintf(stderr, "port: only 2-D disks with NUM_C = 5 and NUM_Q <= %d are restated\n", PORT_MAXQ);
    return 1;
  }
  p->NQ = 5 + p->NUM_N;
  set_grid(p);
  for (q = 0; q < p->NQ; ++q) {
    p->prim[q] = calloc((size_t)p->N, sizeof(double));
    p->cons[q] = calloc((size_t)p->N, sizeof(double));
    p->rkcons[q] = calloc((size_t)p->N, sizeof(double));
    p->grad[q] = calloc((size_t)p->N, sizeof(double));
    p->gradp[q] = calloc((size_t)p->N, sizeof(double));
  }
  p->tiph = calloc((size_t)p->N, sizeof(double));
  p->rktiph = calloc((size_t)p->N, sizeof(double));
  p->dphi = calloc((size_t)p->N, sizeof(double));
  p->wiph = calloc((size_t)p->N, sizeof(double));
  p->nri = calloc((size_t)p->NR, sizeof(int));
  p->fcap = 2 * p->N + 8 * p->NR;
  p->fL = malloc(sizeof(int) * (size_t)p->fcap);
  p->fR = malloc(sizeof(int) * (size_t)p->fcap);
  p->fr = malloc(sizeof(double) * (size_t)p->fcap);
  p->fdphi = malloc(sizeof(double) * (size_t)p->fcap);
  p->fdA = malloc(sizeof(double) * (size_t)p->fcap);
  p->fdl = malloc(sizeof(double) * (size_t)p->fcap);
  p->fdr = malloc(sizeof(double) * (size_t)p->fcap);
  p->fcm = malloc(sizeof(double) * (size_t)p->fcap);
  /* cell_create (src/Cell/cell_create_destroy.c:64-91) + cell_clean_pi */
  srand(666);
  for (i = 0; i < p->NR; i++) {
    double tiph_0 = PHIMAX * (double)rand() / (double)RAND_MAX;
    double dphi = PHIMAX / (double)p->N_p[i];
    for (j = 0; j < p->N_p[i]; j++) {
      int g = p->off[i] + j;
      double tiph = tiph_0 + (double)j * dphi;
      while (tiph > PHIMAX) tiph -= PHIMAX;
      while (tiph < 0.0) tiph += PHIMAX;
      p->tiph[g] = tiph;
      p->rktiph[g] = tiph;
      p->dphi[g] = dphi;
    }
  }
  /* gravMass_init_* (src/GravMass/GravMass_init.c:9-84) */
  memset(p->gr, 0, sizeof(p->gr)); memset(p->gphi, 0, sizeof(p->gphi));
  memset(p->gM, 0, sizeof(p->gM)); memset(p->gom, 0, sizeof(p->gom));
  memset(p->mdot, 0, sizeof(p->mdot)); memset(p->macc, 0, sizeof(p->macc));
  if (p->GravMassType == 1) {
    p->gM[0] = 1.0;
    p->gr[1] = 1.0;
  } else if (p->GravMassType == 2) {
    double Mtotal = 1.0, sep = 1.0, q2 = p->MassRatio;
    double M0 = Mtotal / (1. + q2), M1 = Mtotal / (1. + 1. / q2);
    double om2 = 1. / sep / sep / sep;
    p->gM[0] = M0; p->gr[0] = M1 / Mtotal * sep; p->gphi[0] = 0.0; p->gom[0] = sqrt(om2);
    p->gM[1] = M1; p->gr[1] = M0 / Mtotal * sep; p->gphi[1] = M_PI; p->gom[1] = sqrt(om2);
  }
  /* initial data (cell_init_*; ref_newic.c for 7..9) */
  srand(666); /* cell_init_torus re-seeds */
  for (i = 0; i < p->NR; i++) {
    double rm = FP(p, i - 1), rp = FP(p, i), r = 0.5 * (rm + rp);
    double prof[5];
    int st = single_init(p, i, prof);
    if (p->InitialDataType == SHEAR || p->InitialDataType == TORUS || p->InitialDataType == MILOS_MACFADYEN ||
        p->InitialDataType == MIDDLE) {
      for (j = 0; j < p->N_p[i]; j++, idx++) {
        int g = p->off[i] + j;
        double c[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        grid_cell(p, i, g, c);
        for (q = 0; q < 5; ++q) p->prim[q][g] = c[q];
      }
      continue;
    }
    if (st < 0) {
      fprintf(stderr, "port: InitialDataType %d is not restated\n", p->InitialDataType);
      return 1;
    }
    for (j = 0; j < p->N_p[i]; j++, idx++) {
      int g = p->off[i] + j;
      if (st == 0) continue; /* vortex leaves r >= R at cell_create's zeros */
      for (q = 0; q < 5; ++q) p->prim[q][g] = prof[q];
      /* cell_init_vortex's dye: 1 where cos(phi) >= 0 (cell_init_vortex.c:64-68);
         the other families leave passive scalars at zero */
      if (p->InitialDataType == VORTEX && p->NQ > 5)
        p->prim[5][g] = cos(p->tiph[g] - .5 * p->dphi[g]) < 0.0 ? 0.0 : 1.0;
      if (p->InitialDataType >= GRESHO) {
        double f = 1. + p->IC_Noise * noise_u(p->IC_Seed, idx);
        p->prim[RHO][g] = prof[RHO] * f;
        if (p->InitialDataType != GRESHO)
          p->prim[PPP][g] = p->prim[RHO][g] * (p->IC_HoR * p->IC_HoR / r) / p->Adiabatic_Index;
      }
    }
  }
  {
    int k;
    for (k = 0; k < 2; ++k) { /* gravMass_clean_pi */
      while (p->gphi[k] > 2. * M_PI) p->gphi[k] -= 2. * M_PI;
      while (p->gphi[k] < 0.0) p->gphi[k] += 2. * M_PI;
    }
  }
  p->t = 0.0;
  p->dt = 0.0;
  port_calc_cons(p);
  return 0;
}

void port_free(Port *p) {
  int q;
  for (q = 0; q < p->NQ; ++q) {
    free(p->prim[q]); free(p->cons[q]); free(p->rkcons[q]); free(p->grad[q]); free(p->gradp[q]);
  }
  free(p->tiph); free(p->rktiph); free(p->dphi); free(p->wiph); free(p->nri);
  free(p->fL); free(p->fR); free(p->fr); free(p->fdphi); free(p->fdA); free(p->fdl); free(p->fdr);
  free(p->fcm); free(p->rf); free(p->N_p); free(p->off);
}

/* ---------------- faces (src/Face/face_create_destroy.c:11-193) ---------------- */
static void add_face(Port *p, int n, int L, int R, double r, double dl, double dr, double dphi, double tp,
                     double dperp) {
  if (n >= p->fcap) {
    fprintf(stderr, "port: face buffer overflow\n");
    exit(4);
  }
  p->fL[n] = L; p->fR[n] = R; p->fr[n] = r; p->fdl[n] = dl; p->fdr[n] = dr;
  p->fdphi[n] = dphi;
  p->fdA[n] = r * dphi * dperp;
  p->fcm[n] = tp - .5 * dphi;
}

void port_build_faces(Port *p) {
  int n = 0, i, j, jp;
  double dperp = p->zf[1] - p->zf[0];
  for (i = 0; i < p->NR - 1; ++i) {
    int a = p->off[i], b = p->off[i + 1], Ni = p->N_p[i], No = p->N_p[i + 1];
    double deltaL = .5 * (FP(p, i) - FP(p, i - 1));
    double deltaR = .5 * (FP(p, i + 1) - FP(p, i));
    double r = FP(p, i);
    double p0 = p->tiph[a + Ni - 1];
    int jpmin = 0;
    double dpmin = PHIMAX;
    p->nri[i] = n;
    for (jp = 0; jp < No; ++jp) {
      double dp = p->tiph[b + jp] - p0;
      while (dp > PHIMAX) dp -= PHIMAX;
      while (dp < 0.0) dp += PHIMAX;
      if (dpmin > dp) { dpmin = dp; jpmin = jp; }
    }
    jp = jpmin;
    for (j = 0; j < Ni; ++j) {
      int jm = j - 1;
      double dp;
      if (jm < 0) jm = Ni - 1;
      dp = p->tiph[b + jp] - p->tiph[a + jm];
      while (dp > PHIMAX) dp -= PHIMAX;
      while (dp < 0.0) dp += PHIMAX;
      if (p->dphi[a + j] < dp) {
        add_face(p, n++, a + j, b + jp, r, deltaL, deltaR, p->dphi[a + j], p->tiph[a + j], dperp);
      } else {
        add_face(p, n++, a + j, b + jp, r, deltaL, deltaR, dp, p->tiph[b + jp], dperp);
        ++jp;
        if (jp == No) jp = 0;
        dp = p->tiph[a + j] - p->tiph[b + jp];
        while (dp > PHIMAX / 2.) dp -= PHIMAX;
        while (dp < -PHIMAX / 2.) dp += PHIMAX;
        while (dp > 0.0) {
          add_face(p, n++, a + j, b + jp, r, deltaL, deltaR, p->dphi[b + jp], p->tiph[b + jp], dperp);
          ++jp;
          if (jp == No) jp = 0;
          dp = p->tiph[a + j] - p->tiph[b + jp];
          while (dp > PHIMAX / 2.) dp -= PHIMAX;
          while (dp < -PHIMAX / 2.) dp += PHIMAX;
        }
        dp = p->dphi[b + jp] + dp;
        add_face(p, n++, a + j, b + jp, r, deltaL, deltaR, dp, p->tiph[a + j], dperp);
      }
    }
  }
  p->nri[p->NR - 1] = n;
  p->nf = n;
}

/* ---------------- mesh motion, w, RK helpers (src/Cell/cell_misc.c, cell_set_w.c) ---------------- */
static void clean_pi(Port *p) {
  int g;
  for (g = 0; g < p->N; ++g) {
    double phi = p->tiph[g];
    while (phi > PHIMAX) phi -= PHIMAX;
    while (phi < 0.0) phi += PHIMAX;
    p->tiph[g] = phi;
  }
}
static void set_w(Port *p) {
  int i, j;
  for (i = 0; i < p->NR; ++i) {
    double rp = FP(p, i), rm = FP(p, i - 1), r = 0.5 * (rm + rp), w = 0.0;
    switch (p->w_numeric_type) {
      case C_RIGID: {
        double Mring = 0.0;
        for (j = 0; j < p->N_p[i]; ++j) {
          int g = p->off[i] + j;
          double vp = r * p->prim[UPP][g], m = p->cons[DDD][g];
          Mring += m;
          w += vp * m;
        }
        w = w / Mring;
        break;
      }
      case C_KEPLER: w = pow(r, -0.5); break;
      case C_OMEGA20: w = r * 20.; break;
      case C_MILOS: w = (1. - exp(-pow(r, 1.5))) / sqrt(r); break;
      case C_POWERLAW: w = pow(r, -1.0); break;
      default: w = 0.0;
    }
    for (j = 0; j < p->N_p[i]; ++j) p->wiph[p->off[i] + j] = w;
  }
}

static double gm_dist(const Port *p, int k, double r, double phi) {
  double xbh = p->gr[k] * cos(p->gphi[k]), ybh = p->gr[k] * sin(p->gphi[k]);
  double x = r * cos(phi), y = r * sin(phi), z = 0.;
  return (sqrt((x - xbh) * (x - xbh) + (y - ybh) * (y - ybh) + z * z));
}

/* cell_mindt (src/Cell/cell_mindt.c:10-100) + timestep_set_dt */
static void set_dt(Port *p) {
  double dz = p->zf[1] - p->zf[0], dt_m = 1.e100;
  int i, j;
  for (i = p->ng_min; i < p->NR - p->ng_max; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i), dr = rp - rm, r = .5 * (rp + rm);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j, jm = j == 0 ? p->N_p[i] - 1 : j - 1;
      double w = .5 * (p->wiph[g] + p->wiph[p->off[i] + jm]);
      double dx = dr, rdphi = .5 * (rp + rm) * p->dphi[g];
      double Pp = p->prim[PPP][g], rho = p->prim[RHO][g];
      double vp = p->prim[UPP][g] * r - w, vr = p->prim[URR][g], vz = p->prim[UZZ][g];
      double cs, cf2, maxv, dt;
      if (rdphi < dr) dx = rdphi;
      if (dx > dz) dx = dz;
      cs = sqrt(p->Adiabatic_Index * Pp / rho);
      cf2 = cs * cs;
      maxv = sqrt(cf2) + sqrt(vr * vr + vp * vp + vz * vz);
      dt = p->CFL * dx / maxv;
      if (p->Explicit_Viscosity > 0.0) {
        double nu;
        if (p->ViscConst == 1) {
          nu = p->Explicit_Viscosity;
        } else {
          double tc = p->tiph[g] - 0.5 * p->dphi[g];
          double d0 = gm_dist(p, 0, r, tc), d1 = gm_dist(p, 1, r, tc), eps = p->G_EPS;
          nu = p->Explicit_Viscosity * Pp / rho /
               sqrt(pow(d0 * d0 + eps * eps, -1.5) * p->gM[0] + pow(d1 * d1 + eps * eps, -1.5) * p->gM[1]);
        }
        {
          double dt_visc = .25 * dx * dx / nu;
          dt = dt / (1. + dt / dt_visc);
        }
      }
      if (dt_m > dt) dt_m = dt;
    }
  }
  p->dt = dt_m;
  if (p->t + p->dt > p->Time_Max) p->dt = p->Time_Max - p->t;
}

/* ---------------- PLM (src/Cell/cell_plm.c) ---------------- */
static void plm_p(Port *p) {
  int i, j, q;
  for (i = 0; i < p->NR; ++i) {
    int a = p->off[i], n = p->N_p[i];
    for (j = 0; j < n; ++j) {
      int c = a + j, cL = a + (j == 0 ? n - 1 : j - 1), cR = a + (j == n - 1 ? 0 : j + 1);
      double dpL = .5 * (p->dphi[c] + p->dphi[cL]), dpR = .5 * (p->dphi[c] + p->dphi[cR]);
      for (q = 0; q < p->NQ; ++q) {
        double sL = (p->prim[q][c] - p->prim[q][cL]) / dpL;
        double sR = (p->prim[q][cR] - p->prim[q][c]) / dpR;
        double sM = (p->prim[q][cR] - p->prim[q][cL]) / (dpL + dpR);
        double s = p->PLM * sL;
        if (fabs(s) > p->PLM * fabs(sR)) s = p->PLM * sR;
        if (fabs(s) > fabs(sM)) s = sM;
        if (sL * sR < 0.0) s = 0.0;
        p->gradp[q][c] = s;
      }
    }
  }
}

static void face_dps(const Port *p, int n, double *dpL, double *dpR) {
  int cL = p->fL[n], cR = p->fR[n];
  double pL = p->tiph[cL] - .5 * p->dphi[cL], pR = p->tiph[cR] - .5 * p->dphi[cR];
  double a = p->fcm[n] - pL, b = pR - p->fcm[n];
  while (a > PHIMAX / 2.) a -= PHIMAX;
  while (a < -PHIMAX / 2.) a += PHIMAX;
  while (b > PHIMAX / 2.) b -= PHIMAX;
  while (b < -PHIMAX / 2.) b += PHIMAX;
  *dpL = a;
  *dpR = b;
}

static void plm_rz(Port *p) {
  double dz = p->zf[1] - p->zf[0];
  int n, q, i, j;
  for (q = 0; q < p->NQ; ++q) memset(p->grad[q], 0, sizeof(double) * (size_t)p->N);
  for (n = 0; n < p->nf; ++n) {
    int cL = p->fL[n], cR = p->fR[n];
    double dpL, dpR;
    face_dps(p, n, &dpL, &dpR);
    for (q = 0; q < p->NQ; ++q) {
      double WL = p->prim[q][cL] + dpL * p->gradp[q][cL];
      double WR = p->prim[q][cR] - dpR * p->gradp[q][cR];
      double S = (WR - WL) / (p->fdr[n] + p->fdl[n]);
      p->grad[q][cL] += S * p->fdA[n];
      p->grad[q][cR] += S * p->fdA[n];
    }
  }
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double dp = p->dphi[g], dAtot;
      if (i == 0) dAtot = dz * rp * dp;
      else if (i == p->NR - 1) dAtot = dz * rm * dp;
      else dAtot = dz * (rp + rm) * dp;
      for (q = 0; q < p->NQ; ++q) p->grad[q][g] /= dAtot;
    }
  }
  for (n = 0; n < p->nf; ++n) {
    int cL = p->fL[n], cR = p->fR[n];
    double dpL, dpR;
    face_dps(p, n, &dpL, &dpR);
    for (q = 0; q < p->NQ; ++q) {
      double WL = p->prim[q][cL] + dpL * p->gradp[q][cL];
      double WR = p->prim[q][cR] - dpR * p->gradp[q][cR];
      double S = (WR - WL) / (p->fdr[n] + p->fdl[n]);
      double SL = p->grad[q][cL], SR = p->grad[q][cR];
      if (S * SL < 0.0) p->grad[q][cL] = 0.0;
      else if (fabs(p->PLM * S) < fabs(SL)) p->grad[q][cL] = p->PLM * S;
      if (S * SR < 0.0) p->grad[q][cR] = 0.0;
      else if (fabs(p->PLM * S) < fabs(SR)) p->grad[q][cR] = p->PLM * S;
    }
  }
}

/* ---------------- Riemann (src/Riemann/Riemann_routines.c) ---------------- */
typedef struct {
  int cL, cR, n[3];
  double r, r_cell_L, r_cell_R, dA, cm;
  double primL[PORT_MAXQ], primR[PORT_MAXQ], UL[PORT_MAXQ], UR[PORT_MAXQ], Ustar[PORT_MAXQ], FL[PORT_MAXQ],
      FR[PORT_MAXQ], Fstar[PORT_MAXQ], F[PORT_MAXQ], Fvisc[PORT_MAXQ];
  double Sl, Sr, Ss;
  int state;
} Rm;

static void LR_speed(const double *prim, double r, const int *n, double G, double *vn, double *cf2) {
  double P = prim[PPP], rho = prim[RHO], vr = prim[URR], vp = r * prim[UPP], vz = prim[UZZ];
  *vn = vr * n[0] + vp * n[1] + vz * n[2];
  *cf2 = G * (P / rho);
}
static void set_flux(const Port *p, Rm *R, int side) {
  double r = R->r, G = p->Adiabatic_Index;
  double *prim = side == LEFT ? R->primL : R->primR, *F = side == LEFT ? R->FL : R->FR;
  double rho = prim[RHO], Pp = prim[PPP], vr = prim[URR], vp = prim[UPP] * r, vz = prim[UZZ];
  double vn = vr * R->n[0] + vp * R->n[1] + vz * R->n[2];
  double rhoe = Pp / (G - 1.), v2 = vr * vr + vp * vp + vz * vz;
  F[DDD] = rho * vn;
  F[SRR] = rho * vr * vn + Pp * R->n[0];
  F[LLL] = r * (rho * vp * vn + Pp * R->n[1]);
  F[SZZ] = rho * vz * vn + Pp * R->n[2];
  F[TAU] = (.5 * rho * v2 + rhoe + Pp) * vn;
  for (int q = 5; q < p->NQ; ++q) F[q] = prim[q] * F[DDD]; /* passive scalars */
}
static void star_hllc(const Port *p, Rm *R) {
  double r = R->r, G = p->Adiabatic_Index;
  double *prim, Sk, *Uk, *Fk;
  int q;
  if (R->state == LEFTSTAR) { prim = R->primL; Sk = R->Sl; Uk = R->UL; Fk = R->FL; }
  else { prim = R->primR; Sk = R->Sr; Uk = R->UR; Fk = R->FR; }
  {
    double Ss = R->Ss, rho = prim[RHO], vr = prim[URR], vp = prim[UPP] * r, vz = prim[UZZ], Pp = prim[PPP];
    double v2 = vr * vr + vp * vp + vz * vz;
    double vn = vr * R->n[0] + vp * R->n[1] + vz * R->n[2];
    double rhoe = Pp / (G - 1.);
    double D = rho, mr = rho * vr, mp = rho * vp, mz = rho * vz;
    double E_hydro = .5 * rho * v2 + rhoe;
    double Ps = rho * (Sk - vn) * (Ss - vn) + Pp;
    double Dstar = (Sk - vn) * D / (Sk - Ss);
    double Msn = Dstar * Ss;
    double Msr = (Sk - vn) * mr / (Sk - Ss);
    double Msp = (Sk - vn) * mp / (Sk - Ss);
    double Msz = (Sk - vn) * mz / (Sk - Ss);
    double Estar = ((Sk - vn) * E_hydro + Ps * Ss - Pp * vn) / (Sk - Ss);
    double mn = Msr * R->n[0] + Msp * R->n[1] + Msz * R->n[2];
    Msr += R->n[0] * (Msn - mn);
    Msp += R->n[1] * (Msn - mn);
    Msz += R->n[2] * (Msn - mn);
    R->Ustar[DDD] = Dstar; R->Ustar[SRR] = Msr; R->Ustar[LLL] = r * Msp; R->Ustar[SZZ] = Msz;
    R->Ustar[TAU] = Estar;
  }
  for (q = 5; q < p->NQ; ++q) R->Ustar[q] = prim[q] * R->Ustar[DDD];
  for (q = 0; q < p->NQ; ++q) R->Fstar[q] = Fk[q] + Sk * (R->Ustar[q] - Uk[q]);
}

static void visc_flux(const Port *p, Rm *R) {
  double r = R->r, tiph = R->cm, M0 = p->gM[0], M1 = p->gM[1], a = p->gr[0] + p->gr[1];
  double d0 = gm_dist(p, 0, r, tiph), d1 = gm_dist(p, 1, r, tiph);
  double Avg[5], Gr[5], Gp[5], nu, alpha = p->Explicit_Viscosity;
  int q, cL = R->cL, cR = R->cR;
  for (q = 0; q < 5; ++q) {
    Avg[q] = .5 * (R->primL[q] + R->primR[q]);
    Gp[q] = .5 * (p->gradp[q][cL] + p->gradp[q][cR]) / r;
    Gr[q] = .5 * (p->grad[q][cL] + p->grad[q][cR]);
    if (R->n[0] == 1) {
      double pL = p->tiph[cL] - .5 * p->dphi[cL], pR = p->tiph[cR] - .5 * p->dphi[cR];
      double dpL = R->cm - pL, dpR = -R->cm + pR;
      double WL, WR, deltaL, deltaR;
      while (dpL > PHIMAX / 2.) dpL -= PHIMAX;
      while (dpL < -PHIMAX / 2.) dpL += PHIMAX;
      while (dpR > PHIMAX / 2.) dpR -= PHIMAX;
      while (dpR < -PHIMAX / 2.) dpR += PHIMAX;
      WL = p->prim[q][cL] + dpL * p->gradp[q][cL];
      WR = p->prim[q][cR] - dpR * p->gradp[q][cR];
      deltaL = R->r - R->r_cell_L;
      deltaR = R->r_cell_R - R->r;
      Avg[q] = 0.5 * (WL + WR);
      Gr[q] = (WR - WL) / (deltaR + deltaL);
    }
    if (R->n[1] == 1) {
      Avg[q] = 0.5 * (p->prim[q][cR] + p->prim[q][cL]);
      Gp[q] = (p->prim[q][cR] - p->prim[q][cL]) / (p->tiph[cR] - p->tiph[cL]) / r;
    }
  }
  if (p->ViscConst == 1) {
    nu = alpha;
  } else {
    double eps = p->G_EPS;
    nu = alpha * Avg[PPP] / Avg[RHO] / sqrt(pow(d0 * d0 + eps * eps, -1.5) * M0 + pow(d1 * d1 + eps * eps, -1.5) * M1);
  }
  {
    double rho = Avg[RHO], vr = Avg[URR], om = Avg[UPP], vz = Avg[UZZ];
    double Gr_vr = Gr[URR], Gr_om = Gr[UPP], Gp_vr = Gp[URR], Gp_om = Gp[UPP];
    double rdr = rdrOm_a(p, r, a);
    if (fabs(vz) > 1.e-12) {
      fprintf(stderr, "port: viscosity with nonzero v_z\n");
      exit(5);
    }
    for (q = 0; q < 5; ++q) R->Fvisc[q] = 0.0;
    if (R->n[0] == 1) {
      R->Fvisc[SRR] = -nu * rho * (r * Gr_vr - vr - r * r * Gp_om);
      R->Fvisc[LLL] = -nu * rho * (r * (r * Gr_om + rdr) + r * Gp_vr);
      R->Fvisc[TAU] = -nu * rho * (vr * (Gr_vr - vr / r - r * Gp_om) + r * om * (Gp_vr + (rdr + r * Gr_om)));
    }
    if (R->n[1] == 1) {
      R->Fvisc[SRR] = -nu * rho * (r * (r * Gr_om + rdr) + r * Gp_vr);
      R->Fvisc[LLL] = -nu * rho * (-r * Gr_vr + vr + r * r * Gp_om);
      R->Fvisc[TAU] = -nu * rho * (-r * om * (Gr_vr - vr / r - r * Gp_om) + vr * (Gp_vr + (rdr + r * Gr_om)));
    }
  }
}

/* riemann_AddFlux (Riemann_routines.c:314-397) */
static void add_flux(Port *p, Rm *R, double dt) {
  double G = p->Adiabatic_Index, w, vnL, cf2L, vnR, cf2R;
  int q;
  LR_speed(R->primL, R->r, R->n, G, &vnL, &cf2L);
  R->Sl = vnL - sqrt(cf2L);
  R->Sr = vnL + sqrt(cf2L);
  LR_speed(R->primR, R->r, R->n, G, &vnR, &cf2R);
  if (R->Sl > vnR - sqrt(cf2R)) R->Sl = vnR - sqrt(cf2R);
  if (R->Sr < vnR + sqrt(cf2R)) R->Sr = vnR + sqrt(cf2R);
  R->Ss = (R->primR[RHO] * vnR * (R->Sr - vnR) - R->primL[RHO] * vnL * (R->Sl - vnL) + R->primL[PPP] - R->primR[PPP]) /
          (R->primR[RHO] * (R->Sr - vnR) - R->primL[RHO] * (R->Sl - vnL));
  w = R->n[1] ? p->wiph[R->cL] : 0.0;
  if (w < R->Sl) R->state = LEFT;
  else if (w > R->Sr) R->state = RIGHT;
  else if (w < R->Ss) R->state = LEFTSTAR;
  else R->state = RIGHTSTAR;
  if (R->state == LEFT) {
    set_flux(p, R, LEFT);
    prim2cons(p, R->primL, R->UL, R->r, 1.0);
    for (q = 0; q < p->NQ; ++q) R->F[q] = R->FL[q] - w * R->UL[q];
  } else if (R->state == RIGHT) {
    set_flux(p, R, RIGHT);
    prim2cons(p, R->primR, R->UR, R->r, 1.0);
    for (q = 0; q < p->NQ; ++q) R->F[q] = R->FR[q] - w * R->UR[q];
  } else {
    if (p->RiemannSolver == HLL) {
      set_flux(p, R, LEFT);
      set_flux(p, R, RIGHT);
      prim2cons(p, R->primL, R->UL, R->r, 1.0);
      prim2cons(p, R->primR, R->UR, R->r, 1.0);
      for (q = 0; q < p->NQ; ++q) {
        R->Ustar[q] = (R->Sr * R->UR[q] - R->Sl * R->UL[q] + R->FL[q] - R->FR[q]) / (R->Sr - R->Sl);
        R->Fstar[q] = (R->Sr * R->FL[q] - R->Sl * R->FR[q] - R->Sr * R->Sl * (R->UL[q] - R->UR[q])) / (R->Sr - R->Sl);
      }
    } else if (R->state == LEFTSTAR) {
      set_flux(p, R, LEFT);
      prim2cons(p, R->primL, R->UL, R->r, 1.0);
      star_hllc(p, R);
    } else {
      set_flux(p, R, RIGHT);
      prim2cons(p, R->primR, R->UR, R->r, 1.0);
      star_hllc(p, R);
    }
    for (q = 0; q < p->NQ; ++q) R->F[q] = R->Fstar[q] - w * R->Ustar[q];
  }
  if (p->Explicit_Viscosity > 0.0) visc_flux(p, R);
  for (q = 0; q < p->NQ; ++q) {
    p->cons[q][R->cL] += -dt * R->dA * R->F[q];
    p->cons[q][R->cR] += dt * R->dA * R->F[q];
  }
  if (p->Explicit_Viscosity > 0.) {
    p->cons[SRR][R->cL] += -dt * R->dA * R->Fvisc[SRR] / R->r_cell_L;
    p->cons[SRR][R->cR] += dt * R->dA * R->Fvisc[SRR] / R->r_cell_R;
    p->cons[LLL][R->cL] += -dt * R->dA * R->Fvisc[LLL];
    p->cons[LLL][R->cR] += dt * R->dA * R->Fvisc[LLL];
    p->cons[TAU][R->cL] += -dt * R->dA * R->Fvisc[TAU];
    p->cons[TAU][R->cR] += +dt * R->dA * R->Fvisc[TAU];
  }
}

static void phi_fluxes(Port *p, double dt) {
  double dz = p->zf[1] - p->zf[0];
  int i, j, q;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i), dr = rp - rm, r = .5 * (rp + rm);
    int a = p->off[i], n = p->N_p[i];
    for (j = 0; j < n; ++j) {
      Rm R;
      memset(&R, 0, sizeof(R));
      R.n[1] = 1;
      R.cL = a + j;
      R.cR = a + (j == n - 1 ? 0 : j + 1);
      R.dA = dr * dz;
      R.r = r;
      R.cm = p->tiph[R.cL];
      R.r_cell_L = r;
      R.r_cell_R = r;
      for (q = 0; q < p->NQ; ++q) {
        R.primL[q] = p->prim[q][R.cL] + 0.5 * p->gradp[q][R.cL] * p->dphi[R.cL];
        R.primR[q] = p->prim[q][R.cR] - 0.5 * p->gradp[q][R.cR] * p->dphi[R.cR];
      }
      add_flux(p, &R, dt);
    }
  }
}

static void r_fluxes(Port *p, double dt) {
  int n, q;
  for (n = 0; n < p->nf; ++n) {
    Rm R;
    double dpL, dpR;
    memset(&R, 0, sizeof(R));
    R.n[0] = 1;
    R.cL = p->fL[n];
    R.cR = p->fR[n];
    {
      double pL = p->tiph[R.cL] - .5 * p->dphi[R.cL], pR = p->tiph[R.cR] - .5 * p->dphi[R.cR];
      dpL = p->fcm[n] - pL;
      dpR = -p->fcm[n] + pR;
      while (dpL > PHIMAX / 2.) dpL -= PHIMAX;
      while (dpL < -PHIMAX / 2.) dpL += PHIMAX;
      while (dpR > PHIMAX / 2.) dpR -= PHIMAX;
      while (dpR < -PHIMAX / 2.) dpR += PHIMAX;
    }
    R.r = p->fr[n];
    R.dA = p->fdA[n];
    R.cm = p->fcm[n];
    R.r_cell_L = R.r - p->fdl[n];
    R.r_cell_R = R.r + p->fdr[n];
    for (q = 0; q < p->NQ; ++q) {
      R.primL[q] = p->prim[q][R.cL] + p->grad[q][R.cL] * p->fdl[n] + p->gradp[q][R.cL] * dpL;
      R.primR[q] = p->prim[q][R.cR] - p->grad[q][R.cR] * p->fdr[n] - p->gradp[q][R.cR] * dpR;
    }
    add_flux(p, &R, dt);
  }
}

/* ---------------- sources (src/Cell/cell_source.c, cell_add_split_fictitious.c) ---------------- */
static double fgrav(double M, double r, double eps, int n) {
  return (M * pow(r, n - 1.) / pow(pow(r, n) + pow(eps, n), 1. + 1. / n));
}

static void add_src(Port *p, double dt) {
  double dz = p->zf[1] - p->zf[0];
  double a = p->gr[0] + p->gr[1];
  double xbh0 = p->gr[0] * cos(p->gphi[0]), ybh0 = p->gr[0] * sin(p->gphi[0]);
  double xbh1 = p->gr[1] * cos(p->gphi[1]), ybh1 = p->gr[1] * sin(p->gphi[1]);
  double Md[2] = {0.0, 0.0};
  int imin = p->ng_min == 1 ? 0 : p->ng_min, imax = p->NR - p->ng_max;
  int i, j, k;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double phi = p->tiph[g] - .5 * p->dphi[g], dphi = p->dphi[g];
      double rho = p->prim[RHO][g], Pp = p->prim[PPP][g], r = .5 * (rp + rm);
      double vr = p->prim[URR][g], vz = p->prim[UZZ][g], vp = p->prim[UPP][g] * r;
      double dV = dphi * .5 * (rp * rp - rm * rm) * dz;
      double xpos = r * cos(phi), ypos = r * sin(phi);
      double r0 = sqrt((xpos - xbh0) * (xpos - xbh0) + (ypos - ybh0) * (ypos - ybh0));
      double r1 = sqrt((xpos - xbh1) * (xpos - xbh1) + (ypos - ybh1) * (ypos - ybh1));
      double z = .5 * (p->zf[1] + p->zf[0]), R = sqrt(r * r + z * z);
      double sint, cost, gravdist, Fr = 0.0, Fp = 0.0;
      double w_a, rdr, F_cent, dtOm, F_euler;
      if (p->Grav_2D == 1) { sint = 1.0; cost = 0.0; gravdist = r; }
      else { sint = r / R; cost = z / R; gravdist = R; }
      for (k = 0; k < 2; ++k) { /* gravMassForce (cell_source.c:49-71) */
        double cosp = cos(phi), sinp = sin(phi);
        double dx = gravdist * cosp - p->gr[k] * cos(p->gphi[k]);
        double dy = gravdist * sinp - p->gr[k] * sin(p->gphi[k]);
        double script_r = sqrt(dx * dx + dy * dy);
        double cosa = dx / script_r, sina = dy / script_r;
        double cosap = cosa * cosp + sina * sinp, sinap = sina * cosp - cosa * sinp;
        double f1 = -fgrav(p->gM[k], script_r, p->G_EPS, p->PHI_ORDER);
        Fr += cosap * f1;
        Fp += sinap * f1;
      }
      w_a = rOm_a(p, r, a);
      rdr = rdrOm_a(p, r, a);
      F_cent = w_a * w_a / r;
      dtOm = dtOm_a(p, r, a);
      F_euler = -(r * dtOm + vr * rdr);
      p->cons[SRR][g] += dt * dV * (rho * vp * vp + Pp) / r;
      p->cons[SRR][g] += dt * dV * rho * (Fr * sint + F_cent);
      p->cons[LLL][g] += dt * dV * rho * (Fp - r * dtOm) * r;
      p->cons[SZZ][g] += dt * dV * rho * Fr * cost;
      p->cons[TAU][g] += dt * dV * rho * ((Fr * sint + F_cent) * vr + Fr * vz * cost + (Fp + F_euler) * vp);
      if (p->RhoSinkOn == 1) { /* get_rho_sink (cell_source.c:15-47) */
        double M0 = p->gM[0], M1 = p->gM[1], Mt = M0 + M1, al = p->Explicit_Viscosity;
        double one_o_nu = 1.0 / (al * Pp / rho) * sqrt(pow(r0, -3) * M0 / Mt + pow(r1, -3) * M1 / Mt);
        double tv0 = TVISC_FAC * 2. / 3. * r0 * r0 * one_o_nu, tv1 = TVISC_FAC * 2. / 3. * r1 * r1 * one_o_nu;
        if (tv0 < 10. * dt) tv0 = 10. * dt;
        if (tv1 < 10. * dt) tv1 = 10. * dt;
        for (k = 0; k < p->GravMassType; ++k) {
          double dr = 0.0;
          if (k == 0) { if (r0 < 0.5) dr = rho / tv0; }
          else { if (r1 < 0.5) dr = rho / tv1; }
          p->cons[DDD][g] -= dr * dt * dV;
          if (i >= imin && i < imax) Md[k] += dr * dV;
        }
      }
      if (p->Cooling == 1 && p->InitialDataType == SHEAR) { /* cell_source.c:189-193 */
        double ct = (Pp - .01) / (p->Adiabatic_Index - 1.) * dV / 1.e-2;
        if (ct < 0.0) ct = 0.0;
        p->cons[TAU][g] -= ct * dt;
      } else if (p->Cooling == 1) { /* cell_source.c:195-201 */
        double cap = p->cons[TAU][g] * 1.0;
        double ct = 9. / 4. * p->Explicit_Viscosity * pow(p->PoRho_r1, -3) / rho * pow(Pp / rho, 4.) * dt * dV;
        if (ct > cap) ct = cap;
        p->cons[TAU][g] -= ct;
      }
    }
  }
  p->mdot[0] = Md[0];
  p->mdot[1] = Md[1];
}

static void add_visc_src(Port *p, double dt) {
  double dz = p->zf[1] - p->zf[0], a = p->gr[0] + p->gr[1];
  double xbh0 = p->gr[0] * cos(p->gphi[0]), ybh0 = p->gr[0] * sin(p->gphi[0]);
  double xbh1 = p->gr[1] * cos(p->gphi[1]), ybh1 = p->gr[1] * sin(p->gphi[1]);
  int i, j;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double dphi = p->dphi[g], rho = p->prim[RHO][g], P = p->prim[PPP][g], r = .5 * (rp + rm);
      double dV = dphi * .5 * (rp * rp - rm * rm) * dz;
      double phi = p->tiph[g] - 0.5 * p->dphi[g];
      double xpos = r * cos(phi), ypos = r * sin(phi);
      double d0 = sqrt((xpos - xbh0) * (xpos - xbh0) + (ypos - ybh0) * (ypos - ybh0));
      double d1 = sqrt((xpos - xbh1) * (xpos - xbh1) + (ypos - ybh1) * (ypos - ybh1));
      double alpha = p->Explicit_Viscosity, rdr = rdrOm_a(p, r, a), eps = p->G_EPS, Sn;
      if (p->ViscConst == 1) Sn = rho * alpha;
      else Sn = alpha * P / sqrt(pow(d0 * d0 + eps * eps, -1.5) * p->gM[0] + pow(d1 * d1 + eps * eps, -1.5) * p->gM[1]);
      p->cons[TAU][g] += dt * dV * Sn * rdr * (rdr + r * p->grad[UPP][g] + p->gradp[URR][g]);
    }
  }
}

static void split_fictitious(Port *p, double dt) {
  double a = p->gr[0] + p->gr[1];
  int i, j;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i), r = 0.5 * (rm + rp);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double Omega = rOm_a(p, r, a) / r;
      double dr_r2Om = 2. * rOm_a(p, r, a) + r * rdrOm_a(p, r, a);
      double kappa2 = 2. * Omega / r * dr_r2Om;
      if (kappa2 > 0.) {
        double kappa = sqrt(kappa2), l0 = p->cons[LLL][g], rhov0 = p->cons[SRR][g];
        double l = l0 * cos(kappa * dt) - p->cons[SRR][g] * dr_r2Om / kappa * sin(kappa * dt);
        double rhov = rhov0 * cos(kappa * dt) + 2.0 * Omega * p->cons[LLL][g] / r / kappa * sin(kappa * dt);
        p->cons[LLL][g] = l;
        p->cons[SRR][g] = rhov;
      }
    }
  }
}

static void update_phi(Port *p, double RK, double dt) {
  double a = p->gr[0] + p->gr[1];
  int i, j;
  for (i = 0; i < p->NR; ++i) {
    double rm = FP(p, i - 1), rp = FP(p, i), r = .5 * (rm + rp);
    for (j = 0; j < p->N_p[i]; ++j) {
      int g = p->off[i] + j;
      double w_total;
      while (p->tiph[g] - p->rktiph[g] > PHIMAX / 2.) p->rktiph[g] += PHIMAX;
      while (p->tiph[g] - p->rktiph[g] < -PHIMAX / 2.) p->rktiph[g] -= PHIMAX;
      p->tiph[g] = (1.0 - RK) * p->tiph[g] + RK * p->rktiph[g];
      w_total = p->wiph[g] + rOm_a(p, r, a);
      p->tiph[g] += w_total * dt / r;
    }
  }
}

static void update_dphi(Port *p) {
  int i, j;
  for (i = 0; i < p->NR; ++i) {
    int a = p->off[i], n = p->N_p[i];
    for (j = 0; j < n; ++j) {
      int jm = j == 0 ? n - 1 : j - 1;
      double dphi = p->tiph[a + j] - p->tiph[a + jm];
      while (dphi > PHIMAX) dphi -= PHIMAX;
      while (dphi < 0.0) dphi += PHIMAX;
      p->dphi[a + j] = dphi;
    }
  }
}

static void gm_update_RK(Port *p, double RK) {
  int k;
  for (k = 0; k < 2; ++k) {
    while (p->gphi[k] - p->grk_phi[k] > M_PI) p->grk_phi[k] += 2. * M_PI;
    while (p->gphi[k] - p->grk_phi[k] < -M_PI) p->grk_phi[k] -= 2. * M_PI;
    p->gr[k] = (1.0 - RK) * p->gr[k] + RK * p->grk_r[k];
    p->gphi[k] = (1.0 - RK) * p->gphi[k] + RK * p->grk_phi[k];
    p->gM[k] = (1.0 - RK) * p->gM[k] + RK * p->grk_M[k];
    p->gom[k] = (1.0 - RK) * p->gom[k] + RK * p->grk_om[k];
  }
}

static void gm_move(Port *p, double t, double dt) { /* gravMass_move (GravMass_misc.c:31-64) */
  double m0 = p->gM[0], m1 = p->gM[1], M = m0 + m1, a_0 = 1.0;
  double tau_0 = p->OrbShrinkTscale, T0 = p->OrbShrinkT0, a, omega, r0, r1;
  if ((t - T0) / tau_0 < 1.) {
    a = a_0 * pow((1.0 - (t - T0) / tau_0), 0.25);
    omega = pow(a / M, -1.5);
  } else {
    a = 0.0;
    omega = 0.0;
  }
  if (M < 1.e-12) { r0 = 0.0; r1 = 0.0; }
  else { r0 = m1 / M * a; r1 = m0 / M * a; }
  p->gphi[0] += omega * dt;
  p->gphi[1] += omega * dt;
  p->gr[0] = r0;
  p->gr[1] = r1;
  p->gom[0] = omega;
  p->gom[1] = omega;
}

/* cell_boundary_outflow_r (cell_boundary.c:14-139) with the reference's build
 * constants EXTRAP_BC = SS_BCS = diode = KEP_BNDRY = 0 (header.h): a boundary
 * cell takes the dA-weighted sum of its neighbours' prims over the r faces of
 * the substep's face list, divided by dz * r_face * dphi.  The extrapolation
 * term 0 * grad * (...) / 2 is +-0 for a finite slope, and x - (+-0) == x, so
 * the inner sum is prim * dA like the outer one.  The inner ghost annulus 0
 * (unless NoInnerBC == 1) comes from annulus 1; then annulus NR-2 from NR-3,
 * then NR-1 from the new NR-2 -- also when NR-2 is not a ghost annulus. */
static void outflow_pair(Port *p, int i, int outer) {
  int n, q, j;
  const int dst = outer ? i + 1 : i;
  const double dz = p->zf[1] - p->zf[0];
  for (n = p->nri[i]; n < p->nri[i + 1]; ++n)
    for (q = 0; q < p->NQ; ++q) p->prim[q][outer ? p->fR[n] : p->fL[n]] = 0.0;
  for (n = p->nri[i]; n < p->nri[i + 1]; ++n) {
    const int to = outer ? p->fR[n] : p->fL[n], from = outer ? p->fL[n] : p->fR[n];
    for (q = 0; q < p->NQ; ++q) p->prim[q][to] += p->prim[q][from] * p->fdA[n];
  }
  for (j = 0; j < p->N_p[dst]; ++j) {
    const int g = p->off[dst] + j;
    const double dA = dz * FP(p, i) * p->dphi[g];
    for (q = 0; q < p->NQ; ++q) p->prim[q][g] /= dA;
  }
}

static void boundary_and_damp(Port *p, double dt) {
  int i, j, q;
  if (p->BoundTypeR == 1) {
    if (p->NoInnerBC != 1) outflow_pair(p, 0, 0);
    outflow_pair(p, p->NR - 3, 1);
    outflow_pair(p, p->NR - 2, 1);
  }
  /* cell_boundary_fixed_r (cell_boundary.c:208-231) */
  if (p->BoundTypeR == 0) {
    for (i = 0; i < p->NR; ++i) {
      double prof[5];
      if (!((p->NoInnerBC != 1 && i < p->ng_min) || i > p->NR - p->ng_max - 1)) continue;
      if (single_init(p, i, prof) != 1) continue;
      for (j = 0; j < p->N_p[i]; ++j) {
        int g = p->off[i] + j;
        for (q = 0; q < 5; ++q) p->prim[q][g] = prof[q];
        /* cell_single_init_vortex's dye at the cell's current phi */
        if (p->InitialDataType == VORTEX && p->NQ > 5)
          p->prim[5][g] = cos(p->tiph[g] - .5 * p->dphi[g]) < 0.0 ? 0.0 : 1.0;
      }
    }
  }
  /* cell_bc_damp (cell_misc.c:98-132) */
  if (p->DAMP_TIME > 0.0) {
    double RMIN = p->R_Min, RMAX = p->R_Max, R0 = 1. / p->DAMP_TIME / 2. / M_PI;
    for (i = 0; i < p->NR; ++i) {
      double rp = FP(p, i), rm = FP(p, i - 1), r = .5 * (rp + rm);
      if (r < p->RDAMP_INNER || r > p->RDAMP_OUTER) {
        double rate = R0 * (r - p->RDAMP_INNER) / (RMIN - p->RDAMP_INNER), prof[5];
        if (r > p->RDAMP_OUTER) rate = R0 * (r - p->RDAMP_OUTER) / (RMAX - p->RDAMP_OUTER);
        if (single_init(p, i, prof) != 1) continue;
        for (j = 0; j < p->N_p[i]; ++j)
          for (q = 0; q < 5; ++q) {
            int g = p->off[i] + j;
            double dprim = prof[q] - p->prim[q][g];
            p->prim[q][g] += (1. - exp(-rate * dt)) * dprim;
          }
      }
    }
  }
}

/* ---------------- step (src/TimeStep/timestep_routines.c:16-113, timestep_algorithm.c:11-41) ---------------- */
void port_substep(Port *p, double fac, int stop) {
  double dt = fac * p->dt;
  int g, q, k;
  ULP_NOISE_START();
  port_build_faces(p);
  clean_pi(p);
  for (k = 0; k < 2; ++k) {
    while (p->gphi[k] > 2. * M_PI) p->gphi[k] -= 2. * M_PI;
    while (p->gphi[k] < 0.0) p->gphi[k] += 2. * M_PI;
  }
  set_w(p);
  for (g = 0; g < p->N; ++g)
    for (q = 0; q < p->NQ; ++q) p->cons[q][g] = (1.0 - p->RK) * p->cons[q][g] + p->RK * p->rkcons[q][g];
  if (stop == 0) return;
  plm_p(p);
  plm_rz(p);
  if (stop == 1) return;
  phi_fluxes(p, dt);
  if (stop == 2) return;
  r_fluxes(p, dt);
  if (stop == 3) return;
  add_src(p, dt);
  if (p->Explicit_Viscosity > 0.0) add_visc_src(p, dt);
  split_fictitious(p, dt);
  if (stop == 4) return;
  update_phi(p, p->RK, dt);
  update_dphi(p);
  gm_update_RK(p, p->RK);
  calc_prim(p);
  if (stop == 5) return;
  boundary_and_damp(p, dt);
  if (stop == 6) return;
  port_calc_cons(p);
}

void port_prologue(Port *p) {
  int g, q, k;
  for (g = 0; g < p->N; ++g) p->wiph[g] = 0.0;
  set_w(p);
  set_dt(p);
  for (g = 0; g < p->N; ++g) {
    for (q = 0; q < p->NQ; ++q) p->rkcons[q][g] = p->cons[q][g];
    p->rktiph[g] = p->tiph[g];
  }
  for (k = 0; k < 2; ++k) {
    p->grk_r[k] = p->gr[k];
    p->grk_phi[k] = p->gphi[k];
    p->grk_M[k] = p->gM[k];
    p->grk_om[k] = p->gom[k];
  }
  p->RK = 0.0;
}

void port_stage(Port *p, int phase) {
  port_prologue(p);
  if (phase >= 8) {
    port_substep(p, 1.0, 7);
    gm_move(p, p->t, 1.0 * p->dt);
    p->RK = 0.5;
    port_substep(p, 0.5, phase - 8);
  } else {
    port_substep(p, 1.0, phase);
  }
}

void port_step_rk2(Port *p) {
  int k;
  port_prologue(p);
  port_substep(p, 1.0, 7);
  gm_move(p, p->t, 1.0 * p->dt);
  p->RK = 0.5;
  port_substep(p, 0.5, 7);
  gm_move(p, p->t, 0.5 * p->dt);
  p->t += p->dt;
  for (k = 0; k < 2; ++k) p->macc[k] = p->macc[k] + p->mdot[k] * p->dt;
}
