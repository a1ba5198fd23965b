// Dot-product checks of the hand-written adjoints of the per-face and per-cell
// physics against the Dual tangent of the same templated forward code, on the
// host (nvcc compiles the __host__ __device__ functions for the CPU).
//
// For each function f and random inputs x, tangent direction v and output
// weights l:   <l, J v>  (Dual forward)  ==  <J^T l, v>  (reverse).
// Prints one line per function: name, trials, branch counts, max relative
// mismatch.  Exit status 1 if any mismatch exceeds the tolerance.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../disco2_b200/csrc/dgpu_adjoint.cuh"

static unsigned long long rng_state = 0x9e3779b97f4a7c15ull;
static double urand() {  // splitmix64 -> [0, 1)
  unsigned long long z = (rng_state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
static double urange(double a, double b) { return a + (b - a) * urand(); }

static double worst = 0.0;
static int failed = 0;
static void report(const char *name, int n, double maxrel, const char *extra) {
  printf("%-16s trials=%d max_rel=%.3e %s\n", name, n, maxrel, extra);
  if (maxrel > 1e-10) failed = 1;
  if (maxrel > worst) worst = maxrel;
}
static double rel(double a, double b, double scale) {
  double d = fabs(a - b);
  double s = fabs(a) + fabs(b) + scale;
  return d / s;
}

static DiskParams base_params() {
  DiskParams P;
  memset(&P, 0, sizeof(P));
  P.gamma = 5.0 / 3.0;
  P.plm = 1.5;
  P.visc = 0.1;
  P.g_eps = 0.05;
  P.phi_order = 2;
  P.has_visc = 1;
  P.visc_const = 0;
  P.init_type = DI_CIRCUMBINARY;
  P.rho_floor = 1e-8;
  P.cs_floor = 1e-6;
  P.cs_cap = 10.0;
  P.vel_cap = 10.0;
  P.grav2d = 1;
  P.dz = 2.0;
  return P;
}

static void rand_prim(double *p) {
  p[D_RHO] = urange(0.3, 2.0);
  p[D_PPP] = urange(0.3, 2.0);
  p[D_URR] = urange(-1.0, 1.0);
  p[D_UPP] = urange(-1.0, 1.0);
  p[D_UZZ] = 0.0;
}

static void check_riemann() {
  int counts[4] = {0, 0, 0, 0};
  double mx = 0.0;
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    double pL[5], pR[5], vL[5], vR[5], aF[5];
    rand_prim(pL);
    rand_prim(pR);
    for (int q = 0; q < 5; ++q) {
      vL[q] = urange(-1, 1);
      vR[q] = urange(-1, 1);
      aF[q] = urange(-1, 1);
    }
    const double r = urange(0.5, 2.0), w = urange(-4.0, 4.0), gam = 5.0 / 3.0;
    const int dir = t & 1, solver = (t >> 1) & 1 ? DR_HLL : DR_HLLC;
    Dual dL[5], dR[5], F[5];
    for (int q = 0; q < 5; ++q) {
      dL[q] = Dual(pL[q], vL[q]);
      dR[q] = Dual(pR[q], vR[q]);
    }
    riemann_flux(dL, dR, r, dir, w, gam, solver, F);
    double lhs = 0.0, scale = 0.0;
    for (int q = 0; q < 5; ++q) {
      lhs += aF[q] * F[q].d;
      scale += fabs(aF[q] * F[q].d);
    }
    double aL[5] = {0}, aR[5] = {0};
    riemann_flux_rev(pL, pR, r, dir, w, gam, solver, aF, aL, aR);
    double rhs = 0.0;
    for (int q = 0; q < 5; ++q) rhs += aL[q] * vL[q] + aR[q] * vR[q];
    // state of this trial (same selection as the forward)
    {
      double fl[5];
      riemann_flux(pL, pR, r, dir, w, gam, solver, fl);
      const double n0 = dir == 0 ? 1.0 : 0.0, n1 = dir == 1 ? 1.0 : 0.0;
      double vnL = pL[D_URR] * n0 + r * pL[D_UPP] * n1, vnR = pR[D_URR] * n0 + r * pR[D_UPP] * n1;
      double cL = sqrt(gam * (pL[D_PPP] / pL[D_RHO])), cR = sqrt(gam * (pR[D_PPP] / pR[D_RHO]));
      double Sl = fmin(vnL - cL, vnR - cR), Sr = fmax(vnL + cL, vnR + cR);
      counts[w < Sl ? 0 : (w > Sr ? 3 : 1)]++;
    }
    double e = rel(lhs, rhs, 1e-12 * scale + 1e-300);
    if (e > mx) mx = e;
  }
  char buf[128];
  snprintf(buf, sizeof(buf), "(left %d, star %d, right %d)", counts[0], counts[1], counts[3]);
  report("riemann_flux", n, mx, buf);
}

static void check_visc() {
  double mx = 0.0;
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    DiskParams P = base_params();
    P.visc_const = (t % 3 == 0) ? 1 : 0;
    const int dir = (t >> 1) & 1;
    ViscIn<double> v;
    ViscIn<Dual> vd;
    double tc[6][5];
    double *dst[6] = {v.cL, v.cR, v.gpL, v.gpR, v.grL, v.grR};
    Dual *dd[6] = {vd.cL, vd.cR, vd.gpL, vd.gpR, vd.grL, vd.grR};
    for (int k = 0; k < 6; ++k) {
      if (k < 2) rand_prim(dst[k]);
      else
        for (int q = 0; q < 5; ++q) dst[k][q] = urange(-1, 1);
      dst[k][D_UZZ] = 0.0;
      for (int q = 0; q < 5; ++q) {
        tc[k][q] = urange(-1, 1);
        dd[k][q] = Dual(dst[k][q], tc[k][q]);
      }
    }
    v.r = vd.r = urange(0.5, 3.0);
    v.tL = vd.tL = urange(0, 6);
    v.tR = vd.tR = v.tL + urange(0.01, 0.2);
    v.dpL = vd.dpL = urange(-0.1, 0.1);
    v.dpR = vd.dpR = urange(-0.1, 0.1);
    v.cm = vd.cm = urange(0, 6.28);
    v.r_cell_L = vd.r_cell_L = v.r - urange(0.01, 0.1);
    v.r_cell_R = vd.r_cell_R = v.r + urange(0.01, 0.1);
    v.rdr_om = vd.rdr_om = urange(-1, 1);
    GravT<double> G;
    GravT<Dual> GD;
    double tg[7];
    for (int p = 0; p < 2; ++p) {
      G.gx[p] = urange(-0.6, 0.6);
      G.gy[p] = urange(-0.6, 0.6);
      G.gM[p] = urange(0.1, 0.9);
    }
    G.alpha = urange(0.01, 0.1);
    for (int k = 0; k < 7; ++k) tg[k] = urange(-1, 1);
    for (int p = 0; p < 2; ++p) {
      GD.gx[p] = Dual(G.gx[p], tg[p]);
      GD.gy[p] = Dual(G.gy[p], tg[2 + p]);
      GD.gM[p] = Dual(G.gM[p], tg[4 + p]);
    }
    GD.alpha = Dual(G.alpha, tg[6]);
    Dual Fv[3];
    int err = 0;
    visc_flux(vd, dir, P, GD, Fv, &err);
    double aFv[3] = {urange(-1, 1), urange(-1, 1), urange(-1, 1)};
    double lhs = 0.0, scale = 0.0;
    for (int k = 0; k < 3; ++k) {
      lhs += aFv[k] * Fv[k].d;
      scale += fabs(aFv[k] * Fv[k].d);
    }
    ViscAdj a;
    visc_adj_zero(a);
    GravAdj ag;
    grav_adj_zero(ag);
    visc_flux_rev(v, dir, P, G, aFv, a, ag);
    double *aa[6] = {a.cL, a.cR, a.gpL, a.gpR, a.grL, a.grR};
    double rhs = 0.0;
    for (int k = 0; k < 6; ++k)
      for (int q = 0; q < 5; ++q) rhs += aa[k][q] * tc[k][q];
    for (int p = 0; p < 2; ++p) rhs += ag.gx[p] * tg[p] + ag.gy[p] * tg[2 + p] + ag.gM[p] * tg[4 + p];
    rhs += ag.alpha * tg[6];
    double e = rel(lhs, rhs, 1e-12 * scale + 1e-300);
    if (e > mx) mx = e;
  }
  report("visc_flux", n, mx, "(alpha-law and constant nu, r and phi faces)");
}

static void check_source() {
  double mx = 0.0;
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    DiskParams P = base_params();
    P.visc_const = (t % 3 == 0) ? 1 : 0;
    P.has_visc = (t % 5 != 0);
    SrcGeom g;
    g.r = urange(0.5, 3.0);
    g.dV = urange(0.01, 0.1);
    g.dt = urange(0.001, 0.01);
    double ph = urange(0, 6.28);
    g.cosp = cos(ph);
    g.sinp = sin(ph);
    g.xpos = g.r * g.cosp;
    g.ypos = g.r * g.sinp;
    g.sint = 1.0;
    g.cost = 0.0;
    g.gravdist = g.r;
    g.Fc = urange(-1, 1);
    g.dtOm = urange(-1, 1);
    g.rdrOm = urange(-1, 1);
    double pm[5], tp[5];
    rand_prim(pm);
    pm[D_UZZ] = urange(-0.5, 0.5);
    Dual pd[5];
    for (int q = 0; q < 5; ++q) {
      tp[q] = urange(-1, 1);
      pd[q] = Dual(pm[q], tp[q]);
    }
    double gu = urange(-1, 1), gpu = urange(-1, 1), tgu = urange(-1, 1), tgpu = urange(-1, 1);
    GravT<double> G;
    GravT<Dual> GD;
    double tg[7];
    for (int p = 0; p < 2; ++p) {
      G.gx[p] = urange(-0.6, 0.6);
      G.gy[p] = urange(-0.6, 0.6);
      G.gM[p] = urange(0.1, 0.9);
    }
    G.alpha = urange(0.01, 0.1);
    for (int k = 0; k < 7; ++k) tg[k] = urange(-1, 1);
    for (int p = 0; p < 2; ++p) {
      GD.gx[p] = Dual(G.gx[p], tg[p]);
      GD.gy[p] = Dual(G.gy[p], tg[2 + p]);
      GD.gM[p] = Dual(G.gM[p], tg[4 + p]);
    }
    GD.alpha = Dual(G.alpha, tg[6]);
    Dual s[6];
    source_cell(g, P, pd, Dual(gu, tgu), Dual(gpu, tgpu), GD, s);
    double as[6], lhs = 0.0, scale = 0.0;
    for (int k = 0; k < 6; ++k) {
      as[k] = urange(-1, 1);
      lhs += as[k] * s[k].d;
      scale += fabs(as[k] * s[k].d);
    }
    double apm[5] = {0}, agu = 0.0, agpu = 0.0;
    GravAdj ag;
    grav_adj_zero(ag);
    source_cell_rev(g, P, pm, gu, gpu, G, as, apm, agu, agpu, ag);
    double rhs = agu * tgu + agpu * tgpu;
    for (int q = 0; q < 5; ++q) rhs += apm[q] * tp[q];
    for (int p = 0; p < 2; ++p) rhs += ag.gx[p] * tg[p] + ag.gy[p] * tg[2 + p] + ag.gM[p] * tg[4 + p];
    rhs += ag.alpha * tg[6];
    double e = rel(lhs, rhs, 1e-12 * scale + 1e-300);
    if (e > mx) mx = e;
  }
  report("source_cell", n, mx, "(binary gravity, frame terms, viscous heating)");
}

static void check_update_chain() {
  // split_rotate -> cons2prim -> damping -> prim2cons, with the floors active
  // on part of the trials
  double mx = 0.0;
  int nfloor = 0, ncap = 0;
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    DiskParams P = base_params();
    if (t % 4 == 1) P.rho_floor = 1.5;   // density floor often active
    if (t % 4 == 2) P.cs_floor = 2.0;    // pressure floor often active
    if (t % 4 == 3) P.vel_cap = 0.5;     // velocity cap often active
    double c[5], tc[5];
    const double dV = urange(0.05, 0.2), r = urange(0.5, 3.0);
    double pm[5];
    rand_prim(pm);
    pm[D_UZZ] = urange(-0.3, 0.3);
    prim2cons(pm, c, r, dV, P.gamma);
    Dual cd[5];
    for (int q = 0; q < 5; ++q) {
      tc[q] = urange(-1, 1);
      cd[q] = Dual(c[q], tc[q]);
    }
    const double ck = urange(-1, 1), sk = urange(-1, 1), dr2 = urange(0.1, 2), kap = urange(0.1, 2),
                 Om = urange(-1, 1), f = (t & 1) ? urange(0, 0.5) : 0.0;
    double ic[5];
    rand_prim(ic);
    const double dV2 = urange(0.05, 0.2);
    // forward (Dual)
    Dual prd[5], cout[5];
    split_rotate(cd, ck, sk, dr2, kap, Om, r);
    cons2prim(cd, dV2, r, P, prd);
    for (int q = 0; q < 5; ++q) {
      Dual dprim = ic[q] - prd[q];
      prd[q] += f * dprim;
    }
    prim2cons(prd, cout, r, dV2, P.gamma);
    double apo[5], aco[5], lhs = 0.0, scale = 0.0;
    for (int q = 0; q < 5; ++q) {
      apo[q] = urange(-1, 1);
      aco[q] = urange(-1, 1);
      lhs += apo[q] * prd[q].d + aco[q] * cout[q].d;
      scale += fabs(apo[q] * prd[q].d) + fabs(aco[q] * cout[q].d);
    }
    // reverse: recompute the forward values
    double cv[5], prv[5];
    for (int q = 0; q < 5; ++q) cv[q] = c[q];
    split_rotate(cv, ck, sk, dr2, kap, Om, r);
    cons2prim(cv, dV2, r, P, prv);
    {
      double rho = cv[D_DDD] / dV2;
      if (rho < P.rho_floor) ++nfloor;
      double Ppre = prv[D_PPP];
      if (Ppre <= P.cs_floor * P.cs_floor * prv[D_RHO] / P.gamma * (1 + 1e-12)) ++ncap;
    }
    for (int q = 0; q < 5; ++q) {
      double dprim = ic[q] - prv[q];
      prv[q] += f * dprim;
    }
    double apr[5];
    for (int q = 0; q < 5; ++q) apr[q] = apo[q];
    prim2cons_rev(prv, r, dV2, P.gamma, aco, apr);
    for (int q = 0; q < 5; ++q) apr[q] *= (1.0 - f);
    double ac[5] = {0, 0, 0, 0, 0};
    double cpre[5];
    for (int q = 0; q < 5; ++q) cpre[q] = c[q];
    split_rotate(cpre, ck, sk, dr2, kap, Om, r);
    cons2prim_rev(cpre, dV2, r, P, apr, ac);
    split_rotate_rev(ac, ck, sk, dr2, kap, Om, r);
    double rhs = 0.0;
    for (int q = 0; q < 5; ++q) rhs += ac[q] * tc[q];
    double e = rel(lhs, rhs, 1e-12 * scale + 1e-300);
    if (e > mx) mx = e;
  }
  char buf[128];
  snprintf(buf, sizeof(buf), "(rotation, cons2prim, damping, prim2cons; rho floor %d, P floor %d)", nfloor, ncap);
  report("update_chain", n, mx, buf);
}

static void check_plm_p() {
  double mx = 0.0;
  int br[4] = {0, 0, 0, 0};
  const int n = 20000;
  for (int t = 0; t < n; ++t) {
    double pl = urange(-1, 1), pc = urange(-1, 1), pr = urange(-1, 1);
    double vl = urange(-1, 1), vc = urange(-1, 1), vr = urange(-1, 1);
    double dpL = urange(0.01, 0.1), dpR = urange(0.01, 0.1), plm = (t & 1) ? 1.5 : 1.0;
    Dual s = plm_p_slope(Dual(pl, vl), Dual(pc, vc), Dual(pr, vr), dpL, dpR, plm);
    double kl, kc, kr;
    plm_p_slope_coef(pl, pc, pr, dpL, dpR, plm, &kl, &kc, &kr);
    double rhs = kl * vl + kc * vc + kr * vr;
    double e = rel(s.d, rhs, 1e-12 * fabs(s.d) + 1e-300);
    if (e > mx) mx = e;
    br[(kl == 0 && kc == 0 && kr == 0) ? 3 : (kr == 0 ? 0 : (kl == 0 ? 1 : 2))]++;
  }
  char buf[128];
  snprintf(buf, sizeof(buf), "(branches: left %d, right %d, centred %d, zero %d)", br[0], br[1], br[2], br[3]);
  report("plm_p_slope", n, mx, buf);
}

int main() {
  check_riemann();
  check_visc();
  check_source();
  check_update_chain();
  check_plm_p();
  printf("worst %.3e\n", worst);
  return failed;
}
