// Hand-written reverse-mode (adjoint) versions of the per-face and per-cell
// physics in dgpu_device.cuh.
//
// Each *_rev function takes the forward inputs (values), recomputes the
// forward intermediates it needs and adds (d out / d in)^T a_out to the
// adjoints of the inputs.  Branches are replayed from the recomputed values:
// the HLLC state and wave-speed choices, the limiter branches and the
// floor/cap clamps follow the forward pass exactly, so the result is the
// transpose of the tangent of the same branch.  All of them are __host__
// __device__: a host build checks each against the Dual tangent with
// dot-product tests.
#ifndef DGPU_ADJOINT_CUH
#define DGPU_ADJOINT_CUH

#include "dgpu_device.cuh"

namespace {

// Adjoints of the binary's masses and positions and of alpha.
struct GravAdj {
  double gx[2], gy[2], gM[2], alpha;
};
HD void grav_adj_zero(GravAdj &a) {
  for (int p = 0; p < 2; ++p) a.gx[p] = a.gy[p] = a.gM[p] = 0.0;
  a.alpha = 0.0;
}

// phys_flux: ap += (dF/dp)^T aF
HD void phys_flux_rev(const double *p, double r, double n0, double n1, double n2, double gam, const double *aF,
                      double *ap) {
  const double rho = p[D_RHO], Pp = p[D_PPP], vr = p[D_URR], vp = p[D_UPP] * r, vz = p[D_UZZ];
  const double vn = vr * n0 + vp * n1 + vz * n2;
  const double rhoe = Pp / (gam - 1.);
  const double v2 = vr * vr + vp * vp + vz * vz;
  const double aD = aF[D_DDD], aS = aF[D_SRR], aL = aF[D_LLL], aZ = aF[D_SZZ], aT = aF[D_TAU];
  const double arho = aD * vn + aS * vr * vn + aL * r * vp * vn + aZ * vz * vn + aT * .5 * v2 * vn;
  const double avn = aD * rho + aS * rho * vr + aL * r * rho * vp + aZ * rho * vz + aT * (.5 * rho * v2 + rhoe + Pp);
  const double av2 = aT * .5 * rho * vn;
  const double aP = aS * n0 + aL * r * n1 + aZ * n2 + aT * vn + aT * vn / (gam - 1.);
  const double avr = aS * rho * vn + avn * n0 + 2. * vr * av2;
  const double avp = aL * r * rho * vn + avn * n1 + 2. * vp * av2;
  const double avz = aZ * rho * vn + avn * n2 + 2. * vz * av2;
  ap[D_RHO] += arho;
  ap[D_PPP] += aP;
  ap[D_URR] += avr;
  ap[D_UPP] += avp * r;
  ap[D_UZZ] += avz;
}

// prim2cons: ap += (dU/dp)^T aU
HD void prim2cons_rev(const double *p, double r, double dV, double gam, const double *aU, double *ap) {
  const double rho = p[D_RHO], vr = p[D_URR], vp = p[D_UPP] * r, vz = p[D_UZZ];
  const double v2 = vr * vr + vp * vp + vz * vz;
  const double aD = aU[D_DDD], aS = aU[D_SRR], aL = aU[D_LLL], aZ = aU[D_SZZ], aT = aU[D_TAU];
  ap[D_RHO] += dV * (aD + aS * vr + aL * r * vp + aZ * vz + aT * .5 * v2);
  ap[D_PPP] += dV * aT / (gam - 1.);
  ap[D_URR] += dV * (aS * rho + aT * rho * vr);
  ap[D_UPP] += dV * (aL * r * rho + aT * rho * vp) * r;
  ap[D_UZZ] += dV * (aZ * rho + aT * rho * vz);
}

// riemann_flux: apL += (dF/dpL)^T aF, apR += (dF/dpR)^T aF
HD void riemann_flux_rev(const double *pL, const double *pR, double r, int dir, double w, double gam, int solver,
                         const double *aF, double *apL, double *apR) {
  const double n0 = dir == 0 ? 1.0 : 0.0, n1 = dir == 1 ? 1.0 : 0.0, n2 = 0.0;
  const double vnL = pL[D_URR] * n0 + (r * pL[D_UPP]) * n1 + pL[D_UZZ] * n2;
  const double vnR = pR[D_URR] * n0 + (r * pR[D_UPP]) * n1 + pR[D_UZZ] * n2;
  const double cf2L = gam * (pL[D_PPP] / pL[D_RHO]);
  const double cf2R = gam * (pR[D_PPP] / pR[D_RHO]);
  const double cL = sqrt(cf2L), cR = sqrt(cf2R);
  double Sl = vnL - cL, Sr = vnL + cL;
  const bool slR = Sl > vnR - cR;
  if (slR) Sl = vnR - cR;
  const bool srR = Sr < vnR + cR;
  if (srR) Sr = vnR + cR;
  const double NumS = pR[D_RHO] * vnR * (Sr - vnR) - pL[D_RHO] * vnL * (Sl - vnL) + pL[D_PPP] - pR[D_PPP];
  const double DenS = pR[D_RHO] * (Sr - vnR) - pL[D_RHO] * (Sl - vnL);
  const double Ss = NumS / DenS;
  int state;
  if (w < Sl) state = DS_LEFT;
  else if (w > Sr) state = DS_RIGHT;
  else if (w < Ss) state = DS_LEFTSTAR;
  else state = DS_RIGHTSTAR;

  if (state == DS_LEFT || state == DS_RIGHT) {
    const double *p = state == DS_LEFT ? pL : pR;
    double *ap = state == DS_LEFT ? apL : apR;
    double aU[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) aU[q] = -w * aF[q];
    phys_flux_rev(p, r, n0, n1, n2, gam, aF, ap);
    prim2cons_rev(p, r, 1.0, gam, aU, ap);
    return;
  }
  double aSl = 0.0, aSr = 0.0;
  if (solver == DR_HLL) {
    double FL[5], FR[5], UL[5], UR[5];
    phys_flux(pL, r, n0, n1, n2, gam, FL);
    phys_flux(pR, r, n0, n1, n2, gam, FR);
    prim2cons(pL, UL, r, 1.0, gam);
    prim2cons(pR, UR, r, 1.0, gam);
    const double dS = Sr - Sl;
    double aFL[5], aFR[5], aUL[5], aUR[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const double Ustar = (Sr * UR[q] - Sl * UL[q] + FL[q] - FR[q]) / dS;
      const double Fstar = (Sr * FL[q] - Sl * FR[q] - Sr * Sl * (UL[q] - UR[q])) / dS;
      const double aUs = -w * aF[q], aFs = aF[q];
      aUR[q] = aUs * Sr / dS + aFs * Sr * Sl / dS;
      aUL[q] = -aUs * Sl / dS - aFs * Sr * Sl / dS;
      aFL[q] = aUs / dS + aFs * Sr / dS;
      aFR[q] = -aUs / dS - aFs * Sl / dS;
      aSr += aUs * (UR[q] - Ustar) / dS + aFs * ((FL[q] - Sl * (UL[q] - UR[q])) - Fstar) / dS;
      aSl += aUs * (Ustar - UL[q]) / dS + aFs * ((-FR[q] - Sr * (UL[q] - UR[q])) + Fstar) / dS;
    }
    phys_flux_rev(pL, r, n0, n1, n2, gam, aFL, apL);
    phys_flux_rev(pR, r, n0, n1, n2, gam, aFR, apR);
    prim2cons_rev(pL, r, 1.0, gam, aUL, apL);
    prim2cons_rev(pR, r, 1.0, gam, aUR, apR);
  } else {
    const bool left = state == DS_LEFTSTAR;
    const double *prim = left ? pL : pR;
    double *ap = left ? apL : apR;
    const double Sk = left ? Sl : Sr;
    double Fk[5], Uk[5];
    phys_flux(prim, r, n0, n1, n2, gam, Fk);
    prim2cons(prim, Uk, r, 1.0, gam);
    const double rho = prim[D_RHO], vr = prim[D_URR], vp = prim[D_UPP] * r, vz = prim[D_UZZ];
    const double Pp = prim[D_PPP];
    const double v2 = vr * vr + vp * vp + vz * vz;
    const double vn = vr * n0 + vp * n1 + vz * n2;
    const double rhoe = Pp / (gam - 1.);
    const double D = rho, mr = rho * vr, mp = rho * vp, mz = rho * vz;
    const double E_h = .5 * rho * v2 + rhoe;
    const double K = Sk - vn, Dn = Sk - Ss;
    const double Ps = rho * K * (Ss - vn) + Pp;
    const double Dstar = K * D / Dn;
    const double Msr = K * mr / Dn, Msp = K * mp / Dn, Msz = K * mz / Dn;
    const double Estar = (K * E_h + Ps * Ss - Pp * vn) / Dn;
    const double Msn = Dstar * Ss;
    const double mn = Msr * n0 + Msp * n1 + Msz * n2;
    double Ust[5];
    Ust[D_DDD] = Dstar;
    Ust[D_SRR] = Msr + n0 * (Msn - mn);
    Ust[D_LLL] = r * (Msp + n1 * (Msn - mn));
    Ust[D_SZZ] = Msz + n2 * (Msn - mn);
    Ust[D_TAU] = Estar;
    // F = Fk + Sk (Ust - Uk) - w Ust
    double aUk[5], aSk = 0.0;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      aUk[q] = -Sk * aF[q];
      aSk += aF[q] * (Ust[q] - Uk[q]);
    }
    const double aDstar0 = (Sk - w) * aF[D_DDD];
    const double aEstar = (Sk - w) * aF[D_TAU];
    const double aMsrF = (Sk - w) * aF[D_SRR];
    const double aMspF = r * (Sk - w) * aF[D_LLL];
    const double aMszF = (Sk - w) * aF[D_SZZ];
    const double aMsn = n0 * aMsrF + n1 * aMspF + n2 * aMszF;
    const double amn = -aMsn;
    const double aMsr = aMsrF + amn * n0, aMsp = aMspF + amn * n1, aMsz = aMszF + amn * n2;
    const double aDstar = aDstar0 + aMsn * Ss;
    double aSs = aMsn * Dstar;
    // Estar
    const double aNumE = aEstar / Dn;
    double aDn = -aEstar * Estar / Dn;
    double aK = aNumE * E_h;
    const double aEh = aNumE * K;
    const double aPs = aNumE * Ss;
    aSs += aNumE * Ps;
    double aPp = -aNumE * vn;
    double avn = -aNumE * Pp;
    // Msr, Msp, Msz, Dstar
    aK += (aMsr * mr + aMsp * mp + aMsz * mz + aDstar * D) / Dn;
    const double amr = aMsr * K / Dn, amp = aMsp * K / Dn, amz = aMsz * K / Dn, aD = aDstar * K / Dn;
    aDn -= (aMsr * Msr + aMsp * Msp + aMsz * Msz + aDstar * Dstar) / Dn;
    // Ps
    double arho = aPs * K * (Ss - vn);
    aK += aPs * rho * (Ss - vn);
    aSs += aPs * rho * K;
    avn -= aPs * rho * K;
    aPp += aPs;
    // K = Sk - vn, Dn = Sk - Ss
    aSk += aK + aDn;
    avn -= aK;
    aSs -= aDn;
    // E_h, momenta, D, rhoe
    arho += aEh * .5 * v2 + amr * vr + amp * vp + amz * vz + aD;
    const double av2 = aEh * .5 * rho;
    aPp += aEh / (gam - 1.);
    const double avr = amr * rho + avn * n0 + 2. * vr * av2;
    const double avp = amp * rho + avn * n1 + 2. * vp * av2;
    const double avz = amz * rho + avn * n2 + 2. * vz * av2;
    ap[D_RHO] += arho;
    ap[D_PPP] += aPp;
    ap[D_URR] += avr;
    ap[D_UPP] += avp * r;
    ap[D_UZZ] += avz;
    phys_flux_rev(prim, r, n0, n1, n2, gam, aF, ap);
    prim2cons_rev(prim, r, 1.0, gam, aUk, ap);
    if (left) aSl += aSk;
    else aSr += aSk;
    // Ss = NumS / DenS
    const double aNumS = aSs / DenS, aDenS = -aSs * Ss / DenS;
    apR[D_RHO] += aNumS * vnR * (Sr - vnR) + aDenS * (Sr - vnR);
    apL[D_RHO] -= aNumS * vnL * (Sl - vnL) + aDenS * (Sl - vnL);
    apL[D_PPP] += aNumS;
    apR[D_PPP] -= aNumS;
    aSr += aNumS * pR[D_RHO] * vnR + aDenS * pR[D_RHO];
    aSl -= aNumS * pL[D_RHO] * vnL + aDenS * pL[D_RHO];
    const double avnR = aNumS * pR[D_RHO] * (Sr - 2. * vnR) - aDenS * pR[D_RHO];
    const double avnL = -aNumS * pL[D_RHO] * (Sl - 2. * vnL) + aDenS * pL[D_RHO];
    apR[D_URR] += avnR * n0;
    apR[D_UPP] += avnR * r * n1;
    apR[D_UZZ] += avnR * n2;
    apL[D_URR] += avnL * n0;
    apL[D_UPP] += avnL * r * n1;
    apL[D_UZZ] += avnL * n2;
  }
  // wave speeds: Sl = min(vnL - cL, vnR - cR), Sr = max(vnL + cL, vnR + cR)
  double avnL = 0.0, avnR = 0.0, acL = 0.0, acR = 0.0;
  if (slR) {
    avnR += aSl;
    acR -= aSl;
  } else {
    avnL += aSl;
    acL -= aSl;
  }
  if (srR) {
    avnR += aSr;
    acR += aSr;
  } else {
    avnL += aSr;
    acL += aSr;
  }
  const double acf2L = acL / (2. * cL), acf2R = acR / (2. * cR);
  apL[D_PPP] += acf2L * gam / pL[D_RHO];
  apL[D_RHO] -= acf2L * gam * pL[D_PPP] / (pL[D_RHO] * pL[D_RHO]);
  apR[D_PPP] += acf2R * gam / pR[D_RHO];
  apR[D_RHO] -= acf2R * gam * pR[D_PPP] / (pR[D_RHO] * pR[D_RHO]);
  apL[D_URR] += avnL * n0;
  apL[D_UPP] += avnL * r * n1;
  apL[D_UZZ] += avnL * n2;
  apR[D_URR] += avnR * n0;
  apR[D_UPP] += avnR * r * n1;
  apR[D_UZZ] += avnR * n2;
}

// Adjoints of the cell inputs of visc_flux.
struct ViscAdj {
  double cL[5], cR[5], gpL[5], gpR[5], grL[5], grR[5];
};
HD void visc_adj_zero(ViscAdj &a) {
  for (int q = 0; q < 5; ++q) a.cL[q] = a.cR[q] = a.gpL[q] = a.gpR[q] = a.grL[q] = a.grR[q] = 0.0;
}

// visc_flux: adds (dFv/d inputs)^T aFv to a (cell inputs) and ag (binary, alpha)
HD void visc_flux_rev(const ViscIn<double> &v, int dir, const DiskParams &P, const GravT<double> &G,
                      const double *aFv, ViscAdj &a, GravAdj &ag) {
  const double r = v.r;
  double Avg[4], Gr[4], Gp[4];
  double den = 0.0;
  if (dir == 0) {
    double deltaL = v.r - v.r_cell_L;
    double deltaR = v.r_cell_R - v.r;
    den = deltaR + deltaL;
    for (int q = 0; q < 4; ++q) {
      double WL = v.cL[q] + v.dpL * v.gpL[q];
      double WR = v.cR[q] - v.dpR * v.gpR[q];
      Avg[q] = 0.5 * (WL + WR);
      Gr[q] = (WR - WL) / den;
      Gp[q] = .5 * (v.gpL[q] + v.gpR[q]) / r;
    }
  } else {
    for (int q = 0; q < 4; ++q) {
      Avg[q] = 0.5 * (v.cR[q] + v.cL[q]);
      Gp[q] = (v.cR[q] - v.cL[q]) / (v.tR - v.tL) / r;
      Gr[q] = .5 * (v.grL[q] + v.grR[q]);
    }
  }
  // nu and its inputs
  double nu;
  double x = 0.0, y = 0.0, d0 = 0.0, d1 = 0.0, s0 = 0.0, s1 = 0.0, Q0 = 0.0, Q1 = 0.0, sq = 1.0, t2 = 0.0;
  double shear_c = 0.0;
  const int law = P.visc_const == 1 ? 0 : (P.init_type == DI_SHEAR ? 1 : 2);
  if (law == 0) {
    nu = G.alpha;
  } else if (law == 1) {
    shear_c = dpow(fabs(r * cos(v.cm)), 2.0);
    nu = G.alpha * P.gamma * Avg[D_PPP] / Avg[D_RHO] * shear_c;
    if (r * cos(v.cm) > 20.) nu = 0.0;
  } else {
    double sc, cc;
    sincos(v.cm, &sc, &cc);
    x = r * cc;
    y = r * sc;
    d0 = gm_dist_xy(x, y, G.gx[0], G.gy[0]);
    d1 = gm_dist_xy(x, y, G.gx[1], G.gy[1]);
    const double eps = P.g_eps;
    s0 = d0 * d0 + eps * eps;
    s1 = d1 * d1 + eps * eps;
    Q0 = dpow(s0, -1.5);
    Q1 = dpow(s1, -1.5);
    sq = sqrt(Q0 * G.gM[0] + Q1 * G.gM[1]);
    t2 = G.alpha * Avg[D_PPP] / Avg[D_RHO];
    nu = t2 / sq;
  }
  const double rho = Avg[D_RHO], vr = Avg[D_URR], om = Avg[D_UPP];
  const double Gr_vr = Gr[D_URR], Gr_om = Gr[D_UPP], Gp_vr = Gp[D_URR], Gp_om = Gp[D_UPP];
  const double rdr = v.rdr_om;
  double B[3];
  if (dir == 0) {
    B[0] = r * Gr_vr - vr - r * r * Gp_om;
    B[1] = r * (r * Gr_om + rdr) + r * Gp_vr;
    B[2] = vr * (Gr_vr - vr / r - r * Gp_om) + r * om * (Gp_vr + (rdr + r * Gr_om));
  } else {
    B[0] = r * (r * Gr_om + rdr) + r * Gp_vr;
    B[1] = -r * Gr_vr + vr + r * r * Gp_om;
    B[2] = -r * om * (Gr_vr - vr / r - r * Gp_om) + vr * (Gp_vr + (rdr + r * Gr_om));
  }
  // Fv_k = A B_k, A = -nu rho
  const double A = -nu * rho;
  const double aA = aFv[0] * B[0] + aFv[1] * B[1] + aFv[2] * B[2];
  const double aB0 = aFv[0] * A, aB1 = aFv[1] * A, aB2 = aFv[2] * A;
  double anu = -aA * rho;
  double aAvg[4] = {-aA * nu, 0.0, 0.0, 0.0};
  double aGr[4] = {0.0, 0.0, 0.0, 0.0}, aGp[4] = {0.0, 0.0, 0.0, 0.0};
  if (dir == 0) {
    aGr[D_URR] += r * aB0 + aB2 * vr;
    aAvg[D_URR] += -aB0 + aB2 * (Gr_vr - vr / r - r * Gp_om) - aB2 * vr / r;
    aGp[D_UPP] += -r * r * aB0 - aB2 * vr * r;
    aGr[D_UPP] += r * r * aB1 + aB2 * r * om * r;
    aGp[D_URR] += r * aB1 + aB2 * r * om;
    aAvg[D_UPP] += aB2 * r * (Gp_vr + (rdr + r * Gr_om));
  } else {
    aGr[D_UPP] += r * r * aB0 + aB2 * vr * r;
    aGp[D_URR] += r * aB0 + aB2 * vr;
    aGr[D_URR] += -r * aB1 - aB2 * r * om;
    aAvg[D_URR] += aB1 + aB2 * om + aB2 * (Gp_vr + (rdr + r * Gr_om));
    aGp[D_UPP] += r * r * aB1 + aB2 * r * om * r;
    aAvg[D_UPP] += -aB2 * r * (Gr_vr - vr / r - r * Gp_om);
  }
  // nu
  if (law == 0) {
    ag.alpha += anu;
  } else if (law == 1) {
    if (!(r * cos(v.cm) > 20.)) {
      ag.alpha += anu * P.gamma * Avg[D_PPP] / Avg[D_RHO] * shear_c;
      aAvg[D_PPP] += anu * G.alpha * P.gamma / Avg[D_RHO] * shear_c;
      aAvg[D_RHO] -= anu * nu / Avg[D_RHO];
    }
  } else {
    const double at2 = anu / sq;
    const double asq = -anu * nu / sq;
    const double at1 = at2 / Avg[D_RHO];
    aAvg[D_RHO] -= at2 * t2 / Avg[D_RHO];
    ag.alpha += at1 * Avg[D_PPP];
    aAvg[D_PPP] += at1 * G.alpha;
    const double aQ = asq / (2. * sq);
    ag.gM[0] += aQ * Q0;
    ag.gM[1] += aQ * Q1;
    const double ad0 = 2. * d0 * aQ * G.gM[0] * dpow_dx(s0, -1.5, Q0);
    const double ad1 = 2. * d1 * aQ * G.gM[1] * dpow_dx(s1, -1.5, Q1);
    ag.gx[0] -= ad0 * (x - G.gx[0]) / d0;
    ag.gy[0] -= ad0 * (y - G.gy[0]) / d0;
    ag.gx[1] -= ad1 * (x - G.gx[1]) / d1;
    ag.gy[1] -= ad1 * (y - G.gy[1]) / d1;
  }
  // face average and gradients
  if (dir == 0) {
    for (int q = 0; q < 4; ++q) {
      const double aWL = .5 * aAvg[q] - aGr[q] / den;
      const double aWR = .5 * aAvg[q] + aGr[q] / den;
      a.cL[q] += aWL;
      a.gpL[q] += v.dpL * aWL + .5 * aGp[q] / r;
      a.cR[q] += aWR;
      a.gpR[q] += -v.dpR * aWR + .5 * aGp[q] / r;
    }
  } else {
    const double k = 1.0 / (v.tR - v.tL) / r;
    for (int q = 0; q < 4; ++q) {
      a.cR[q] += .5 * aAvg[q] + aGp[q] * k;
      a.cL[q] += .5 * aAvg[q] - aGp[q] * k;
      a.grL[q] += .5 * aGr[q];
      a.grR[q] += .5 * aGr[q];
    }
  }
}

// source_cell: adds (ds/d inputs)^T as to apm (prims), agu (grad[UPP]),
// agpu (gradp[URR]) and ag (binary, alpha)
HD void source_cell_rev(const SrcGeom &g, const DiskParams &P, const double *pm, double grad_upp, double gradp_urr,
                        const GravT<double> &G, const double *as, double *apm, double &agu, double &agpu,
                        GravAdj &ag) {
  const double rho = pm[D_RHO], Pp = pm[D_PPP], vr = pm[D_URR], vz = pm[D_UZZ];
  const double vp = pm[D_UPP] * g.r;
  double Fr = 0.0, Fp = 0.0;
  double dx[2], dy[2], sr[2], cosa[2], sina[2], cosap[2], sinap[2], f1[2];
  for (int p = 0; p < 2; ++p) {
    dx[p] = g.gravdist * g.cosp - G.gx[p];
    dy[p] = g.gravdist * g.sinp - G.gy[p];
    sr[p] = sqrt(dx[p] * dx[p] + dy[p] * dy[p]);
    cosa[p] = dx[p] / sr[p];
    sina[p] = dy[p] / sr[p];
    cosap[p] = cosa[p] * g.cosp + sina[p] * g.sinp;
    sinap[p] = sina[p] * g.cosp - cosa[p] * g.sinp;
    f1[p] = -fgrav(G.gM[p], sr[p], P.g_eps, P.phi_order);
    Fr += cosap[p] * f1[p];
    Fp += sinap[p] * f1[p];
  }
  const double Feul = -(g.r * g.dtOm + vr * g.rdrOm);
  const double k = g.dt * g.dV;
  double arho = 0.0, aP = 0.0, avr = 0.0, avp = 0.0, avz = 0.0, aFr = 0.0, aFp = 0.0;
  // s0 = k (rho vp^2 + P) / r
  arho += k * as[0] * vp * vp / g.r;
  avp += k * as[0] * rho * 2. * vp / g.r;
  aP += k * as[0] / g.r;
  // s1 = k rho (Fr sint + Fc)
  arho += k * as[1] * (Fr * g.sint + g.Fc);
  aFr += k * as[1] * rho * g.sint;
  // s2 = k rho (Fp - r dtOm) r
  arho += k * as[2] * (Fp - g.r * g.dtOm) * g.r;
  aFp += k * as[2] * rho * g.r;
  // s3 = k rho Fr cost
  arho += k * as[3] * Fr * g.cost;
  aFr += k * as[3] * rho * g.cost;
  // s4 = k rho ((Fr sint + Fc) vr + Fr vz cost + (Fp + Feul) vp)
  {
    const double E4 = (Fr * g.sint + g.Fc) * vr + Fr * vz * g.cost + (Fp + Feul) * vp;
    const double R4 = k * as[4] * rho;
    arho += k * as[4] * E4;
    aFr += R4 * (g.sint * vr + vz * g.cost);
    avr += R4 * (Fr * g.sint + g.Fc);
    avz += R4 * Fr * g.cost;
    aFp += R4 * vp;
    avp += R4 * (Fp + Feul);
    avr -= R4 * vp * g.rdrOm;  // Feul = -(r dtOm + vr rdrOm)
  }
  // gravity
  for (int p = 0; p < 2; ++p) {
    const double acosap = aFr * f1[p], asinap = aFp * f1[p];
    const double af1 = aFr * cosap[p] + aFp * sinap[p];
    const double acosa = acosap * g.cosp - asinap * g.sinp;
    const double asina = acosap * g.sinp + asinap * g.cosp;
    // f1 = -M q(sr): d/dM = f1/M computed as -q; d/dsr = f1 ((n-1)/sr - (n+1) sr^(n-1)/(sr^n + eps^n))
    const int n = P.phi_order;
    const double qv = fgrav(1.0, sr[p], P.g_eps, n);
    ag.gM[p] += -af1 * qv;
    const double srn = dpow(sr[p], (double)n), epn = dpow(P.g_eps, (double)n);
    const double dln = (n - 1.) / sr[p] - (n + 1.) * dpow(sr[p], n - 1.) / (srn + epn);
    double asr = af1 * f1[p] * dln;
    asr -= (acosa * dx[p] + asina * dy[p]) / (sr[p] * sr[p]);
    const double adx = acosa / sr[p] + asr * dx[p] / sr[p];
    const double ady = asina / sr[p] + asr * dy[p] / sr[p];
    ag.gx[p] -= adx;
    ag.gy[p] -= ady;
  }
  // viscous heating
  if (P.has_visc) {
    const double eps = P.g_eps;
    double db[2], sb[2], Qb[2], sqQ = 1.0, Sigma_nu;
    for (int p = 0; p < 2; ++p) {
      db[p] = sqrt((g.xpos - G.gx[p]) * (g.xpos - G.gx[p]) + (g.ypos - G.gy[p]) * (g.ypos - G.gy[p]));
      sb[p] = db[p] * db[p] + eps * eps;
      Qb[p] = dpow(sb[p], -1.5);
    }
    if (P.visc_const == 1) {
      Sigma_nu = rho * G.alpha;
    } else {
      sqQ = sqrt(Qb[0] * G.gM[0] + Qb[1] * G.gM[1]);
      Sigma_nu = G.alpha * Pp / sqQ;
    }
    const double B5 = g.rdrOm + g.r * grad_upp + gradp_urr;
    const double aSn = k * as[5] * g.rdrOm * B5;
    const double aB5 = k * as[5] * Sigma_nu * g.rdrOm;
    agu += aB5 * g.r;
    agpu += aB5;
    if (P.visc_const == 1) {
      arho += aSn * G.alpha;
      ag.alpha += aSn * rho;
    } else {
      ag.alpha += aSn * Pp / sqQ;
      aP += aSn * G.alpha / sqQ;
      const double asq = -aSn * Sigma_nu / sqQ;
      const double aQ = asq / (2. * sqQ);
      for (int p = 0; p < 2; ++p) {
        ag.gM[p] += aQ * Qb[p];
        const double ad = 2. * db[p] * aQ * G.gM[p] * dpow_dx(sb[p], -1.5, Qb[p]);
        ag.gx[p] -= ad * (g.xpos - G.gx[p]) / db[p];
        ag.gy[p] -= ad * (g.ypos - G.gy[p]) / db[p];
      }
    }
  }
  apm[D_RHO] += arho;
  apm[D_PPP] += aP;
  apm[D_URR] += avr;
  apm[D_UPP] += avp * g.r;
  apm[D_UZZ] += avz;
}

// split_rotate: ac += (d c_out / d c_in)^T ac_out  (in place: ac holds a of the
// output on entry and a of the input on return)
HD void split_rotate_rev(double *ac, double ck, double sk, double dr_r2Om, double kappa, double Omega, double r) {
  const double al = ac[D_LLL], arv = ac[D_SRR];
  const double fa = dr_r2Om / kappa * sk;       // l = l0 ck - rv0 fa
  const double fb = 2.0 * Omega / r / kappa * sk; // rv = rv0 ck + l0 fb
  ac[D_LLL] = al * ck + arv * fb;
  ac[D_SRR] = -al * fa + arv * ck;
}

// cons2prim: ac += (d pr / d c)^T apr
HD void cons2prim_rev(const double *c, double dV, double r, const DiskParams &P, const double *apr, double *ac) {
  double rho = c[D_DDD] / dV;
  const bool rho_floor = rho < P.rho_floor;
  if (rho_floor) rho = P.rho_floor;
  const double Sr = c[D_SRR] / dV, Sp = c[D_LLL] / dV / r, Sz = c[D_SZZ] / dV;
  const double vr0 = Sr / rho, vp0 = Sp / rho, vz0 = Sz / rho;
  const double KE = .5 * (Sr * vr0 + Sp * vp0 + Sz * vz0);
  const double vmag = sqrt(2. * KE / rho);
  const double rhoe = c[D_TAU] / dV - KE;
  double Pp = (P.gamma - 1.) * rhoe;
  int pclamp = 0;
  if (Pp < P.cs_floor * P.cs_floor * rho / P.gamma) {
    Pp = P.cs_floor * P.cs_floor * rho / P.gamma;
    pclamp = 1;
  }
  if (Pp > P.cs_cap * P.cs_cap * rho / P.gamma) pclamp = 2;
  const bool vcap = vmag > P.vel_cap;
  double arho = apr[D_RHO];
  const double aPp = apr[D_PPP];
  double avr = apr[D_URR], avp = apr[D_UPP] / r, avz = apr[D_UZZ];
  // velocity cap: v = v0 cap / vmag
  double aKE = 0.0;
  if (vcap) {
    const double s = P.vel_cap / vmag;
    const double avmag = -(avr * vr0 + avp * vp0 + avz * vz0) * P.vel_cap / (vmag * vmag);
    avr *= s;
    avp *= s;
    avz *= s;
    // vmag = sqrt(2 KE / rho)
    aKE += avmag / (vmag * rho);
    arho -= avmag * vmag / (2. * rho);
  }
  // pressure
  double arhoe = 0.0;
  if (pclamp == 1) arho += aPp * P.cs_floor * P.cs_floor / P.gamma;
  else if (pclamp == 2) arho += aPp * P.cs_cap * P.cs_cap / P.gamma;
  else arhoe = (P.gamma - 1.) * aPp;
  const double aE = arhoe;
  aKE -= arhoe;
  // KE = .5 (Sr vr0 + Sp vp0 + Sz vz0)
  double aSr = .5 * aKE * vr0, aSp = .5 * aKE * vp0, aSz = .5 * aKE * vz0;
  avr += .5 * aKE * Sr;
  avp += .5 * aKE * Sp;
  avz += .5 * aKE * Sz;
  // v0 = S / rho
  aSr += avr / rho;
  aSp += avp / rho;
  aSz += avz / rho;
  arho -= (avr * vr0 + avp * vp0 + avz * vz0) / rho;
  ac[D_DDD] += rho_floor ? 0.0 : arho / dV;
  ac[D_SRR] += aSr / dV;
  ac[D_LLL] += aSp / dV / r;
  ac[D_SZZ] += aSz / dV;
  ac[D_TAU] += aE / dV;
}

// plm_p_slope: derivative coefficients of the returned slope with respect to
// (pl, pc, pr) on the branch the forward takes.
HD void plm_p_slope_coef(double pl, double pc, double pr, double dpL, double dpR, double plm, double *kl, double *kc,
                         double *kr) {
  const double sL = (pc - pl) / dpL;
  const double sR = (pr - pc) / dpR;
  const double sM = (pr - pl) / (dpL + dpR);
  double sv = plm * sL;
  int br = 0;  // 0: plm sL, 1: plm sR, 2: sM, 3: zero
  if (fabs(sv) > plm * fabs(sR)) {
    sv = plm * sR;
    br = 1;
  }
  if (fabs(sv) > fabs(sM)) {
    sv = sM;
    br = 2;
  }
  if (sL * sR < 0.0) br = 3;
  *kl = *kc = *kr = 0.0;
  if (br == 0) {
    *kc = plm / dpL;
    *kl = -plm / dpL;
  } else if (br == 1) {
    *kr = plm / dpR;
    *kc = -plm / dpR;
  } else if (br == 2) {
    *kr = 1.0 / (dpL + dpR);
    *kl = -1.0 / (dpL + dpR);
  }
}

}  // namespace

#endif
