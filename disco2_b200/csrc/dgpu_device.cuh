// Device helpers shared by the forward, tangent and adjoint kernels.
//
// The per-face and per-cell physics (phys_flux, prim2cons, riemann_flux,
// visc_flux, fgrav) is written once, templated on the scalar type T:
//   T = double : the forward step (every expression in the reference's
//                operation order; built with -fmad=false, so the rounding is
//                the reference's),
//   T = Dual   : the forward-mode tangent.  A Dual carries a value and one
//                directional derivative; its value part is computed by
//                exactly the double expressions, so a tangent run reproduces
//                the forward trajectory bit for bit while carrying d/de.
// Branches (HLLC state, limiters, floors) compare values, so the tangent
// differentiates the branch the forward took.
//
// Everything here is __host__ __device__ so that a host build of the same
// source can check the hand-written adjoints against the tangent on the CPU.
#ifndef DGPU_DEVICE_CUH
#define DGPU_DEVICE_CUH

#include <cuda_runtime.h>
#include <climits>
#include <math.h>
#include <stdint.h>

#include "dgpu_internal.h"

#define PHIMAX (2.0 * M_PI)
// threads per block of every kernel
#ifndef DGPU_BLK
#define DGPU_BLK 256
#endif
#define BLK DGPU_BLK

#define HD __host__ __device__ __forceinline__

namespace {

// the Dual overloads below sit beside, not in place of, the double functions
using ::exp;
using ::fabs;
using ::pow;
using ::sqrt;

// ---------------------------------------------------------------------------
// Dual numbers (value, derivative)
// ---------------------------------------------------------------------------
struct Dual {
  double v, d;
  HD Dual() {}
  HD Dual(double x) : v(x), d(0.0) {}
  HD Dual(double x, double y) : v(x), d(y) {}
};

HD double val(double x) { return x; }
HD double val(const Dual &x) { return x.v; }

HD Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
HD Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.d + b.d); }
HD Dual operator+(const Dual &a, double b) { return Dual(a.v + b, a.d); }
HD Dual operator+(double a, const Dual &b) { return Dual(a + b.v, b.d); }
HD Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.d - b.d); }
HD Dual operator-(const Dual &a, double b) { return Dual(a.v - b, a.d); }
HD Dual operator-(double a, const Dual &b) { return Dual(a - b.v, -b.d); }
HD Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
HD Dual operator*(const Dual &a, double b) { return Dual(a.v * b, a.d * b); }
HD Dual operator*(double a, const Dual &b) { return Dual(a * b.v, a * b.d); }
HD Dual operator/(const Dual &a, const Dual &b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
HD Dual operator/(const Dual &a, double b) { return Dual(a.v / b, a.d / b); }
HD Dual operator/(double a, const Dual &b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
HD Dual &operator+=(Dual &a, const Dual &b) { a = a + b; return a; }
HD Dual &operator+=(Dual &a, double b) { a.v += b; return a; }
HD Dual &operator-=(Dual &a, const Dual &b) { a = a - b; return a; }
HD Dual &operator-=(Dual &a, double b) { a.v -= b; return a; }
HD Dual &operator*=(Dual &a, const Dual &b) { a = a * b; return a; }
HD Dual &operator*=(Dual &a, double b) { a = a * b; return a; }
HD Dual &operator/=(Dual &a, const Dual &b) { a = a / b; return a; }
HD Dual &operator/=(Dual &a, double b) { a = a / b; return a; }
#define DGPU_DUAL_CMP(op)                                                  \
  HD bool operator op(const Dual &a, const Dual &b) { return a.v op b.v; } \
  HD bool operator op(const Dual &a, double b) { return a.v op b; }        \
  HD bool operator op(double a, const Dual &b) { return a op b.v; }
DGPU_DUAL_CMP(<)
DGPU_DUAL_CMP(>)
DGPU_DUAL_CMP(<=)
DGPU_DUAL_CMP(>=)
DGPU_DUAL_CMP(==)
DGPU_DUAL_CMP(!=)
#undef DGPU_DUAL_CMP

HD Dual sqrt(const Dual &a) {
  const double s = ::sqrt(a.v);
  return Dual(s, a.d / (2.0 * s));
}
HD Dual fabs(const Dual &a) { return a.v < 0.0 ? Dual(-a.v, -a.d) : a; }
HD Dual pow(const Dual &a, double y) {
  const double p = ::pow(a.v, y);
  return Dual(p, y * ::pow(a.v, y - 1.0) * a.d);
}
HD Dual exp(const Dual &a) {
  const double e = ::exp(a.v);
  return Dual(e, e * a.d);
}

// ---------------------------------------------------------------------------
// Loads and stores of a per-cell / per-face variable with its tangent
// ---------------------------------------------------------------------------
template <typename T> struct Fld;
template <> struct Fld<double> {
  static HD double ld(const double *v, const double *, size_t i) { return v[i]; }
  static HD void st(double *v, double *, size_t i, double x) { v[i] = x; }
  static HD double mk(double v, double) { return v; }
};
template <> struct Fld<Dual> {
  static HD Dual ld(const double *v, const double *d, size_t i) { return Dual(v[i], d[i]); }
  static HD void st(double *v, double *d, size_t i, const Dual &x) {
    v[i] = x.v;
    d[i] = x.d;
  }
  static HD Dual mk(double v, double d) { return Dual(v, d); }
};

HD double ld(const double *p, int q, int n, int g) { return p[(size_t)q * n + g]; }
template <typename T>
HD T ldq(const double *v, const double *d, int q, int n, int g) {
  return Fld<T>::ld(v, d, (size_t)q * n + g);
}

// Loads of data that no thread of the running kernel writes (or that only
// the loading thread writes, after the load).  On the device they take the
// read-only path (ld.global.nc), so the compiler may issue them ahead of the
// kernel's stores instead of one dependent round trip after another.
template <typename X>
HD X rd(const X *p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
HD double ldr(const double *p, int q, int n, int g) { return rd(p + (size_t)q * n + g); }

// Starts moving the line holding *p into L2 without waiting for it (no
// register, no effect on results): the later load of the same line then
// waits on L2 instead of HBM.  Every address given here is inside its array.
__device__ __forceinline__ void pf(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// The same for the n-plane SoA value of cell g in each plane.
__device__ __forceinline__ void pf_planes(const double *p, int planes, int n, int g) {
  for (int q = 0; q < planes; ++q) pf(p + (size_t)q * n + g);
}
template <typename T> struct FldR;
template <> struct FldR<double> {
  static HD double ld(const double *v, const double *, size_t i) { return rd(v + i); }
};
template <> struct FldR<Dual> {
  static HD Dual ld(const double *v, const double *d, size_t i) { return Dual(rd(v + i), rd(d + i)); }
};
template <typename T>
HD T ldqr(const double *v, const double *d, int q, int n, int g) {
  return FldR<T>::ld(v, d, (size_t)q * n + g);
}
template <typename T>
HD void stq(double *v, double *d, int q, int n, int g, const T &x) {
  Fld<T>::st(v, d, (size_t)q * n + g, x);
}

// ---------------------------------------------------------------------------
// Error flags and the reference's bounded phi loops
// ---------------------------------------------------------------------------
HD void set_err(int *err, int flag) {
#ifdef __CUDA_ARCH__
  atomicOr(err, flag);
#else
  *err |= flag;
#endif
}

// while(dp > PHIMAX) dp -= PHIMAX; while(dp < 0.0) dp += PHIMAX;  (bounded)
HD double wrap_pos(double dp, int *err) {
  int it = 0;
  while (dp > PHIMAX) {
    dp -= PHIMAX;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return dp; }
  }
  while (dp < 0.0) {
    dp += PHIMAX;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return dp; }
  }
  return dp;
}
// while(dp > PHIMAX/2.) dp -= PHIMAX; while(dp < -PHIMAX/2.) dp += PHIMAX;  (bounded)
HD double wrap_pm(double dp, int *err) {
  int it = 0;
  while (dp > PHIMAX / 2.) {
    dp -= PHIMAX;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return dp; }
  }
  while (dp < -PHIMAX / 2.) {
    dp += PHIMAX;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return dp; }
  }
  return dp;
}

// while (x - y > h) y += p; while (x - y < -h) y -= p;  (bounded: the RK phase
// adjustments of cell_update_phi and gravMass_update_RK)
HD double adjust_toward(double x, double y, double h, double per, int *err) {
  int it = 0;
  while (x - y > h) {
    y += per;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return y; }
  }
  while (x - y < -h) {
    y -= per;
    if (++it > DGPU_WRAP_LIMIT) { set_err(err, DGPU_EF_WRAP_LIMIT); return y; }
  }
  return y;
}

// pow for the exponents the step uses: x^1 = x and x^2 = x*x are the correctly
// rounded values; x^1.5 = x*sqrt(x) and x^-1.5 = 1/(x*sqrt(x)) are within 2 ulp
// (like CUDA's pow, which also differs from the host libm in the last ulp).
HD double dpow(double x, double y) {
  if (y == 1.0) return x;
  if (y == 2.0) return x * x;
  if (y == 1.5) return x * sqrt(x);
  if (y == -1.5) return 1.0 / (x * sqrt(x));
  return pow(x, y);
}
HD Dual dpow(const Dual &x, double y) {
  const double p = dpow(x.v, y);
  double dp;
  if (y == 1.0) dp = x.d;
  else if (y == 2.0) dp = 2.0 * x.v * x.d;
  else dp = y * (p / x.v) * x.d;
  return Dual(p, dp);
}
// d/dx of dpow(x, y) given p = dpow(x, y) (x > 0 for the fractional exponents)
HD double dpow_dx(double x, double y, double p) {
  if (y == 1.0) return 1.0;
  if (y == 2.0) return 2.0 * x;
  return y * (p / x);
}

// sim_rOm_a / sim_rdrOm_a / sim_dtOm_a for A_MILOS (src/Sim/sim_w_a.c:8-72);
// other frame types use the host-computed annulus tables.
HD double milos_rom(double r, double a) {
  const int n = 8;
  return r * (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
}
HD double milos_rdrom(double r, double a) {
  const int n = 8;
  double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
  double arn = pow(a / r, n);
  return ((-1.5 + n * arn / (1. + arn)) * Omega_a +
          (1.5 - n) * pow(a / r, n - 1.5) / (1. + arn) * pow(r, -1.5));
}
HD double milos_dtom(double r, double a, double tau) {
  const int n = 8;
  double a0 = 1.0;
  double dta_o_a = -.25 * pow(a / a0, -4) / tau;
  double Omega_a = (pow(r, n - 1.5) + pow(a, n - 1.5)) / (pow(r, n) + pow(a, n));
  double arn = pow(a / r, n);
  if (a > 0.0) return (dta_o_a * (Omega_a * (-1.5 + n / (1. + arn)) + (1.5 - n) * pow(r, -1.5) / (1. + arn)));
  return 0.0;
}
HD double frame_rom(const DiskParams &P, double tab, double r, double a) {
  return P.w_analytic == DA_MILOS ? milos_rom(r, a) : tab;
}
HD double frame_rdrom(const DiskParams &P, double tab, double r, double a) {
  return P.w_analytic == DA_MILOS ? milos_rdrom(r, a) : tab;
}
HD double frame_dtom(const DiskParams &P, double tab, double r, double a) {
  return P.w_analytic == DA_MILOS ? milos_dtom(r, a, P.orb_tscale) : tab;
}

// gravMass_dist (src/GravMass/GravMass_access.c:25-31) from the point's
// x = r cos(phi), y = r sin(phi) and the mass position (xbh, ybh).
template <typename T>
HD T gm_dist_xy(double x, double y, const T &xbh, const T &ybh) {
  double z = 0.;
  return sqrt((x - xbh) * (x - xbh) + (y - ybh) * (y - ybh) + z * z);
}

// fgrav (src/Cell/cell_source.c:11-13)
template <typename T>
HD T fgrav(const T &M, const T &r, double eps, int n) {
  return (M * dpow(r, n - 1.) / dpow(dpow(r, n) + dpow(eps, n), 1. + 1. / n));
}

// ---------------------------------------------------------------------------
// Riemann solver: riemann_set_vel / _set_state / _set_flux / _set_star_hll /
// _set_star_hllc and the flux choice of riemann_AddFlux
// (src/Riemann/Riemann_routines.c:14-191,314-371).  dir 0 = r face, 1 = phi, 2 = z.
// ---------------------------------------------------------------------------
template <typename T>
HD void phys_flux(const T *p, double r, double n0, double n1, double n2, double gam, T *F) {
  T rho = p[D_RHO];
  T Pp = p[D_PPP];
  T vr = p[D_URR];
  T vp = p[D_UPP] * r;
  T vz = p[D_UZZ];
  T vn = vr * n0 + vp * n1 + vz * n2;
  T rhoe = Pp / (gam - 1.);
  T v2 = vr * vr + vp * vp + vz * vz;
  F[D_DDD] = rho * vn;
  F[D_SRR] = rho * vr * vn + Pp * n0;
  F[D_LLL] = r * (rho * vp * vn + Pp * n1);
  F[D_SZZ] = rho * vz * vn + Pp * n2;
  F[D_TAU] = (.5 * rho * v2 + rhoe + Pp) * vn;
}
// cell_prim2cons (src/Cell/cell_conversion.c:11-33)
template <typename T>
HD void prim2cons(const T *p, T *U, double r, double dV, double gam) {
  T rho = p[D_RHO];
  T Pp = p[D_PPP];
  T vr = p[D_URR];
  T vp = p[D_UPP] * r;
  T vz = p[D_UZZ];
  T v2 = vr * vr + vp * vp + vz * vz;
  T rhoe = Pp / (gam - 1.);
  U[D_DDD] = rho * dV;
  U[D_SRR] = rho * vr * dV;
  U[D_LLL] = r * rho * vp * dV;
  U[D_SZZ] = rho * vz * dV;
  U[D_TAU] = (.5 * rho * v2 + rhoe) * dV;
}

template <typename T>
// np passive scalars (face states qL, qR) ride on the mass flux: their
// physical flux and conserved value are q F_D and q U_D (riemann_set_flux,
// Riemann_routines.c:184-189; cell_prim2cons, cell_conversion.c:28-31), their
// HLL star state follows Toro's formulas like the others and their HLLC star
// state is q U*_D (riemann_set_star_hllc, Riemann_routines.c:143-146).  The
// differentiated runs carry no passive scalar (np = 0).
HD void riemann_flux(const T *pL, const T *pR, double r, int dir, double w, double gam, int solver, T *F,
                     int np = 0, const double *qL = nullptr, const double *qR = nullptr, double *Fq = nullptr) {
  const double n0 = dir == 0 ? 1.0 : 0.0, n1 = dir == 1 ? 1.0 : 0.0, n2 = dir == 2 ? 1.0 : 0.0;
  T vnL, cf2L, vnR, cf2R;
  {
    T P = pL[D_PPP], rho = pL[D_RHO], vr = pL[D_URR], vp = r * pL[D_UPP], vz = pL[D_UZZ];
    vnL = vr * n0 + vp * n1 + vz * n2;
    cf2L = gam * (P / rho);
  }
  {
    T P = pR[D_PPP], rho = pR[D_RHO], vr = pR[D_URR], vp = r * pR[D_UPP], vz = pR[D_UZZ];
    vnR = vr * n0 + vp * n1 + vz * n2;
    cf2R = gam * (P / rho);
  }
  T Sl = vnL - sqrt(cf2L);
  T Sr = vnL + sqrt(cf2L);
  if (Sl > vnR - sqrt(cf2R)) Sl = vnR - sqrt(cf2R);
  if (Sr < vnR + sqrt(cf2R)) Sr = vnR + sqrt(cf2R);
  T Ss = (pR[D_RHO] * vnR * (Sr - vnR) - pL[D_RHO] * vnL * (Sl - vnL) + pL[D_PPP] - pR[D_PPP]) /
         (pR[D_RHO] * (Sr - vnR) - pL[D_RHO] * (Sl - vnL));
  int state;
  if (w < Sl) state = DS_LEFT;
  else if (w > Sr) state = DS_RIGHT;
  else if (w < Ss) state = DS_LEFTSTAR;
  else state = DS_RIGHTSTAR;

  T Fk[5], Uk[5];
  if (state == DS_LEFT || state == DS_RIGHT) {
    const T *p = state == DS_LEFT ? pL : pR;
    phys_flux(p, r, n0, n1, n2, gam, Fk);
    prim2cons(p, Uk, r, 1.0, gam);
#pragma unroll
    for (int q = 0; q < 5; ++q) F[q] = Fk[q] - w * Uk[q];
    for (int k = 0; k < np; ++k) {
      const double qk = state == DS_LEFT ? qL[k] : qR[k];
      const double Fkq = qk * val(Fk[D_DDD]), Ukq = qk * val(Uk[D_DDD]);
      Fq[k] = Fkq - w * Ukq;
    }
    return;
  }
  T Ustar[5], Fstar[5];
  if (solver == DR_HLL) {
    T FL[5], FR[5], UL[5], UR[5];
    phys_flux(pL, r, n0, n1, n2, gam, FL);
    phys_flux(pR, r, n0, n1, n2, gam, FR);
    prim2cons(pL, UL, r, 1.0, gam);
    prim2cons(pR, UR, r, 1.0, gam);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      Ustar[q] = (Sr * UR[q] - Sl * UL[q] + FL[q] - FR[q]) / (Sr - Sl);
      Fstar[q] = (Sr * FL[q] - Sl * FR[q] - Sr * Sl * (UL[q] - UR[q])) / (Sr - Sl);
    }
    for (int k = 0; k < np; ++k) {
      const double sr = val(Sr), sl = val(Sl);
      const double FLq = qL[k] * val(FL[D_DDD]), FRq = qR[k] * val(FR[D_DDD]);
      const double ULq = qL[k] * val(UL[D_DDD]), URq = qR[k] * val(UR[D_DDD]);
      const double Usq = (sr * URq - sl * ULq + FLq - FRq) / (sr - sl);
      const double Fsq = (sr * FLq - sl * FRq - sr * sl * (ULq - URq)) / (sr - sl);
      Fq[k] = Fsq - w * Usq;
    }
  } else {
    const T *prim = state == DS_LEFTSTAR ? pL : pR;
    T Sk = state == DS_LEFTSTAR ? Sl : Sr;
    phys_flux(prim, r, n0, n1, n2, gam, Fk);
    prim2cons(prim, Uk, r, 1.0, gam);
    T rho = prim[D_RHO];
    T vr = prim[D_URR];
    T vp = prim[D_UPP] * r;
    T vz = prim[D_UZZ];
    T Pp = prim[D_PPP];
    T v2 = vr * vr + vp * vp + vz * vz;
    T vn = vr * n0 + vp * n1 + vz * n2;
    T rhoe = Pp / (gam - 1.);
    T D = rho;
    T mr = rho * vr;
    T mp = rho * vp;
    T mz = rho * vz;
    T E_hydro = .5 * rho * v2 + rhoe;
    T Ps = rho * (Sk - vn) * (Ss - vn) + Pp;
    T Dstar = (Sk - vn) * D / (Sk - Ss);
    T Msn = Dstar * Ss;
    T Msr = (Sk - vn) * mr / (Sk - Ss);
    T Msp = (Sk - vn) * mp / (Sk - Ss);
    T Msz = (Sk - vn) * mz / (Sk - Ss);
    T Estar = ((Sk - vn) * E_hydro + Ps * Ss - Pp * vn) / (Sk - Ss);
    T mn = Msr * n0 + Msp * n1 + Msz * n2;
    Msr += n0 * (Msn - mn);
    Msp += n1 * (Msn - mn);
    Msz += n2 * (Msn - mn);
    Ustar[D_DDD] = Dstar;
    Ustar[D_SRR] = Msr;
    Ustar[D_LLL] = r * Msp;
    Ustar[D_SZZ] = Msz;
    Ustar[D_TAU] = Estar;
#pragma unroll
    for (int q = 0; q < 5; ++q) Fstar[q] = Fk[q] + Sk * (Ustar[q] - Uk[q]);
    for (int k = 0; k < np; ++k) {
      const double qk = state == DS_LEFTSTAR ? qL[k] : qR[k];
      const double Fkq = qk * val(Fk[D_DDD]), Ukq = qk * val(Uk[D_DDD]);
      const double Usq = qk * val(Ustar[D_DDD]);
      const double Fsq = Fkq + val(Sk) * (Usq - Ukq);
      Fq[k] = Fsq - w * Usq;
    }
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) F[q] = Fstar[q] - w * Ustar[q];
}

// Inputs of riemann_visc_flux (src/Riemann/Riemann_routines.c:193-311).
template <typename T>
struct ViscIn {
  T cL[5], cR[5];               // cell prims
  T gpL[5], gpR[5];             // cell gradp
  T grL[5], grR[5];             // cell grad
  double tL, tR;                // cell tiph (wrapped)
  double dpL, dpR;              // r faces: wrapped offsets of the face centre (k_rslope)
  double r, cm, r_cell_L, r_cell_R;
  double rdr_om;                // sim_rdrOm_a at r
};
// Binary point-mass positions and masses of the substep, and alpha, as T
// (the tangent carries their derivatives with respect to q and alpha).
template <typename T>
struct GravT {
  T gx[2], gy[2], gM[2], alpha;
};

// The reference forms the face average and the gradients of the viscous flux
// from the reconstructed states first and then overwrites them (r faces: Avg
// and Gr from the cell prims offset to the face centre; phi faces: Avg and Gp
// from the cell prims), so the reconstructed states never reach the flux.
template <typename T>
HD void visc_flux(const ViscIn<T> &v, int dir, const DiskParams &P, const GravT<T> &G, T *Fv, int *err) {
  const double r = v.r;
  T Avg[5], Gr[5], Gp[5];
  if (dir == 0) {
    const double dpL = v.dpL, dpR = v.dpR;
    double deltaL = v.r - v.r_cell_L;
    double deltaR = v.r_cell_R - v.r;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      T WL = v.cL[q] + dpL * v.gpL[q];
      T WR = v.cR[q] - dpR * v.gpR[q];
      Avg[q] = 0.5 * (WL + WR);
      Gr[q] = (WR - WL) / (deltaR + deltaL);
      Gp[q] = .5 * (v.gpL[q] + v.gpR[q]) / r;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Avg[q] = 0.5 * (v.cR[q] + v.cL[q]);
      Gp[q] = (v.cR[q] - v.cL[q]) / (v.tR - v.tL) / r;
      Gr[q] = .5 * (v.grL[q] + v.grR[q]);
    }
  }
  {
    // the v_z check of the reference (Riemann_routines.c:271-274)
    double vz = dir == 0 ? .5 * ((val(v.cL[D_UZZ]) + v.dpL * val(v.gpL[D_UZZ])) +
                                 (val(v.cR[D_UZZ]) - v.dpR * val(v.gpR[D_UZZ])))
                         : .5 * (val(v.cR[D_UZZ]) + val(v.cL[D_UZZ]));
    if (fabs(vz) > 1.e-12) set_err(err, DGPU_EF_VISC_VZ);
  }
  T nu;
  if (P.visc_const == 1) {
    nu = G.alpha;
  } else if (P.init_type == DI_SHEAR) {
    nu = G.alpha * P.gamma * Avg[D_PPP] / Avg[D_RHO] * dpow(fabs(r * cos(v.cm)), 2.0);
    if (r * cos(v.cm) > 20.) nu = 0.0;
  } else {
    double sc, cc;
    sincos(v.cm, &sc, &cc);
    const double x = r * cc, y = r * sc;
    T d0 = gm_dist_xy(x, y, G.gx[0], G.gy[0]);
    T d1 = gm_dist_xy(x, y, G.gx[1], G.gy[1]);
    double eps = P.g_eps;
    nu = G.alpha * Avg[D_PPP] / Avg[D_RHO] /
         sqrt(dpow(d0 * d0 + eps * eps, -1.5) * G.gM[0] + dpow(d1 * d1 + eps * eps, -1.5) * G.gM[1]);
  }
  T rho = Avg[D_RHO];
  T vr = Avg[D_URR];
  T om = Avg[D_UPP];
  T Gr_vr = Gr[D_URR], Gr_om = Gr[D_UPP];
  T Gp_vr = Gp[D_URR], Gp_om = Gp[D_UPP];
  double rdr = v.rdr_om;
  if (dir == 0) {
    Fv[0] = -nu * rho * (r * Gr_vr - vr - r * r * Gp_om);
    Fv[1] = -nu * rho * (r * (r * Gr_om + rdr) + r * Gp_vr);
    Fv[2] = -nu * rho * (vr * (Gr_vr - vr / r - r * Gp_om) + r * om * (Gp_vr + (rdr + r * Gr_om)));
  } else {
    Fv[0] = -nu * rho * (r * (r * Gr_om + rdr) + r * Gp_vr);
    Fv[1] = -nu * rho * (-r * Gr_vr + vr + r * r * Gp_om);
    Fv[2] = -nu * rho * (-r * om * (Gr_vr - vr / r - r * Gp_om) + vr * (Gp_vr + (rdr + r * Gr_om)));
  }
}

// ---------------------------------------------------------------------------
// Per-cell pieces of the substep shared by the forward, tangent and adjoint
// ---------------------------------------------------------------------------
// cell_plm_p slope of one variable (src/Cell/cell_plm.c:116-161): theta-
// generalised minmod of the left, right and centred differences.
template <typename T>
HD T plm_p_slope(const T &pl, const T &pc, const T &pr, double dpL, double dpR, double plm) {
  T sL = (pc - pl) / dpL;
  T sR = (pr - pc) / dpR;
  T sM = (pr - pl) / (dpL + dpR);
  T sv = plm * sL;
  if (fabs(sv) > plm * fabs(sR)) sv = plm * sR;
  if (fabs(sv) > fabs(sM)) sv = sM;
  if (sL * sR < 0.0) sv = 0.0;
  return sv;
}

// Geometry and frame terms of cell_add_src / cell_add_visc_src for one cell
// (src/Cell/cell_source.c:73-277): everything that does not depend on the state.
struct SrcGeom {
  double r, dV, dt, cosp, sinp, xpos, ypos, sint, cost, gravdist;
  double Fc;     // centrifugal w_a^2 / r
  double dtOm;   // sim_dtOm_a
  double rdrOm;  // sim_rdrOm_a
};
// Source increments s[0..5] (S_r pressure/centrifugal, S_r gravity + frame, L,
// S_z, tau, viscous heating) from the prims, grad[UPP], gradp[URR] and the
// binary; sinks are handled by the caller.
template <typename T>
HD void source_cell(const SrcGeom &g, const DiskParams &P, const T *pm, const T &grad_upp, const T &gradp_urr,
                    const GravT<T> &G, T *s) {
  T rho = pm[D_RHO];
  T Pp = pm[D_PPP];
  T vr = pm[D_URR];
  T vz = pm[D_UZZ];
  T vp = pm[D_UPP] * g.r;
  T Fr = 0.0, Fp = 0.0;
  for (int p = 0; p < 2; ++p) {
    // gravMassForce (src/Cell/cell_source.c:49-71)
    T dx = g.gravdist * g.cosp - G.gx[p];
    T dy = g.gravdist * g.sinp - G.gy[p];
    T script_r = sqrt(dx * dx + dy * dy);
    T cosa = dx / script_r;
    T sina = dy / script_r;
    T cosap = cosa * g.cosp + sina * g.sinp;
    T sinap = sina * g.cosp - cosa * g.sinp;
    T f1 = -fgrav(G.gM[p], script_r, P.g_eps, P.phi_order);
    Fr += cosap * f1;
    Fp += sinap * f1;
  }
  T F_euler_phi = -(g.r * g.dtOm + vr * g.rdrOm);
  s[0] = g.dt * g.dV * (rho * vp * vp + Pp) / g.r;
  s[1] = g.dt * g.dV * rho * (Fr * g.sint + g.Fc);
  s[2] = g.dt * g.dV * rho * (Fp - g.r * g.dtOm) * g.r;
  s[3] = g.dt * g.dV * rho * Fr * g.cost;
  s[4] = g.dt * g.dV * rho * ((Fr * g.sint + g.Fc) * vr + Fr * vz * g.cost + (Fp + F_euler_phi) * vp);
  s[5] = 0.0;
  if (P.has_visc) {
    T dist_bh0 = sqrt((g.xpos - G.gx[0]) * (g.xpos - G.gx[0]) + (g.ypos - G.gy[0]) * (g.ypos - G.gy[0]));
    T dist_bh1 = sqrt((g.xpos - G.gx[1]) * (g.xpos - G.gx[1]) + (g.ypos - G.gy[1]) * (g.ypos - G.gy[1]));
    double eps = P.g_eps;
    T Sigma_nu;
    if (P.visc_const == 1) {
      Sigma_nu = rho * G.alpha;
    } else {
      Sigma_nu = G.alpha * Pp /
                 sqrt(dpow(dist_bh0 * dist_bh0 + eps * eps, -1.5) * G.gM[0] +
                      dpow(dist_bh1 * dist_bh1 + eps * eps, -1.5) * G.gM[1]);
    }
    s[5] = g.dt * g.dV * Sigma_nu * g.rdrOm * (g.rdrOm + g.r * grad_upp + gradp_urr);
  }
}

// Exact epicyclic rotation of (S_r, L) of cell_add_split_fictitious
// (src/Cell/cell_add_split_fictitious.c:26-38), kappa > 0.
template <typename T>
HD void split_rotate(T *c, double ck, double sk, double dr_r2Om, double kappa, double Omega, double r) {
  T l0 = c[D_LLL];
  T rhov0 = c[D_SRR];
  T l = l0 * ck - c[D_SRR] * dr_r2Om / kappa * sk;
  T rhov = rhov0 * ck + 2.0 * Omega * c[D_LLL] / r / kappa * sk;
  c[D_LLL] = l;
  c[D_SRR] = rhov;
}

// cell_cons2prim (src/Cell/cell_conversion.c:57-122): density floor, sound-
// speed floor and cap, velocity cap.
template <typename T>
HD void cons2prim(const T *c, double dV, double r, const DiskParams &P, T *pr) {
  T rho = c[D_DDD] / dV;
  if (rho < P.rho_floor) rho = P.rho_floor;
  T Sr = c[D_SRR] / dV;
  T Sp = c[D_LLL] / dV / r;
  T Sz = c[D_SZZ] / dV;
  T E = c[D_TAU] / dV;
  T vr = Sr / rho;
  T vp = Sp / rho;
  T vz = Sz / rho;
  T KE = .5 * (Sr * vr + Sp * vp + Sz * vz);
  T v_magnitude = sqrt(2. * KE / rho);
  T rhoe = E - KE;
  T Pp = (P.gamma - 1.) * rhoe;
  if (Pp < P.cs_floor * P.cs_floor * rho / P.gamma) Pp = P.cs_floor * P.cs_floor * rho / P.gamma;
  if (Pp > P.cs_cap * P.cs_cap * rho / P.gamma) Pp = P.cs_cap * P.cs_cap * rho / P.gamma;
  if (v_magnitude > P.vel_cap) {
    vr = vr * P.vel_cap / v_magnitude;
    vp = vp * P.vel_cap / v_magnitude;
    vz = vz * P.vel_cap / v_magnitude;
  }
  pr[D_RHO] = rho;
  pr[D_PPP] = Pp;
  pr[D_URR] = vr;
  pr[D_UPP] = vp / r;
  pr[D_UZZ] = vz;
}

// ---------------------------------------------------------------------------
// r faces of a cell in the reference's accumulation order
// ---------------------------------------------------------------------------
struct RFace {
  int cL, cR;
  double dphi, cm;
  double r, dl, dr, dperp;
};

// Calls f(face) for every r face of cell g in the reference's face order:
// first the faces of pair (i-1, i) where g is the outer cell, then the faces
// of pair (i, i+1) where g is the inner cell.
template <typename Fn>
__device__ __forceinline__ void for_cell_rfaces(const DevPtrs &d, const Annulus &A, int a, int g, int NR,
                                                Fn f) {
  const int j = g - A.cell_off;
  if (A.i > 0) {
    const Annulus &Q = d.ann[a - 1];
    const int4 rr = rd(reinterpret_cast<const int4 *>(d.rr) + g);
    auto one = [&](int n) {
      RFace F;
      F.cL = rd(d.fL + Q.face_base + n);
      F.cR = g;
      F.dphi = rd(d.fdphi + Q.face_base + n);
      F.cm = rd(d.fcm + Q.face_base + n);
      F.r = Q.f_r;
      F.dl = Q.f_dl;
      F.dr = Q.f_dr;
      F.dperp = Q.f_dperp;
      f(F, Q.face_base + n, 1);
    };
    if (rr.z != INT_MIN) {
      for (int n = rr.x; n < rr.y; ++n) one(n);
      for (int n = rr.z; n < rr.w; ++n) one(n);
    } else {
      // three or more runs (the outer pointer went round more than twice)
      const int T = rd(d.pair_T + a - 1);
      const int jpmin = rd(d.pair_jpmin + a - 1);
      int dd = j - jpmin;
      if (dd < 0) dd += A.np;
      const int *runs = d.runs + Q.run_base;
      for (int s = dd; s <= T; s += A.np)
        for (int n = rd(runs + s); n < rd(runs + s + 1); ++n) one(n);
    }
  }
  if (A.i < NR - 1) {
    const int nf = rd(d.pair_nf + a);
    int n0 = rd(d.fstart + g);
    int n1 = (j + 1 < A.np) ? rd(d.fstart + g + 1) : nf;
    if (nf <= 0) n1 = n0;
    for (int n = n0; n < n1; ++n) {
      RFace F;
      F.cL = g;
      F.cR = rd(d.fR + A.face_base + n);
      F.dphi = rd(d.fdphi + A.face_base + n);
      F.cm = rd(d.fcm + A.face_base + n);
      F.r = A.f_r;
      F.dl = A.f_dl;
      F.dr = A.f_dr;
      F.dperp = A.f_dperp;
      f(F, A.face_base + n, 0);
    }
  }
}


// The same faces as for_cell_rfaces, in the same order, as contiguous slot
// ranges: f(first slot, end slot, side) with side 1 for the faces of pair
// (i-1, i) (the cell is their outer cell) and 0 for those of pair (i, i+1).
template <typename Fn>
__device__ __forceinline__ void for_cell_rface_ranges(const DevPtrs &d, const Annulus &A, int a, int g, int NR,
                                                      Fn f) {
  const int j = g - A.cell_off;
  if (A.i > 0) {
    const Annulus &Q = d.ann[a - 1];
    const int4 rr = rd(reinterpret_cast<const int4 *>(d.rr) + g);
    if (rr.z != INT_MIN) {
      f(Q.face_base + rr.x, Q.face_base + rr.y, 1);
      f(Q.face_base + rr.z, Q.face_base + rr.w, 1);
    } else {
      const int T = rd(d.pair_T + a - 1);
      const int jpmin = rd(d.pair_jpmin + a - 1);
      int dd = j - jpmin;
      if (dd < 0) dd += A.np;
      const int *runs = d.runs + Q.run_base;
      for (int s = dd; s <= T; s += A.np) f(Q.face_base + rd(runs + s), Q.face_base + rd(runs + s + 1), 1);
    }
  }
  if (A.i < NR - 1) {
    const int nf = rd(d.pair_nf + a);
    int n0 = rd(d.fstart + g);
    int n1 = (j + 1 < A.np) ? rd(d.fstart + g + 1) : nf;
    if (nf <= 0) n1 = n0;
    f(A.face_base + n0, A.face_base + n1, 0);
  }
}

// The z faces of cell g of ring a (3-D disks) in the reference's face order
// (face_create with direction 1 lists them layer pair after layer pair):
// those of the z pair (a-NR, a), where g is the upper cell, then those of
// (a, a+NR), where it is the lower cell, as contiguous slot ranges:
// f(first slot, end slot, side), side 1 for the upper cell, 0 for the lower.
template <typename Fn>
__device__ __forceinline__ void for_cell_zface_ranges(const DevPtrs &d, const Annulus &A, int a, int g, int NR,
                                                      int NZ, Fn f) {
  const int j = g - A.cell_off;
  if (A.k > 0) {
    const Annulus &Q = d.ann[a - NR];
    const int4 rr = rd(reinterpret_cast<const int4 *>(d.zrr) + g);
    if (rr.z != INT_MIN) {
      f(Q.zface_base + rr.x, Q.zface_base + rr.y, 1);
      f(Q.zface_base + rr.z, Q.zface_base + rr.w, 1);
    } else {
      const int T = rd(d.zpair_T + a - NR);
      const int jpmin = rd(d.zpair_jpmin + a - NR);
      int dd = j - jpmin;
      if (dd < 0) dd += A.np;
      const int *runs = d.zruns + Q.zrun_base;
      for (int s = dd; s <= T; s += A.np) f(Q.zface_base + rd(runs + s), Q.zface_base + rd(runs + s + 1), 1);
    }
  }
  if (A.k < NZ - 1) {
    const int nf = rd(d.zpair_nf + a);
    int n0 = rd(d.zfstart + g);
    int n1 = (j + 1 < A.np) ? rd(d.zfstart + g + 1) : nf;
    if (nf <= 0) n1 = n0;
    f(A.zface_base + n0, A.zface_base + n1, 0);
  }
}

}  // namespace

#endif
