// Device functions of the substep shared by the forward/tangent kernels
// (dgpu_kernels.cu) and the adjoint kernels (dgpu_adjoint.cu).
#ifndef DGPU_STEP_CUH
#define DGPU_STEP_CUH

#include <type_traits>

#include "dgpu_device.cuh"

namespace {

// GravMass positions and masses of the substep and alpha as T: the tangent
// seeds of TanPtrs give d/de of M_p and of the orbit radius r_p (the positions
// are r_p (cos, sin) of the orbit phase, which has no tangent).
template <typename T>
__device__ __forceinline__ void grav_t(GravT<T> &G, const InstState &S, const DiskParams &P, const TanPtrs &tp,
                                       int inst) {
  if constexpr (std::is_same<T, Dual>::value) {
    const double *sd = tp.seed + (size_t)DGPU_TP_N * inst;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      G.gM[p] = Dual(S.gM[p], sd[DGPU_TP_DM0 + p]);
      G.gx[p] = Dual(S.gx[p], sd[DGPU_TP_DR0 + p] * S.gc[p]);
      G.gy[p] = Dual(S.gy[p], sd[DGPU_TP_DR0 + p] * S.gs[p]);
    }
    G.alpha = Dual(P.visc, sd[DGPU_TP_DALPHA]);
  } else {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      G.gM[p] = S.gM[p];
      G.gx[p] = S.gx[p];
      G.gy[p] = S.gy[p];
    }
    G.alpha = P.visc;
  }
}

// Advanced phi edge of a cell (cell_update_phi, src/Cell/cell_misc.c:59-79).
__device__ __forceinline__ double new_tiph(double tw, double &rk, double RK, double w_total, double dt, double r,
                                           int *err) {
  rk = adjust_toward(tw, rk, PHIMAX / 2., PHIMAX, err);
  double t = (1.0 - RK) * tw + RK * rk;
  t += w_total * dt / r;
  return t;
}

// A face or source increment: through the read-only path (NC) when an earlier
// kernel wrote it, by a plain load when another block of the running kernel
// did.
template <typename T, bool NC>
__device__ __forceinline__ T ldinc(const double *v, const double *dv, int q, int n, int g) {
  if constexpr (NC) return ldqr<T>(v, dv, q, n, g);
  else return ldq<T>(v, dv, q, n, g);
}

// The conserved sum of a cell before cons2prim: cell_adjust_RK_cons, the phi
// and r face increments in the reference's order, cell_add_src, cooling,
// cell_add_visc_src and cell_add_split_fictitious (the forward stops after
// `stop` like the stage-parity path; returns false when it stopped early).
// Writes rkcons in substep 1 when `write_rk`.  NC: the increments and the
// annulus constants come from earlier kernels (see ldinc).
template <typename T, bool NC = true>
__device__ __forceinline__ bool update_sum(const DevPtrs &d, const TanPtrs &tp, const Annulus &A, int a, int g,
                                           int substep, int stop, double dt, bool write_rk, T *c) {
  const int N = d.n_cells;
  const DiskParams &P = d.par[A.inst];
  const InstState &S = d.ist[A.inst];
  const int j = g - A.cell_off;
  const int np = A.np;
  const double RK = substep == 1 ? 0.0 : 0.5;
  // cell_copy (substep 1) + cell_adjust_RK_cons (cell_misc.c:28-57)
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    T cq = ldqr<T>(d.cons, tp.cons, q, N, g);
    T rk;
    if (substep == 1) {
      rk = cq;
      if (write_rk) stq<T>(d.rkcons, tp.rkcons, q, N, g, cq);
    } else {
      rk = ldqr<T>(d.rkcons, tp.rkcons, q, N, g);
    }
    c[q] = (1.0 - RK) * cq + RK * rk;
  }
  if (stop <= 1) return false;
  // phi faces: for j = 0 the face (0,1) comes before (N-1,0)
  {
    const int gl = j == 0 ? A.cell_off + np - 1 : g - 1;
    const double r = .5 * (A.rp + A.rm);
    auto addL = [&](int f) {
#pragma unroll
      for (int q = 0; q < 5; ++q) c[q] -= ldinc<T, NC>(d.fphi, tp.fphi, q, N, f);
      if (P.has_visc) {
        c[D_SRR] -= ldinc<T, NC>(d.fphi, tp.fphi, 5, N, f) / r;
        c[D_LLL] -= ldinc<T, NC>(d.fphi, tp.fphi, 6, N, f);
        c[D_TAU] -= ldinc<T, NC>(d.fphi, tp.fphi, 7, N, f);
      }
    };
    auto addR = [&](int f) {
#pragma unroll
      for (int q = 0; q < 5; ++q) c[q] += ldinc<T, NC>(d.fphi, tp.fphi, q, N, f);
      if (P.has_visc) {
        c[D_SRR] += ldinc<T, NC>(d.fphi, tp.fphi, 5, N, f) / r;
        c[D_LLL] += ldinc<T, NC>(d.fphi, tp.fphi, 6, N, f);
        c[D_TAU] += ldinc<T, NC>(d.fphi, tp.fphi, 7, N, f);
      }
    };
    if (j == 0) {
      addL(g);
      addR(gl);
    } else {
      addR(gl);
      addL(g);
    }
  }
  if (stop == 2) return false;
  // r faces in face-list order, one face's increments at a time (two at a time
  // spill more at the kernel's 64-register budget)
  {
    const int NS = d.n_slots;
    const bool visc = P.has_visc;
    for_cell_rface_ranges(d, A, a, g, P.NR, [&](int s, int e, int asR) {
      // the outer cell's faces divide the viscous S_r part by its own radius
      const Annulus &Q = asR ? d.ann[a - 1] : A;
      const double rv = asR ? Q.f_r + Q.f_dr : Q.f_r - Q.f_dl;
      auto apply = [&](const T *u) {
        if (asR) {
#pragma unroll
          for (int q = 0; q < 5; ++q) c[q] += u[q];
          if (visc) {
            c[D_SRR] += u[5] / rv;
            c[D_LLL] += u[6];
            c[D_TAU] += u[7];
          }
        } else {
#pragma unroll
          for (int q = 0; q < 5; ++q) c[q] -= u[q];
          if (visc) {
            c[D_SRR] -= u[5] / rv;
            c[D_LLL] -= u[6];
            c[D_TAU] -= u[7];
          }
        }
      };
      for (int n = s; n < e; ++n) {
        T u[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < 5 || visc) u[q] = ldinc<T, NC>(d.frf, tp.frf, q, NS, n);
        apply(u);
      }
    });
  }
  // z faces of a 3-D disk, after the r faces (timestep_routines.c:63-71): the
  // increments of pair (a-NR, a) are added, those of (a, a+NR) subtracted.  Their
  // viscous flux is zero (riemann_visc_flux sets neither the r nor the phi
  // terms); adding its +0 to the upper cell keeps the reference's signed zeros.
  if constexpr (std::is_same<T, double>::value) {
    if (d.has_z && P.NZ > 1) {
      const int NSZ = d.n_zslots;
      const bool visc = P.has_visc;
      for_cell_zface_ranges(d, A, a, g, P.NR, P.NZ, [&](int s, int e, int up) {
        for (int n = s; n < e; ++n) {
          double u[5];
#pragma unroll
          for (int q = 0; q < 5; ++q) u[q] = NC ? ldr(d.zfrf, q, NSZ, n) : ld(d.zfrf, q, NSZ, n);
          if (up) {
#pragma unroll
            for (int q = 0; q < 5; ++q) c[q] += u[q];
            if (visc) {
              c[D_SRR] += 0.0;
              c[D_LLL] += 0.0;
              c[D_TAU] += 0.0;
            }
          } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) c[q] -= u[q];
          }
        }
      });
    }
  }
  if (stop == 3) return false;
  // cell_add_src, cell_add_visc_src, cell_add_split_fictitious: the source
  // increments come from k_source; added here in the reference's order
  c[D_SRR] += ldinc<T, NC>(d.src, tp.src, 0, N, g);
  c[D_SRR] += ldinc<T, NC>(d.src, tp.src, 1, N, g);
  c[D_LLL] += ldinc<T, NC>(d.src, tp.src, 2, N, g);
  c[D_SZZ] += ldinc<T, NC>(d.src, tp.src, 3, N, g);
  c[D_TAU] += ldinc<T, NC>(d.src, tp.src, 4, N, g);
  if (P.rho_sink_on == 1) {
    for (int p = 0; p < P.num_sinks && p < 2; ++p) c[D_DDD] -= ldinc<T, NC>(d.src, tp.src, 6 + p, N, g);
  }
  const double rm = A.rm, rp = A.rp;
  const double r = .5 * (rp + rm);
  if (P.cooling == 1) {
    // cooling reads the running tau (cell_source.c:187-203)
    const T rho = ldqr<T>(d.prim, tp.prim, D_RHO, N, g), Pp = ldqr<T>(d.prim, tp.prim, D_PPP, N, g);
    const double dV = rd(d.dphi + g) * .5 * A.dv_diff * A.dz;
    if (P.init_type == DI_SHEAR) {
      T cooling_term = (Pp - .01) / (P.gamma - 1.) * dV / 1.e-2;
      if (cooling_term < 0.0) cooling_term = 0.0;
      c[D_TAU] -= cooling_term * dt;
    } else {
      double numfac = 1.0;
      double alpha = P.visc;
      T cooling_cap = c[D_TAU] * numfac;
      T cooling_term = 9. / 4. * alpha * pow(P.poro_r1, -3) / rho * pow(Pp / rho, 4.) * dt * dV;
      if (cooling_term > cooling_cap) cooling_term = cooling_cap;
      c[D_TAU] -= cooling_term;
    }
  }
  if (P.has_visc) c[D_TAU] += ldinc<T, NC>(d.src, tp.src, 5, N, g);
  // cell_add_split_fictitious (src/Cell/cell_add_split_fictitious.c:11-44)
  {
    const double a_sep = S.gr[0] + S.gr[1];
    const double rom = frame_rom(P, A.rom, r, a_sep);
    const double Omega = rom / r;
    const double dr_r2Om = 2. * rom + r * frame_rdrom(P, A.rdrom, r, a_sep);
    const int NA = d.n_ann;
    const double kappa = NC ? rd(d.ann_c + a) : d.ann_c[a];  // sqrt(kappa2) when kappa2 > 0, else 0
    if (kappa > 0.)
      split_rotate(c, NC ? rd(d.ann_c + NA + a) : d.ann_c[NA + a], NC ? rd(d.ann_c + 2 * NA + a) : d.ann_c[2 * NA + a],
                   dr_r2Om, kappa, Omega, r);
  }
  return stop > 4;
}

// The conserved sums of a cell's passive scalars (planes 5.. of cons): the RK
// blend and the phi and r face increments (planes 8.. of fphi and frf) in the
// same order as update_sum; no source acts on them.  Writes rkcons in
// substep 1.
__device__ __forceinline__ void passive_sum(const DevPtrs &d, const Annulus &A, int a, int g, int substep,
                                            int stop, int np, double *cp) {
  const int N = d.n_cells, NS = d.n_slots;
  const int j = g - A.cell_off;
  const double RK = substep == 1 ? 0.0 : 0.5;
  for (int k = 0; k < np; ++k) {
    const double cq = ld(d.cons, 5 + k, N, g);
    double rk;
    if (substep == 1) {
      rk = cq;
      d.rkcons[(size_t)(5 + k) * N + g] = cq;
    } else {
      rk = ld(d.rkcons, 5 + k, N, g);
    }
    cp[k] = (1.0 - RK) * cq + RK * rk;
  }
  if (stop <= 1) return;
  {
    const int gl = j == 0 ? A.cell_off + A.np - 1 : g - 1;
    for (int k = 0; k < np; ++k) {
      if (j == 0) {
        cp[k] -= ld(d.fphi, 8 + k, N, g);
        cp[k] += ld(d.fphi, 8 + k, N, gl);
      } else {
        cp[k] += ld(d.fphi, 8 + k, N, gl);
        cp[k] -= ld(d.fphi, 8 + k, N, g);
      }
    }
  }
  if (stop == 2) return;
  for_cell_rface_ranges(d, A, a, g, d.par[A.inst].NR, [&](int s, int e, int asR) {
    for (int n = s; n < e; ++n)
      for (int k = 0; k < np; ++k) {
        if (asR) cp[k] += ld(d.frf, 8 + k, NS, n);
        else cp[k] -= ld(d.frf, 8 + k, NS, n);
      }
  });
}

// cell_update_phi + cell_update_dphi (src/Cell/cell_misc.c:59-96): the new
// phi edge tn of cell g, its RK copy rk and the new width.
__device__ __forceinline__ double mesh_advance(const DevPtrs &d, const Annulus &A, int a, int g, int substep,
                                               double dt, double &tn, double &rk) {
  const DiskParams &P = d.par[A.inst];
  const InstState &S = d.ist[A.inst];
  const double RK = substep == 1 ? 0.0 : 0.5;
  const int j = g - A.cell_off;
  const double r = .5 * (A.rm + A.rp);
  const double a_sep = S.gr[0] + S.gr[1];
  const double w_total = rd(d.w_ann + a) + frame_rom(P, A.rom, r, a_sep);
  const double *tin = substep == 1 ? d.tiph0 : d.tiph1;
  const int gm1 = j == 0 ? A.cell_off + A.np - 1 : g - 1;
  rk = substep == 1 ? rd(tin + g) : rd(d.rktiph + g);
  double rkm = substep == 1 ? rd(tin + gm1) : rd(d.rktiph + gm1);
  tn = new_tiph(rd(d.tiphw + g), rk, RK, w_total, dt, r, d.err);
  double tnm = new_tiph(rd(d.tiphw + gm1), rkm, RK, w_total, dt, r, d.err);
  double dphi_n = tn - tnm;
  return wrap_pos(dphi_n, d.err);
}

// cell_boundary_fixed_r (src/Cell/cell_boundary.c:208-231) and cell_bc_damp
// (src/Cell/cell_misc.c:98-132) on the new prims of a cell.
template <typename T>
__device__ __forceinline__ void bc_damp(const DevPtrs &d, const Annulus &A, int a, T *pr) {
  const DiskParams &P = d.par[A.inst];
  if ((A.kind & DGPU_AK_BC_FIXED) && (A.kind & DGPU_AK_IC)) {
#pragma unroll
    for (int q = 0; q < 5; ++q) pr[q] = A.ic[q];
  }
  if (P.has_damp && (A.kind & DGPU_AK_DAMP) && (A.kind & DGPU_AK_IC)) {
    double f = d.ann_c[3 * d.n_ann + a];  // 1.-exp(-rate*dt), k_source
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      T dprim = A.ic[q] - pr[q];
      pr[q] += f * dprim;
    }
  }
}

}  // namespace

#endif
