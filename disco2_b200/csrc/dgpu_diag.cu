// Diagnostics reductions of diagnostics_set (src/Diagnostics/diagnostics_set.c:
// 13-298) on the device: the per-annulus phi-averaged radial profiles
// (VectorDiag), their area-weighted integrals (ScalarDiag), the equatorial
// dump (EquatDiag) and the quantities of the DiagMdot line, for the current
// state of one disk, before the reference's time weighting by dtout.
//
//   k_diag_annulus  CTA per annulus : one profile row and the mass partials of
//                                     the annulus (fixed-shape tree over its
//                                     cells), the equatorial rows of its cells
//   k_diag_finish   one CTA         : rows scaled, scalars and masses summed
//                                     over the annuli in order
#include "dgpu_device.cuh"

#define DIAG_NVEC 17   // NUM_DIAG + 1 (diagnostics_create_destroy.c:14)
#define DIAG_NEQ 18    // NUM_DIAG + 2
#define DIAG_NMASS 7   // mass inside r = 1, mass within 0.1 / 0.2 / 0.4 of each mass
#define DIAG_NROW (DIAG_NVEC + DIAG_NMASS)
#define DIAG_NEXTRA 14
#define DIAG_BLK 128   // threads of k_diag_annulus (its tree holds DIAG_NROW x DIAG_BLK doubles)

namespace {

// Row of annulus a (rows[a][DIAG_NROW]) of one disk; non-ghost annuli only
// contribute (the reference loops i over [Nghost_min, N - Nghost_max)).
__global__ void __launch_bounds__(DIAG_BLK) k_diag_annulus(DevPtrs d, int inst, double *rows, double *equat,
                                                           int eq_first) {
  __shared__ double sh[DIAG_NROW][DIAG_BLK];
  const DiskParams &P = d.par[inst];
  const InstState &S = d.ist[inst];
  const int a = P.ann_base + blockIdx.x;
  const Annulus &A = d.ann[a];
  const int N = d.n_cells;
  double acc[DIAG_NROW];
#pragma unroll
  for (int n = 0; n < DIAG_NROW; ++n) acc[n] = 0.0;
  const bool live = (A.kind & DGPU_AK_CFL) != 0;
  if (live) {
    const double rm = A.rm, rp = A.rp, r = 0.5 * (rm + rp), dz = P.dz;
    const double r_bh0 = S.gr[0], r_bh1 = S.gr[1];
    const double xb0 = r_bh0 * cos(S.gphi[0]), yb0 = r_bh0 * sin(S.gphi[0]);
    const double xb1 = r_bh1 * cos(S.gphi[1]), yb1 = r_bh1 * sin(S.gphi[1]);
    const double a_sep = r_bh0 + r_bh1;
    const double rom = frame_rom(P, A.rom, r, a_sep);
    const double Np = (double)A.np;
    for (int j = threadIdx.x; j < A.np; j += blockDim.x) {
      const int g = A.cell_off + j;
      const double dphi = d.dphi[g];
      const double phi = d.tiph0[g] - 0.5 * dphi;
      const double rho = ld(d.prim, D_RHO, N, g);
      const double press = ld(d.prim, D_PPP, N, g);
      const double vr = ld(d.prim, D_URR, N, g);
      const double vp_minus_w = ld(d.prim, D_UPP, N, g) * r;
      const double vp = ld(d.prim, D_UPP, N, g) * r + rom;
      const double vz = ld(d.prim, D_UZZ, N, g);
      const double v2 = vr * vr + vp * vp + vz * vz;
      const double rhoe = press / (P.gamma - 1.);
      const double KE = 0.5 * rho * v2;
      const double E_hydro = rhoe + KE;
      const double dV = 0.5 * (rp * rp - rm * rm) * dphi;
      // cells with no cooling keep Cool = 0; the passive column is prim[NUM_C]
      // (with NUM_Q = 5 the reference reads past prim[] there; zero here)
      const double cool = 0.0, passive = P.num_n > 0 ? ld(d.prim, 5, N, g) : 0.0;
      const double col[DIAG_NVEC] = {r, rho, press, vr, vp, vz, vp_minus_w, cool, passive, E_hydro, KE, rhoe,
                                     0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int n = 0; n < DIAG_NVEC; ++n) acc[n] += col[n] / Np * dz;
      if (rp <= 1.0) acc[DIAG_NVEC] += rho * dV;
      // gravMass_dist (src/GravMass/GravMass_access.c:25-31)
      const double x = r * cos(phi), y = r * sin(phi);
      const double d0 = sqrt((x - xb0) * (x - xb0) + (y - yb0) * (y - yb0) + 0.0);
      const double d1 = sqrt((x - xb1) * (x - xb1) + (y - yb1) * (y - yb1) + 0.0);
      const double dM = rho * dV;
      if (d0 < 0.1) acc[DIAG_NVEC + 1] += dM;
      if (d1 < 0.1) acc[DIAG_NVEC + 2] += dM;
      if (d0 < 0.2) acc[DIAG_NVEC + 3] += dM;
      if (d1 < 0.2) acc[DIAG_NVEC + 4] += dM;
      if (d0 < 0.4) acc[DIAG_NVEC + 5] += dM;
      if (d1 < 0.4) acc[DIAG_NVEC + 6] += dM;
      if (equat) {
        // the equatorial row of the cell (every cell of a 2-D disk sits at z = 0)
        double *e = equat + (size_t)(g - eq_first) * DIAG_NEQ;
        const double er[DIAG_NEQ] = {r, phi, rho, press, vr, vp, vz, vp_minus_w, cool, passive, E_hydro, KE, rhoe,
                                     0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int n = 0; n < DIAG_NEQ; ++n) e[n] = er[n];
      }
    }
  }
#pragma unroll
  for (int n = 0; n < DIAG_NROW; ++n) sh[n][threadIdx.x] = acc[n];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int n = 0; n < DIAG_NROW; ++n) sh[n][threadIdx.x] += sh[n][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < DIAG_NROW) rows[(size_t)blockIdx.x * DIAG_NROW + threadIdx.x] = sh[threadIdx.x][0];
}

// vector[nr][17] = rows / (Z_Max - Z_Min) over the non-ghost annuli;
// scalar[16] = sum_i row_i[n + 1] (rp^2 - rm^2) / ((Z_Max - Z_Min)(R_Max^2 - R_Min^2));
// extra[14] = Mdot_near_req1, r_near_req1, mass_inside_1, mass_inner_wedge,
// Mdot_0, Mdot_1, Macc_0, Macc_1, mass within 0.2 of mass 0 / 1, within 0.4
// of mass 0 / 1, within 0.1 of mass 0 / 1.
__global__ void __launch_bounds__(BLK) k_diag_finish(DevPtrs d, int inst, const double *rows, double *vector,
                                                     double *scalar, double *extra, double zspan, double rmin,
                                                     double rmax) {
  const DiskParams &P = d.par[inst];
  const InstState &S = d.ist[inst];
  const int NR = P.NR;
  const int t = threadIdx.x;
  // rows of the non-ghost annuli, in order
  int imin = 0, imax = NR;
  while (imin < NR && !(d.ann[P.ann_base + imin].kind & DGPU_AK_CFL)) ++imin;
  while (imax > imin && !(d.ann[P.ann_base + imax - 1].kind & DGPU_AK_CFL)) --imax;
  for (int k = t; k < (imax - imin) * DIAG_NVEC; k += blockDim.x) {
    const int i = imin + k / DIAG_NVEC, n = k % DIAG_NVEC;
    vector[k] = rows[(size_t)i * DIAG_NROW + n] * (1.0 / zspan);
  }
  if (t < DIAG_NVEC - 1) {
    double s = 0.0;
    for (int i = imin; i < imax; ++i) {
      const Annulus &A = d.ann[P.ann_base + i];
      s += rows[(size_t)i * DIAG_NROW + t + 1] * (A.rp * A.rp - A.rm * A.rm);
    }
    scalar[t] = s * (1.0 / (zspan * (rmax * rmax - rmin * rmin)));
  }
  if (t == 0) {
    double m[DIAG_NMASS];
    for (int n = 0; n < DIAG_NMASS; ++n) m[n] = 0.0;
    for (int i = imin; i < imax; ++i)
      for (int n = 0; n < DIAG_NMASS; ++n) m[n] += rows[(size_t)i * DIAG_NROW + DIAG_NVEC + n];
    // the first annulus whose mean radius exceeds 1
    double mdot = nan(""), rr = nan("");
    for (int i = imin; i < imax; ++i) {
      const double r = rows[(size_t)i * DIAG_NROW] / zspan;
      if (r > 1.0) {
        mdot = rows[(size_t)i * DIAG_NROW + 5] * 2. * M_PI * r / zspan;
        rr = r;
        break;
      }
    }
    // the inner wedge: the reference walks the first N_p(imax) cells of the
    // disk's contiguous cell block with the radii of annulus 0
    double wedge = 0.0;
    {
      const Annulus &A0 = d.ann[P.ann_base];
      const int npw = imax < NR ? d.ann[P.ann_base + imax].np : 0;
      const int N = d.n_cells;
      for (int j = 0; j < npw && j < P.n_cells; ++j) {
        const int g = P.cell_base + j;
        const double dV = 0.5 * (A0.rp * A0.rp - A0.rm * A0.rm) * d.dphi[g];
        wedge += ld(d.prim, D_RHO, N, g) * dV;
      }
    }
    extra[0] = mdot;
    extra[1] = rr;
    extra[2] = m[0];
    extra[3] = wedge;
    extra[4] = S.mdot[0];
    extra[5] = S.mdot[1];
    extra[6] = S.macc[0];
    extra[7] = S.macc[1];
    extra[8] = m[3];
    extra[9] = m[4];
    extra[10] = m[5];
    extra[11] = m[6];
    extra[12] = m[1];
    extra[13] = m[2];
  }
}

}  // namespace

extern "C" {

int dgk_diag_sizes(int *nvec, int *neq, int *nextra, int *nrow) {
  *nvec = DIAG_NVEC;
  *neq = DIAG_NEQ;
  *nextra = DIAG_NEXTRA;
  *nrow = DIAG_NROW;
  return 0;
}

// rows: [NR][DIAG_NROW] scratch; equat: [interior cells][DIAG_NEQ] or NULL,
// indexed from the disk's first non-ghost cell eq_first.
int dgk_diagnostics(const DevPtrs *d, int inst, int n_ann_disk, double *rows, double *vector, double *scalar,
                    double *equat, int eq_first, double *extra, double zspan, double rmin, double rmax, void *stream) {
  k_diag_annulus<<<n_ann_disk, DIAG_BLK, 0, (cudaStream_t)stream>>>(*d, inst, rows, equat, eq_first);
  k_diag_finish<<<1, BLK, 0, (cudaStream_t)stream>>>(*d, inst, rows, vector, scalar, extra, zspan, rmin, rmax);
  return (int)cudaGetLastError();
}

}  // extern "C"
