// Objective, tangent objective and reverse-mode (adjoint) kernels of the
// moving-mesh step.
//
// The adjoint of one substep runs after the forward kernels of that substep
// (all but k_update) have rebuilt its intermediates from a stored state, in
// the reverse order of the forward data flow:
//   a_update      per cell : k_update reversed (RK blend, face and source sums,
//                            epicyclic rotation, cons2prim, boundary, damping,
//                            prim2cons); leaves the adjoint of the conserved
//                            sum lU and of the substep's input cons / rkcons
//   a_source      per cell : k_source reversed -> prim, grad[UPP], gradp[URR]
//   a_flux_phi    per phi face, a_flux_r per r face : the Riemann solver, the
//                            viscous flux and the reconstruction reversed; the
//                            adjoints of each face's cell inputs are stored per
//                            face side (no atomics)
//   a_gather_plm  per cell : gathers the face-side adjoints (phi faces, then r
//                            faces in the forward order), then reverses the
//                            r-slope limiter of the cell, replaying its branch,
//                            onto the face slopes
//   a_rslope      per cell : the face slopes reversed onto prim and gradp
//   a_cellprep    per cell : the phi limiter reversed -> adjoint of the
//                            substep's input prims
// The binary (masses, orbit radii) and alpha collect per-block partial sums,
// reduced in block order by a_par_reduce: every sum is deterministic.
// The mesh (phi edges, face list) and dt do not depend on the state under the
// frames the differentiated runs accept, so they are constants here.
#include "dgpu_adjoint.cuh"
#include "dgpu_step.cuh"

// minimum resident blocks per SM for the three heavy adjoint kernels (their
// reverse sweeps hold ~170 registers per thread without a bound)
#ifndef DGPU_MINB_ADJ
#define DGPU_MINB_ADJ 2
#endif

namespace {

// Deterministic block sum of K values per thread into out[0..K-1] (every
// thread of the block must call it).
template <int K>
__device__ __forceinline__ void block_partial(const double (&v)[K], double *out) {
  __shared__ double sh[K][BLK / 32];
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(full, x, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < BLK / 32; ++w) s += sh[k][w];
      out[k] = s;
    }
  }
}

// Deterministic sum of rows [0, nrows) of a [rows][stride] array, columns
// [0, K), by one whole block: thread t sums rows t, t + blockDim.x, ... in
// order, then a fixed-shape tree over the threads.  Result in out[0..K-1]
// (written by thread 0).  blockDim.x must be a power of two <= BLK.
template <int K>
__device__ __forceinline__ void block_rows_sum(const double *rows, int nrows, int stride, double *out) {
  __shared__ double sh[K][BLK];
  double s[K];
#pragma unroll
  for (int k = 0; k < K; ++k) s[k] = 0.0;
  for (int b = threadIdx.x; b < nrows; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] += ((volatile const double *)rows)[(size_t)stride * b + k];
#pragma unroll
  for (int k = 0; k < K; ++k) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int k = 0; k < K; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = sh[k][0];
}

// per-thread adjoints of (M0, M1, r0, r1, alpha) from position adjoints
// (positions gx = r cos(phi), gy = r sin(phi) with cosines c, sines s)
__device__ __forceinline__ void grav_adj_part(const GravAdj &ag, const double *c, const double *s, double (&v)[5]) {
  v[DGPU_AP_M0] += ag.gM[0];
  v[DGPU_AP_M1] += ag.gM[1];
  v[DGPU_AP_R0] += ag.gx[0] * c[0] + ag.gy[0] * s[0];
  v[DGPU_AP_R1] += ag.gx[1] * c[1] + ag.gy[1] * s[1];
  v[DGPU_AP_ALPHA] += ag.alpha;
}

// ---------------------------------------------------------------------------
// Objective: binary torque and inner accretion rate of the current state
// ---------------------------------------------------------------------------
// Per cell of the disk: the torque contribution -r rho dV F_phi (non-ghost
// annuli; F_phi of gravMassForce, src/Cell/cell_source.c:49-71) and the
// accretion contribution -rho v_r r dphi dz (innermost non-ghost annulus).
template <typename T>
__device__ __forceinline__ void objective_cell(const DevPtrs &d, const TanPtrs &tp, int g, T &tq, T &md) {
  const int N = d.n_cells;
  const Annulus A = d.ann[d.cell_ann[g]];
  const DiskParams &P = d.par[A.inst];
  const InstState &S = d.ist[A.inst];
  const double dphi = d.dphi[g];
  const double r = .5 * (A.rp + A.rm);
  tq = 0.0;
  md = 0.0;
  if (A.kind & DGPU_AK_CFL) {
    const double phi = d.tiph0[g] - .5 * dphi;
    const T rho = ldq<T>(d.prim, tp.prim, D_RHO, N, g);
    const double dV = dphi * .5 * A.dv_diff * P.dz;
    const double cosp = cos(phi), sinp = sin(phi);
    T Fp = 0.0;
    for (int p = 0; p < 2; ++p) {
      T gr, gM;
      if constexpr (std::is_same<T, Dual>::value) {
        const double *sd = tp.seed + (size_t)DGPU_TP_N * A.inst;
        gr = Dual(S.gr[p], sd[DGPU_TP_DR0 + p]);
        gM = Dual(S.gM[p], sd[DGPU_TP_DM0 + p]);
      } else {
        gr = S.gr[p];
        gM = S.gM[p];
      }
      T dx = r * cosp - gr * cos(S.gphi[p]);
      T dy = r * sinp - gr * sin(S.gphi[p]);
      T script_r = sqrt(dx * dx + dy * dy);
      T cosa = dx / script_r, sina = dy / script_r;
      T sinap = sina * cosp - cosa * sinp;
      Fp += sinap * -fgrav(gM, script_r, P.g_eps, P.phi_order);
    }
    tq = -(r * rho * dV * Fp);
  }
  if (A.kind & DGPU_AK_MDOT) {
    const T rho = ldq<T>(d.prim, tp.prim, D_RHO, N, g);
    const T vr = ldq<T>(d.prim, tp.prim, D_URR, N, g);
    md = -(rho * vr * r * dphi * d.par[A.inst].dz);
  }
}

// Sums over the disk (one context = one disk) into out[0..1] (torque,
// accretion rate) and, for the tangent, their derivatives into out_d[0..1];
// per-block partials reduced in block order by the last block.  With idx,
// out and out_d advance by 2 * (*idx) (the step's slot of a log).
template <typename T>
__global__ void __launch_bounds__(BLK) k_objective(DevPtrs d, TanPtrs tp, double *part, double *out, double *out_d,
                                                   const int *idx) {
  __shared__ bool last;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (g < d.n_cells) {
    T tq, md;
    objective_cell(d, tp, g, tq, md);
    v[0] = val(tq);
    v[1] = val(md);
    if constexpr (std::is_same<T, Dual>::value) {
      v[2] = tq.d;
      v[3] = md.d;
    }
  }
  block_partial<4>(v, part + 4 * (size_t)blockIdx.x);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&d.counters[3], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double s[4];
  block_rows_sum<4>(part, gridDim.x, 4, s);
  if (threadIdx.x != 0) return;
  const size_t o = idx ? 2 * (size_t)(*idx) : 0;
  out[o] = s[0];
  out[o + 1] = s[1];
  if (out_d) {
    out_d[o] = s[2];
    out_d[o + 1] = s[3];
  }
  d.counters[3] = 0;
}

// End of a logged step: dtlog[*idx] = dt of the step, then ++*idx.
__global__ void k_step_end(DevPtrs d, double *dtlog, int *idx) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    dtlog[*idx] = d.ist[0].dt;
    *idx += 1;
  }
}
// A frozen dt schedule: the dt of step *idx in place of the CFL value.
__global__ void k_set_dt(DevPtrs d, const double *dtin, const int *idx) {
  if (threadIdx.x == 0 && blockIdx.x == 0) d.ist[0].dt = dtin[*idx];
}
__global__ void k_set_int(int *p, int v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *p = v;
}
__global__ void k_add_int(int *p, int dv) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *p += dv;
}

// Stored states: 19 doubles per cell (prim, cons, rkcons, tiph0, tiph1,
// rktiph, dphi) and the disk states.  save: context -> store; else back.
// A stored state: prim, cons, rkcons (5 planes each), tiph0, tiph1, rktiph,
// dphi, then the passive-scalar planes of prim, cons and rkcons (n_pass each).
__device__ __forceinline__ void snap_copy_dev(const DevPtrs &d, double *sb, InstState *si, int save) {
  const size_t N = (size_t)d.n_cells, NP = (size_t)d.n_pass * N;
  const size_t n = 19 * N + 3 * NP;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double *c;
    if (i < 5 * N) c = d.prim + i;
    else if (i < 10 * N) c = d.cons + (i - 5 * N);
    else if (i < 15 * N) c = d.rkcons + (i - 10 * N);
    else if (i < 16 * N) c = d.tiph0 + (i - 15 * N);
    else if (i < 17 * N) c = d.tiph1 + (i - 16 * N);
    else if (i < 18 * N) c = d.rktiph + (i - 17 * N);
    else if (i < 19 * N) c = d.dphi + (i - 18 * N);
    else if (i < 19 * N + NP) c = d.prim + 5 * N + (i - 19 * N);
    else if (i < 19 * N + 2 * NP) c = d.cons + 5 * N + (i - 19 * N - NP);
    else c = d.rkcons + 5 * N + (i - 19 * N - 2 * NP);
    if (save) sb[i] = *c;
    else *c = sb[i];
  }
  if (blockIdx.x == 0) {
    const int nw = (int)(sizeof(InstState) / sizeof(unsigned long long)) * d.n_inst;
    unsigned long long *a = reinterpret_cast<unsigned long long *>(d.ist);
    unsigned long long *b = reinterpret_cast<unsigned long long *>(si);
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
      if (save) b[w] = a[w];
      else a[w] = b[w];
    }
  }
}
__global__ void __launch_bounds__(BLK) k_snap_ptr(DevPtrs d, double *sb, InstState *si, int save) {
  snap_copy_dev(d, sb, si, save);
}
// the store of slot *idx + off of a table of stores (slot 0 below 0: the
// reverse sweep's look-ahead rebuild past a segment's first step)
__global__ void __launch_bounds__(BLK) k_snap_tab(DevPtrs d, double *const *bufs, InstState *const *ists,
                                                  const int *idx, int off, int save) {
  const int k = max(*idx + off, 0);
  snap_copy_dev(d, bufs[k], ists[k], save);
}

// Adjoint of wT * torque + wM * accretion on the stored state of slot
// *idx + off (prims, phi edges, widths, disk state), added to lW; binary
// adjoints to part rows [row0, row0 + gridDim.x).  The weights of the step
// are wts[2 n], wts[2 n + 1] with n = *base + *idx.
__global__ void __launch_bounds__(BLK) a_objective(DevPtrs d, AdjPtrs J, double *const *bufs,
                                                   InstState *const *ists, const int *idx, int off,
                                                   const double *wts, const int *base, int row0) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  const double *sb = bufs[*idx + off];
  const double *prim = sb, *tiph0 = sb + 15 * (size_t)N, *dphiv = sb + 18 * (size_t)N;
  const int n = *base + *idx;
  const double wT = wts[2 * n], wM = wts[2 * n + 1];
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (g < N) {
    const Annulus A = d.ann[d.cell_ann[g]];
    const DiskParams &P = d.par[A.inst];
    const InstState &S = ists[*idx + off][A.inst];
    const double dphi = dphiv[g];
    const double r = .5 * (A.rp + A.rm);
    if ((A.kind & DGPU_AK_CFL) && wT != 0.0) {
      const double phi = tiph0[g] - .5 * dphi;
      const double rho = ld(prim, D_RHO, N, g);
      const double dV = dphi * .5 * A.dv_diff * P.dz;
      const double cosp = cos(phi), sinp = sin(phi);
      double Fp = 0.0, f1[2], sinap[2], dx[2], dy[2], sr[2], cosa[2], sina[2], cg[2], sg[2];
      for (int p = 0; p < 2; ++p) {
        cg[p] = cos(S.gphi[p]);
        sg[p] = sin(S.gphi[p]);
        dx[p] = r * cosp - S.gr[p] * cg[p];
        dy[p] = r * sinp - S.gr[p] * sg[p];
        sr[p] = sqrt(dx[p] * dx[p] + dy[p] * dy[p]);
        cosa[p] = dx[p] / sr[p];
        sina[p] = dy[p] / sr[p];
        sinap[p] = sina[p] * cosp - cosa[p] * sinp;
        f1[p] = -fgrav(S.gM[p], sr[p], P.g_eps, P.phi_order);
        Fp += sinap[p] * f1[p];
      }
      // tq = -(r rho dV Fp)
      J.lW[(size_t)D_RHO * N + g] += -wT * r * dV * Fp;
      const double aFp = -wT * r * rho * dV;
      for (int p = 0; p < 2; ++p) {
        const double asinap = aFp * f1[p], af1 = aFp * sinap[p];
        const double asina = asinap * cosp, acosa = -asinap * sinp;
        const int no = P.phi_order;
        const double qv = fgrav(1.0, sr[p], P.g_eps, no);
        v[DGPU_AP_M0 + p] += -af1 * qv;
        const double srn = dpow(sr[p], (double)no), epn = dpow(P.g_eps, (double)no);
        const double dln = (no - 1.) / sr[p] - (no + 1.) * dpow(sr[p], no - 1.) / (srn + epn);
        double asr = af1 * f1[p] * dln - (acosa * dx[p] + asina * dy[p]) / (sr[p] * sr[p]);
        const double adx = acosa / sr[p] + asr * dx[p] / sr[p];
        const double ady = asina / sr[p] + asr * dy[p] / sr[p];
        // dx = r cosp - r_p cos(phi_p)
        v[DGPU_AP_R0 + p] += -adx * cg[p] - ady * sg[p];
      }
    }
    if ((A.kind & DGPU_AK_MDOT) && wM != 0.0) {
      const double rho = ld(prim, D_RHO, N, g), vr = ld(prim, D_URR, N, g);
      const double k = r * dphi * P.dz;
      J.lW[(size_t)D_RHO * N + g] += -wM * vr * k;
      J.lW[(size_t)D_URR * N + g] += -wM * rho * k;
    }
  }
  block_partial<5>(v, J.part + DGPU_AP_N * (size_t)(row0 + blockIdx.x));
}

// Sums part rows [row0, row0 + nrows) (one block, deterministic order) and
// adds dJ/dq and dJ/dalpha to acc.
__global__ void __launch_bounds__(BLK) a_par_reduce(AdjPtrs J, int row0, int nrows) {
  __shared__ double s[5];
  block_rows_sum<5>(J.part + DGPU_AP_N * (size_t)row0, nrows, DGPU_AP_N, s);
  if (threadIdx.x != 0) return;
  J.acc[0] += s[DGPU_AP_M0] * J.dq[0] + s[DGPU_AP_M1] * J.dq[1] + s[DGPU_AP_R0] * J.dq[2] + s[DGPU_AP_R1] * J.dq[3];
  J.acc[1] += s[DGPU_AP_ALPHA];
}

// ---------------------------------------------------------------------------
// Substep adjoint
// ---------------------------------------------------------------------------
// k_update reversed, then k_source reversed on the same cell (it reads only
// the cell's own lU): lU, the substep's input lC / lCrk, and the source part
// of lWt, lG[UPP], lGp[URR]; binary adjoints to part rows [row0, ...).
__global__ void __launch_bounds__(BLK, DGPU_MINB_ADJ) a_update_source(DevPtrs d, AdjPtrs J, int substep, int row0,
                                                                     const double *rec, const int *idx) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (g < N) {
    const int a = d.cell_ann[g];
    const Annulus A = d.ann[a];
    const DiskParams &P = d.par[A.inst];
    const InstState &S = d.ist[A.inst];
    const double fac = substep == 1 ? 1.0 : 0.5, RK = substep == 1 ? 0.0 : 0.5;
    const double dt = fac * S.dt;
    const TanPtrs none = {};
    const double r = .5 * (A.rm + A.rp);
    double ac[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    {
      // the conserved sum before cons2prim and the new width, recorded by the
      // segment replay's k_update
      const double *rs = rec + (size_t)(2 * (*idx) + substep - 1) * 6 * N;
      double c[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) c[q] = rs[(size_t)q * N + g];
      const double dphi_n = rs[(size_t)5 * N + g];
      const double dV = A.dv_half * dphi_n * P.dz;
      double pr[5];
      cons2prim(c, dV, r, P, pr);
      bc_damp<double>(d, A, a, pr);
      double apr[5], alc[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        apr[q] = J.lW[(size_t)q * N + g];
        alc[q] = J.lC[(size_t)q * N + g];
      }
      prim2cons_rev(pr, r, dV, P.gamma, alc, apr);
      if (P.has_damp && (A.kind & DGPU_AK_DAMP) && (A.kind & DGPU_AK_IC)) {
        const double f = d.ann_c[3 * d.n_ann + a];
#pragma unroll
        for (int q = 0; q < 5; ++q) apr[q] *= (1.0 - f);
      }
      if ((A.kind & DGPU_AK_BC_FIXED) && (A.kind & DGPU_AK_IC)) {
#pragma unroll
        for (int q = 0; q < 5; ++q) apr[q] = 0.0;
      }
      cons2prim_rev(c, dV, r, P, apr, ac);
    }
    const double a_sep = S.gr[0] + S.gr[1];
    {
      const double rom = frame_rom(P, A.rom, r, a_sep);
      const double Omega = rom / r;
      const double dr_r2Om = 2. * rom + r * frame_rdrom(P, A.rdrom, r, a_sep);
      const int NA = d.n_ann;
      const double kappa = d.ann_c[a];
      if (kappa > 0.) split_rotate_rev(ac, d.ann_c[NA + a], d.ann_c[2 * NA + a], dr_r2Om, kappa, Omega, r);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      J.lU[(size_t)q * N + g] = ac[q];
      double lc = (1.0 - RK) * ac[q];
      if (substep == 1) lc += J.lCrk[(size_t)q * N + g];
      else J.lCrk[(size_t)q * N + g] = RK * ac[q];
      J.lC[(size_t)q * N + g] = lc;
    }
    // k_source reversed
    const double dphi = d.dphi[g];
    SrcGeom sg;
    sg.r = r;
    sg.dt = dt;
    sg.dV = dphi * .5 * A.dv_diff * P.dz;
    sincos(d.tiphw[g] - .5 * dphi, &sg.sinp, &sg.cosp);
    sg.xpos = r * sg.cosp;
    sg.ypos = r * sg.sinp;
    {
      double z = P.z;
      double R = sqrt(r * r + z * z);
      if (P.grav2d == 1) {
        sg.sint = 1.0;
        sg.cost = 0.0;
        sg.gravdist = r;
      } else {
        sg.sint = r / R;
        sg.cost = z / R;
        sg.gravdist = R;
      }
    }
    double w_a = frame_rom(P, A.rom, r, a_sep);
    sg.rdrOm = frame_rdrom(P, A.rdrom, r, a_sep);
    sg.Fc = w_a * w_a / r;
    sg.dtOm = frame_dtom(P, A.dtom, r, a_sep);
    GravT<double> G;
    grav_t(G, S, P, none, A.inst);
    double pm[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) pm[q] = ld(d.prim, q, N, g);
    double gu = 0.0, gpu = 0.0;
    if (P.has_visc) {
      gu = ld(d.grad, D_UPP, N, g);
      gpu = ld(d.gradp, D_URR, N, g);
    }
    double as[6];
    as[0] = as[1] = ac[D_SRR];
    as[2] = ac[D_LLL];
    as[3] = ac[D_SZZ];
    as[4] = ac[D_TAU];
    as[5] = P.has_visc ? ac[D_TAU] : 0.0;
    double apm[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, agu = 0.0, agpu = 0.0;
    GravAdj ag;
    grav_adj_zero(ag);
    source_cell_rev(sg, P, pm, gu, gpu, G, as, apm, agu, agpu, ag);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      J.lWt[(size_t)q * N + g] = apm[q];
      J.lG[(size_t)q * N + g] = q == D_UPP ? agu : 0.0;
      J.lGp[(size_t)q * N + g] = q == D_URR ? agpu : 0.0;
    }
    grav_adj_part(ag, S.gc, S.gs, v);
  }
  block_partial<5>(v, J.part + DGPU_AP_N * (size_t)(row0 + blockIdx.x));
}

__device__ __forceinline__ void store15(double *arr, int n, int i, const double *w, const double *gp, const double *gr) {
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    arr[(size_t)q * n + i] = w[q];
    arr[(size_t)(5 + q) * n + i] = gp[q];
    arr[(size_t)(10 + q) * n + i] = gr[q];
  }
}

__global__ void __launch_bounds__(BLK, DGPU_MINB_ADJ) a_flux_phi(DevPtrs d, AdjPtrs J, int substep, int row0) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (g < N) {
    const int a = d.cell_ann[g];
    const Annulus A = d.ann[a];
    const DiskParams &P = d.par[A.inst];
    const InstState &S = d.ist[A.inst];
    const double fac = substep == 1 ? 1.0 : 0.5;
    const int j = g - A.cell_off;
    const int cL = g, cR = (j == A.np - 1) ? A.cell_off : g + 1;
    const double dpL = d.dphi[cL], dpR = d.dphi[cR];
    const double r = .5 * (A.rp + A.rm);
    const double k = fac * S.dt * ((A.rp - A.rm) * P.dz);
    double pL[5], pR[5], aF[5], aFv[3];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      pL[q] = ld(d.prim, q, N, cL) + 0.5 * ld(d.gradp, q, N, cL) * dpL;
      pR[q] = ld(d.prim, q, N, cR) - 0.5 * ld(d.gradp, q, N, cR) * dpR;
      aF[q] = k * (ld(J.lU, q, N, cR) - ld(J.lU, q, N, cL));
    }
    aFv[0] = k * ((ld(J.lU, D_SRR, N, cR) - ld(J.lU, D_SRR, N, cL)) / r);
    aFv[1] = k * (ld(J.lU, D_LLL, N, cR) - ld(J.lU, D_LLL, N, cL));
    aFv[2] = k * (ld(J.lU, D_TAU, N, cR) - ld(J.lU, D_TAU, N, cL));
    double apL[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, apR[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    riemann_flux_rev(pL, pR, r, 1, d.w_ann[a], P.gamma, P.riemann, aF, apL, apR);
    double wL[5], wR[5], gpL[5], gpR[5], grL[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, grR[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      wL[q] = apL[q];
      wR[q] = apR[q];
      gpL[q] = 0.5 * dpL * apL[q];
      gpR[q] = -0.5 * dpR * apR[q];
    }
    if (P.has_visc) {
      ViscIn<double> vi;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        vi.cL[q] = ld(d.prim, q, N, cL);
        vi.cR[q] = ld(d.prim, q, N, cR);
        vi.gpL[q] = vi.gpR[q] = 0.0;
        vi.grL[q] = ld(d.grad, q, N, cL);
        vi.grR[q] = ld(d.grad, q, N, cR);
      }
      vi.tL = d.tiphw[cL];
      vi.tR = d.tiphw[cR];
      vi.dpL = vi.dpR = 0.0;
      vi.r = r;
      vi.cm = d.tiphw[cL];
      vi.r_cell_L = r;
      vi.r_cell_R = r;
      vi.rdr_om = frame_rdrom(P, A.rdrom, r, S.gr[0] + S.gr[1]);
      const TanPtrs none = {};
      GravT<double> G;
      grav_t(G, S, P, none, A.inst);
      ViscAdj va;
      visc_adj_zero(va);
      GravAdj ag;
      grav_adj_zero(ag);
      visc_flux_rev(vi, 1, P, G, aFv, va, ag);
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        wL[q] += va.cL[q];
        wR[q] += va.cR[q];
        grL[q] += va.grL[q];
        grR[q] += va.grR[q];
      }
      grav_adj_part(ag, S.gc, S.gs, v);
    }
    store15(J.aphiL, N, g, wL, gpL, grL);
    store15(J.aphiR, N, g, wR, gpR, grR);
  }
  block_partial<5>(v, J.part + DGPU_AP_N * (size_t)(row0 + blockIdx.x));
}

__global__ void __launch_bounds__(BLK, DGPU_MINB_ADJ) a_flux_r(DevPtrs d, AdjPtrs J, int substep, int row0) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells, NS = d.n_slots;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int cL = slot < NS ? d.fL[slot] : -1;
  if (cL >= 0) {
    const int cR = d.fR[slot];
    const int a = d.slot_ann[slot];
    const Annulus &A = d.ann[a];
    const DiskParams &P = d.par[A.inst];
    const InstState &S = d.ist[A.inst];
    const double fac = substep == 1 ? 1.0 : 0.5;
    const double deltaL = A.f_dl, deltaR = A.f_dr;
    const double dpL = d.fdp[slot], dpR = d.fdp[(size_t)NS + slot];
    const double r = A.f_r;
    const double k = fac * S.dt * (r * d.fdphi[slot] * A.f_dperp);
    const double rL = r - deltaL, rR = r + deltaR;
    double pL[5], pR[5], aF[5], aFv[3];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      pL[q] = ld(d.prim, q, N, cL) + ld(d.grad, q, N, cL) * deltaL + ld(d.gradp, q, N, cL) * dpL;
      pR[q] = ld(d.prim, q, N, cR) - ld(d.grad, q, N, cR) * deltaR - ld(d.gradp, q, N, cR) * dpR;
      aF[q] = k * (ld(J.lU, q, N, cR) - ld(J.lU, q, N, cL));
    }
    aFv[0] = k * (ld(J.lU, D_SRR, N, cR) / rR - ld(J.lU, D_SRR, N, cL) / rL);
    aFv[1] = k * (ld(J.lU, D_LLL, N, cR) - ld(J.lU, D_LLL, N, cL));
    aFv[2] = k * (ld(J.lU, D_TAU, N, cR) - ld(J.lU, D_TAU, N, cL));
    double apL[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, apR[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    riemann_flux_rev(pL, pR, r, 0, 0.0, P.gamma, P.riemann, aF, apL, apR);
    double wL[5], wR[5], gpL[5], gpR[5], grL[5], grR[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      wL[q] = apL[q];
      wR[q] = apR[q];
      grL[q] = deltaL * apL[q];
      grR[q] = -deltaR * apR[q];
      gpL[q] = dpL * apL[q];
      gpR[q] = -dpR * apR[q];
    }
    if (P.has_visc) {
      ViscIn<double> vi;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        vi.cL[q] = ld(d.prim, q, N, cL);
        vi.cR[q] = ld(d.prim, q, N, cR);
        vi.gpL[q] = ld(d.gradp, q, N, cL);
        vi.gpR[q] = ld(d.gradp, q, N, cR);
        vi.grL[q] = vi.grR[q] = 0.0;
      }
      vi.tL = d.tiphw[cL];
      vi.tR = d.tiphw[cR];
      vi.dpL = dpL;
      vi.dpR = dpR;
      vi.r = r;
      vi.cm = d.fcm[slot];
      vi.r_cell_L = rL;
      vi.r_cell_R = rR;
      vi.rdr_om = frame_rdrom(P, A.f_rdrom, r, S.gr[0] + S.gr[1]);
      const TanPtrs none = {};
      GravT<double> G;
      grav_t(G, S, P, none, A.inst);
      ViscAdj va;
      visc_adj_zero(va);
      GravAdj ag;
      grav_adj_zero(ag);
      visc_flux_rev(vi, 0, P, G, aFv, va, ag);
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        wL[q] += va.cL[q];
        wR[q] += va.cR[q];
        gpL[q] += va.gpL[q];
        gpR[q] += va.gpR[q];
      }
      grav_adj_part(ag, S.gc, S.gs, v);
    }
    store15(J.arL, NS, slot, wL, gpL, grL);
    store15(J.arR, NS, slot, wR, gpR, grR);
  }
  block_partial<5>(v, J.part + DGPU_AP_N * (size_t)(row0 + blockIdx.x));
}

// Gathers the face-side adjoints of each cell (phi faces, then its r faces),
// completing the adjoint of grad; then reverses cell_plm_rz's limiter
// (src/Cell/cell_plm.c:81-113) onto the face slopes, replaying its branch.
__global__ void __launch_bounds__(BLK) a_gather_plm(DevPtrs d, AdjPtrs J) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells, NS = d.n_slots;
  if (g >= N) return;
  const int a = d.cell_ann[g];
  const Annulus A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const int j = g - A.cell_off;
  const int gl = j == 0 ? A.cell_off + A.np - 1 : g - 1;
  double acc[15];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    acc[q] = ld(J.lWt, q, N, g);
    acc[5 + q] = ld(J.lGp, q, N, g);
    acc[10 + q] = ld(J.lG, q, N, g);
  }
#pragma unroll
  for (int q = 0; q < 15; ++q) acc[q] += ld(J.aphiL, q, N, g) + ld(J.aphiR, q, N, gl);
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int asR) {
    const double *src = asR ? J.arR : J.arL;
#pragma unroll
    for (int q = 0; q < 15; ++q) acc[q] += ld(src, q, NS, slot);
  });
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    J.lWt[(size_t)q * N + g] = acc[q];
    J.lGp[(size_t)q * N + g] = acc[5 + q];
  }
  // limiter replay: gq = sum S dA / dAtot, then per face (forward order):
  // zero if the face slope opposes, clip to plm * S if smaller
  double gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int sel[5] = {-1, -1, -1, -1, -1};  // -1 average, -2 zero, else the clipping slot
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
    double dA = F.r * F.dphi * F.dperp;
#pragma unroll
    for (int q = 0; q < 5; ++q) gq[q] += ld(d.fS, q, NS, slot) * dA;
  });
  double dAtot;
  {
    double dz = P.dz, dp = d.dphi[g];
    if (A.i == 0) dAtot = dz * A.rp * dp;
    else if (A.i == P.NR - 1) dAtot = dz * A.rm * dp;
    else dAtot = dz * (A.rp + A.rm) * dp;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) gq[q] /= dAtot;
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      double Sq = ld(d.fS, q, NS, slot);
      if (Sq * gq[q] < 0.0) {
        gq[q] = 0.0;
        sel[q] = -2;
      } else if (fabs(P.plm * Sq) < fabs(gq[q])) {
        gq[q] = P.plm * Sq;
        sel[q] = slot;
      }
    }
  });
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int asR) {
    double dA = F.r * F.dphi * F.dperp;
    double *dst = asR ? J.fsR : J.fsL;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const double lg = acc[10 + q];
      double w = 0.0;
      if (sel[q] == -1) w = lg * dA / dAtot;
      else if (sel[q] == slot) w = P.plm * lg;
      dst[(size_t)q * NS + slot] = w;
    }
  });
}

// The face slopes fS = (WR - WL) / (deltaR + deltaL) reversed onto the prims
// and phi slopes of each cell (its faces in the forward order).
__global__ void __launch_bounds__(BLK) a_rslope(DevPtrs d, AdjPtrs J) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells, NS = d.n_slots;
  if (g >= N) return;
  const int a = d.cell_ann[g];
  const Annulus A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  double lw[5], lgp[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    lw[q] = ld(J.lWt, q, N, g);
    lgp[q] = ld(J.lGp, q, N, g);
  }
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int asR) {
    const double den = F.dr + F.dl;
    const double dp = asR ? d.fdp[(size_t)NS + slot] : d.fdp[slot];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const double ls = (ld(J.fsL, q, NS, slot) + ld(J.fsR, q, NS, slot)) / den;
      if (asR) lw[q] += ls;
      else lw[q] -= ls;
      lgp[q] -= dp * ls;
    }
  });
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    J.lWt[(size_t)q * N + g] = lw[q];
    J.lGp[(size_t)q * N + g] = lgp[q];
  }
}

// cell_plm_p reversed: the adjoint of each cell's prims from the phi slopes of
// itself and its two neighbours (each on the branch its limiter took).
__global__ void __launch_bounds__(BLK) a_cellprep(DevPtrs d, AdjPtrs J) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  if (g >= N) return;
  const int a = d.cell_ann[g];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const int off = A.cell_off, np = A.np, j = g - off;
  auto left = [&](int x) { return off + ((x - off) == 0 ? np - 1 : (x - off) - 1); };
  auto right = [&](int x) { return off + ((x - off) == np - 1 ? 0 : (x - off) + 1); };
  int ks[3] = {g, left(g), right(g)};
  const int nk = ks[1] == ks[2] ? 2 : 3;
  (void)j;
  double lw[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) lw[q] = ld(J.lWt, q, N, g);
  for (int m = 0; m < nk; ++m) {
    const int kk = ks[m], kl = left(kk), kr = right(kk);
    const double dc = d.dphi[kk];
    const double dpL = .5 * (dc + d.dphi[kl]);
    const double dpR = .5 * (dc + d.dphi[kr]);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      double cl, cc, cr;
      plm_p_slope_coef(ld(d.prim, q, N, kl), ld(d.prim, q, N, kk), ld(d.prim, q, N, kr), dpL, dpR, P.plm, &cl, &cc,
                       &cr);
      const double w = (kk == g ? cc : 0.0) + (kl == g ? cl : 0.0) + (kr == g ? cr : 0.0);
      lw[q] += w * ld(J.lGp, q, N, kk);
    }
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) J.lW[(size_t)q * N + g] = lw[q];
}

// cell_calc_cons reversed: lW += (d cons / d prim)^T lC on the current state.
__global__ void __launch_bounds__(BLK) a_calc_cons(DevPtrs d, AdjPtrs J) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  if (g >= N) return;
  const Annulus A = d.ann[d.cell_ann[g]];
  const DiskParams &P = d.par[A.inst];
  const double r = .5 * (A.rp + A.rm);
  const double dV = A.dv_half * d.dphi[g] * P.dz;
  double p[5], ac[5], ap[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    p[q] = ld(d.prim, q, N, g);
    ac[q] = ld(J.lC, q, N, g);
    ap[q] = 0.0;
  }
  prim2cons_rev(p, r, dV, P.gamma, ac, ap);
#pragma unroll
  for (int q = 0; q < 5; ++q) J.lW[(size_t)q * N + g] += ap[q];
}

}  // namespace

extern "C" {

int dgk_objective(const DevPtrs *d, const TanPtrs *t, double *part, double *out, double *out_d, const int *idx,
                  void *stream) {
  const int nb = (d->n_cells + BLK - 1) / BLK;
  static const TanPtrs none = {};
  if (t) k_objective<Dual><<<nb, BLK, 0, (cudaStream_t)stream>>>(*d, *t, part, out, out_d, idx);
  else k_objective<double><<<nb, BLK, 0, (cudaStream_t)stream>>>(*d, none, part, out, out_d, idx);
  return (int)cudaGetLastError();
}

int dgk_step_end(const DevPtrs *d, double *dtlog, int *idx, void *stream) {
  k_step_end<<<1, 32, 0, (cudaStream_t)stream>>>(*d, dtlog, idx);
  return (int)cudaGetLastError();
}
int dgk_set_dt(const DevPtrs *d, const double *dtin, const int *idx, void *stream) {
  k_set_dt<<<1, 32, 0, (cudaStream_t)stream>>>(*d, dtin, idx);
  return (int)cudaGetLastError();
}
int dgk_set_int(int *p, int v, void *stream) {
  k_set_int<<<1, 32, 0, (cudaStream_t)stream>>>(p, v);
  return (int)cudaGetLastError();
}
int dgk_add_int(int *p, int dv, void *stream) {
  k_add_int<<<1, 32, 0, (cudaStream_t)stream>>>(p, dv);
  return (int)cudaGetLastError();
}

static int snap_grid(const DevPtrs *d) {
  long long n = (19LL + 3LL * d->n_pass) * d->n_cells;
  long long b = (n + BLK - 1) / BLK;
  return (int)(b < 148 * 8 ? b : 148 * 8);
}
int dgk_snap(const DevPtrs *d, double *buf, InstState *ist, int save, void *stream) {
  k_snap_ptr<<<snap_grid(d), BLK, 0, (cudaStream_t)stream>>>(*d, buf, ist, save);
  return (int)cudaGetLastError();
}
int dgk_snap_tab(const DevPtrs *d, double *const *bufs, InstState *const *ists, const int *idx, int off, int save,
                 void *stream) {
  k_snap_tab<<<snap_grid(d), BLK, 0, (cudaStream_t)stream>>>(*d, bufs, ists, idx, off, save);
  return (int)cudaGetLastError();
}

int dgk_adj_rows(const DevPtrs *d) {
  const int nbC = (d->n_cells + BLK - 1) / BLK, nbS = (d->n_slots + BLK - 1) / BLK;
  return 3 * nbC + nbS;
}

int dgk_adj_objective(const DevPtrs *d, const AdjPtrs *J, double *const *bufs, InstState *const *ists,
                      const int *idx, int off, const double *wts, const int *base, void *stream) {
  const int nbC = (d->n_cells + BLK - 1) / BLK, nbS = (d->n_slots + BLK - 1) / BLK;
  const int row0 = 2 * nbC + nbS;
  a_objective<<<nbC, BLK, 0, (cudaStream_t)stream>>>(*d, *J, bufs, ists, idx, off, wts, base, row0);
  a_par_reduce<<<1, BLK, 0, (cudaStream_t)stream>>>(*J, row0, nbC);
  return (int)cudaGetLastError();
}

int dgk_adj_substep(const DevPtrs *d, const AdjPtrs *J, int substep, const double *rec, const int *idx,
                    void *stream, void *side, void *ev_fork, void *ev_join) {
  cudaStream_t s = (cudaStream_t)stream, s2 = (cudaStream_t)side;
  const int nbC = (d->n_cells + BLK - 1) / BLK, nbS = (d->n_slots + BLK - 1) / BLK;
  cudaError_t e;
  a_update_source<<<nbC, BLK, 0, s>>>(*d, *J, substep, 0, rec, idx);
  /* the phi faces beside the r faces */
  if ((e = cudaEventRecord((cudaEvent_t)ev_fork, s)) != cudaSuccess) return (int)e;
  if ((e = cudaStreamWaitEvent(s2, (cudaEvent_t)ev_fork, 0)) != cudaSuccess) return (int)e;
  a_flux_phi<<<nbC, BLK, 0, s2>>>(*d, *J, substep, nbC);
  if (nbS > 0) a_flux_r<<<nbS, BLK, 0, s>>>(*d, *J, substep, 2 * nbC);
  if ((e = cudaEventRecord((cudaEvent_t)ev_join, s2)) != cudaSuccess) return (int)e;
  if ((e = cudaStreamWaitEvent(s, (cudaEvent_t)ev_join, 0)) != cudaSuccess) return (int)e;
  a_par_reduce<<<1, BLK, 0, s>>>(*J, 0, 2 * nbC + nbS);
  a_gather_plm<<<nbC, BLK, 0, s>>>(*d, *J);
  a_rslope<<<nbC, BLK, 0, s>>>(*d, *J);
  a_cellprep<<<nbC, BLK, 0, s>>>(*d, *J);
  return (int)cudaGetLastError();
}

int dgk_adj_calc_cons(const DevPtrs *d, const AdjPtrs *J, void *stream) {
  a_calc_cons<<<(d->n_cells + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, *J);
  return (int)cudaGetLastError();
}

}  // extern "C"
