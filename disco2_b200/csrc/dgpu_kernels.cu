// sm_100a kernels of the moving-mesh finite-volume step.
//
// One RK substep is eight launches in a CUDA graph:
//   k_merge    per annulus pair : the r-face list of pair (i, i+1) (face_create
//                                 / build_jloop) as a checked parallel merge of
//                                 the two sorted phi-edge lists, and
//                                 cell_set_w
//   k_cellprep per cell         : cell_clean_pi, cell_plm_p, GravMass copy /
//                                 clean_pi
//   k_rslope   per r face       : the face slope S and the wrapped offsets of
//                                 cell_plm_rz / riemann_setup_rz
//   k_plm_r    per cell         : cell_plm_rz (face-weighted slope + limiter)
//                                 and, in substep 1, the CFL minimum
//                                 (cell_mindt); k_dt then forms dt
//                                 (timestep_set_dt)
//   k_source   per cell         : the increments of cell_add_src and
//                                 cell_add_visc_src; per-annulus constants
//   k_flux_phi per phi face     : riemann_setup_p + riemann_AddFlux
//   k_flux_r   per r face       : riemann_setup_rz + riemann_AddFlux; both
//                                 flux kernels store dt*dA*F per face
//   k_update   per cell         : gathers the increments in the reference's
//                                 accumulation order, cell_add_split_fictitious,
//                                 cell_update_phi/_dphi, cell_calc_prim, the
//                                 fixed radial boundary, cell_bc_damp and
//                                 cell_calc_cons; its last block advances the
//                                 GravMass state
// and, for disks with the outflow radial boundary, k_outflow per disk
// (cell_boundary_outflow_r).  k_merge runs beside k_cellprep on a second
// stream, and k_source then k_flux_phi beside k_flux_r.
//
// Built with -fmad=false: every expression keeps the reference's operation
// order and rounding (double '/' and sqrt are IEEE-rounded on the GPU), so
// paths without transcendentals reproduce the reference bit for bit.
#include <cuda_runtime.h>
#include <climits>
#include <math.h>
#include <stdint.h>

#include "dgpu_step.cuh"

// minimum resident blocks per SM requested from the register allocator
// (measured on B200, circumbinary disk: these kernels are latency-bound, so
// occupancy beats the extra spills)
#ifndef DGPU_MINB_FACE
#define DGPU_MINB_FACE 6
#endif
#ifndef DGPU_MINB_PLM
#define DGPU_MINB_PLM 4
#endif
#ifndef DGPU_MINB_FLUX
#define DGPU_MINB_FLUX 4
#endif
#ifndef DGPU_MINB_FLUXR
#define DGPU_MINB_FLUXR 3
#endif
#ifndef DGPU_MINB_SOURCE
#define DGPU_MINB_SOURCE 3
#endif
#ifndef DGPU_MINB_UPDATE
#define DGPU_MINB_UPDATE 4
#endif
#ifndef DGPU_MINB_PREP
#define DGPU_MINB_PREP 4
#endif
#ifndef DGPU_MINB_SWEEP
#define DGPU_MINB_SWEEP 3
#endif

namespace {


// ---------------------------------------------------------------------------
// r-face list of one annulus pair (build_jloop, face_create_destroy.c:22-128)
// ---------------------------------------------------------------------------
struct FaceCtx {
  const double *tin, *din, *tout, *dout;
  int Nin, Nout;
  int *fL, *fR;
  double *fdphi, *fcm;
  int *runs;
  int *sruns;   // copy of runs the rr pass reads (shared memory when staged)
  int *fstart;  // fstart of the inner annulus cells (indexed by j)
  int cap, rcap;
  int *err;
  int offL, offR;  // global cell numbers of inner/outer cell 0 (face records hold global cells)
};

// The body of the reference's j loop for inner cell j starting at outer cell
// jp: emits its faces and advances jp.  n = running face number, s = running
// count of jp advances (the run index of the next face).  FILL writes.
template <bool FILL>
__device__ void face_cell(const FaceCtx &c, int j, int &jp, int &n, int &s) {
  int jm = j - 1;
  if (jm < 0) jm = c.Nin - 1;
  bool mark = false;
  auto emit = [&](double dphi, double tp) {
    if (FILL) {
      if (n < c.cap) {
        c.fL[n] = c.offL + j;
        c.fR[n] = c.offR + jp;
        c.fdphi[n] = dphi;
        c.fcm[n] = tp - .5 * dphi;
      }
      if (mark && s < c.rcap) c.runs[s] = c.sruns[s] = n;
    }
    mark = false;
    ++n;
  };
  auto advance = [&]() {
    ++jp;
    if (jp == c.Nout) jp = 0;
    ++s;
    mark = true;
  };
  if (FILL) c.fstart[j] = n;
  double dp = c.tout[jp] - c.tin[jm];
  dp = wrap_pos(dp, c.err);
  if (c.din[j] < dp) {
    emit(c.din[j], c.tin[j]);
    return;
  }
  emit(dp, c.tout[jp]);
  advance();
  dp = c.tin[j] - c.tout[jp];
  dp = wrap_pm(dp, c.err);
  int guard = 0;
  while (dp > 0.0) {
    emit(c.dout[jp], c.tout[jp]);
    advance();
    dp = c.tin[j] - c.tout[jp];
    dp = wrap_pm(dp, c.err);
    if (++guard > c.Nout + 2) {
      set_err(c.err, DGPU_EF_FACE_OVERFLOW);
      break;
    }
  }
  dp = c.dout[jp] + dp;
  emit(dp, c.tin[j]);
}

// Exclusive scan of one value per thread over the block (blockDim.x a multiple
// of 32, at most 1024); sh needs blockDim.x / 32 entries.
template <typename T>
__device__ T block_excl_scan(T v, T *sh, T &total) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(full, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    T t = lane < nw ? sh[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(full, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) sh[lane] = t;
  }
  __syncthreads();
  T pre = w > 0 ? sh[w - 1] : T(0);
  total = sh[nw - 1];
  __syncthreads();
  return pre + x - v;
}

// Per cell, once per substep: cell_clean_pi of the phi edge
// (src/Cell/cell_misc.c:12-26) and cell_plm_p (src/Cell/cell_plm.c:116-161).
template <typename T, bool PS>
__device__ __forceinline__ void cellprep_cell(const DevPtrs &d, const TanPtrs &tp, int g, int substep) {
  const int N = d.n_cells;
  const double *traw = substep == 1 ? d.tiph0 : d.tiph1;
  pf_planes(d.prim, 5, N, g);
  pf(d.dphi + g);
  pf(traw + g);
  const int a = d.cell_ann[g];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const int np = A.np, off = A.cell_off, j = g - off;
  d.tiphw[g] = wrap_pos(traw[g], d.err);
  const int gl = off + (j == 0 ? np - 1 : j - 1);
  const int gr = off + (j == np - 1 ? 0 : j + 1);
  const double dc = d.dphi[g];
  const double dpL = .5 * (dc + d.dphi[gl]);
  const double dpR = .5 * (dc + d.dphi[gr]);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    T pc = ldq<T>(d.prim, tp.prim, q, N, g), pl = ldq<T>(d.prim, tp.prim, q, N, gl),
      pr = ldq<T>(d.prim, tp.prim, q, N, gr);
    stq<T>(d.gradp, tp.gradp, q, N, g, plm_p_slope(pl, pc, pr, dpL, dpR, P.plm));
  }
  for (int q = 5; q < 5 + (PS ? P.num_n : 0); ++q)
    d.gradp[(size_t)q * N + g] = plm_p_slope(ld(d.prim, q, N, gl), ld(d.prim, q, N, g), ld(d.prim, q, N, gr), dpL, dpR, P.plm);
}

// cellprep_cell for every cell and, for the first cell of each disk,
// gravMass_copy at the start of a step (GravMass_misc.c:20-28) and
// gravMass_clean_pi (GravMass_misc.c:9-17).  Runs concurrently with k_merge.
template <typename T, bool PS = false>
__global__ void __launch_bounds__(BLK, DGPU_MINB_FACE) k_cellprep(DevPtrs d, TanPtrs tp, int substep) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.n_cells) return;
  cellprep_cell<T, PS>(d, tp, g, substep);
  const Annulus &A = d.ann[d.cell_ann[g]];
  const DiskParams &P = d.par[A.inst];
  if (g == P.cell_base) {
    InstState &S = d.ist[A.inst];
    if (substep == 1) {
      for (int p = 0; p < 2; ++p) {
        S.grk_r[p] = S.gr[p];
        S.grk_phi[p] = S.gphi[p];
        S.grk_M[p] = S.gM[p];
        S.grk_om[p] = S.gom[p];
        // gravMass_dist of the step-start positions (the CFL's viscosity)
        S.rkx[p] = S.gr[p] * cos(S.gphi[p]);
        S.rky[p] = S.gr[p] * sin(S.gphi[p]);
      }
      S.dtkey = (unsigned long long)__double_as_longlong(1.e100);
    }
    for (int p = 0; p < 2; ++p) S.gphi[p] = wrap_pos(S.gphi[p], d.err);  // 2.*M_PI == PHIMAX
  }
}

// Per annulus pair (i, i+1) of a disk, one block: the r-face list of
// face_create/build_jloop (src/Face/face_create_destroy.c:22-193) as a checked
// parallel merge, and cell_set_w (src/Cell/cell_set_w.c:12-102) of annulus i.
// Z: the z pair (ring a, ring a+NR) of a 3-D disk (build_jloop with zDir:
// both rings have N_p cells of annulus i) into the z-face arrays; no
// cell_set_w then.
template <bool Z>
__device__ __forceinline__ void merge_pair(const DevPtrs &d, int a, int substep) {
  __shared__ int sh_i[BLK / 32];
  __shared__ int sh_j[BLK];
  __shared__ double sh_v[BLK / 32];
  __shared__ unsigned long long sh_u[BLK / 32];
  __shared__ int sh_flag, sh_nf, sh_T;
  // staged phi edges and widths of the pair, then the runs
  extern __shared__ double sm[];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const double *traw = substep == 1 ? d.tiph0 : d.tiph1;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int np = A.np, off = A.cell_off;
  const int N = d.n_cells;
  const bool rigid = P.w_numeric == DC_RIGID;
  if (!Z && tid == 0 && !rigid) d.w_ann[a] = A.wnum;
  // the pair's arrays: r faces of (a, a+1), or z faces of (a, a+NR)
  int *const pfL = Z ? d.zfL : d.fL, *const pfR = Z ? d.zfR : d.fR;
  double *const pfdphi = Z ? d.zfdphi : d.fdphi, *const pfcm = Z ? d.zfcm : d.fcm;
  int *const pruns = Z ? d.zruns : d.runs, *const pfstart = Z ? d.zfstart : d.fstart;
  int *const prr = Z ? d.zrr : d.rr;
  int *const p_nf = Z ? d.zpair_nf : d.pair_nf, *const p_jpmin = Z ? d.zpair_jpmin : d.pair_jpmin;
  int *const p_T = Z ? d.zpair_T : d.pair_T, *const p_seq = Z ? d.zpair_seq : d.pair_seq;
  const int fbase = Z ? A.zface_base : A.face_base, fcap = Z ? A.zface_cap : A.face_cap;
  const int rbase = Z ? A.zrun_base : A.run_base;
  const int partner = Z ? a + P.NR : a + 1;
  if (Z ? A.k < P.NZ - 1 : A.i < P.NR - 1) {
    const int npo = d.ann[partner].np;
    const int offo = d.ann[partner].cell_off;
    const int rcap = Z ? A.zrun_cap : A.run_cap;
    const bool staged = d.smem_face >= (int)sizeof(double) * 2 * (np + npo) + (int)sizeof(int) * rcap;
    const double *tin = traw + off, *din = d.dphi + off;
    const double *tout = traw + offo, *dout = d.dphi + offo;
    if (staged) {
      double *s_tin = sm, *s_din = sm + np, *s_tout = sm + 2 * np, *s_dout = sm + 2 * np + npo;
      for (int j = tid; j < np; j += nt) {
        s_tin[j] = tin[j];
        s_din[j] = din[j];
      }
      for (int j = tid; j < npo; j += nt) {
        s_tout[j] = tout[j];
        s_dout[j] = dout[j];
      }
      __syncthreads();
      tin = s_tin;
      din = s_din;
      tout = s_tout;
      dout = s_dout;
    }
    FaceCtx c;
    c.tin = tin;
    c.din = din;
    c.tout = tout;
    c.dout = dout;
    c.Nin = np;
    c.Nout = npo;
    c.fL = pfL + fbase;
    c.fR = pfR + fbase;
    c.fdphi = pfdphi + fbase;
    c.fcm = pfcm + fbase;
    c.runs = pruns + rbase;
    c.sruns = staged ? reinterpret_cast<int *>(sm + 2 * (np + npo)) : c.runs;
    c.fstart = pfstart + off;
    c.cap = fcap;
    c.rcap = rcap;
    c.err = d.err;
    c.offL = off;
    c.offR = offo;
    const double p0 = c.tin[np - 1];

    // jpmin: first outer cell with the smallest wrap(tiph - p0), start (PHIMAX, 0)
    double bv = PHIMAX;
    int bi = 0;
    {
      for (int jp = tid; jp < c.Nout; jp += nt) {
        double dp = wrap_pos(c.tout[jp] - p0, d.err);
        if (dp < bv || (dp == bv && jp < bi)) {
          bv = dp;
          bi = jp;
        }
      }
      // the (value, index) minimum is the same in any order of combination:
      // per warp by shuffles, then over the warps
      const unsigned full = 0xffffffffu;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_down_sync(full, bv, o);
        int i2 = __shfl_down_sync(full, bi, o);
        if (v2 < bv || (v2 == bv && i2 < bi)) {
          bv = v2;
          bi = i2;
        }
      }
      if ((tid & 31) == 0) {
        sh_v[tid >> 5] = bv;
        sh_i[tid >> 5] = bi;
      }
      __syncthreads();
      bv = sh_v[0];
      bi = sh_i[0];
      for (int w = 1; w < (nt >> 5); ++w) {
        const double v2 = sh_v[w];
        const int i2 = sh_i[w];
        if (v2 < bv || (v2 == bv && i2 < bi)) {
          bv = v2;
          bi = i2;
        }
      }
    }
    const int jpmin = bi;

    // contiguous chunk of inner cells per thread; speculative start outer cell
    const int chunk = (np + nt - 1) / nt;
    const int j0 = min(np, tid * chunk), j1 = min(np, j0 + chunk);
    int jp_start = jpmin;
    if (j0 > 0 && j0 < np) {
      // lower bound of the left edge of inner cell j0 among the outer edges,
      // both measured as wrap(edge - p0); verified below
      double L = wrap_pos(c.tin[j0 - 1] - p0, d.err);
      int lo = 0, hi = c.Nout;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int k = jpmin + mid;
        if (k >= c.Nout) k -= c.Nout;
        double e = wrap_pos(c.tout[k] - p0, d.err);
        if (e < L) lo = mid + 1;
        else hi = mid;
      }
      jp_start = jpmin + lo;
      if (jp_start >= c.Nout) jp_start -= c.Nout;
    }
    int cnt = 0, steps = 0, jp = jp_start;
    {
      int n = 0, s = 0;
      for (int j = j0; j < j1; ++j) face_cell<false>(c, j, jp, n, s);
      cnt = n;
      steps = s;
    }
    if (tid == 0) sh_flag = 0;
    sh_j[tid] = (j0 < j1) ? jp_start : -1;
    __syncthreads();
    if (j0 < j1 && tid + 1 < nt && sh_j[tid + 1] >= 0 && sh_j[tid + 1] != jp) sh_flag = 1;
    __syncthreads();
    const bool sequential = sh_flag != 0;

    if (!sequential) {
      // one scan of (faces, advances) packed in a 64-bit word: the advances
      // of a pair stay far below 2^32, so no carry reaches the face count
      unsigned long long tot;
      const unsigned long long pre =
          block_excl_scan<unsigned long long>(((unsigned long long)cnt << 32) | (unsigned)steps, sh_u, tot);
      const int fo = (int)(pre >> 32), so = (int)(pre & 0xffffffffu);
      const int ntot = (int)(tot >> 32), stot = (int)(tot & 0xffffffffu);
      if (ntot > c.cap || stot + 2 > c.rcap) {
        if (tid == 0) {
          set_err(d.err, DGPU_EF_FACE_OVERFLOW);
          p_nf[a] = 0;
          p_T[a] = 0;
          sh_nf = 0;
          sh_T = 0;
        }
      } else {
        int n = fo, s = so;
        jp = jp_start;
        for (int j = j0; j < j1; ++j) face_cell<true>(c, j, jp, n, s);
        if (tid == 0) {
          c.runs[0] = c.sruns[0] = 0;
          c.runs[stot + 1] = c.sruns[stot + 1] = ntot;
          p_nf[a] = ntot;
          p_jpmin[a] = jpmin;
          p_T[a] = stot;
          p_seq[a] = 0;
          sh_nf = ntot;
          sh_T = stot;
        }
      }
    } else if (tid == 0) {
      // exact sequential replay of build_jloop from jpmin
      int n = 0, s = 0;
      jp = jpmin;
      for (int j = 0; j < np; ++j) face_cell<true>(c, j, jp, n, s);
      if (n > c.cap || s + 2 > c.rcap) {
        set_err(d.err, DGPU_EF_FACE_OVERFLOW);
        p_nf[a] = 0;
        p_T[a] = 0;
        sh_nf = 0;
        sh_T = 0;
      } else {
        c.runs[0] = c.sruns[0] = 0;
        c.runs[s + 1] = c.sruns[s + 1] = n;
        p_nf[a] = n;
        p_jpmin[a] = jpmin;
        p_T[a] = s;
        p_seq[a] = 1;
        sh_nf = n;
        sh_T = s;
      }
    }
    __syncthreads();
    // per outer cell, the face ranges of its runs s = jp - jpmin (mod Nout) and
    // s + Nout (the cell at the wrap point); z = INT_MIN flags a third run
    {
      const int nf = sh_nf, T = sh_T;
      for (int jq = tid; jq < npo; jq += nt) {
        int4 rr = make_int4(0, 0, 0, 0);
        if (nf > 0) {
          int s0 = jq - jpmin;
          if (s0 < 0) s0 += npo;
          if (s0 <= T) rr.x = c.sruns[s0], rr.y = c.sruns[s0 + 1];
          if (s0 + npo <= T) rr.z = c.sruns[s0 + npo], rr.w = c.sruns[s0 + npo + 1];
          if (s0 + 2 * npo <= T) rr.z = INT_MIN;
        }
        reinterpret_cast<int4 *>(prr)[offo + jq] = rr;
      }
      // slab slots past the list hold no face
      for (int n = nf + tid; n < c.cap; n += nt) c.fL[n] = -1;
    }
  }
  // C_RIGID: the mass-weighted mean v_phi of the annulus, summed in j order
  // like the reference (cell_set_w.c:41-49); one lane, after the merge
  if (!Z && rigid && tid == nt - 32) {
    double w = 0.0, Mring = 0.0;
    for (int j = 0; j < np; ++j) {
      double vp = A.r * ld(d.prim, D_UPP, N, off + j);
      double m = ld(d.cons, D_DDD, N, off + j);
      Mring += m;
      w += vp * m;
    }
    d.w_ann[a] = w / Mring;
  }
}

__global__ void __launch_bounds__(BLK, DGPU_MINB_FACE) k_merge(DevPtrs d, int substep) {
  merge_pair<false>(d, blockIdx.x, substep);
}

// The z-face lists of a 3-D disk: one block per ring a with k < NZ-1.
__global__ void __launch_bounds__(BLK, DGPU_MINB_FACE) k_zmerge(DevPtrs d, int substep) {
  merge_pair<true>(d, blockIdx.x, substep);
}

// ---------------------------------------------------------------------------
// cell_plm_rz (src/Cell/cell_plm.c:13-114) per cell + CFL (cell_mindt.c:32-100)
// ---------------------------------------------------------------------------
// r-face slope and reconstruction offsets, once per face: the S of
// cell_plm_rz (src/Cell/cell_plm.c:31-53) and the wrapped dpL, dpR that
// cell_plm_rz, riemann_setup_rz (Riemann_setup.c:18-25) and riemann_visc_flux
// (Riemann_routines.c:220-228) all form the same way.
template <typename T, bool PS>
__device__ __forceinline__ void rslope_face(const DevPtrs &d, const TanPtrs &tp, int slot) {
  const int cL = rd(d.fL + slot);
  if (cL < 0) return;  // slot past the face list of its pair
  const int cR = rd(d.fR + slot);
  pf_planes(d.prim, 5, d.n_cells, cL);
  pf_planes(d.prim, 5, d.n_cells, cR);
  pf_planes(d.gradp, 5, d.n_cells, cL);
  pf_planes(d.gradp, 5, d.n_cells, cR);
  const int a = rd(d.slot_ann + slot);
  const Annulus &A = d.ann[a];
  const int N = d.n_cells, NS = d.n_slots;
  const double cm = rd(d.fcm + slot);
  double pL = rd(d.tiphw + cL) - .5 * rd(d.dphi + cL);
  double pR = rd(d.tiphw + cR) - .5 * rd(d.dphi + cR);
  double dpL = cm - pL;
  dpL = wrap_pm(dpL, d.err);
  double dpR = pR - cm;
  dpR = wrap_pm(dpR, d.err);
  d.fdp[slot] = dpL;
  d.fdp[(size_t)NS + slot] = dpR;
  const double den = A.f_dr + A.f_dl;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    T WL = ldqr<T>(d.prim, tp.prim, q, N, cL) + dpL * ldqr<T>(d.gradp, tp.gradp, q, N, cL);
    T WR = ldqr<T>(d.prim, tp.prim, q, N, cR) - dpR * ldqr<T>(d.gradp, tp.gradp, q, N, cR);
    stq<T>(d.fS, tp.fS, q, NS, slot, (WR - WL) / den);
  }
  for (int q = 5; q < 5 + (PS ? d.par[A.inst].num_n : 0); ++q) {
    const double WL = ldr(d.prim, q, N, cL) + dpL * ldr(d.gradp, q, N, cL);
    const double WR = ldr(d.prim, q, N, cR) - dpR * ldr(d.gradp, q, N, cR);
    d.fS[(size_t)q * NS + slot] = (WR - WL) / den;
  }
}

template <typename T, bool PS = false>
__global__ void __launch_bounds__(BLK) k_rslope(DevPtrs d, TanPtrs tp) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= d.n_slots) return;
  rslope_face<T, PS>(d, tp, slot);
}

// cell_plm_rz's r slope of cell g (src/Cell/cell_plm.c:56-114): the
// face-area-weighted mean of the face slopes S, then the theta limiter against
// each face's S in face order.
template <typename T, bool PS>
__device__ __forceinline__ void plm_r_grad(const DevPtrs &d, const TanPtrs &tp, int g) {
  const int N = d.n_cells, NS = d.n_slots;
  pf(d.rr + 4 * (size_t)g);
  pf(d.fstart + g);
  pf(d.dphi + g);
  const int a = d.cell_ann[g];
  const Annulus A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  T gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
    double dA = F.r * F.dphi * F.dperp;
#pragma unroll
    for (int q = 0; q < 5; ++q) gq[q] += ldq<T>(d.fS, tp.fS, q, NS, slot) * dA;
  });
  double dAtot;
  {
    double dz = A.dz, dp = d.dphi[g];
    if (A.i == 0) dAtot = dz * A.rp * dp;
    else if (A.i == P.NR - 1) dAtot = dz * A.rm * dp;
    else dAtot = dz * (A.rp + A.rm) * dp;
#pragma unroll
    for (int q = 0; q < 5; ++q) gq[q] /= dAtot;
  }
  for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      T Sq = ldq<T>(d.fS, tp.fS, q, NS, slot);
      if (Sq * gq[q] < 0.0) gq[q] = 0.0;
      else if (fabs(P.plm * Sq) < fabs(gq[q])) gq[q] = P.plm * Sq;
    }
  });
  // passive scalars: the same face-weighted slope and limiter
  for (int q = 5; q < 5 + (PS ? P.num_n : 0); ++q) {
    double gs = 0.0;
    for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
      double dA = F.r * F.dphi * F.dperp;
      gs += ld(d.fS, q, NS, slot) * dA;
    });
    gs /= dAtot;
    for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int slot, int) {
      const double Sq = ld(d.fS, q, NS, slot);
      if (Sq * gs < 0.0) gs = 0.0;
      else if (fabs(P.plm * Sq) < fabs(gs)) gs = P.plm * Sq;
    });
    d.grad[(size_t)q * N + g] = gs;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) stq<T>(d.grad, tp.grad, q, N, g, gq[q]);
}

// The CFL step of non-ghost cell g (cell_mindt, src/Cell/cell_mindt.c:10-100)
// as the bit pattern of the positive double (~0: no candidate, also for a NaN,
// which is reported).  rkx/rky/rkM: the step-start GravMass positions and
// masses (the viscous limit's nu); wa = wiph of the annulus.
__device__ __forceinline__ unsigned long long cfl_key(const DevPtrs &d, const Annulus &A, const DiskParams &P,
                                                      int g, double wa, const double *rkx, const double *rky,
                                                      const double *rkM) {
  const int N = d.n_cells;
  const double *traw = d.tiph0;
  double w = .5 * (wa + wa);
  double dr = A.rp - A.rm;
  double r = .5 * (A.rp + A.rm);
  double dx = dr;
  double rdphi = .5 * (A.rp + A.rm) * d.dphi[g];
  if (rdphi < dr) dx = rdphi;
  if (dx > A.dz) dx = A.dz;
  double Pp = ld(d.prim, D_PPP, N, g), rho = ld(d.prim, D_RHO, N, g);
  double vp = ld(d.prim, D_UPP, N, g) * r - w;
  double vr = ld(d.prim, D_URR, N, g), vz = ld(d.prim, D_UZZ, N, g);
  double cs = sqrt(P.gamma * Pp / rho);
  double cf2 = cs * cs;
  double maxv = sqrt(cf2) + sqrt(vr * vr + vp * vp + vz * vz);
  double dt = P.cfl * dx / maxv;
  if (P.has_visc) {
    double nu;
    if (P.visc_const == 1) {
      nu = P.visc;
    } else {
      double tc = traw[g] - 0.5 * d.dphi[g];
      if (P.init_type == DI_SHEAR) {
        nu = P.visc * P.gamma * Pp / rho * dpow(fabs(r * cos(tc)), 2.0);
        if (r * cos(tc) > 20.) nu = 0.000000001;
      } else {
        double sc, cc;
        sincos(tc, &sc, &cc);
        const double x = r * cc, y = r * sc;
        double d0 = gm_dist_xy(x, y, rkx[0], rky[0]);
        double d1 = gm_dist_xy(x, y, rkx[1], rky[1]);
        double eps = P.g_eps;
        nu = P.visc * Pp / rho /
             sqrt(dpow(d0 * d0 + eps * eps, -1.5) * rkM[0] + dpow(d1 * d1 + eps * eps, -1.5) * rkM[1]);
      }
    }
    double dt_visc = .25 * dx * dx / nu;
    dt = dt / (1. + dt / dt_visc);
  }
  unsigned long long key = (unsigned long long)__double_as_longlong(dt);
  if (__longlong_as_double((long long)key) < 0.0 || dt != dt) key = ~0ull;
  // the reference's minimum skips such a cell too (cell_mindt.c); here it
  // is also reported
  if (dt != dt) set_err(d.err, DGPU_EF_NONFINITE);
  return key;
}

template <typename T, int MB = DGPU_MINB_PLM, bool PS = false>
__global__ void __launch_bounds__(BLK, MB) k_plm_r(DevPtrs d, TanPtrs tp, int substep) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  unsigned long long key = ~0ull;
  int inst = -1;
  if (g < d.n_inst) {
    // GravMass positions of this substep (gravMass_dist, cell_source.c:103-107)
    InstState &S = d.ist[g];
    for (int p = 0; p < 2; ++p) {
      S.gc[p] = cos(S.gphi[p]);
      S.gs[p] = sin(S.gphi[p]);
      S.gx[p] = S.gr[p] * S.gc[p];
      S.gy[p] = S.gr[p] * S.gs[p];
    }
  }
  if (g < N) {
    plm_r_grad<T, PS>(d, tp, g);
    const int a = d.cell_ann[g];
    const Annulus &A = d.ann[a];
    inst = A.inst;
    // CFL candidate (cell_mindt), substep 1 only, non-ghost annuli
    if (substep == 1 && (A.kind & DGPU_AK_CFL)) {
      const InstState &S = d.ist[A.inst];
      key = cfl_key(d, A, d.par[A.inst], g, d.w_ann[a], S.rkx, S.rky, S.grk_M);
    }
  }
  if (substep != 1) return;

  // minimum per disk: warp reduction when the warp holds one disk
  const unsigned full = 0xffffffffu;
  int inst0 = __shfl_sync(full, inst, 0);
  bool uniform = __all_sync(full, inst == inst0);
  if (uniform) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long k2 = __shfl_down_sync(full, key, o);
      key = k2 < key ? k2 : key;
    }
    if ((threadIdx.x & 31) == 0 && inst0 >= 0 && key != ~0ull) atomicMin(&d.ist[inst0].dtkey, key);
  } else if (inst >= 0 && key != ~0ull) {
    atomicMin(&d.ist[inst].dtkey, key);
  }
}

// dt of each disk once k_plm_r has formed the CFL minimum: the minimum,
// clipped to Time_Max (timestep_set_dt, timestep_set.c:16-21).  A kernel of
// its own, so that no block of k_plm_r has to wait for its stores to land
// before a last block is elected.
__global__ void k_dt(DevPtrs d) {
  for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
    InstState &S = d.ist[k];
    double dt = __longlong_as_double((long long)S.dtkey);
    if (S.t + dt > d.par[k].t_max) dt = d.par[k].t_max - S.t;
    S.dt = dt;
  }
}

// ---------------------------------------------------------------------------
// Face increments: one thread per phi face (at its left cell) and per r-face slot
// ---------------------------------------------------------------------------
// phi faces: thread per cell j, face (j, j+1) (riemann_setup_p, Riemann_setup.c:46-80)
// S: the disk's state with this substep's GravMass positions; dt: the
// substep's fac * dt.
template <typename T, bool PS>
__device__ __forceinline__ void flux_phi_cell(const DevPtrs &d, const TanPtrs &tp, int g, const InstState &S,
                                              double dt) {
  const int N = d.n_cells;
  // the cell's own planes (its right neighbour's share the lines) ahead of
  // the annulus lookups
  pf_planes(d.prim, 5, N, g);
  pf_planes(d.gradp, 5, N, g);
  pf_planes(d.grad, 5, N, g);
  pf(d.tiphw + g);
  pf(d.dphi + g);
  const int a = d.cell_ann[g];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const int j = g - A.cell_off;
  const int cL = g, cR = (j == A.np - 1) ? A.cell_off : g + 1;
  const double dpL = d.dphi[cL], dpR = d.dphi[cR];
  const double dz = A.dz;
  const double dr = A.rp - A.rm;
  const double r = .5 * (A.rp + A.rm);
  const double dA = dr * dz;
  T pL[5], pR[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    pL[q] = ldq<T>(d.prim, tp.prim, q, N, cL) + 0.5 * ldq<T>(d.gradp, tp.gradp, q, N, cL) * dpL;
    pR[q] = ldq<T>(d.prim, tp.prim, q, N, cR) - 0.5 * ldq<T>(d.gradp, tp.gradp, q, N, cR) * dpR;
  }
  const double w = d.w_ann[a];
  T F[5];
  double qL[DGPU_MAX_PASSIVE], qR[DGPU_MAX_PASSIVE], Fq[DGPU_MAX_PASSIVE];
  const int np = PS ? P.num_n : 0;
  for (int s = 0; s < np; ++s) {
    qL[s] = ld(d.prim, 5 + s, N, cL) + 0.5 * ld(d.gradp, 5 + s, N, cL) * dpL;
    qR[s] = ld(d.prim, 5 + s, N, cR) - 0.5 * ld(d.gradp, 5 + s, N, cR) * dpR;
  }
  riemann_flux(pL, pR, r, 1, w, P.gamma, P.riemann, F, np, qL, qR, Fq);
  const double k = dt * dA;
#pragma unroll
  for (int q = 0; q < 5; ++q) stq<T>(d.fphi, tp.fphi, q, N, g, k * F[q]);
  for (int s = 0; s < np; ++s) d.fphi[(size_t)(8 + s) * N + g] = k * Fq[s];
  if (P.has_visc) {
    ViscIn<T> v;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      v.cL[q] = ldq<T>(d.prim, tp.prim, q, N, cL);
      v.cR[q] = ldq<T>(d.prim, tp.prim, q, N, cR);
      v.grL[q] = ldq<T>(d.grad, tp.grad, q, N, cL);
      v.grR[q] = ldq<T>(d.grad, tp.grad, q, N, cR);
    }
    v.tL = d.tiphw[cL];
    v.tR = d.tiphw[cR];
    v.dpL = v.dpR = 0.0;
    v.r = r;
    v.cm = d.tiphw[cL];
    v.r_cell_L = r;
    v.r_cell_R = r;
    double a_sep = S.gr[0] + S.gr[1];
    v.rdr_om = frame_rdrom(P, A.rdrom, r, a_sep);
    GravT<T> G;
    grav_t(G, S, P, tp, A.inst);
    T Fv[3];
    visc_flux(v, 1, P, G, Fv, d.err);
#pragma unroll
    for (int q = 0; q < 3; ++q) stq<T>(d.fphi, tp.fphi, 5 + q, N, g, k * Fv[q]);
  }
}

template <typename T, int MB = DGPU_MINB_FLUX, bool PS = false>
__global__ void __launch_bounds__(BLK, MB) k_flux_phi(DevPtrs d, TanPtrs tp, int substep) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.n_cells) return;
  const InstState &S = d.ist[d.ann[d.cell_ann[g]].inst];
  flux_phi_cell<T, PS>(d, tp, g, S, (substep == 1 ? 1.0 : 0.5) * S.dt);
}

// r faces: thread per face slot (riemann_setup_rz, Riemann_setup.c:11-44)
template <typename T, bool PS>
__device__ __forceinline__ void flux_r_face(const DevPtrs &d, const TanPtrs &tp, int slot, const InstState &S,
                                            double dt) {
  const int N = d.n_cells;
  const int cL = d.fL[slot];
  if (cL < 0) return;  // slot past the face list of its pair
  const int cR = d.fR[slot];
  const int a = d.slot_ann[slot];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const double fdphi = d.fdphi[slot], cm = d.fcm[slot];
  const double deltaL = A.f_dl, deltaR = A.f_dr;
  const double dpL = d.fdp[slot];
  const double dpR = d.fdp[(size_t)d.n_slots + slot];
  const double r = A.f_r;
  const double dA = r * fdphi * A.f_dperp;
  const double r_cell_L = r - deltaL;
  const double r_cell_R = r + deltaR;
  T pL[5], pR[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    pL[q] = ldq<T>(d.prim, tp.prim, q, N, cL) + ldq<T>(d.grad, tp.grad, q, N, cL) * deltaL +
            ldq<T>(d.gradp, tp.gradp, q, N, cL) * dpL;
    pR[q] = ldq<T>(d.prim, tp.prim, q, N, cR) - ldq<T>(d.grad, tp.grad, q, N, cR) * deltaR -
            ldq<T>(d.gradp, tp.gradp, q, N, cR) * dpR;
  }
  T F[5];
  double qL[DGPU_MAX_PASSIVE], qR[DGPU_MAX_PASSIVE], Fq[DGPU_MAX_PASSIVE];
  const int np = PS ? P.num_n : 0;
  for (int s = 0; s < np; ++s) {
    qL[s] = ld(d.prim, 5 + s, N, cL) + ld(d.grad, 5 + s, N, cL) * deltaL + ld(d.gradp, 5 + s, N, cL) * dpL;
    qR[s] = ld(d.prim, 5 + s, N, cR) - ld(d.grad, 5 + s, N, cR) * deltaR - ld(d.gradp, 5 + s, N, cR) * dpR;
  }
  riemann_flux(pL, pR, r, 0, 0.0, P.gamma, P.riemann, F, np, qL, qR, Fq);
  const double k = dt * dA;
  const int NS = d.n_slots;
#pragma unroll
  for (int q = 0; q < 5; ++q) stq<T>(d.frf, tp.frf, q, NS, slot, k * F[q]);
  for (int s = 0; s < np; ++s) d.frf[(size_t)(8 + s) * NS + slot] = k * Fq[s];
  if (P.has_visc) {
    ViscIn<T> v;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      v.cL[q] = ldq<T>(d.prim, tp.prim, q, N, cL);
      v.cR[q] = ldq<T>(d.prim, tp.prim, q, N, cR);
      v.gpL[q] = ldq<T>(d.gradp, tp.gradp, q, N, cL);
      v.gpR[q] = ldq<T>(d.gradp, tp.gradp, q, N, cR);
    }
    v.tL = d.tiphw[cL];
    v.tR = d.tiphw[cR];
    v.dpL = dpL;
    v.dpR = dpR;
    v.r = r;
    v.cm = cm;
    v.r_cell_L = r_cell_L;
    v.r_cell_R = r_cell_R;
    double a_sep = S.gr[0] + S.gr[1];
    v.rdr_om = frame_rdrom(P, A.f_rdrom, r, a_sep);
    GravT<T> G;
    grav_t(G, S, P, tp, A.inst);
    T Fv[3];
    visc_flux(v, 0, P, G, Fv, d.err);
#pragma unroll
    for (int q = 0; q < 3; ++q) stq<T>(d.frf, tp.frf, 5 + q, NS, slot, k * Fv[q]);
  }
}

template <typename T, int MB = DGPU_MINB_FLUXR, bool PS = false>
__global__ void __launch_bounds__(BLK, MB) k_flux_r(DevPtrs d, TanPtrs tp, int substep) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= d.n_slots) return;
  if (d.fL[slot] < 0) return;  // slot past the face list of its pair
  const InstState &S = d.ist[d.ann[d.slot_ann[slot]].inst];
  flux_r_face<T, PS>(d, tp, slot, S, (substep == 1 ? 1.0 : 0.5) * S.dt);
}

// ---------------------------------------------------------------------------
// z faces of 3-D disks (face_create with direction 1, cell_plm_rz with
// Z_DIR, the z-face riemann_setup_rz + riemann_AddFlux of
// src/TimeStep/timestep_routines.c:63-71)
// ---------------------------------------------------------------------------
// z-face slope and reconstruction offsets, once per face: as k_rslope, with
// the half heights of the two layers in place of the radial half widths.
__global__ void __launch_bounds__(BLK) k_zslope(DevPtrs d) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= d.n_zslots) return;
  const int cL = rd(d.zfL + slot);
  if (cL < 0) return;  // slot past the face list of its pair
  const int cR = rd(d.zfR + slot);
  const int a = rd(d.zslot_ann + slot);
  const Annulus &A = d.ann[a];
  const int N = d.n_cells, NS = d.n_zslots;
  const double cm = rd(d.zfcm + slot);
  double pL = rd(d.tiphw + cL) - .5 * rd(d.dphi + cL);
  double pR = rd(d.tiphw + cR) - .5 * rd(d.dphi + cR);
  double dpL = cm - pL;
  dpL = wrap_pm(dpL, d.err);
  double dpR = pR - cm;
  dpR = wrap_pm(dpR, d.err);
  d.zfdp[slot] = dpL;
  d.zfdp[(size_t)NS + slot] = dpR;
  const double den = A.zf_dr + A.zf_dl;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const double WL = ldr(d.prim, q, N, cL) + dpL * ldr(d.gradp, q, N, cL);
    const double WR = ldr(d.prim, q, N, cR) - dpR * ldr(d.gradp, q, N, cR);
    d.zfS[(size_t)q * NS + slot] = (WR - WL) / den;
  }
}

// cell_plm_rz with Z_DIR (src/Cell/cell_plm.c:13-114) per cell of a 3-D disk:
// the face-area-weighted mean of the z-face slopes over
// dAtot = 2*.5*(rp^2 - rm^2)*dphi, then the limiter in face order.  The
// reference overwrites grad with it; here it goes to gradz, which the z
// fluxes and (in 3-D) the viscous source read.
__global__ void __launch_bounds__(BLK) k_plm_z(DevPtrs d) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells, NS = d.n_zslots;
  if (g >= N) return;
  const int a = d.cell_ann[g];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  if (P.NZ == 1) return;
  const double rm = A.rm, rp = A.rp;
  const double zr = .5 * (rp + rm), zperp = rp - rm;  // build_jloop's r and deltaPerp of a z face
  double gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for_cell_zface_ranges(d, A, a, g, P.NR, P.NZ, [&](int s, int e, int) {
    for (int n = s; n < e; ++n) {
      const double dA = zr * rd(d.zfdphi + n) * zperp;
#pragma unroll
      for (int q = 0; q < 5; ++q) gq[q] += ld(d.zfS, q, NS, n) * dA;
    }
  });
  const double dp = d.dphi[g];
  const double dAtot = 2. * .5 * (rp * rp - rm * rm) * dp;
#pragma unroll
  for (int q = 0; q < 5; ++q) gq[q] /= dAtot;
  for_cell_zface_ranges(d, A, a, g, P.NR, P.NZ, [&](int s, int e, int) {
    for (int n = s; n < e; ++n) {
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const double Sq = ld(d.zfS, q, NS, n);
        if (Sq * gq[q] < 0.0) gq[q] = 0.0;
        else if (fabs(P.plm * Sq) < fabs(gq[q])) gq[q] = P.plm * Sq;
      }
    }
  });
#pragma unroll
  for (int q = 0; q < 5; ++q) d.gradz[(size_t)q * N + g] = gq[q];
}

// z faces: thread per face slot (riemann_setup_rz with ZDIRECTION,
// Riemann_setup.c:11-44, and riemann_AddFlux with w = 0): the states are
// reconstructed with the z slopes; the viscous flux of a z face is zero, and
// only the reference's v_z check remains.
__global__ void __launch_bounds__(BLK) k_flux_z(DevPtrs d, int substep) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= d.n_zslots) return;
  const int cL = d.zfL[slot];
  if (cL < 0) return;
  const int cR = d.zfR[slot];
  const int a = d.zslot_ann[slot];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  const InstState &S = d.ist[A.inst];
  const int N = d.n_cells, NS = d.n_zslots;
  const double fac = substep == 1 ? 1.0 : 0.5;
  const double deltaL = A.zf_dl, deltaR = A.zf_dr;
  const double dpL = d.zfdp[slot], dpR = d.zfdp[(size_t)NS + slot];
  const double r = A.zf_r;
  const double dA = r * d.zfdphi[slot] * A.zf_dperp;
  double pL[5], pR[5], F[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    pL[q] = ld(d.prim, q, N, cL) + ld(d.gradz, q, N, cL) * deltaL + ld(d.gradp, q, N, cL) * dpL;
    pR[q] = ld(d.prim, q, N, cR) - ld(d.gradz, q, N, cR) * deltaR - ld(d.gradp, q, N, cR) * dpR;
  }
  riemann_flux(pL, pR, r, 2, 0.0, P.gamma, P.riemann, F);
  const double k = fac * S.dt * dA;
#pragma unroll
  for (int q = 0; q < 5; ++q) d.zfrf[(size_t)q * NS + slot] = k * F[q];
  if (P.has_visc) {
    // riemann_visc_flux averages the reconstructed states on a z face and
    // exits on a nonzero v_z (Riemann_routines.c:271-274)
    const double vz = .5 * (pL[D_UZZ] + pR[D_UZZ]);
    if (fabs(vz) > 1.e-12) set_err(d.err, DGPU_EF_VISC_VZ);
  }
}

// The single-rank cell_syncproc_z (src/Cell/cell_sync.c:156-205) at the end
// of a substep of a 3-D disk, then cell_calc_cons of the cells it wrote: the
// ng lowest layers take prim, RKcons and tiph of layers NZ-2ng .. NZ-ng-1, the
// ng highest those of layers ng .. 2ng-1 (dphi stays the cell's own).  Runs
// after k_update and the radial boundary, which have finished every layer.
__global__ void __launch_bounds__(BLK) k_zsync(DevPtrs d, int substep) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells, zg = d.zghost;
  // zghost > 0: threads cover the ng lowest layers' cells, then the ng highest
  const int g = zg > 0 ? (t < zg ? t : N - 2 * zg + t) : t;
  if (zg > 0 ? t >= 2 * zg : g >= N) return;
  const int a = d.cell_ann[g];
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  if (P.NZ == 1) return;
  const int ng = P.ngz, shift = P.NZ - 2 * ng;
  int ks;
  if (A.k < ng) ks = A.k + shift;
  else if (A.k >= P.NZ - ng) ks = A.k - shift;
  else return;
  const Annulus &Sr = d.ann[a + (ks - A.k) * P.NR];
  const int gs = Sr.cell_off + (g - A.cell_off);
  double *tout = substep == 1 ? d.tiph1 : d.tiph0;
  double pr[5], c[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    pr[q] = d.prim[(size_t)q * N + gs];
    d.prim[(size_t)q * N + g] = pr[q];
    d.rkcons[(size_t)q * N + g] = d.rkcons[(size_t)q * N + gs];
  }
  tout[g] = tout[gs];
  const double r = .5 * (A.rm + A.rp);
  const double dV = A.dv_half * d.dphi[g] * A.dz;
  prim2cons(pr, c, r, dV, P.gamma);
#pragma unroll
  for (int q = 0; q < 5; ++q) d.cons[(size_t)q * N + g] = c[q];
}

// ---------------------------------------------------------------------------
// Per-cell update: flux gather + sources + mesh motion + prim/cons + BC + damping
// ---------------------------------------------------------------------------

// Source increments of cell_add_src (src/Cell/cell_source.c:73-214) and
// cell_add_visc_src (cell_source.c:216-277), per cell, for k_update to add in
// the reference's order: src[0..4] = S_r (pressure/centrifugal), S_r (gravity
// + frame), L, S_z, tau; src[5] = viscous heating; src[6+p] = sink mass of mass
// p.  They read only the substep's primitives, slopes and GravMass positions,
// so this kernel runs concurrently with k_flux_r.  Its first n_ann threads also
// form the per-annulus constants of the substep (epicyclic rotation of
// cell_add_split_fictitious.c:26-38, relaxation factor of cell_misc.c:121).
// Per-annulus constants of the substep for the update of annulus t: the
// epicyclic rotation of cell_add_split_fictitious
// (cell_add_split_fictitious.c:26-38) and the relaxation factor of
// cell_bc_damp (cell_misc.c:121), identical for every cell of the annulus.
__device__ __forceinline__ void ann_consts(const DevPtrs &d, int t, const InstState &S, double dt) {
  const Annulus &A = d.ann[t];
  const DiskParams &P = d.par[A.inst];
  const double r = 0.5 * (A.rm + A.rp);
  const double a_sep = S.gr[0] + S.gr[1];
  const double rom = frame_rom(P, A.rom, r, a_sep);
  const double Omega = rom / r;
  const double dr_r2Om = 2. * rom + r * frame_rdrom(P, A.rdrom, r, a_sep);
  const double kappa2 = 2. * Omega / r * dr_r2Om;
  double kappa = 0.0, ck = 1.0, sk = 0.0;
  if (kappa2 > 0.) {
    kappa = sqrt(kappa2);
    ck = cos(kappa * dt);
    sk = sin(kappa * dt);
  }
  const int NA = d.n_ann;
  d.ann_c[t] = kappa;
  d.ann_c[NA + t] = ck;
  d.ann_c[2 * NA + t] = sk;
  d.ann_c[3 * NA + t] = (A.kind & DGPU_AK_DAMP) ? (1. - exp(-A.damp_rate * dt)) : 0.0;
}

// The source increments of cell g (see k_source); the sink masses of the
// cells counted in Mdot are added to md0 / md1.
template <typename T, bool PS>
__device__ __forceinline__ void source_cell_k(const DevPtrs &d, const TanPtrs &tp, int g, const InstState &S,
                                              double dt, double &md0, double &md1) {
  const int N = d.n_cells;
  {
    pf_planes(d.prim, 5, N, g);
    pf(d.grad + (size_t)D_UPP * N + g);
    pf(d.gradp + (size_t)D_URR * N + g);
    pf(d.tiphw + g);
    pf(d.dphi + g);
    const int a = d.cell_ann[g];
    const Annulus &A = d.ann[a];
    const DiskParams &P = d.par[A.inst];
    const double a_sep = S.gr[0] + S.gr[1];
    const double dphi = d.dphi[g];
    const double rm = A.rm, rp = A.rp;
    double phi = d.tiphw[g] - .5 * dphi;
    double r = .5 * (rp + rm);
    T pm[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) pm[q] = ldq<T>(d.prim, tp.prim, q, N, g);
    SrcGeom sg;
    sg.r = r;
    sg.dt = dt;
    sg.dV = dphi * .5 * A.dv_diff * A.dz;
    sincos(phi, &sg.sinp, &sg.cosp);
    sg.xpos = r * sg.cosp;
    sg.ypos = r * sg.sinp;
    {
      double z = A.z;
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
    GravT<T> G;
    grav_t(G, S, P, tp, A.inst);
    T gu = 0.0, gpu = 0.0;
    if (P.has_visc) {
      // in 3-D cell_plm_rz(Z_DIR) has overwritten grad with the z slopes by the
      // time cell_add_visc_src reads it (timestep_routines.c:63-81)
      gu = (d.has_z && P.NZ > 1) ? T(d.gradz[(size_t)D_UPP * N + g]) : ldq<T>(d.grad, tp.grad, D_UPP, N, g);
      gpu = ldq<T>(d.gradp, tp.gradp, D_URR, N, g);
    }
    T sv[6];
    source_cell(sg, P, pm, gu, gpu, G, sv);
#pragma unroll
    for (int q = 0; q < 5; ++q) stq<T>(d.src, tp.src, q, N, g, sv[q]);
    if (P.has_visc) stq<T>(d.src, tp.src, 5, N, g, sv[5]);
    const double xpos = sg.xpos, ypos = sg.ypos, dV = sg.dV;
    const T rho = pm[D_RHO], Pp = pm[D_PPP];
    if (P.rho_sink_on == 1) {
      // get_rho_sink (src/Cell/cell_source.c:15-47); no tangent (refused by the
      // differentiated runs)
      const double rhov = val(rho), Pv = val(Pp);
      double r0 = sqrt((xpos - S.gx[0]) * (xpos - S.gx[0]) + (ypos - S.gy[0]) * (ypos - S.gy[0]));
      double r1 = sqrt((xpos - S.gx[1]) * (xpos - S.gx[1]) + (ypos - S.gy[1]) * (ypos - S.gy[1]));
      double M0 = S.gM[0], M1 = S.gM[1];
      double Mtotal = M0 + M1;
      double alpha = P.visc;
      double one_o_nu = 1.0 / (alpha * Pv / rhov) * sqrt(pow(r0, -3) * M0 / Mtotal + pow(r1, -3) * M1 / Mtotal);
      double t_visc0 = 1.0 * 2. / 3. * r0 * r0 * one_o_nu;
      double t_visc1 = 1.0 * 2. / 3. * r1 * r1 * one_o_nu;
      if (t_visc0 < 10. * dt) t_visc0 = 10. * dt;
      if (t_visc1 < 10. * dt) t_visc1 = 10. * dt;
      double sink_size = 0.5;
      for (int p = 0; p < P.num_sinks && p < 2; ++p) {
        double drho = 0.0;
        if (p == 0) { if (r0 < sink_size) drho = rhov / t_visc0; }
        else { if (r1 < sink_size) drho = rhov / t_visc1; }
        stq<T>(d.src, tp.src, 6 + p, N, g, T(drho * dt * dV));
        if (A.kind & DGPU_AK_SINK_SUM) {
          if (p == 0) md0 += drho * dV;
          else md1 += drho * dV;
        }
      }
    }
  }
}

template <typename T, int MB = DGPU_MINB_SOURCE, bool PS = false>
__global__ void __launch_bounds__(BLK, MB) k_source(DevPtrs d, TanPtrs tp, int substep, int cells) {
  __shared__ double sh_md[2][BLK / 32];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  const double fac = substep == 1 ? 1.0 : 0.5;
  if (t < d.n_ann) {
    const InstState &S = d.ist[d.ann[t].inst];
    ann_consts(d, t, S, fac * S.dt);
  }
  double md0 = 0.0, md1 = 0.0;
  if (t < N && cells) {
    const InstState &S = d.ist[d.ann[d.cell_ann[t]].inst];
    source_cell_k<T, PS>(d, tp, t, S, fac * S.dt, md0, md1);
  }
  // deterministic per-block Mdot partial sums (reduced in block order by k_update)
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    md0 += __shfl_down_sync(full, md0, o);
    md1 += __shfl_down_sync(full, md1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh_md[0][threadIdx.x >> 5] = md0;
    sh_md[1][threadIdx.x >> 5] = md1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && (size_t)blockIdx.x * BLK < (size_t)N) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < BLK / 32; ++w) {
      s0 += sh_md[0][w];
      s1 += sh_md[1][w];
    }
    d.mdot_part[2 * blockIdx.x] = s0;
    d.mdot_part[2 * blockIdx.x + 1] = s1;
  }
}

// The update of cell g after its face and source increments are in place:
// the conserved sum in the reference's order (update_sum),
// cell_update_phi/_dphi, cell_calc_prim, the fixed radial boundary,
// cell_bc_damp and cell_calc_cons.  dt: the substep's fac * dt.  XC: the
// increments were written by other blocks of the running kernel (plain loads,
// not the read-only path).  rec (the adjoint's segment replay, else NULL): the
// conserved sum before cons2prim and the new width of each cell go to slot
// 2 * (*rec_idx) + substep - 1 of rec ([slot][6][n_cells]).
template <typename T, bool PS, bool XC = false>
__device__ __forceinline__ void update_cell(const DevPtrs &d, const TanPtrs &tp, int g, int substep, int stop,
                                            double dt, double *rec, const int *rec_idx) {
  const int N = d.n_cells;
  {
    // the cell's own planes, before the annulus lookups they do not depend on
    pf_planes(d.cons, 5, N, g);
    if (substep == 2) {
      pf_planes(d.rkcons, 5, N, g);
      pf(d.rktiph + g);
    }
    pf_planes(d.fphi, 8, N, g);
    pf_planes(d.src, 6, N, g);
    pf(d.tiphw + g);
    pf((substep == 1 ? d.tiph0 : d.tiph1) + g);
    // and its r-face run ranges and first face, which k_merge just wrote
    pf(d.rr + 4 * (size_t)g);
    pf(d.fstart + g);
    const int a = d.cell_ann[g];
    const Annulus &A = d.ann[a];
    const DiskParams &P = d.par[A.inst];
    T c[5];
    double cp[DGPU_MAX_PASSIVE], pp[DGPU_MAX_PASSIVE];
    const int np = PS ? P.num_n : 0;
    if (np > 0) passive_sum(d, A, a, g, substep, stop, np, cp);
    if (!update_sum<T, !XC>(d, tp, A, a, g, substep, stop, dt, true, c)) {
#pragma unroll
      for (int q = 0; q < 5; ++q) stq<T>(d.cons, tp.cons, q, N, g, c[q]);
      for (int k = 0; k < np; ++k) d.cons[(size_t)(5 + k) * N + g] = cp[k];
    } else {
      double tn, rk;
      const double dphi_n = mesh_advance(d, A, a, g, substep, dt, tn, rk);
      if (substep == 1) d.rktiph[g] = rk;
      (substep == 1 ? d.tiph1 : d.tiph0)[g] = tn;
      d.dphi[g] = dphi_n;
      if (rec) {
        double *rs = rec + (size_t)(2 * (*rec_idx) + substep - 1) * 6 * N;
#pragma unroll
        for (int q = 0; q < 5; ++q) rs[(size_t)q * N + g] = val(c[q]);
        rs[(size_t)5 * N + g] = dphi_n;
      }
      // cell_calc_prim -> cell_cons2prim (src/Cell/cell_conversion.c:57-122)
      const double r = .5 * (A.rm + A.rp);
      const double dV = A.dv_half * dphi_n * A.dz;
      T pr[5];
      cons2prim(c, dV, r, P, pr);
      // passive scalars: prim = cons / cons[DDD] (cell_conversion.c:98-101)
      for (int k = 0; k < np; ++k) pp[k] = cp[k] / val(c[D_DDD]);
      // the outflow boundary reads these prims before any damping; the
      // annuli it rewrites are damped and converted by k_outflow
      if (A.ob_off >= 0 && stop >= 6) {
#pragma unroll
        for (int q = 0; q < 5; ++q) d.obuf[(size_t)q * d.n_ob + A.ob_off + (g - A.cell_off)] = val(pr[q]);
        for (int k = 0; k < np; ++k) d.obuf[(size_t)(5 + k) * d.n_ob + A.ob_off + (g - A.cell_off)] = pp[k];
      }
      const bool own = !(A.kind & DGPU_AK_OUT_DST);
      if (stop >= 6 && own) {
        bc_damp(d, A, a, pr);
        // cell_single_init_vortex's dye at the cell's new phi, in the fixed
        // boundary (cell_init_vortex.c:22-35); no other family sets one
        if (np > 0 && P.init_type == DI_VORTEX && (A.kind & DGPU_AK_BC_FIXED) && (A.kind & DGPU_AK_IC))
          pp[0] = cos(tn - .5 * dphi_n) < 0.0 ? 0.0 : 1.0;
      }
      // cell_calc_cons (src/Cell/cell_conversion.c:35-55)
      if (stop >= 7 && own) {
        prim2cons(pr, c, r, dV, P.gamma);
        for (int k = 0; k < np; ++k) cp[k] = pp[k] * val(c[D_DDD]);
      }
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        stq<T>(d.prim, tp.prim, q, N, g, pr[q]);
        stq<T>(d.cons, tp.cons, q, N, g, c[q]);
      }
      for (int k = 0; k < np; ++k) {
        d.prim[(size_t)(5 + k) * N + g] = pp[k];
        d.cons[(size_t)(5 + k) * N + g] = cp[k];
      }
    }
  }
}

// GravMass after the substep for disk k: gravMass_update_RK
// (GravMass_misc.c:66-77), then gravMass_move(t, fac*dt) (GravMass_misc.c:31-64);
// after substep 2 also t += dt and Macc += Mdot*dt (timestep_algorithm.c:27-39).
// S.gphi holds the substep's wrapped phases (gravMass_clean_pi) and S.mdot
// the substep's sink rates.
__device__ __forceinline__ void gm_tail(const DevPtrs &d, InstState &S, const DiskParams &P, int substep,
                                        int tail) {
  const double RK = substep == 1 ? 0.0 : 0.5;
  const double fac = substep == 1 ? 1.0 : 0.5;
  for (int p = 0; p < 2; ++p) {
    S.grk_phi[p] = adjust_toward(S.gphi[p], S.grk_phi[p], M_PI, 2. * M_PI, d.err);
    S.gr[p] = (1.0 - RK) * S.gr[p] + RK * S.grk_r[p];
    S.gphi[p] = (1.0 - RK) * S.gphi[p] + RK * S.grk_phi[p];
    S.gM[p] = (1.0 - RK) * S.gM[p] + RK * S.grk_M[p];
    S.gom[p] = (1.0 - RK) * S.gom[p] + RK * S.grk_om[p];
  }
  if (tail >= 2) {
    double t = S.t, dtm = fac * S.dt;
    double m0 = S.gM[0], m1 = S.gM[1];
    double M = m0 + m1;
    double a_0 = 1.0, tau_0 = P.orb_tscale, T0 = P.orb_t0;
    double asep, omega;
    if ((t - T0) / tau_0 < 1.) {
      asep = a_0 * pow((1.0 - (t - T0) / tau_0), 0.25);
      omega = pow(asep / M, -1.5);
    } else {
      asep = 0.0;
      omega = 0.0;
    }
    double r0, r1;
    if (M < 1.e-12) {
      r0 = 0.0;
      r1 = 0.0;
    } else {
      r0 = m1 / M * asep;
      r1 = m0 / M * asep;
    }
    S.gphi[0] += omega * dtm;
    S.gphi[1] += omega * dtm;
    S.gr[0] = r0;
    S.gr[1] = r1;
    S.gom[0] = omega;
    S.gom[1] = omega;
    if (substep == 2) {
      S.t += S.dt;
      for (int p = 0; p < 2; ++p) S.macc[p] = S.macc[p] + S.mdot[p] * S.dt;
    }
  }
}

template <typename T, int MB = DGPU_MINB_UPDATE, bool PS = false>
__global__ void __launch_bounds__(BLK, MB) k_update(DevPtrs d, TanPtrs tp, int substep, int stop,
                                                                  int tail, double *rec, const int *rec_idx) {
  __shared__ bool last;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  const double fac = substep == 1 ? 1.0 : 0.5;
  if (g < N) {
    const InstState &S = d.ist[d.ann[d.cell_ann[g]].inst];
    update_cell<T, PS>(d, tp, g, substep, stop, fac * S.dt, rec, rec_idx);
  }
  if (tail == 0) return;
  // the last block reads nothing the other blocks write (mdot_part comes from
  // k_source), so no fence is needed before the count
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&d.counters[1], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
    InstState &S = d.ist[k];
    const DiskParams &P = d.par[k];
    // Mdot of this disk: block partials in block order
    {
      int c0 = P.cell_base, c1 = P.cell_base + P.n_cells;
      int b0 = c0 / BLK, b1 = (c1 + BLK - 1) / BLK;
      double s0 = 0.0, s1 = 0.0;
      if (P.rho_sink_on == 1) {
        for (int b = b0; b < b1; ++b) {
          s0 += d.mdot_part[2 * b];
          s1 += d.mdot_part[2 * b + 1];
        }
      }
      S.mdot[0] = s0;
      S.mdot[1] = s1;
    }
    gm_tail(d, S, P, substep, tail);
  }
  if (threadIdx.x == 0) d.counters[1] = 0;
}

// ---------------------------------------------------------------------------
// The fused substep: k_prep then k_sweep
// ---------------------------------------------------------------------------
// k_prep: one block per annulus a of every disk.  The face list of pair
// (a, a+1) and cell_set_w (merge_pair), cell_clean_pi and cell_plm_p of the
// annulus's cells and, in substep 1, gravMass_copy and the annulus's CFL
// minimum (cell_mindt, src/Cell/cell_mindt.c:10-100), from which every block of
// k_sweep forms the disk's dt (timestep_set_dt).  It also clears the sweep's
// progress flags and work counters.
template <int MB>
__global__ void __launch_bounds__(BLK, MB) k_prep(DevPtrs d, int substep) {
  __shared__ unsigned long long sh_k[BLK / 32];
  __shared__ double sh_rk[6];
  const int a = blockIdx.x;
  const TanPtrs tp = {};
  merge_pair<false>(d, a, substep);
  __syncthreads();  // w_ann[a] (one lane) before the CFL
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  for (int j = threadIdx.x; j < A.np; j += BLK) cellprep_cell<double, false>(d, tp, A.cell_off + j, substep);
  if (threadIdx.x == 0) {
    d.sweep_flag[a] = 0;
    if (a == 0) {
      d.counters[3] = 0;
      d.counters[4] = 0;
    }
  }
  if (substep != 1) return;
  if (threadIdx.x == 0) {
    InstState &S = d.ist[A.inst];
    // gravMass_dist of the step-start positions, for the CFL's viscosity
    for (int p = 0; p < 2; ++p) {
      sh_rk[p] = S.gr[p] * cos(S.gphi[p]);
      sh_rk[2 + p] = S.gr[p] * sin(S.gphi[p]);
      sh_rk[4 + p] = S.gM[p];
    }
    if (A.i == 0) {
      // gravMass_copy (GravMass_misc.c:20-28); no block of this kernel reads
      // these copies
      for (int p = 0; p < 2; ++p) {
        S.grk_r[p] = S.gr[p];
        S.grk_phi[p] = S.gphi[p];
        S.grk_M[p] = S.gM[p];
        S.grk_om[p] = S.gom[p];
      }
    }
  }
  __syncthreads();
  unsigned long long key = ~0ull;
  if (A.kind & DGPU_AK_CFL) {
    const double wa = d.w_ann[a];
    for (int j = threadIdx.x; j < A.np; j += BLK) {
      const unsigned long long k = cfl_key(d, A, P, A.cell_off + j, wa, sh_rk, sh_rk + 2, sh_rk + 4);
      key = k < key ? k : key;
    }
  }
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long k2 = __shfl_down_sync(full, key, o);
    key = k2 < key ? k2 : key;
  }
  if ((threadIdx.x & 31) == 0) sh_k[threadIdx.x >> 5] = key;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < BLK / 32; ++w) key = sh_k[w] < key ? sh_k[w] : key;
    d.cfl_ann[a] = key;
  }
}

// dt of a disk from k_prep's per-annulus CFL minima: the minimum (1e100 when
// no cell has a candidate), clipped to Time_Max (timestep_set_dt,
// src/TimeStep/timestep_set.c:16-21).  The same value as k_plm_r + k_dt form.
__device__ __forceinline__ double sweep_dt(const DevPtrs &d, const DiskParams &P, double t) {
  unsigned long long key = (unsigned long long)__double_as_longlong(1.e100);
  for (int k = P.ann_base; k < P.ann_base + P.NR; ++k) {
    const unsigned long long v = d.cfl_ann[k];
    key = v < key ? v : key;
  }
  double dt = __longlong_as_double((long long)key);
  if (t + dt > P.t_max) dt = P.t_max - t;
  return dt;
}

// Progress flags of k_sweep: after a __syncthreads, thread 0 publishes that
// this block's phase v of annulus a is done (its stores ordered before the
// flag), or waits until the block of annulus a has published v (the block's
// later loads ordered after the flag).  A wait gives up after
// DGPU_SWEEP_SPIN_LIMIT polls, reports DGPU_EF_SWEEP_WAIT and returns.
#define DGPU_SWEEP_SPIN_LIMIT (1 << 18)
__device__ __forceinline__ void sweep_publish(const DevPtrs &d, int a, int v) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(d.sweep_flag + a), "r"(v) : "memory");
  }
}
__device__ __forceinline__ void sweep_wait(const DevPtrs &d, int a, int v) {
  if (threadIdx.x == 0) {
    int it = 0, f;
    for (;;) {
      asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(f) : "l"(d.sweep_flag + a) : "memory");
      if (f >= v) break;
      if (++it > DGPU_SWEEP_SPIN_LIMIT) {
        set_err(d.err, DGPU_EF_SWEEP_WAIT);
        break;
      }
      __nanosleep(100);
    }
  }
  __syncthreads();
}

// The phases of k_sweep for the block's annulus (the block's threads stride
// over the annulus's faces or cells).  Inlined: as separate calls they spill
// more across the call boundaries and run slower (measured).
#define SWEEP_FN __device__ __forceinline__
SWEEP_FN void sweep_slopes(const DevPtrs &d, int a) {
  const TanPtrs tp = {};
  const Annulus &A = d.ann[a];
  const int nf = d.pair_nf[a];
  for (int n = threadIdx.x; n < nf; n += BLK) rslope_face<double, false>(d, tp, A.face_base + n);
}
SWEEP_FN void sweep_grad(const DevPtrs &d, int a) {
  const TanPtrs tp = {};
  const Annulus &A = d.ann[a];
  for (int j = threadIdx.x; j < A.np; j += BLK) plm_r_grad<double, false>(d, tp, A.cell_off + j);
}
SWEEP_FN void sweep_flux_r(const DevPtrs &d, int b, const InstState &S, double dt) {
  const TanPtrs tp = {};
  const Annulus &Q = d.ann[b];
  const int nf = d.pair_nf[b];
  for (int n = threadIdx.x; n < nf; n += BLK) flux_r_face<double, false>(d, tp, Q.face_base + n, S, dt);
}
SWEEP_FN void sweep_cells(const DevPtrs &d, int a, const InstState &S, double dt) {
  const TanPtrs tp = {};
  const Annulus &A = d.ann[a];
  double md0 = 0.0, md1 = 0.0;
  for (int j = threadIdx.x; j < A.np; j += BLK) {
    const int g = A.cell_off + j;
    flux_phi_cell<double, false>(d, tp, g, S, dt);
    source_cell_k<double, false>(d, tp, g, S, dt, md0, md1);
  }
}
SWEEP_FN void sweep_update_cells(const DevPtrs &d, int b, int substep, double dt) {
  const TanPtrs tp = {};
  const Annulus &B = d.ann[b];
  for (int j = threadIdx.x; j < B.np; j += BLK)
    update_cell<double, false, true>(d, tp, B.cell_off + j, substep, 7, dt, nullptr, nullptr);
}

// The update of annulus b's cells (update_cell) once its increments are in
// place, with the annulus's constants of the substep.
__device__ __forceinline__ void sweep_update(const DevPtrs &d, int b, int substep, const InstState &S, double dt) {
  if (threadIdx.x == 0) ann_consts(d, b, S, dt);
  __syncthreads();
  sweep_update_cells(d, b, substep, dt);
}

// k_sweep: the rest of the substep as one wavefront over the annuli.  Each
// block takes the next annulus a in order (a work counter, so every earlier
// annulus is held by a block that is already running) and does, waiting only
// on the block of annulus a-1 of the same disk:
//   1. the face slopes S and offsets of the faces of pair (a, a+1) (k_rslope);
//   2. the r slopes of annulus a (cell_plm_rz) -- needs 1. of a-1;
//   3. the fluxes of the faces of pair (a-1, a) (riemann_setup_rz +
//      riemann_AddFlux) -- needs 2. of a-1 -- and the phi faces and source
//      increments of annulus a;
//   4. the update of annulus a-1 (and of a itself when it is the disk's last),
//      whose increments are then all in place -- needs 3. of a-1.
// A block never waits for a later annulus, so the wavefront always advances.
// The last block to finish advances the GravMass state (gm_tail).  The
// increments pass between neighbouring annuli through L2 instead of HBM round
// trips between eight kernels, and phases of different annuli overlap on the
// SMs.
template <int MB>
__global__ void __launch_bounds__(BLK, MB) k_sweep(const __grid_constant__ DevPtrs d, int substep) {
  __shared__ int s_a;
  __shared__ InstState s_S;
  __shared__ bool s_last;
  if (threadIdx.x == 0) s_a = (int)atomicAdd(&d.counters[3], 1u);
  __syncthreads();
  const int a = s_a;
  const Annulus &A = d.ann[a];
  const DiskParams &P = d.par[A.inst];
  if (threadIdx.x == 0) {
    // the disk's state with the substep's GravMass positions (gravMass_clean_pi,
    // then gravMass_dist's r cos(phi), r sin(phi)) and, in substep 1, its dt
    s_S = d.ist[A.inst];
    for (int p = 0; p < 2; ++p) {
      const double ph = wrap_pos(s_S.gphi[p], d.err);
      s_S.gphi[p] = ph;
      s_S.gc[p] = cos(ph);
      s_S.gs[p] = sin(ph);
      s_S.gx[p] = s_S.gr[p] * s_S.gc[p];
      s_S.gy[p] = s_S.gr[p] * s_S.gs[p];
    }
    if (substep == 1) s_S.dt = sweep_dt(d, P, s_S.t);
  }
  __syncthreads();
  const double dt = (substep == 1 ? 1.0 : 0.5) * s_S.dt;
  const int first = A.i == 0, last = A.i == P.NR - 1;
  // 1. face slopes of pair (a, a+1)
  if (!last) sweep_slopes(d, a);
  sweep_publish(d, a, 1);
  // 2. r slopes of annulus a
  if (!first) sweep_wait(d, a - 1, 1);
  sweep_grad(d, a);
  sweep_publish(d, a, 2);
  // 3. fluxes of pair (a-1, a); phi faces and sources of annulus a
  if (!first) {
    sweep_wait(d, a - 1, 2);
    sweep_flux_r(d, a - 1, s_S, dt);
  }
  sweep_cells(d, a, s_S, dt);
  sweep_publish(d, a, 3);
  // 4. update of annulus a-1, then of the disk's last annulus
  if (!first) {
    sweep_wait(d, a - 1, 3);
    sweep_update(d, a - 1, substep, s_S, dt);
  }
  if (last) {
    __syncthreads();
    sweep_update(d, a, substep, s_S, dt);
  }
  // the last block: the GravMass of every disk.  It reads nothing that
  // another block of this kernel writes.
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&d.counters[4], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  for (int k = threadIdx.x; k < d.n_inst; k += BLK) {
    InstState &S = d.ist[k];
    const DiskParams &Pk = d.par[k];
    if (substep == 1) S.dt = sweep_dt(d, Pk, S.t);
    for (int p = 0; p < 2; ++p) S.gphi[p] = wrap_pos(S.gphi[p], d.err);
    S.mdot[0] = 0.0;  // no sink on this path
    S.mdot[1] = 0.0;
    gm_tail(d, S, Pk, substep, 2);
  }
  if (threadIdx.x == 0) {
    d.counters[3] = 0;
    d.counters[4] = 0;
  }
}

// cell_calc_cons over all cells (set-up and state upload)
template <typename T, bool PS = false>
__global__ void __launch_bounds__(BLK) k_calc_cons(DevPtrs d, TanPtrs tp) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = d.n_cells;
  if (g >= N) return;
  const Annulus &A = d.ann[d.cell_ann[g]];
  const DiskParams &P = d.par[A.inst];
  double r = .5 * (A.rp + A.rm);
  double dV = A.dv_half * d.dphi[g] * A.dz;
  T p[5], c[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) p[q] = ldq<T>(d.prim, tp.prim, q, N, g);
  prim2cons(p, c, r, dV, P.gamma);
#pragma unroll
  for (int q = 0; q < 5; ++q) stq<T>(d.cons, tp.cons, q, N, g, c[q]);
  for (int q = 5; q < 5 + (PS ? P.num_n : 0); ++q) d.cons[(size_t)q * N + g] = ld(d.prim, q, N, g) * val(c[D_DDD]);
}

// One pass of cell_boundary_outflow_r (src/Cell/cell_boundary.c:14-139) over
// the r faces of annulus pair (i, i+1) of the substep's face list: every cell
// of the rewritten annulus (i when outer == 0, else i+1) takes the sum, in face
// order, of prim * dA of the cells across its faces, divided by
// dz * FacePos(i) * dphi.  The reference's build constants EXTRAP_BC, SS_BCS,
// diode and KEP_BNDRY are 0 (header.h); its inner term
// (prim - 0 * grad * (...) / 2.) * dA is prim * dA for a finite slope.  A cell
// with no face keeps its own value, divided (the reference zeroes only the
// cells its face loop visits).
__device__ __forceinline__ void outflow_pass(const DevPtrs &d, const DiskParams &P, int base, int i, int outer) {
  const int a = base + i + outer;
  const Annulus &A = d.ann[a];
  const Annulus &S = d.ann[base + i + 1 - outer];  // the annulus read
  const double rf = d.ann[base + i].f_r;           // FacePos(i)
  const size_t NB = d.n_ob;
  const int nq = 5 + P.num_n;
  const int np = nq - 5;
  for (int j = threadIdx.x; j < A.np; j += blockDim.x) {
    const int g = A.cell_off + j;
    // the five hydro sums in registers, the passive scalars' apart
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, sp[DGPU_MAX_PASSIVE];
    for (int k = 0; k < np; ++k) sp[k] = 0.0;
    int nface = 0;
    for_cell_rfaces(d, A, a, g, P.NR, [&](const RFace &F, int, int side) {
      if (side != outer) return;
      const int o = S.ob_off + ((outer ? F.cL : F.cR) - S.cell_off);
      const double dA = F.r * F.dphi * F.dperp;
#pragma unroll
      for (int q = 0; q < 5; ++q) s[q] += d.obuf[q * NB + o] * dA;
      for (int k = 0; k < np; ++k) sp[k] += d.obuf[(5 + k) * NB + o] * dA;
      ++nface;
    });
    const double dA = A.dz * rf * d.dphi[g];
    const size_t self = (size_t)A.ob_off + j;
#pragma unroll
    for (int q = 0; q < 5; ++q) d.obuf[q * NB + self] = (nface ? s[q] : d.obuf[q * NB + self]) / dA;
    for (int k = 0; k < np; ++k)
      d.obuf[(5 + k) * NB + self] = (nface ? sp[k] : d.obuf[(5 + k) * NB + self]) / dA;
  }
}

// The outflow radial boundary of one layer of a disk per block (blockIdx.x:
// the disk, blockIdx.y: the layer), in the reference's order: annulus 0 from
// annulus 1 (unless NoInnerBC == 1), NR-2 from NR-3, NR-1 from the new NR-2;
// each pass reads the previous one's results.  The r faces join rings of one
// layer, so the layers are independent.  Then the rewritten annuli get
// cell_bc_damp and, for stop 7, cell_calc_cons.
__global__ void __launch_bounds__(BLK) k_outflow(DevPtrs d, int stop) {
  const DiskParams &P = d.par[blockIdx.x];
  if (!(P.outflow & 1) || (int)blockIdx.y >= P.NZ) return;
  const int NR = P.NR, N = d.n_cells;
  const int base = P.ann_base + (int)blockIdx.y * NR;
  const size_t NB = d.n_ob;
  if (P.outflow & 2) outflow_pass(d, P, base, 0, 0);
  __syncthreads();
  outflow_pass(d, P, base, NR - 3, 1);
  __syncthreads();
  outflow_pass(d, P, base, NR - 2, 1);
  __syncthreads();
  for (int k = 0; k < 3; ++k) {
    const int i = k == 0 ? 0 : NR - 3 + k;
    const int a = base + i;
    const Annulus &A = d.ann[a];
    if (!(A.kind & DGPU_AK_OUT_DST)) continue;
    const double r = .5 * (A.rm + A.rp);
    for (int j = threadIdx.x; j < A.np; j += blockDim.x) {
      const int g = A.cell_off + j;
      double pr[5], c[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) pr[q] = d.obuf[q * NB + A.ob_off + j];
      bc_damp(d, A, a, pr);
#pragma unroll
      for (int q = 0; q < 5; ++q) d.prim[(size_t)q * N + g] = pr[q];
      for (int q = 5; q < 5 + P.num_n; ++q) d.prim[(size_t)q * N + g] = d.obuf[q * NB + A.ob_off + j];
      if (stop >= 7) {
        const double dV = A.dv_half * d.dphi[g] * A.dz;
        prim2cons(pr, c, r, dV, P.gamma);
#pragma unroll
        for (int q = 0; q < 5; ++q) d.cons[(size_t)q * N + g] = c[q];
        for (int q = 5; q < 5 + P.num_n; ++q) d.cons[(size_t)q * N + g] = d.obuf[q * NB + A.ob_off + j] * c[D_DDD];
      }
    }
  }
}

// Torque on the binary: -sum over non-ghost cells of r*rho*dV*F_phi, with the
// gas state's cell-centre phi and F_phi from gravMassForce; per-block partial
// sums, reduced in block order by the last block.
__global__ void __launch_bounds__(BLK) k_torque(DevPtrs d, int inst, double *part, double *out) {
  __shared__ double sh[BLK / 32];
  __shared__ bool last;
  const DiskParams &P = d.par[inst];
  const InstState &S = d.ist[inst];
  const int N = d.n_cells;
  const int g = P.cell_base + blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (g < P.cell_base + P.n_cells) {
    const Annulus &A = d.ann[d.cell_ann[g]];
    if (A.kind & DGPU_AK_CFL) {
      double dphi = d.dphi[g];
      double phi = d.tiph0[g] - .5 * dphi;
      double r = .5 * (A.rp + A.rm);
      double rho = ld(d.prim, D_RHO, N, g);
      double dV = dphi * .5 * A.dv_diff * P.dz;
      double cosp = cos(phi), sinp = sin(phi);
      double Fp = 0.0;
      for (int p = 0; p < 2; ++p) {
        double dx = r * cosp - S.gr[p] * cos(S.gphi[p]);
        double dy = r * sinp - S.gr[p] * sin(S.gphi[p]);
        double script_r = sqrt(dx * dx + dy * dy);
        double cosa = dx / script_r, sina = dy / script_r;
        double sinap = sina * cosp - cosa * sinp;
        Fp += sinap * -fgrav(S.gM[p], script_r, P.g_eps, P.phi_order);
      }
      v = -(r * rho * dV * Fp);
    }
  }
  const unsigned full = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < BLK / 32; ++w) s += sh[w];
    part[blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&d.counters[2], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double s = 0.0;
  for (int b = 0; b < (int)gridDim.x; ++b) s += ((volatile double *)part)[b];
  *out = s;
  d.counters[2] = 0;
}

// AoS rows [n][nq] (the boundary format) <-> SoA columns X[q*stride + base + c]
__global__ void k_aos_to_soa(double *soa, int nq, int stride, int base, const double *aos, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = 0; q < nq; ++q) soa[(size_t)q * stride + base + c] = aos[(size_t)c * nq + q];
}
__global__ void k_soa_to_aos(double *aos, int nq, int stride, int base, const double *soa, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int q = 0; q < nq; ++q) aos[(size_t)c * nq + q] = soa[(size_t)q * stride + base + c];
}

}  // namespace

extern "C" {

int dgk_aos_to_soa(double *soa, int nq, int stride, int base, const double *aos, int n, void *stream) {
  if (n <= 0) return 0;
  k_aos_to_soa<<<(n + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(soa, nq, stride, base, aos, n);
  return (int)cudaGetLastError();
}
int dgk_soa_to_aos(double *aos, int nq, int stride, int base, const double *soa, int n, void *stream) {
  if (n <= 0) return 0;
  k_soa_to_aos<<<(n + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(aos, nq, stride, base, soa, n);
  return (int)cudaGetLastError();
}

int dgk_update_blocks(int n_cells) { return (n_cells + BLK - 1) / BLK; }
int dgk_block_size(void) { return BLK; }

// t == NULL: the forward kernels; otherwise their tangent instances.
// Contexts with passive scalars take the instances that carry them (PS).
#define DGK_LAUNCH(kern, grid, smem, stream, ...)                                                  \
  do {                                                                                            \
    static const TanPtrs none_ = {};                                                              \
    if (t) kern<Dual><<<(grid), BLK, (smem), (cudaStream_t)(stream)>>>(*d, *t, __VA_ARGS__);       \
    else if (d->n_pass > 0)                                                                       \
      kern<double, true><<<(grid), BLK, (smem), (cudaStream_t)(stream)>>>(*d, none_, __VA_ARGS__); \
    else kern<double><<<(grid), BLK, (smem), (cudaStream_t)(stream)>>>(*d, none_, __VA_ARGS__);    \
  } while (0)
// The same for the kernels the autotuner sizes: the forward instance with
// d->tune[which] resident blocks per SM (0: the built-in choice).
#define DGK_LAUNCH_TUNED(kern, which, mbdef, grid, stream, ...)                           \
  do {                                                                                   \
    static const TanPtrs none_ = {};                                                     \
    cudaStream_t s_ = (cudaStream_t)(stream);                                            \
    if (t) {                                                                             \
      kern<Dual><<<(grid), BLK, 0, s_>>>(*d, *t, __VA_ARGS__);                            \
    } else if (d->n_pass > 0) {                                                          \
      kern<double, mbdef, true><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__);          \
    } else {                                                                             \
      switch (d->tune[which]) {                                                          \
        case 2: kern<double, 2><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__); break;   \
        case 3: kern<double, 3><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__); break;   \
        case 4: kern<double, 4><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__); break;   \
        case 5: kern<double, 5><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__); break;   \
        default: kern<double><<<(grid), BLK, 0, s_>>>(*d, none_, __VA_ARGS__);           \
      }                                                                                  \
    }                                                                                    \
  } while (0)

int dgk_cellprep(const DevPtrs *d, const TanPtrs *t, int substep, void *stream) {
  DGK_LAUNCH(k_cellprep, (d->n_cells + BLK - 1) / BLK, 0, stream, substep);
  return (int)cudaGetLastError();
}
int dgk_merge(const DevPtrs *d, int substep, void *stream) {
  k_merge<<<d->n_ann, d->merge_nt > 0 ? d->merge_nt : BLK, d->smem_face, (cudaStream_t)stream>>>(*d, substep);
  return (int)cudaGetLastError();
}
int dgk_rslope(const DevPtrs *d, const TanPtrs *t, void *stream) {
  if (d->n_slots <= 0) return 0;
  static const TanPtrs none = {};
  if (t) k_rslope<Dual><<<(d->n_slots + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, *t);
  else if (d->n_pass > 0) k_rslope<double, true><<<(d->n_slots + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, none);
  else k_rslope<double><<<(d->n_slots + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, none);
  return (int)cudaGetLastError();
}
int dgk_plm_r(const DevPtrs *d, const TanPtrs *t, int substep, void *stream) {
  DGK_LAUNCH_TUNED(k_plm_r, DGPU_TUNE_PLM, DGPU_MINB_PLM, (d->n_cells + BLK - 1) / BLK, stream, substep);
  if (substep == 1) k_dt<<<1, BLK, 0, (cudaStream_t)stream>>>(*d);
  return (int)cudaGetLastError();
}
int dgk_flux_phi(const DevPtrs *d, const TanPtrs *t, int substep, void *stream) {
  DGK_LAUNCH_TUNED(k_flux_phi, DGPU_TUNE_FLUXPHI, DGPU_MINB_FLUX, (d->n_cells + BLK - 1) / BLK, stream, substep);
  return (int)cudaGetLastError();
}
int dgk_flux_r(const DevPtrs *d, const TanPtrs *t, int substep, void *stream) {
  if (d->n_slots <= 0) return 0;
  DGK_LAUNCH_TUNED(k_flux_r, DGPU_TUNE_FLUXR, DGPU_MINB_FLUXR, (d->n_slots + BLK - 1) / BLK, stream, substep);
  return (int)cudaGetLastError();
}
int dgk_source(const DevPtrs *d, const TanPtrs *t, int substep, void *stream) {
  int n = d->n_cells > d->n_ann ? d->n_cells : d->n_ann;
  DGK_LAUNCH_TUNED(k_source, DGPU_TUNE_SOURCE, DGPU_MINB_SOURCE, (n + BLK - 1) / BLK, stream, substep, 1);
  return (int)cudaGetLastError();
}
int dgk_update(const DevPtrs *d, const TanPtrs *t, int substep, int stop, void *stream) {
  int tail = stop >= 7 ? 2 : (stop >= 5 ? 1 : 0);
  DGK_LAUNCH_TUNED(k_update, DGPU_TUNE_UPDATE, DGPU_MINB_UPDATE, dgk_update_blocks(d->n_cells), stream, substep, stop, tail,
                   (double *)NULL, (const int *)NULL);
  return (int)cudaGetLastError();
}
int dgk_update_rec(const DevPtrs *d, int substep, double *rec, const int *rec_idx, void *stream) {
  static const TanPtrs none = {};
  k_update<double><<<dgk_update_blocks(d->n_cells), BLK, 0, (cudaStream_t)stream>>>(*d, none, substep, 7, 2, rec,
                                                                                      rec_idx);
  return (int)cudaGetLastError();
}
int dgk_ann_consts(const DevPtrs *d, int substep, void *stream) {
  static const TanPtrs none = {};
  k_source<double><<<(d->n_ann + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, none, substep, 0);
  return (int)cudaGetLastError();
}
int dgk_update_stage(const DevPtrs *d, int substep, int stop, void *stream) {
  int tail = stop >= 5 ? 1 : 0;
  static const TanPtrs none = {};
  if (d->n_pass > 0)
    k_update<double, DGPU_MINB_UPDATE, true><<<dgk_update_blocks(d->n_cells), BLK, 0, (cudaStream_t)stream>>>(
        *d, none, substep, stop, tail, nullptr, nullptr);
  else
    k_update<double><<<dgk_update_blocks(d->n_cells), BLK, 0, (cudaStream_t)stream>>>(*d, none, substep, stop,
                                                                                        tail, nullptr, nullptr);
  return (int)cudaGetLastError();
}
int dgk_zmerge(const DevPtrs *d, int substep, void *stream) {
  if (!d->has_z) return 0;
  k_zmerge<<<d->n_ann, d->merge_nt > 0 ? d->merge_nt : BLK, d->smem_face, (cudaStream_t)stream>>>(*d, substep);
  return (int)cudaGetLastError();
}
int dgk_zslope(const DevPtrs *d, void *stream) {
  if (!d->has_z || d->n_zslots <= 0) return 0;
  k_zslope<<<(d->n_zslots + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d);
  return (int)cudaGetLastError();
}
int dgk_plm_z(const DevPtrs *d, void *stream) {
  if (!d->has_z) return 0;
  k_plm_z<<<(d->n_cells + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d);
  return (int)cudaGetLastError();
}
int dgk_flux_z(const DevPtrs *d, int substep, void *stream) {
  if (!d->has_z || d->n_zslots <= 0) return 0;
  k_flux_z<<<(d->n_zslots + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, substep);
  return (int)cudaGetLastError();
}
int dgk_zsync(const DevPtrs *d, int substep, void *stream) {
  if (!d->has_z) return 0;
  const int n = d->zghost > 0 ? 2 * d->zghost : d->n_cells;
  k_zsync<<<(n + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, substep);
  return (int)cudaGetLastError();
}
int dgk_prep(const DevPtrs *d, int substep, void *stream) {
  k_prep<DGPU_MINB_PREP><<<d->n_ann, BLK, d->smem_face, (cudaStream_t)stream>>>(*d, substep);
  return (int)cudaGetLastError();
}
int dgk_sweep(const DevPtrs *d, int substep, void *stream) {
  cudaStream_t s_ = (cudaStream_t)stream;
  switch (d->tune[DGPU_TUNE_SWEEP]) {
    case 2: k_sweep<2><<<d->n_ann, BLK, 0, s_>>>(*d, substep); break;
    case 4: k_sweep<4><<<d->n_ann, BLK, 0, s_>>>(*d, substep); break;
    default: k_sweep<DGPU_MINB_SWEEP><<<d->n_ann, BLK, 0, s_>>>(*d, substep);
  }
  return (int)cudaGetLastError();
}
int dgk_outflow(const DevPtrs *d, int stop, void *stream) {
  if (d->n_ob <= 0 || stop < 6) return 0;
  k_outflow<<<dim3(d->n_inst, d->max_nz), BLK, 0, (cudaStream_t)stream>>>(*d, stop);
  return (int)cudaGetLastError();
}
int dgk_calc_cons(const DevPtrs *d, const TanPtrs *t, void *stream) {
  static const TanPtrs none = {};
  if (t) k_calc_cons<Dual><<<(d->n_cells + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, *t);
  else if (d->n_pass > 0) k_calc_cons<double, true><<<(d->n_cells + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, none);
  else k_calc_cons<double><<<(d->n_cells + BLK - 1) / BLK, BLK, 0, (cudaStream_t)stream>>>(*d, none);
  return (int)cudaGetLastError();
}
int dgk_torque(const DevPtrs *d, int inst, double *part, double *out, int n_inst_cells, void *stream) {
  int nb = (n_inst_cells + BLK - 1) / BLK;
  k_torque<<<nb, BLK, 0, (cudaStream_t)stream>>>(*d, inst, part, out);
  return (int)cudaGetLastError();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Face list without allocation (dgpu_face_list_noalloc).
//
// For callers that cannot allocate device memory: the face list of one disk is
// built from the caller's device arrays into the caller's device arrays, and
// the only working memory is g_noalloc_scratch below, a fixed static array
// that every GPU loading this library holds until the process exits.  Per
// annulus pair it keeps only counts and offsets, so its size is set by the
// number of annuli (DGPU_NOALLOC_MAX_ANNULI), not by the number of cells.
// ---------------------------------------------------------------------------
extern "C" {
#include "dgpu_sim.h"
}

#define NOALLOC_MAXA DGPU_NOALLOC_MAX_ANNULI

struct NoallocScratch {
  int np[NOALLOC_MAXA];        // N_p per annulus
  int off[NOALLOC_MAXA];       // first cell of each annulus
  int cnt[NOALLOC_MAXA];       // faces per pair
  int base[NOALLOC_MAXA + 1];  // first face of each pair; base[NR-1] = total
  double rface[NOALLOC_MAXA + 1];
  double dperp;
  int err;                     // DGPU_EF_* flags of this call
  int total;
  int fill_ok;                 // written only by k_noalloc_offsets: 1 when total <= cap
};
static_assert(sizeof(NoallocScratch) <= DGPU_NOALLOC_SCRATCH_BYTES, "scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[DGPU_NOALLOC_SCRATCH_BYTES];

namespace {

__global__ void k_noalloc_setup(NoallocScratch *S, int NR) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int o = 0;
  for (int i = 0; i < NR; ++i) {
    S->off[i] = o;
    o += S->np[i];
  }
  S->err = 0;
  S->total = 0;
  S->fill_ok = 0;
}

// Chunk start, count and verification of one pair; the same decisions as k_merge.
struct PairPlan {
  int jpmin, jp_start, j0, j1, cnt, sequential;
};

__device__ PairPlan noalloc_plan(const FaceCtx &c, int *sh_i, int *sh_j, double *sh_v, int *sh_flag) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int np = c.Nin;
  const double p0 = c.tin[np - 1];
  PairPlan pl;
  double bv = PHIMAX;
  int bi = 0;
  for (int jp = tid; jp < c.Nout; jp += nt) {
    double dp = wrap_pos(c.tout[jp] - p0, c.err);
    if (dp < bv || (dp == bv && jp < bi)) {
      bv = dp;
      bi = jp;
    }
  }
  sh_v[tid] = bv;
  sh_i[tid] = bi;
  __syncthreads();
  for (int o = nt / 2; o > 0; o >>= 1) {
    if (tid < o) {
      double v2 = sh_v[tid + o];
      int i2 = sh_i[tid + o];
      if (v2 < sh_v[tid] || (v2 == sh_v[tid] && i2 < sh_i[tid])) {
        sh_v[tid] = v2;
        sh_i[tid] = i2;
      }
    }
    __syncthreads();
  }
  pl.jpmin = sh_i[0];
  __syncthreads();
  const int chunk = (np + nt - 1) / nt;
  pl.j0 = min(np, tid * chunk);
  pl.j1 = min(np, pl.j0 + chunk);
  pl.jp_start = pl.jpmin;
  if (pl.j0 > 0 && pl.j0 < np) {
    double L = wrap_pos(c.tin[pl.j0 - 1] - p0, c.err);
    int lo = 0, hi = c.Nout;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      int k = pl.jpmin + mid;
      if (k >= c.Nout) k -= c.Nout;
      double e = wrap_pos(c.tout[k] - p0, c.err);
      if (e < L) lo = mid + 1;
      else hi = mid;
    }
    pl.jp_start = pl.jpmin + lo;
    if (pl.jp_start >= c.Nout) pl.jp_start -= c.Nout;
  }
  int jp = pl.jp_start, n = 0, s = 0;
  for (int j = pl.j0; j < pl.j1; ++j) face_cell<false>(c, j, jp, n, s);
  pl.cnt = n;
  if (tid == 0) *sh_flag = 0;
  sh_j[tid] = (pl.j0 < pl.j1) ? pl.jp_start : -1;
  __syncthreads();
  if (pl.j0 < pl.j1 && tid + 1 < nt && sh_j[tid + 1] >= 0 && sh_j[tid + 1] != jp) *sh_flag = 1;
  __syncthreads();
  pl.sequential = *sh_flag;
  __syncthreads();
  return pl;
}

__device__ FaceCtx noalloc_ctx(const NoallocScratch *S, int i, const double *tiph, const double *dphi,
                               int *err) {
  FaceCtx c;
  c.tin = tiph + S->off[i];
  c.din = dphi + S->off[i];
  c.tout = tiph + S->off[i + 1];
  c.dout = dphi + S->off[i + 1];
  c.Nin = S->np[i];
  c.Nout = S->np[i + 1];
  c.fL = c.fR = nullptr;
  c.fdphi = c.fcm = nullptr;
  c.runs = c.sruns = c.fstart = nullptr;
  c.cap = c.rcap = 0;
  c.err = err;
  c.offL = c.offR = 0;
  return c;
}

__global__ void __launch_bounds__(BLK) k_noalloc_count(NoallocScratch *S, const double *tiph,
                                                       const double *dphi) {
  __shared__ int sh_i[BLK];
  __shared__ int sh_j[BLK];
  __shared__ double sh_v[BLK];
  __shared__ int sh_flag;
  const int i = blockIdx.x;
  FaceCtx c = noalloc_ctx(S, i, tiph, dphi, &S->err);
  PairPlan pl = noalloc_plan(c, sh_i, sh_j, sh_v, &sh_flag);
  if (!pl.sequential) {
    int tot;
    block_excl_scan<int>(pl.cnt, sh_i, tot);
    if (threadIdx.x == 0) S->cnt[i] = tot;
  } else if (threadIdx.x == 0) {
    int jp = pl.jpmin, n = 0, s = 0;
    for (int j = 0; j < c.Nin; ++j) face_cell<false>(c, j, jp, n, s);
    S->cnt[i] = n;
  }
}

__global__ void k_noalloc_offsets(NoallocScratch *S, int NR, int cap, int *nri) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int o = 0;
  for (int i = 0; i < NR - 1; ++i) {
    S->base[i] = o;
    nri[i] = o;
    o += S->cnt[i];
  }
  S->base[NR - 1] = o;
  nri[NR - 1] = o;
  S->total = o;
  S->fill_ok = o <= cap ? 1 : 0;
  if (o > cap) S->err |= DGPU_EF_FACE_OVERFLOW;
}

// One inner cell of build_jloop writing the reference's face records
// (addFace, face_create_destroy.c:11-20) straight into the caller's arrays.
struct NoallocOut {
  int *L, *R;
  double *dphi, *dA, *cm;
  int offL, offR;
  int limit;                   // faces this pair may write (its count)
  double r, dperp;
  int *err;
};

__device__ void noalloc_cell(const FaceCtx &c, const NoallocOut &o, int j, int &jp, int &n) {
  int jm = j - 1;
  if (jm < 0) jm = c.Nin - 1;
  auto emit = [&](double dphi, double tp) {
    if (n >= 0 && n < o.limit) {
      o.L[n] = o.offL + j;
      o.R[n] = o.offR + jp;
      o.dphi[n] = dphi;
      o.dA[n] = o.r * dphi * o.dperp;
      o.cm[n] = tp - .5 * dphi;
    } else {
      set_err(o.err, DGPU_EF_FACE_OVERFLOW);
    }
    ++n;
  };
  double dp = c.tout[jp] - c.tin[jm];
  dp = wrap_pos(dp, c.err);
  if (c.din[j] < dp) {
    emit(c.din[j], c.tin[j]);
    return;
  }
  emit(dp, c.tout[jp]);
  ++jp;
  if (jp == c.Nout) jp = 0;
  dp = c.tin[j] - c.tout[jp];
  dp = wrap_pm(dp, c.err);
  int guard = 0;
  while (dp > 0.0) {
    emit(c.dout[jp], c.tout[jp]);
    ++jp;
    if (jp == c.Nout) jp = 0;
    dp = c.tin[j] - c.tout[jp];
    dp = wrap_pm(dp, c.err);
    if (++guard > c.Nout + 2) {
      set_err(c.err, DGPU_EF_FACE_OVERFLOW);
      break;
    }
  }
  dp = c.dout[jp] + dp;
  emit(dp, c.tin[j]);
}

__global__ void __launch_bounds__(BLK) k_noalloc_fill(NoallocScratch *S, const double *tiph, const double *dphi,
                                                      int *L, int *R, double *fdphi, double *fdA,
                                                      double *fcm) {
  __shared__ int sh_i[BLK];
  __shared__ int sh_j[BLK];
  __shared__ double sh_v[BLK];
  __shared__ int sh_flag;
  // fill_ok, base, cnt and total were written by the earlier kernels and are
  // only read here, so these early exits are uniform across the block
  if (!S->fill_ok) return;
  const int i = blockIdx.x;
  const int b = S->base[i];
  if (b < 0 || S->cnt[i] < 0 || b + S->cnt[i] > S->total) return;
  FaceCtx c = noalloc_ctx(S, i, tiph, dphi, &S->err);
  PairPlan pl = noalloc_plan(c, sh_i, sh_j, sh_v, &sh_flag);
  NoallocOut o;
  o.L = L + b;
  o.R = R + b;
  o.dphi = fdphi + b;
  o.dA = fdA + b;
  o.cm = fcm + b;
  o.offL = S->off[i];
  o.offR = S->off[i + 1];
  o.limit = S->cnt[i];
  o.r = S->rface[i + 1];
  o.dperp = S->dperp;
  o.err = &S->err;
  if (!pl.sequential) {
    int tot;
    int fo = block_excl_scan<int>(pl.cnt, sh_i, tot);
    if (tot != S->cnt[i]) {
      if (threadIdx.x == 0) set_err(&S->err, DGPU_EF_FACE_OVERFLOW);
      return;
    }
    int jp = pl.jp_start, n = fo;
    for (int j = pl.j0; j < pl.j1; ++j) noalloc_cell(c, o, j, jp, n);
  } else if (threadIdx.x == 0) {
    int jp = pl.jpmin, n = 0;
    for (int j = 0; j < c.Nin; ++j) noalloc_cell(c, o, j, jp, n);
  }
}

}  // namespace

// The device address of the scratch array is looked up on every call, in the
// calling thread's current context, so it stays valid after a device reset or
// from another context on the same device.  Every pointer argument must be
// memory of that current device.

extern "C" __attribute__((visibility("default"))) int dgpu_face_list_noalloc(const dgpu_sim *sim, const double *tiph, const double *dphi, int cap,
                                      int *nri, int *L, int *R, double *fdphi, double *fdA, double *fcm,
                                      int *nf, void *stream) {
  int dev = -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (!sim || !tiph || !dphi || !nri || !L || !R || !fdphi || !fdA || !fcm || !nf || cap < 0)
    return DGPU_ERR_ARG;
  const int NR = sim->NR;
  if (NR > NOALLOC_MAXA || NR < 3) return DGPU_ERR_ARG;  // more annuli than the static scratch holds
  if (sim->NumZ != 1) return DGPU_ERR_UNSUPPORTED;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return DGPU_ERR_CUDA;
  void *sp = nullptr;
  if (cudaGetSymbolAddress(&sp, g_noalloc_scratch) != cudaSuccess || !sp) return DGPU_ERR_CUDA;
  NoallocScratch *S = (NoallocScratch *)sp;
  const double dperp = dsim_zface(sim, 0) - dsim_zface(sim, -1);
  if (cudaMemcpyAsync(S->np, sim->N_p, sizeof(int) * (size_t)NR, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(S->rface, sim->r_faces, sizeof(double) * (size_t)(NR + 1), cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyAsync(&S->dperp, &dperp, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return DGPU_ERR_CUDA;
  k_noalloc_setup<<<1, 1, 0, st>>>(S, NR);
  k_noalloc_count<<<NR - 1, BLK, 0, st>>>(S, tiph, dphi);
  k_noalloc_offsets<<<1, 1, 0, st>>>(S, NR, cap, nri);
  k_noalloc_fill<<<NR - 1, BLK, 0, st>>>(S, tiph, dphi, L, R, fdphi, fdA, fcm);
  if (cudaGetLastError() != cudaSuccess) return DGPU_ERR_CUDA;
  int res[2] = {0, 0};
  if (cudaMemcpyAsync(&res[0], &S->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&res[1], &S->total, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return DGPU_ERR_CUDA;
  *nf = res[1];
  if (res[0] & DGPU_EF_FACE_OVERFLOW) return res[1] > cap ? DGPU_ERR_ARG : DGPU_ERR_FACE_OVERFLOW;
  if (res[0]) return DGPU_ERR_NUMERIC;
  return DGPU_OK;
}
