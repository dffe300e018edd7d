// Face-split schedule of the explicit RK stage (an alternative to
// k_stage_tile, picked per level by the autotuner in cosa_gpu.cu).
//
//   k_halo<true>     BC + cut halos (as for the tile kernel)
//   k_prim           primitive copy of the stage state (visc.cuh)
//   k_faces<P>       one thread per face of all three families of every
//                    block: MUSCL + limiter + Roe flux from the primitive
//                    copy (stencil reads hit L1/L2), face flux to HBM
//   k_cells<P,RMS>   one thread per cell: flux balance in the reference's
//                    order, [viscous balance, HB source], [lambda/deltat],
//                    norms, multigrid forcing, the update
//
// The face and cell arithmetic is the tile kernel's (same device functions,
// same order), so both schedules give the same bits.  The split schedule
// moves 3 x 5 face fluxes per cell through HBM (240 B/cell written and read
// back) but has no shared-memory ring, no barriers and far fewer registers
// per thread, so many more warps hide the FP64 latency chains.
#pragma once
#include "fused.cuh"
#include "visc.cuh"

// MUSCL + limiter + Roe flux of face f along a line of 4 cells w[0..3] =
// cells f-2..f+1 (the tile kernel's `face`)
template <bool MIXED>
__device__ __forceinline__ void split_face(const PhysPar &ph, bool first_order, const double w[4][5], int f, int mx,
                                           bool slo, bool shi, const double *met, double *F) {
  double qr[5], ql[5];
  const bool ovr_lo = (f == 1 && slo), ovr_hi = (f == mx && shi);
  const bool d_lo = (f - 1 == 1 && slo) || (f - 1 == mx && shi);
  const bool d_mid = (f == 1 && slo) || (f == mx && shi);
  const bool d_hi = (f + 1 == 1 && slo) || (f + 1 == mx && shi);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    const double a0 = w[0][m], a1 = w[1][m], a2 = w[2][m], a3 = w[3][m];
    if (first_order) {
      qr[m] = a2; ql[m] = a1;
    } else {
      double dlo = a1 - a0, dmid = a2 - a1, dhi = a3 - a2;
      if (d_lo) dlo = (a1 - a0) * 2;
      if (d_mid) dmid = (a2 - a1) * 2;
      if (d_hi) dhi = (a3 - a2) * 2;
      if (MIXED) {
        float dp, dm;
        limit_face_fast(ph.ilimf, (float)ph.epslimf, (float)ph.rkap, (float)dlo, (float)dmid, (float)dhi, dp, dm);
        qr[m] = a2 + (double)dp; ql[m] = a1 + (double)dm;
      } else {
        double dp, dm;
        limit_face_nr(ph.ilimf, ph.epslimf, ph.rkap, dlo, dmid, dhi, dp, dm);
        qr[m] = a2 + dp; ql[m] = a1 + dm;
      }
    }
    if (ovr_lo) { qr[m] = a1; ql[m] = a1; }
    if (ovr_hi) { qr[m] = a2; ql[m] = a2; }
  }
  if (MIXED) roe_flux_mixed(ph, met[0], met[1], met[2], met[3], qr, ql, F);
  else roe_flux_euler(ph, met[0], met[1], met[2], met[3], qr, ql, F);
}

// grid (x, 3 families, blocks from blk0): the three families of a block run
// one after the other, so the block's state stays in L2 across them; face
// flux of family d into cf + (d-1)*n0*5*S (F0 layout per family)
template <bool MIXED>
__global__ void __launch_bounds__(128, 5) k_faces(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                                               const double *__restrict__ qp, const double *__restrict__ si,
                                               const double *__restrict__ sj, const double *__restrict__ sk,
                                               const uint8_t *__restrict__ strong, const StrongMap *__restrict__ smap,
                                               int first_order, int64_t n0, double *__restrict__ cf, int blk0) {
  const DevBlock b = blocks[blk0 + blockIdx.z];
  const int d = blockIdx.y + 1;
  const cosa_params &P = *Pp;
  const PhysPar ph = make_phys(P);
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const unsigned ni = d == 1 ? b.im : b.im - 1, nj = d == 2 ? b.jm : b.jm - 1, nk = d == 3 ? b.km : b.km - 1;
  const unsigned total = ni * nj * nk * S;  // < 2^31 per block and family (checked on the host)
  const double *s = d == 1 ? si : (d == 2 ? sj : sk);
  double *F0 = cf + (int64_t)(d - 1) * n0 * 5 * S;
  const StrongMap sm = smap[blk0 + blockIdx.z];
  const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  const int64_t step = d == 1 ? 1 : (d == 2 ? (int64_t)b.I3 : (int64_t)b.I3 * b.J3);
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    // 32-bit decomposition (64-bit division costs several times more instructions)
    unsigned r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk), nh = n * P.hbmove;
    const int f = d == 1 ? i : (d == 2 ? j : k);
    const int t2 = d == 1 ? j : i, t3 = d == 3 ? j : k;
    const bool slo = (f <= 2) && strong_at(strong, sm, d - 1, 0, t2, t3);
    const bool shi = (f >= mx - 1) && strong_at(strong, sm, d - 1, 1, t2, t3);
    const double *base = qp + p3_var(b, 5, S, 1, n) + p3_cell(b, i, j, k) - 2 * step;
    double w[4][5];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int m = 0; m < 5; ++m) w[p][m] = __ldg(base + p * step + m * b.P3);
    const int64_t e = p2_idx(b, S2, 1, i, j, k, nh);
    const double2 a = __ldg(reinterpret_cast<const double2 *>(s + e));
    const double2 c = __ldg(reinterpret_cast<const double2 *>(s + e + 2));
    const double met[4] = {a.x, a.y, c.x, c.y};
    double F[5];
    split_face<MIXED>(ph, first_order != 0, w, f, mx, slo, shi, met, F);
#pragma unroll
    for (int m = 0; m < 5; ++m) F0[f0_idx(b, 5, S, i, j, k, m + 1, n)] = F[m];
  }
}

// grid (x, nblocks): local time step of the stage-1 pass (lambdab + bdeltat,
// src/cosa.f90:1293-1323, 4860-4870) from the primitive copy
__global__ void k_dt_euler(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                           const double *__restrict__ qp, const double *__restrict__ si,
                           const double *__restrict__ sj, const double *__restrict__ sk, double *__restrict__ dtv,
                           double *bx, double *by, double *bz) {
  const DevBlock b = blocks[blockIdx.y];
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t rr = t;
    const int i = (int)(rr % ni) + 1; rr /= ni;
    const int j = (int)(rr % nj) + 1; rr /= nj;
    const int k = (int)(rr % nk) + 1;
    const int n = (int)(rr / nk), nh = n * P.hbmove;
    const int64_t cell = p3_cell(b, i, j, k), o1 = p1_idx(b, S, i, j, k, n);
    double qc[5], sim[4], sip[4], sjm[4], sjp[4], skm[4], skp[4];
#pragma unroll
    for (int m = 0; m < 5; ++m) qc[m] = qp[p3_var(b, 5, S, m + 1, n) + cell];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      sim[m] = si[p2_idx(b, S2, m + 1, i, j, k, nh)]; sip[m] = si[p2_idx(b, S2, m + 1, i + 1, j, k, nh)];
      sjm[m] = sj[p2_idx(b, S2, m + 1, i, j, k, nh)]; sjp[m] = sj[p2_idx(b, S2, m + 1, i, j + 1, k, nh)];
      skm[m] = sk[p2_idx(b, S2, m + 1, i, j, k, nh)]; skp[m] = sk[p2_idx(b, S2, m + 1, i, j, k + 1, nh)];
    }
    double li, lj, lk;
    eig_eul(P.gamma, qc, sim, sip, sjm, sjp, skm, skp, li, lj, lk);
    const double dt = P.cfl / (li + lj + lk);
    dtv[o1] = dt;
    if (bx) {
      double ba, bb_, bc;
      irs_beta(P.irsop, P.rat, P.psirs, li, lj, lk, ba, bb_, bc);
      bx[o1] = ba; by[o1] = bb_; bz[o1] = bc;
    }
  }
}

// grid (x, blocks from blk0): flux balance, norms, forcing and update of
// every interior cell (the tile kernel's epilogue; the time step is already
// in dtvol); per-CTA norm partials at part[(block * gridDim.x + blockIdx.x) * 8 + m]
template <bool RMS>
__global__ void __launch_bounds__(256, 2) k_cells(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                                               StageArgs A, const double *__restrict__ qp,
                                               const double *__restrict__ cf, int64_t n0, int blk0) {
  __shared__ double red[8][8];
  const DevBlock b = blocks[blk0 + blockIdx.y];
  const cosa_params &P = *Pp;
  const int npde = 5, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  const double *__restrict__ Fi = cf;
  const double *__restrict__ Fj = cf + n0 * 5 * S;
  const double *__restrict__ Fk = cf + 2 * n0 * 5 * S;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t rr = t;
    const int i = (int)(rr % ni) + 1; rr /= ni;
    const int j = (int)(rr % nj) + 1; rr /= nj;
    const int k = (int)(rr % nk) + 1;
    const int n = (int)(rr / nk);
    const int64_t cell = p3_cell(b, i, j, k);
    const int64_t o1 = p1_idx(b, S, i, j, k, n);
    const double dt = A.dtvol[o1];
    const double *qo = A.qold + p3_var(b, npde, S, 1, n);
    double *qw = A.qout + p3_var(b, npde, S, 1, n);
    // all loads first: the stores below may alias nothing read here, but the
    // compiler cannot know that
    double fl[5][6], q0s[5];
    const int64_t fbase = f0_idx(b, 5, S, i, j, k, 1, n), fv = (int64_t)b.im * b.jm * b.km;
    const int64_t sj_ = b.im, sk_ = (int64_t)b.im * b.jm;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const int64_t o = fbase + m * fv;
      fl[m][0] = __ldg(Fi + o + 1); fl[m][1] = __ldg(Fi + o);
      fl[m][2] = __ldg(Fj + o + sj_); fl[m][3] = __ldg(Fj + o);
      fl[m][4] = __ldg(Fk + o + sk_); fl[m][5] = __ldg(Fk + o);
      if (A.update) q0s[m] = qo[m * b.P3 + cell];
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      // bresid order: i, then j, then k (src/cosa.f90:1800-1876)
      double r = fl[m][0] - fl[m][1];
      r = r + fl[m][2] - fl[m][3];
      r = r + fl[m][4] - fl[m][5];
      if (A.vres) r = r + A.vres[p3_var(b, npde, S, m + 1, n) + cell];
      if (A.vol) {
        // src_bhb (src/src.f90:556-613)
        const double ov = P.omega * A.vol[p1_idx(b, 1, i, j, k, 0)];
        double qhb = 0.0;
        for (int nj2 = 0; nj2 < S; ++nj2)
          qhb = qhb + ov * P.dhb[n * S + nj2] * A.qin[p3_var(b, npde, S, m + 1, nj2) + cell];
        r = r + qhb;
      }
      if (RMS) acc[m] += r * r;
      if (A.rhs_mode) {
        double *rh = A.rhs + p3_var(b, npde, S, m + 1, n) + cell;
        if (A.rhs_mode == 2) {
          const double rn = *rh + r;
          *rh = rn;
          r = r - rn;
        } else {
          r = r - *rh;
        }
      }
      if (A.res_out) A.res_out[p3_var(b, npde, S, m + 1, n) + cell] = r;
      if (A.update) {
        const double q0 = q0s[m];
        if (A.qold_copy) A.qold_copy[p3_var(b, npde, S, m + 1, n) + cell] = q0;
        qw[m * b.P3 + cell] = q0 - A.ar * r * dt;
      }
    }
  }
  if (RMS) {
    // deterministic per-CTA sums: warp shuffle, then fixed-order warp sums
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double x = acc[m];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) == 0) red[m][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
      double x = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[threadIdx.x][w];
      A.part[((int64_t)(blk0 + blockIdx.y) * gridDim.x + blockIdx.x) * 8 + threadIdx.x] = x;
    }
  }
}
