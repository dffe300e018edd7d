// Face-split schedule of the explicit RK stage (an alternative to
// k_stage_tile, picked per level by the autotuner in cosa_gpu.cu).
//
//   k_halo<true>        BC + cut halos (as for the tile kernel)
//   [k_prim]            primitive copy of the stage state, viscous flows
//                       only (their face stencils read it too)
//   k_faces_line<P>     MUSCL + limiter + Roe flux of every face of the three
//                       families, threads marching along face lines
//                       (faces.cuh), face fluxes to HBM
//   [k_dt_euler]        local time step at stage 1
//   k_cells<RMS>        one thread per cell: flux balance in the reference's
//                       order, [viscous balance, HB source], norms, multigrid
//                       forcing, the update
//
// The face and cell arithmetic in FP64 is the tile kernel's (same device
// functions, same order), so both schedules give the same bits.  The split
// schedule moves 3 x 5 face fluxes per cell through HBM (120 B/cell written
// and read back) but has no shared-memory ring and no barriers.
#pragma once
#include "fused.cuh"
#include "visc.cuh"

// grid (x, nblocks): local time step of the stage-1 pass (lambdab + bdeltat,
// src/cosa.f90:1293-1323, 4860-4870) from the primitive copy, or (CONV) from
// the stage input's conservative interior cells converted on load
// cell grid velocities of a moving grid (the reference's xdot, ydot, zdot after
// vert2cell_g: node-array layout, one set per snapshot); null on fixed grids
struct CellVel {
  const double *c[3];
};

template <bool CONV>
__global__ void k_dt_euler(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                           const double *__restrict__ qp, const double *__restrict__ si,
                           const double *__restrict__ sj, const double *__restrict__ sk, double *__restrict__ dtv,
                           double *bx, double *by, double *bz, CellVel cv = CellVel{{nullptr, nullptr, nullptr}}) {
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
    if (CONV) c2p5_nr(P.gamma, qc);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      sim[m] = si[p2_idx(b, S2, m + 1, i, j, k, nh)]; sip[m] = si[p2_idx(b, S2, m + 1, i + 1, j, k, nh)];
      sjm[m] = sj[p2_idx(b, S2, m + 1, i, j, k, nh)]; sjp[m] = sj[p2_idx(b, S2, m + 1, i, j + 1, k, nh)];
      skm[m] = sk[p2_idx(b, S2, m + 1, i, j, k, nh)]; skp[m] = sk[p2_idx(b, S2, m + 1, i, j, k + 1, nh)];
    }
    double li, lj, lk, gv[3];
    if (cv.c[0]) {
      const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
      const int64_t g = b.op2 * S2 + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k);
      gv[0] = cv.c[0][g]; gv[1] = cv.c[1][g]; gv[2] = cv.c[2][g];
    }
    eig_eul(P.gamma, qc, sim, sip, sjm, sjp, skm, skp, li, lj, lk, cv.c[0] ? gv : nullptr);
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
#ifndef COSA_CELLS_MINB
#define COSA_CELLS_MINB 2  // resident CTAs per SM k_cells is compiled for
#endif
__global__ void __launch_bounds__(256, COSA_CELLS_MINB) k_cells(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                                               StageArgs A, const double *__restrict__ cf, int64_t n0,
                                               int blk0) {
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
