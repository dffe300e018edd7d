// Time-accurate runs: dual time stepping (dualt) and the explicit RK
// integration rkuns (rgkuns), one snapshot (S = 1).
//
//   k_src_uns          src_uns_b (src/src.f90:406-451): the BDF term of the
//                      pseudo-time residual, res += 3/2 q V / dt (q V / dt
//                      on a first-order first step, bdf1)
//   k_rhs_uns          rhs_uns_b (src/src.f90:480-527): rhs = (2 q^n -
//                      q^(n-1) / 2) V / dt (q^n V / dt with bdf1)
//   k_rms_dualimp      resg_brms with rkimp, no IRS, one level
//                      (src/cosa.f90:4533-4549): (fact q V / dt + res - rhs)^2
//   k_update_dual      update_b with rkimp (src/update.f90:650-738), the
//                      physical-time term implicit, variables 1..5
//   k_update_kom_dual  its k-omega part
//   k_deltat_urk       bdeltat_urk (src/cosa.f90:2550-2572): dtvol = dt / V
#pragma once
#include "kom.cuh"

__device__ __forceinline__ double bdf_fact(const cosa_params &P) { return P.bdf1 ? 1.0 : 1.5; }

template <class BS>
__global__ void k_src_uns(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                          const double *__restrict__ vol, double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 1;
  KOM_CELL_LOOP
    (void)n;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    for (int m = 1; m <= npde; ++m) {
      const int64_t o = p3_var(b, npde, 1, m, 0) + c;
      if (P.bdf1) res[o] = res[o] + q[o] * v / P.dt;
      else res[o] = res[o] + 3 * q[o] * v / 2 / P.dt;
    }
  }
}

template <class BS>
__global__ void k_rhs_uns(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ rhs,
                          const double *__restrict__ q1, const double *__restrict__ q2,
                          const double *__restrict__ vol) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 1;
  KOM_CELL_LOOP
    (void)n;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    for (int m = 1; m <= npde; ++m) {
      const int64_t o = p3_var(b, npde, 1, m, 0) + c;
      if (P.bdf1) rhs[o] = q1[o] * v / P.dt;
      else rhs[o] = (2 * q1[o] - q2[o] / 2) * v / P.dt;
    }
  }
}

// per-CTA partial sums (8 doubles per CTA) of (fact q V / dt + res - rhs)^2
__global__ void k_rms_dualimp(DevBlock b, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                              const double *__restrict__ rhs, const double *__restrict__ q,
                              const double *__restrict__ vol, double *__restrict__ part) {
  const cosa_params &P = *Pp;
  const int npde = P.npde;
  const double fact = bdf_fact(P);
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1;
    const int k = (int)(r / nj) + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    for (int m = 0; m < npde; ++m) {
      const int64_t o = p3_var(b, npde, 1, m + 1, 0) + c;
      const double tt = fact * q[o] * v / P.dt + res[o] - rhs[o];
      acc[m] += tt * tt;
    }
  }
  __shared__ double red[7][32];
  for (int m = 0; m < npde; ++m) {
    double x = acc[m];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[m][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    for (int m = 0; m < npde; ++m) {
      double x = threadIdx.x < nw ? red[m][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) part[(int64_t)blockIdx.x * 8 + m] = x;
    }
  }
}

// qin: the stage state (src_in_res: the state src_uns saw, whose term the
// smoothed residual holds); qout may be qin (each thread reads its cell's
// values before writing them)
template <class BS>
__global__ void k_update_dual(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                              const double *__restrict__ qold, const double *qin, double *qout,
                              double *__restrict__ qcopy, const double *__restrict__ dtv,
                              const double *__restrict__ vol, double ar, int src_in_res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 1;
  const double fact = bdf_fact(P);
  KOM_CELL_LOOP
    (void)n;
    const int64_t c = p3_cell(b, i, j, k);
    const double dt = dtv[p1_idx(b, 1, i, j, k, 0)], v = vol[p1_idx(b, 1, i, j, k, 0)];
    const double den = 1 + fact * ar * dt * v / P.dt;
    for (int m = 1; m <= 5; ++m) {
      const int64_t o = p3_var(b, npde, 1, m, 0) + c;
      const double q0 = qold[o];
      if (qcopy) qcopy[o] = q0;
      if (src_in_res) qout[o] = (q0 - ar * dt * (-fact * v / P.dt * qin[o] + res[o])) / den;
      else qout[o] = (q0 - ar * res[o] * dt) / den;
    }
  }
}

// k-omega part (rho omega, then rho k), in place on q before k_update_dual
template <class BS>
__global__ void k_update_kom_dual(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                                  double *__restrict__ q, const double *__restrict__ qold,
                                  const double *__restrict__ vol, const double *__restrict__ dtt,
                                  const double *__restrict__ delpls, const double *__restrict__ prd, double ar,
                                  const double *__restrict__ ttrm, int src_in_res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 1;
  const double fact = bdf_fact(P);
  KOM_CELL_LOOP
    const double gav = ttrm ? ttrm[ttrm_idx(b, 1, i, j, k, 2, 0)] : P.gkw;
    const double bav = ttrm ? ttrm[ttrm_idx(b, 1, i, j, k, 3, 0)] : P.bkw;
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, 1, i, j, k, n);
    const int64_t i1 = p3_var(b, npde, 1, 1, 0) + c, i6 = p3_var(b, npde, 1, 6, 0) + c, i7 = p3_var(b, npde, 1, 7, 0) + c;
    const double rho = q[i1], ome = q[i7] / q[i1];
    const double dt = dtt[p1_idx(b, 1, i, j, k, 0)];
    const double dtau = dt * vol[p1_idx(b, 1, i, j, k, 0)];
    const double dp = delpls[o];
    double rhomega;
    if (src_in_res)
      rhomega = (qold[i7] + ar * fact * dtau / P.dt * q[i7] - ar * res[i7] * dt + ar * dtau * q[i7] * (gav * dp + 2 * bav * ome)) /
                (1 + ar * dtau * (gav * dp + 2 * bav * ome) + ar * fact * dtau / P.dt);
    else
      rhomega = (qold[i7] - ar * res[i7] * dt + ar * dtau * q[i7] * (gav * dp + 2 * bav * ome)) /
                (1 + ar * dtau * (gav * dp + 2 * bav * ome) + fact * ar * dtau / P.dt);
    const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
    if (rhomega < rhomegamin) rhomega = rhomegamin;
    q[i7] = rhomega;
    const double drhomega = rhomega - rho * ome;
    if (src_in_res)
      q[i6] = (qold[i6] + ar * fact * dtau / P.dt * q[i6] - ar * res[i6] * dt +
               ar * dtau * q[i6] * (dp + P.bstrkw * ome - P.bstrkw * drhomega / rho)) /
              (1 + ar * dtau * (dp + P.bstrkw * ome) + ar * fact * dtau / P.dt);
    else
      q[i6] = (qold[i6] - ar * res[i6] * dt + ar * dtau * q[i6] * (dp + P.bstrkw * ome - P.bstrkw * drhomega / rho)) /
              (1 + ar * dtau * (dp + P.bstrkw * ome) + ar * fact * dtau / P.dt);
  }
}

template <class BS>
__global__ void k_deltat_urk(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ vol,
                             double *__restrict__ dtv) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int S = 1;
  KOM_CELL_LOOP
    (void)n;
    dtv[p1_idx(b, 1, i, j, k, 0)] = P.dt / vol[p1_idx(b, 1, i, j, k, 0)];
  }
}

// ---- k-omega harmonic balance ---------------------------------------------------------
// update_bhb's k-omega part with rkimp (src/update.f90:1427-1560 without IRS
// on one level, 1633-1768 with IRS or multigrid; src_in_res for the latter):
// per cell the S snapshots of rho omega, then of rho k, through (I (1 + ar
// dtau a_n) + ar omega dtau D) x = rhs, rho omega floored by gav cmu rho
// sqrt(prd); the k equation takes omega before the update and the change of
// rho omega.  In place on q, before k_update_bhb (variables 1..5).
template <class BS>
__global__ void k_update_bhb_kom(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                                 double *__restrict__ q, const double *__restrict__ qold,
                                 const double *__restrict__ vol, const double *__restrict__ dtt,
                                 const double *__restrict__ delpls, const double *__restrict__ prd, double ar,
                                 const double *__restrict__ ttrm, int src_in_res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni_ = b.im - 1, nj_ = b.jm - 1, nk_ = b.km - 1;
  const int64_t ncell = (int64_t)ni_ * nj_ * nk_;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni_) + 1; r /= ni_;
    const int j = (int)(r % nj_) + 1;
    const int k = (int)(r / nj_) + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    auto Q = [&](int m, int n) -> double & { return q[p3_var(b, npde, S, m, n) + c]; };
    auto hbsrc = [&](int m, int n) {
      double qhb = 0.0;
      for (int nj = 0; nj < S; ++nj) qhb = qhb + P.omega * v * P.dhb[n * S + nj] * Q(m, nj);
      return qhb;
    };
    double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP], w7[COSA_MAX_SNAP], xk[COSA_MAX_SNAP];
    double sk[COSA_MAX_SNAP], dw[COSA_MAX_SNAP];
    for (int n = 0; n < S; ++n) {
      const int64_t o = p3s_idx(b, S, i, j, k, n);
      const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
      const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
      const double ome = Q(7, n) / Q(1, n);
      const double dt = dtt[p1_idx(b, S, i, j, k, n)], dtau = dt * v, dps = delpls[o];
      const int64_t i7 = p3_var(b, npde, S, 7, n) + c;
      if (src_in_res)
        x[n] = qold[i7] + ar * dt * (hbsrc(7, n) - res[i7]) + ar * dtau * Q(7, n) * (gav * dps + 2 * bav * ome);
      else
        x[n] = qold[i7] - ar * res[i7] * dt + ar * dtau * Q(7, n) * (gav * dps + 2 * bav * ome);
      w7[n] = Q(7, n);
      sk[n] = src_in_res ? hbsrc(6, n) : 0.0;
      for (int m = 0; m < S; ++m)
        a[n + S * m] = (n == m ? 1.0 : 0.0) * (1 + ar * dtau * (gav * dps + 2 * bav * ome)) +
                       ar * P.omega * dtau * P.dhb[n * S + m];
    }
    hb_lu_solve(S, a, x, 1);
    for (int n = 0; n < S; ++n) {
      const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
      const double rhomegamin = gav * P.cmu * Q(1, n) * sqrt(prd[p3s_idx(b, S, i, j, k, n)]);
      if (x[n] < rhomegamin) x[n] = rhomegamin;
      dw[n] = x[n] - w7[n];
    }
    for (int n = 0; n < S; ++n) {
      const int64_t o = p3s_idx(b, S, i, j, k, n);
      const double rho = Q(1, n), ome = w7[n] / Q(1, n);
      const double dt = dtt[p1_idx(b, S, i, j, k, n)], dtau = dt * v, dps = delpls[o];
      const int64_t i6 = p3_var(b, npde, S, 6, n) + c;
      if (src_in_res)
        xk[n] = qold[i6] + ar * dt * (sk[n] - res[i6]) + ar * dtau * Q(6, n) * (dps + P.bstrkw * ome - P.bstrkw * dw[n] / rho);
      else
        xk[n] = qold[i6] - ar * res[i6] * dt + ar * dtau * Q(6, n) * (dps + P.bstrkw * ome - P.bstrkw * dw[n] / rho);
      for (int m = 0; m < S; ++m)
        a[n + S * m] = (n == m ? 1.0 : 0.0) * (1 + ar * dtau * (dps + P.bstrkw * ome)) +
                       ar * P.omega * dtau * P.dhb[n * S + m];
    }
    hb_lu_solve(S, a, xk, 1);
    for (int n = 0; n < S; ++n) {
      Q(7, n) = x[n];
      Q(6, n) = xk[n];
    }
  }
}

// lim_res_ome_bhb (src/update.f90:2836-2999), without low-speed
// preconditioning: explicit per snapshot; with rkimp through the
// snapshot-coupled system (I (1 + dtau a_n) + omega dtau D)
template <class BS>
__global__ void k_lim_res_ome_bhb(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ res,
                                  const double *__restrict__ q, const double *__restrict__ qold,
                                  const double *__restrict__ vol, const double *__restrict__ dtt,
                                  const double *__restrict__ delpls, const double *__restrict__ prd,
                                  const double *__restrict__ ttrm) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni_ = b.im - 1, nj_ = b.jm - 1, nk_ = b.km - 1;
  const int64_t ncell = (int64_t)ni_ * nj_ * nk_;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni_) + 1; r /= ni_;
    const int j = (int)(r % nj_) + 1;
    const int k = (int)(r / nj_) + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    if (!P.rkimp) {
      for (int n = 0; n < S; ++n) {
        const int64_t o = p3s_idx(b, S, i, j, k, n), i1 = p3_var(b, npde, S, 1, n) + c, i7 = p3_var(b, npde, S, 7, n) + c;
        const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
        const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
        const double rho = q[i1], ome = q[i7] / q[i1];
        const double dt = dtt[p1_idx(b, S, i, j, k, n)], dtau = dt * v;
        const double den = 1 + dtau * (gav * delpls[o] + 2 * bav * ome);
        const double rhomega = qold[i7] - res[i7] * dt / den;
        const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
        res[i7] = res[i7] - den * fmax(0.0, (rhomegamin - rhomega) / dt);
      }
      continue;
    }
    double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP];
    for (int n = 0; n < S; ++n) {
      const int64_t o = p3s_idx(b, S, i, j, k, n), i1 = p3_var(b, npde, S, 1, n) + c, i7 = p3_var(b, npde, S, 7, n) + c;
      const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
      const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
      const double ome = q[i7] / q[i1];
      const double dt = dtt[p1_idx(b, S, i, j, k, n)], dtau = dt * v, dps = delpls[o];
      for (int m = 0; m < S; ++m)
        a[n + S * m] = (n == m ? 1.0 : 0.0) * (1 + dtau * (gav * dps + 2 * bav * ome)) + P.omega * dtau * P.dhb[n * S + m];
      x[n] = res[i7] * dt;
    }
    hb_lu_solve(S, a, x, 1);
    for (int n = 0; n < S; ++n) {
      const int64_t o = p3s_idx(b, S, i, j, k, n), i7 = p3_var(b, npde, S, 7, n) + c;
      const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
      const double rhomegamin = gav * P.cmu * q[p3_var(b, npde, S, 1, n) + c] * sqrt(prd[o]);
      const double rhomeganew = qold[i7] - x[n];
      res[i7] = res[i7] - fmax(0.0, (rhomegamin - rhomeganew)) / dtt[p1_idx(b, S, i, j, k, n)];
    }
  }
}
