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
