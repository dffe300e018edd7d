// Per-routine kernels: one CUDA kernel per reference routine, with the
// reference's array contract (the level drivers of include/cosa_gpu.h).
// Each kernel covers one block; the host loops over the blocks of a level
// exactly like the Fortran drivers' `do iblock = 1,mynblocks`.
#pragma once
#include "physics.cuh"

// IRS coefficients beta of bdeltat (src/cosa.f90:4882-5180), inviscid lambdas
// (irsop 5/6 reduce to 2/3 when the viscous spectral radii are zero)
__device__ __forceinline__ void irs_beta(int irsop, double rat, double psirs, double lami, double lamj, double lamk,
                                         double &bx, double &by, double &bz) {
  if (irsop == 2 || irsop == 5) {
    const double zeta = 0.4;
    const double phixi = 1 + pow(lamj / lami, zeta) + pow(lamk / lami, zeta);
    const double phieta = 1 + pow(lami / lamj, zeta) + pow(lamk / lamj, zeta);
    const double phizeta = 1 + pow(lami / lamk, zeta) + pow(lamj / lamk, zeta);
    double tt;
    tt = (rat * lami * phixi / (lami + lamj + lamk)); bx = fmax(0.0, (tt * tt - 1) / 4);
    tt = (rat * lamj * phieta / (lami + lamj + lamk)); by = fmax(0.0, (tt * tt - 1) / 4);
    tt = (rat * lamk * phizeta / (lami + lamj + lamk)); bz = fmax(0.0, (tt * tt - 1) / 4);
  } else {
    const double rji = lamj / lami, rki = lamk / lami, rij = lami / lamj;
    const double rkj = lamk / lamj, rik = lami / lamk, rjk = lamj / lamk;
    double tt;
    tt = rat / (1 + psirs * (rji + rki)); bx = fmax(0.0, 0.25 * (tt * tt - 1));
    tt = rat / (1 + psirs * (rij + rkj)); by = fmax(0.0, 0.25 * (tt * tt - 1));
    tt = rat / (1 + psirs * (rik + rjk)); bz = fmax(0.0, 0.25 * (tt * tt - 1));
  }
}


// ---- cons2prim_b (src/update.f90:2112-2188) ----------------------------------------
template <class BS>
__global__ void k_cons2prim(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ q, int xtnd) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1 + 2 * xtnd, nj = b.jm - 1 + 2 * xtnd, nk = b.km - 1 + 2 * xtnd;
  const int64_t ncell = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1 - xtnd; r /= ni;
    const int j = (int)(r % nj) + 1 - xtnd; r /= nj;
    const int k = (int)(r % nk) + 1 - xtnd; r /= nk;
    const int n = (int)r;
    const int64_t c = p3_cell(b, i, j, k);
    double v[7];
    for (int m = 0; m < npde; ++m) v[m] = q[p3_var(b, npde, S, m + 1, n) + c];
    if (npde > 5) c2p7(P.gamma, v); else c2p5(P.gamma, v);
    for (int m = 0; m < npde; ++m) q[p3_var(b, npde, S, m + 1, n) + c] = v[m];
  }
}

// ---- prim2cons_b (src/update.f90:1875-2084): interior + face halos ------------------
template <class BS>
__global__ void k_prim2cons(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ q) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  // domain: i in -1..im+1, j,k in -1..jm+1/-1..km+1 restricted to the
  // interior plus the six face-halo slabs (no edges, no corners)
  const int ni = b.im + 3, nj = b.jm + 3, nk = b.km + 3;
  const int64_t ncell = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) - 1; r /= ni;
    const int j = (int)(r % nj) - 1; r /= nj;
    const int k = (int)(r % nk) - 1; r /= nk;
    const int n = (int)r;
    const int oi = (i < 1 || i > b.im - 1), oj = (j < 1 || j > b.jm - 1), ok = (k < 1 || k > b.km - 1);
    if (oi + oj + ok > 1) continue;
    const int64_t c = p3_cell(b, i, j, k);
    double v[7];
    for (int m = 0; m < npde; ++m) v[m] = q[p3_var(b, npde, S, m + 1, n) + c];
    p2c(P.gamma, v, npde);
    for (int m = 0; m < npde; ++m) q[p3_var(b, npde, S, m + 1, n) + c] = v[m];
  }
}

// ---- bprtest (src/cosa.f90:960-1120): status bits instead of stop -----------------
template <class BS>
__global__ void k_prtest(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q, int *status) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im + 3, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk * S;
  int st = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) - 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int n = (int)r;
    const int64_t c = p3_cell(b, i, j, k);
    const double rho = q[p3_var(b, npde, S, 1, n) + c], pr = q[p3_var(b, npde, S, 5, n) + c];
    if (pr <= P.qmin[4]) st |= COSA_ERR_NEG_P;
    else if (rho <= P.qmin[0]) st |= COSA_ERR_NEG_RHO;
  }
  if (st) atomicOr(status, st);
}

// ---- lambdab inviscid (src/cosa.f90:1248-1330) --------------------------------------
template <class BS>
__global__ void k_lambda(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                         const double *__restrict__ si, const double *__restrict__ sj,
                         const double *__restrict__ sk, double *__restrict__ lam, const double *__restrict__ cvx = nullptr,
                         const double *__restrict__ cvy = nullptr, const double *__restrict__ cvz = nullptr,
                         const double *__restrict__ cpg = nullptr, const double *__restrict__ cvs = nullptr,
                         int nl = 1) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int n = (int)r, nh = n * P.hbmove;
    const int64_t c = p3_cell(b, i, j, k);
    double qc[5], sim[4], sip[4], sjm[4], sjp[4], skm[4], skp[4];
    for (int m = 0; m < 5; ++m) qc[m] = q[p3_var(b, npde, S, m + 1, n) + c];
    for (int m = 0; m < 4; ++m) {
      sim[m] = si[p2_idx(b, S2, m + 1, i, j, k, nh)]; sip[m] = si[p2_idx(b, S2, m + 1, i + 1, j, k, nh)];
      sjm[m] = sj[p2_idx(b, S2, m + 1, i, j, k, nh)]; sjp[m] = sj[p2_idx(b, S2, m + 1, i, j + 1, k, nh)];
      skm[m] = sk[p2_idx(b, S2, m + 1, i, j, k, nh)]; skp[m] = sk[p2_idx(b, S2, m + 1, i, j, k + 1, nh)];
    }
    double li, lj, lk, gv[3];
    if (cvx) {
      // cell grid velocity of a moving grid (node-array layout, snapshot nh)
      const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
      const int64_t g = b.op2 * S2 + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k);
      gv[0] = cvx[g]; gv[1] = cvy[g]; gv[2] = cvz[g];
    }
    if (cpg) {
      // low-speed preconditioning: eig_eul_p with the cell's cut-offs (interior layout)
      const int64_t m = b.om1 * S + (int64_t)n * ni * nj * nk + (i - 1) + (int64_t)ni * ((j - 1) + (int64_t)nj * (k - 1));
      eig_eul_p(P.gamma, P.uprv, P.epsp[nl - 1] * P.epsp[nl - 1], fmax(cpg[m], cvs[m]), qc, sim, sip, sjm, sjp, skm,
                skp, li, lj, lk);
    } else {
      eig_eul(P.gamma, qc, sim, sip, sjm, sjp, skm, skp, li, lj, lk, cvx ? gv : nullptr);
    }
    lam[p3_var(b, npde, S, 1, n) + c] = li;
    lam[p3_var(b, npde, S, 2, n) + c] = lj;
    lam[p3_var(b, npde, S, 3, n) + c] = lk;
  }
}

// ---- bdeltat (src/cosa.f90:4733-5203): dtvol and IRS beta, inviscid ---------------
template <class BS>
__global__ void k_deltat(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ dtv,
                         const double *__restrict__ lam, double *bx, double *by, double *bz) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int n = (int)r;
    const int64_t c = p3_cell(b, i, j, k);
    const double lami = lam[p3_var(b, npde, S, 1, n) + c];
    const double lamj = lam[p3_var(b, npde, S, 2, n) + c];
    const double lamk = lam[p3_var(b, npde, S, 3, n) + c];
    const int64_t o = p1_idx(b, S, i, j, k, n);
    dtv[o] = P.cfl / (lami + lamj + lamk);
    if (bx && P.irsop >= 2 && P.irsop != 4) {
      double a, c2, d;
      irs_beta(P.irsop, P.rat, P.psirs, lami, lamj, lamk, a, c2, d);
      bx[o] = a; by[o] = c2; bz[o] = d;
    }
  }
}

// ---- muscl_b{i,j,k} (src/flux.f90:1221-1810) ---------------------------------------
// Pass 1: dq along d over the reference's range, with strong-boundary doubling.
template <class BS>
__global__ void k_muscl_dq(BS bs_, const cosa_params *__restrict__ Pp, int d, const double *__restrict__ q,
                           double *__restrict__ dq, const int *__restrict__ bct, int vs, int ve) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  int lo[3] = {1, 1, 1}, n_[3] = {b.im - 1, b.jm - 1, b.km - 1};
  lo[d - 1] = 0; n_[d - 1] = mx + 2;
  const int nv = ve - vs + 1;
  const int64_t ncell = (int64_t)n_[0] * n_[1] * n_[2] * nv * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % n_[0]) + lo[0]; r /= n_[0];
    const int j = (int)(r % n_[1]) + lo[1]; r /= n_[1];
    const int k = (int)(r % n_[2]) + lo[2]; r /= n_[2];
    const int v = (int)(r % nv) + vs; r /= nv;
    const int n = (int)r;
    const int im1 = i - (d == 1), jm1 = j - (d == 2), km1 = k - (d == 3);
    const int64_t base = p3_var(b, npde, S, v, n);
    double val = q[base + p3_cell(b, i, j, k)] - q[base + p3_cell(b, im1, jm1, km1)];
    const int e = d == 1 ? i : (d == 2 ? j : k);
    if (e == 1 || e == mx) {
      for (int ib = 0; ib < b.nbcs; ++ib) {
        const int *rw = bct + b.obct + 10 * ib;
        if (rw[1] != d || !strong_bc(rw[0])) continue;
        const int bcpt = rw[2] == 1 ? 1 : mx;
        if (e != bcpt) continue;
        const int t2 = d == 1 ? j : i, t3 = d == 3 ? j : k;
        const int s2 = d == 1 ? rw[5] : rw[3], e2 = d == 1 ? rw[6] : rw[4];
        const int s3 = d == 3 ? rw[5] : rw[7], e3 = d == 3 ? rw[6] : rw[8];
        if (t2 >= s2 && t2 <= e2 && t3 >= s3 && t3 <= e3) {
          val = (q[base + p3_cell(b, i, j, k)] - q[base + p3_cell(b, im1, jm1, km1)]) * 2;
          break;
        }
      }
    }
    dq[base + p3_cell(b, i, j, k)] = val;
  }
}

// Pass 2: limiter + construction of qp/qm on the faces, then the
// strong-boundary override (qp = qm = q(halo)).
template <class BS>
__global__ void k_muscl_face(BS bs_, const cosa_params *__restrict__ Pp, int d, int nl,
                             const double *__restrict__ q, double *__restrict__ qp, double *__restrict__ qm,
                             const double *__restrict__ dq, double *__restrict__ dqp, double *__restrict__ dqm,
                             const int *__restrict__ bct, int mixed = 0) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  int n_[3] = {b.im - 1, b.jm - 1, b.km - 1};
  n_[d - 1] = mx;
  const int64_t ncell = (int64_t)n_[0] * n_[1] * n_[2] * npde * S;
  const bool first_all = nl >= P.nl_crs;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % n_[0]) + 1; r /= n_[0];
    const int j = (int)(r % n_[1]) + 1; r /= n_[1];
    const int k = (int)(r % n_[2]) + 1; r /= n_[2];
    const int v = (int)(r % npde) + 1; r /= npde;
    const int n = (int)r;
    const int di = (d == 1), dj = (d == 2), dk = (d == 3);
    const int64_t base = p3_var(b, npde, S, v, n);
    const int64_t c0 = p3_cell(b, i, j, k), cm = p3_cell(b, i - di, j - dj, k - dk);
    const bool fo = first_all || (P.foturb && v >= 6);
    double vp, vm;
    if (fo) {
      vp = q[base + c0];
      vm = q[base + cm];
    } else {
      const double dlo = dq[base + cm], dmid = dq[base + c0], dhi = dq[base + p3_cell(b, i + di, j + dj, k + dk)];
      double a, bq;
      const int ilim = v <= 5 ? P.ilimf : P.ilimt;
      const double eps = v <= 5 ? P.epslimf : P.epslimt;
      if (mixed) {
        // the limited slopes in FP32 on the FP64 differences
        float fa, fb;
        limit_face_fast(ilim, (float)eps, (float)P.rkap, (float)dlo, (float)dmid, (float)dhi, fa, fb);
        a = fa; bq = fb;
      } else {
        limit_face<double>(ilim, eps, P.rkap, dlo, dmid, dhi, a, bq);
      }
      dqp[base + c0] = a;
      dqm[base + c0] = bq;
      vp = q[base + c0] + a;
      vm = q[base + cm] + bq;
    }
    const int e = d == 1 ? i : (d == 2 ? j : k);
    if (e == 1 || e == mx) {
      for (int ib = 0; ib < b.nbcs; ++ib) {
        const int *rw = bct + b.obct + 10 * ib;
        if (rw[1] != d || !strong_bc(rw[0])) continue;
        const int qpm = rw[2] == 1 ? 1 : mx;
        if (e != qpm) continue;
        const int t2 = d == 1 ? j : i, t3 = d == 3 ? j : k;
        const int s2 = d == 1 ? rw[5] : rw[3], e2 = d == 1 ? rw[6] : rw[4];
        const int s3 = d == 3 ? rw[5] : rw[7], e3 = d == 3 ? rw[6] : rw[8];
        if (t2 >= s2 && t2 <= e2 && t3 >= s3 && t3 <= e3) {
          const int64_t cb = rw[2] == 1 ? cm : c0;  // q(0) at the min face, q(mx) at the max face
          vp = q[base + cb];
          vm = q[base + cb];
        }
      }
    }
    qp[base + c0] = vp;
    qm[base + c0] = vm;
  }
}

// ---- roflux_b (src/flux.f90:45-238) --------------------------------------------------
template <class BS>
__global__ void k_roflux(BS bs_, const cosa_params *__restrict__ Pp, int d, const double *__restrict__ qr,
                         const double *__restrict__ ql, double *__restrict__ flux, const double *__restrict__ sijk,
                         int mixed = 0, const double *__restrict__ fv = nullptr) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const PhysPar ph = make_phys(P);
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int ic = d == 1 ? b.im : b.im - 1, jc = d == 2 ? b.jm : b.jm - 1, kc = d == 3 ? b.km : b.km - 1;
  const int64_t ncell = (int64_t)ic * jc * kc * S;
  const bool kom = npde > 5;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ic) + 1; r /= ic;
    const int j = (int)(r % jc) + 1; r /= jc;
    const int k = (int)(r % kc) + 1; r /= kc;
    const int n = (int)r, nh = n * P.hbmove;
    const int64_t c = p3_cell(b, i, j, k);
    double vr[5], vl[5], f[5];
    for (int m = 0; m < 5; ++m) {
      vr[m] = qr[p3_var(b, npde, S, m + 1, n) + c];
      vl[m] = ql[p3_var(b, npde, S, m + 1, n) + c];
    }
    const double tker = kom ? qr[p3_var(b, npde, S, 6, n) + c] : 0.0;
    const double tkel = kom ? ql[p3_var(b, npde, S, 6, n) + c] : 0.0;
    if (mixed)
      roe_flux_mixed_tke(ph, sijk[p2_idx(b, S2, 1, i, j, k, nh)], sijk[p2_idx(b, S2, 2, i, j, k, nh)],
                         sijk[p2_idx(b, S2, 3, i, j, k, nh)], sijk[p2_idx(b, S2, 4, i, j, k, nh)], vr, vl, tker, tkel,
                         f);
    else {
      const double kx = sijk[p2_idx(b, S2, 1, i, j, k, nh)], ky = sijk[p2_idx(b, S2, 2, i, j, k, nh)];
      const double kz = sijk[p2_idx(b, S2, 3, i, j, k, nh)];
      double ubn = 0.0;
      if (fv) {
        // face velocity . normal, roflux_b's order (src/flux.f90:110-113)
        const int64_t e = p2_idx(b, S2, 1, i, j, k, nh) / 4 * 3;
        ubn = fv[e] * kx + fv[e + 1] * ky + fv[e + 2] * kz;
      }
      roe_flux_fp64(ph, kx, ky, kz, sijk[p2_idx(b, S2, 4, i, j, k, nh)], vr, vl, tker, tkel, f, ubn);
    }
    for (int m = 0; m < 5; ++m) flux[f0_idx(b, npde, S, i, j, k, m + 1, n)] = f[m];
    if (kom) {
      // turbulence fluxes (src/flux.f90:249-380) with the mean-flow loop's
      // final h0l/h0r: those of the last face (ic,jc,kc) of this snapshot
      double a7[7], b7[7], tr[7], tl[7];
      const int64_t cl = p3_cell(b, ic, jc, kc);
      for (int m = 0; m < 6; ++m) {
        a7[m] = qr[p3_var(b, npde, S, m + 1, n) + cl];
        b7[m] = ql[p3_var(b, npde, S, m + 1, n) + cl];
      }
      for (int m = 0; m < 7; ++m) {
        tr[m] = qr[p3_var(b, npde, S, m + 1, n) + c];
        tl[m] = ql[p3_var(b, npde, S, m + 1, n) + c];
      }
      double fk, fw;
      roe_turb(P, sijk[p2_idx(b, S2, 1, i, j, k, nh)], sijk[p2_idx(b, S2, 2, i, j, k, nh)],
               sijk[p2_idx(b, S2, 3, i, j, k, nh)], sijk[p2_idx(b, S2, 4, i, j, k, nh)], tr, tl,
               face_h0(P.gamma, a7), face_h0(P.gamma, b7), fk, fw);
      flux[f0_idx(b, npde, S, i, j, k, 6, n)] = fk;
      flux[f0_idx(b, npde, S, i, j, k, 7, n)] = fw;
    }
  }
}

// ---- bresid (src/cosa.f90:1149-1211) --------------------------------------------------
template <class BS>
__global__ void k_resid(BS bs_, const cosa_params *__restrict__ Pp, int d, const double *__restrict__ flux,
                        double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk * npde * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int v = (int)(r % npde) + 1; r /= npde;
    const int n = (int)r;
    const int64_t o = p3_var(b, npde, S, v, n) + p3_cell(b, i, j, k);
    res[o] = res[o] + flux[f0_idx(b, npde, S, i + (d == 1), j + (d == 2), k + (d == 3), v, n)] -
             flux[f0_idx(b, npde, S, i, j, k, v, n)];
  }
}

// ---- update_b explicit, mean flow (src/update.f90:568-640) ---------------------------
template <class BS>
__global__ void k_update(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                         double *__restrict__ q, const double *__restrict__ qold, const double *__restrict__ dtv,
                         double ar) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk * 5 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int v = (int)(r % 5) + 1; r /= 5;
    const int n = (int)r;
    const int64_t o = p3_var(b, npde, S, v, n) + p3_cell(b, i, j, k);
    q[o] = qold[o] - ar * res[o] * dtv[p1_idx(b, S, i, j, k, n)];
  }
}

// ---- zero (src/util.f90), extent 1: 0..imax etc. ---------------------------------------
template <class BS>
__global__ void k_zero_res(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im + 1, nj = b.jm + 1, nk = b.km + 1;
  const int64_t ncell = (int64_t)ni * nj * nk * npde * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni); r /= ni;
    const int j = (int)(r % nj); r /= nj;
    const int k = (int)(r % nk); r /= nk;
    const int v = (int)(r % npde) + 1; r /= npde;
    const int n = (int)r;
    res[p3_var(b, npde, S, v, n) + p3_cell(b, i, j, k)] = 0.0;
  }
}

// ---- resg_brms / resg_brms_hb partial sums (src/cosa.f90:4503-4582, 4629-4697) -------
// One partial per CTA.  Steady flows sum snapshot 0; harmonic balance sums
// every snapshot (resg_brms_hb's loop over n = 0..2*nharms, :4680-4690), and
// the caller divides by ncell * S.
__device__ __forceinline__ void rms_accumulate(const DevBlock &b, int npde, int S, int nsnap,
                                               const double *__restrict__ res, const double *__restrict__ rhs,
                                               double acc[7]) {
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk, nall = ncell * nsnap;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nall; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const int64_t c = p3_cell(b, i, j, k);
    for (int v = 0; v < npde; ++v) {
      const double tt = res[p3_var(b, npde, S, v + 1, n) + c] - (rhs ? rhs[p3_var(b, npde, S, v + 1, n) + c] : 0.0);
      acc[v] += tt * tt;
    }
  }
}

__global__ void k_rms_partial(DevBlock b, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                              const double *__restrict__ rhs, double *__restrict__ part) {
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  rms_accumulate(b, npde, S, P.harbal ? S : 1, res, rhs, acc);
  __shared__ double red[7][32];
  for (int v = 0; v < npde; ++v) {
    double x = acc[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    for (int v = 0; v < npde; ++v) {
      double x = threadIdx.x < nw ? red[v][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) part[(int64_t)blockIdx.x * 8 + v] = x;
    }
  }
}

// Same partial sums as k_rms_partial with npde and the snapshot count passed
// by value (the allocation-free entry point has no device parameter block);
// S > 1 sums every snapshot, as resg_brms_hb does.
__global__ void k_rms_partial_noalloc(DevBlock b, int npde, int S, const double *__restrict__ res,
                                      const double *__restrict__ rhs, double *__restrict__ part) {
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  rms_accumulate(b, npde, S, S, res, rhs, acc);
  __shared__ double red[7][32];
  for (int v = 0; v < npde; ++v) {
    double x = acc[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    for (int v = 0; v < npde; ++v) {
      double x = threadIdx.x < nw ? red[v][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) part[(int64_t)blockIdx.x * 8 + v] = x;
    }
  }
}

// ---- imetrix_b (src/grid.f90:847-1010): face unit normals and areas, fixed grid ----
// One thread per face of family d; x/y/z are P2 grid arrays (0:imax+1, ...).
// S2 snapshots of the grid (node arrays (0:imax+1,...,0:S2-1) per block at
// op2*S2), metrics of snapshot nh
__global__ void k_imetrix(DevBlock b, int d, const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, double *__restrict__ s, int S2 = 1, int nh = 0) {
  const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
  const int ni = d == 1 ? b.im : b.im - 1, nj = d == 2 ? b.jm : b.jm - 1, nk = d == 3 ? b.km : b.km - 1;
  const int64_t nf = (int64_t)ni * nj * nk;
  const int64_t g0 = b.op2 * S2 + (int64_t)nh * I2 * J2 * K2;
  const double *X = x + g0, *Y = y + g0, *Z = z + g0;
  auto at = [&](const double *A, int i, int j, int k) { return A[i + I2 * (j + J2 * (int64_t)k)]; };
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)r + 1;
    // the two diagonals of the face: (p1 -> p3) and (p2 -> p4)
    int a0[3], a1[3], b0[3], b1[3];
    if (d == 1) { a0[0] = i; a0[1] = j; a0[2] = k; a1[0] = i; a1[1] = j + 1; a1[2] = k + 1;
                  b0[0] = i; b0[1] = j + 1; b0[2] = k; b1[0] = i; b1[1] = j; b1[2] = k + 1; }
    else if (d == 2) { a0[0] = i; a0[1] = j; a0[2] = k; a1[0] = i + 1; a1[1] = j; a1[2] = k + 1;
                       b0[0] = i + 1; b0[1] = j; b0[2] = k; b1[0] = i; b1[1] = j; b1[2] = k + 1; }
    else { a0[0] = i; a0[1] = j; a0[2] = k; a1[0] = i + 1; a1[1] = j + 1; a1[2] = k;
           b0[0] = i + 1; b0[1] = j; b0[2] = k; b1[0] = i; b1[1] = j + 1; b1[2] = k; }
    const double dxa = at(X, a1[0], a1[1], a1[2]) - at(X, a0[0], a0[1], a0[2]);
    const double dya = at(Y, a1[0], a1[1], a1[2]) - at(Y, a0[0], a0[1], a0[2]);
    const double dza = at(Z, a1[0], a1[1], a1[2]) - at(Z, a0[0], a0[1], a0[2]);
    const double dxb = at(X, b1[0], b1[1], b1[2]) - at(X, b0[0], b0[1], b0[2]);
    const double dyb = at(Y, b1[0], b1[1], b1[2]) - at(Y, b0[0], b0[1], b0[2]);
    const double dzb = at(Z, b1[0], b1[1], b1[2]) - at(Z, b0[0], b0[1], b0[2]);
    double n1, n2, n3;
    if (d == 2) {  // eta faces: the reference takes the cross product in the other order
      n1 = (dza * dyb - dya * dzb) / 2;
      n2 = (dxa * dzb - dza * dxb) / 2;
      n3 = (dya * dxb - dxa * dyb) / 2;
    } else {
      n1 = (dya * dzb - dza * dyb) / 2;
      n2 = (dza * dxb - dxa * dzb) / 2;
      n3 = (dxa * dyb - dya * dxb) / 2;
    }
    const double area = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
    const int64_t e = (g0 + i + I2 * (j + J2 * (int64_t)k)) * 4;
    s[e] = n1 / area; s[e + 1] = n2 / area; s[e + 2] = n3 / area; s[e + 3] = area;
  }
}

// ---- bvols (src/grid.f90:2160-2230): cell volumes (Kordulla-Vinokur) ---------------------
// the volumes of the first grid snapshot (S2 snapshots stored; rigid motions keep them)
__global__ void k_vols(DevBlock b, const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, double *__restrict__ vol, int S2 = 1) {
  const int64_t I2 = b.im + 2, J2 = b.jm + 2, I1 = b.im + 1, J1 = b.jm + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t nc = (int64_t)ni * nj * nk;
  const double *X = x + b.op2 * S2, *Y = y + b.op2 * S2, *Z = z + b.op2 * S2;
  auto at = [&](const double *A, int i, int j, int k) { return A[i + I2 * (j + J2 * (int64_t)k)]; };
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nc; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)r + 1;
    // components c of the (unnormalised) face vectors of the xi, eta, zeta faces at the cell's min corner
    auto sface = [&](int d, const double *P, const double *Q, int c) {
      // c-th component of the cross product of the two face diagonals
      int a0i = i, a0j = j, a0k = k, a1i, a1j, a1k, b0i, b0j, b0k, b1i, b1j, b1k;
      if (d == 1) { a1i = i; a1j = j + 1; a1k = k + 1; b0i = i; b0j = j + 1; b0k = k; b1i = i; b1j = j; b1k = k + 1; }
      else if (d == 2) { a1i = i + 1; a1j = j; a1k = k + 1; b0i = i + 1; b0j = j; b0k = k; b1i = i; b1j = j; b1k = k + 1; }
      else { a1i = i + 1; a1j = j + 1; a1k = k; b0i = i + 1; b0j = j; b0k = k; b1i = i; b1j = j + 1; b1k = k; }
      const double pa = at(P, a1i, a1j, a1k) - at(P, a0i, a0j, a0k), pb = at(P, b1i, b1j, b1k) - at(P, b0i, b0j, b0k);
      const double qa = at(Q, a1i, a1j, a1k) - at(Q, a0i, a0j, a0k), qb = at(Q, b1i, b1j, b1k) - at(Q, b0i, b0j, b0k);
      (void)c;
      return d == 2 ? (qa * pb - pa * qb) / 2 : (pa * qb - qa * pb) / 2;
    };
    const double dx = (sface(1, Y, Z, 1) + sface(2, Y, Z, 1) + sface(3, Y, Z, 1)) * (at(X, i + 1, j + 1, k + 1) - at(X, i, j, k));
    const double dy = (sface(1, Z, X, 2) + sface(2, Z, X, 2) + sface(3, Z, X, 2)) * (at(Y, i + 1, j + 1, k + 1) - at(Y, i, j, k));
    const double dz = (sface(1, X, Y, 3) + sface(2, X, Y, 3) + sface(3, X, Y, 3)) * (at(Z, i + 1, j + 1, k + 1) - at(Z, i, j, k));
    vol[b.op1 + i + I1 * (j + J1 * (int64_t)k)] = (dx + dy + dz) / 3;
  }
}

// ---- implicit residual smoothing (src/cosa.f90:2035-2443, 5206-5773) -------------
// scalef_b / scaleb_b (src/cosa.f90:5652-5773): res *= or /= dt/V
template <class BS>
__global__ void k_irs_scale(BS bs_, int npde, int S, double *__restrict__ res, const double *__restrict__ dtv,
                            const double *__restrict__ dtvt, int forward) {
  const DevBlock b = bs_.get();
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t n = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int s = (int)r;
    const int64_t c = p3_cell(b, i, j, k), o = p1_idx(b, S, i, j, k, s);
    const double d = dtv[o], dt2 = dtvt ? dtvt[o] : d;
    for (int v = 1; v <= npde; ++v) {
      if (v >= 6 && !dtvt) continue;
      const double f = v >= 6 ? dt2 : d;
      double &x = res[p3_var(b, npde, S, v, s) + c];
      x = forward ? x * f : x / f;
    }
  }
}

// One direction D of cirs_b / ccirs_b: a thread solves every variable vs..ve
// of one grid line with tridi (src/cosa.f90:2418-2443).  The line's pivots
// den(m) = b(m) - r(m-1) a(m) and ratios r(m) depend only on the coefficients,
// so they are computed once into `scr` (2 doubles per cell) and reused for
// each variable.  ores (if set) is the right-hand side of the i sweep of the
// cut variant; with_halo adds eps * res(halo) on the first and last rows.
template <int D, class BS>
__global__ void k_irs_line(BS bs_, int npde, int S, double *__restrict__ res, const double *__restrict__ ores,
                           const double *__restrict__ beta, double eps, int vs, int ve, int with_halo,
                           double *__restrict__ scr) {
  const DevBlock b = bs_.get();
  const int im = b.im - 1, jm = b.jm - 1, km = b.km - 1;
  const int len = D == 1 ? im : (D == 2 ? jm : km);
  const int n2 = D == 1 ? jm : im, n3 = D == 3 ? jm : km;
  const int64_t nlines = (int64_t)n2 * n3 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nlines; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r_ = t;
    const int t2 = (int)(r_ % n2) + 1; r_ /= n2;
    const int t3 = (int)(r_ % n3) + 1; r_ /= n3;
    const int s = (int)r_;
    auto ijk = [&](int m, int &i, int &j, int &k) {
      if (D == 1) { i = m; j = t2; k = t3; }
      else if (D == 2) { i = t2; j = m; k = t3; }
      else { i = t2; j = t3; k = m; }
    };
    auto coef = [&](int m) {
      int i, j, k;
      ijk(m, i, j, k);
      return beta ? beta[p1_idx(b, S, i, j, k, s)] : eps;
    };
    // pivots
    double rprev = 0.0;
    for (int m = 1; m <= len; ++m) {
      int i, j, k;
      ijk(m, i, j, k);
      const double e = coef(m);
      const double a = m == 1 ? 0.0 : -e, bb = 1 + 2 * e, c = m == len ? 0.0 : -e;
      const double den = m == 1 ? bb : bb - rprev * a;
      const double rr = c / den;
      const int64_t o = 2 * (b.op3 * S + (int64_t)s * b.P3 + p3_cell(b, i, j, k));
      scr[o] = rr;
      scr[o + 1] = den;
      rprev = rr;
    }
    for (int v = vs; v <= ve; ++v) {
      const int64_t base = p3_var(b, npde, S, v, s);
      const double *src = ores ? ores + base : res + base;
      double *x = res + base;
      double tprev = 0.0;
      for (int m = 1; m <= len; ++m) {
        int i, j, k;
        ijk(m, i, j, k);
        const int64_t c = p3_cell(b, i, j, k);
        const double e = coef(m);
        double rhs = src[c];
        if (with_halo && (m == 1 || m == len)) {
          // the last-row assignment wins on a single-cell line, as in ccirs_b
          int hi, hj, hk;
          ijk(m == len ? len + 1 : 0, hi, hj, hk);
          rhs = src[c] + e * x[p3_cell(b, hi, hj, hk)];
        }
        const double a = m == 1 ? 0.0 : -e;
        const int64_t o = 2 * (b.op3 * S + (int64_t)s * b.P3 + c);
        const double tt = m == 1 ? rhs / scr[o + 1] : (rhs - tprev * a) / scr[o + 1];
        x[c] = tt;
        tprev = tt;
      }
      double xnext = tprev;
      for (int m = len - 1; m >= 1; --m) {
        int i, j, k;
        ijk(m, i, j, k);
        const int64_t c = p3_cell(b, i, j, k);
        const int64_t o = 2 * (b.op3 * S + (int64_t)s * b.P3 + c);
        const double xm = x[c] - xnext * scr[o];
        x[c] = xm;
        xnext = xm;
      }
    }
  }
}

// The same line solves by parallel cyclic reduction: one warp per (line,
// snapshot, variable), the line's four diagonals/right-hand side in shared
// memory (ping-pong, 8 * nmax doubles per warp).  Row m of the system is
// -e_m x_{m-1} + (1 + 2 e_m) x_m - e_m x_{m+1} = r_m (first and last rows
// without the outer term), as in the Thomas sweeps above; step s eliminates
// x_{m-s} and x_{m+s} from row m, so after ceil(log2 len) steps x_m = r_m /
// b_m.  The chain of dependent steps is log2(len) instead of 2 len; the
// result differs from the Thomas sweeps by rounding only (the matrix is
// strictly diagonally dominant).
template <int D, class BS>
__global__ void __launch_bounds__(128) k_irs_pcr(BS bs_, int npde, int S, double *__restrict__ res,
                                                 const double *__restrict__ ores, const double *__restrict__ beta,
                                                 double eps, int vs, int ve, int with_halo, int nmax) {
  const DevBlock b = bs_.get();
  extern __shared__ double irs_sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int im = b.im - 1, jm = b.jm - 1, km = b.km - 1;
  const int len = D == 1 ? im : (D == 2 ? jm : km);
  const int n2 = D == 1 ? jm : im, n3 = D == 3 ? jm : km;
  const int nv = ve - vs + 1;
  const int64_t nwork = (int64_t)n2 * n3 * S * nv;
  double *buf = irs_sm + (size_t)warp * 8 * nmax;
  for (int64_t w = blockIdx.x * (int64_t)nw + warp; w < nwork; w += (int64_t)gridDim.x * nw) {
    int64_t r_ = w;
    const int t2 = (int)(r_ % n2) + 1; r_ /= n2;
    const int t3 = (int)(r_ % n3) + 1; r_ /= n3;
    const int s = (int)(r_ % S); r_ /= S;
    const int v = vs + (int)r_;
    auto cell = [&](int m) {
      if (D == 1) return p3_cell(b, m, t2, t3);
      if (D == 2) return p3_cell(b, t2, m, t3);
      return p3_cell(b, t2, t3, m);
    };
    auto coef = [&](int m) {
      if (!beta) return eps;
      if (D == 1) return beta[p1_idx(b, S, m, t2, t3, s)];
      if (D == 2) return beta[p1_idx(b, S, t2, m, t3, s)];
      return beta[p1_idx(b, S, t2, t3, m, s)];
    };
    const int64_t base = p3_var(b, npde, S, v, s);
    const double *src = ores ? ores + base : res + base;
    double *x = res + base;
    double *a0 = buf, *b0 = buf + nmax, *c0 = buf + 2 * nmax, *r0 = buf + 3 * nmax;
    double *a1 = buf + 4 * nmax, *b1 = buf + 5 * nmax, *c1 = buf + 6 * nmax, *r1 = buf + 7 * nmax;
    for (int m = lane + 1; m <= len; m += 32) {
      const double e = coef(m);
      double rhs = src[cell(m)];
      if (with_halo && (m == 1 || m == len)) rhs = src[cell(m)] + e * x[cell(m == len ? len + 1 : 0)];
      a0[m - 1] = m == 1 ? 0.0 : -e;
      b0[m - 1] = 1 + 2 * e;
      c0[m - 1] = m == len ? 0.0 : -e;
      r0[m - 1] = rhs;
    }
    __syncwarp();
    for (int st = 1; st < len; st <<= 1) {
      for (int m = lane; m < len; m += 32) {
        double am = a0[m], bm = b0[m], cm = c0[m], rm = r0[m];
        double an = 0.0, cn = 0.0;
        if (m - st >= 0) {
          const double al = -am / b0[m - st];
          an = al * a0[m - st];
          bm += al * c0[m - st];
          rm += al * r0[m - st];
        }
        if (m + st < len) {
          const double ga = -cm / b0[m + st];
          cn = ga * c0[m + st];
          bm += ga * a0[m + st];
          rm += ga * r0[m + st];
        }
        a1[m] = an; b1[m] = bm; c1[m] = cn; r1[m] = rm;
      }
      __syncwarp();
      double *t;
      t = a0; a0 = a1; a1 = t;
      t = b0; b0 = b1; b1 = t;
      t = c0; c0 = c1; c1 = t;
      t = r0; r0 = r1; r1 = t;
    }
    for (int m = lane + 1; m <= len; m += 32) x[cell(m)] = r0[m - 1] / b0[m - 1];
    __syncwarp();
  }
}

// RK update of the stage from a stored residual (IRS path):
// q_out = q^n - alpha dt/V R, optional copy of q^n (stage 1)
__global__ void k_update_stage(DevBlock b, int npde, int S, const double *__restrict__ res,
                               const double *__restrict__ qold, double *__restrict__ qout, double *__restrict__ qcopy,
                               const double *__restrict__ dtv, double ar) {
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t n = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int s = (int)r;
    const int64_t c = p3_cell(b, i, j, k);
    const double dt = dtv[p1_idx(b, S, i, j, k, s)];
    for (int v = 1; v <= 5; ++v) {
      const int64_t o = p3_var(b, npde, S, v, s) + c;
      const double q0 = qold[o];
      if (qcopy) qcopy[o] = q0;
      qout[o] = q0 - ar * res[o] * dt;
    }
  }
}

// ---- src_bhb (src/src.f90:556-613): res(n) += sum_m omega V D(n,m) q(m) -------------
template <class BS>
__global__ void k_src_hb(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                         const double *__restrict__ vol, double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t n = (int64_t)ni * nj * nk * npde;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int v = (int)r + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double ov = P.omega * vol[p1_idx(b, 1, i, j, k, 0)];
    double qs[COSA_MAX_SNAP];
    for (int m = 0; m < S; ++m) qs[m] = q[p3_var(b, npde, S, v, m) + c];
    for (int s = 0; s < S; ++s) {
      double qhb = 0.0;
      for (int m = 0; m < S; ++m) qhb = qhb + ov * P.dhb[s * S + m] * qs[m];
      double &x = res[p3_var(b, npde, S, v, s) + c];
      x = x + qhb;
    }
  }
}

// ---- update_bhb, rkimp branch without IRS on one level (src/update.f90:1564-1604) ----
// LU with partial pivoting of an n x n matrix (column-major a[i + n*j]) and
// the solve for nrhs right-hand sides (b[i + n*m]), in the order of LAPACK's
// unblocked DGETF2 (first largest pivot, whole rows swapped, column scaled by
// the pivot's reciprocal, rank-1 update) and DGETRS 'N'
__device__ __forceinline__ void hb_lu_solve(int n, double *a, double *bm, int nrhs) {
  int ipiv[COSA_MAX_SNAP];
  for (int j = 0; j < n; ++j) {
    int pv = j;
    double amax = fabs(a[j + n * j]);
    for (int i = j + 1; i < n; ++i)
      if (fabs(a[i + n * j]) > amax) { amax = fabs(a[i + n * j]); pv = i; }
    ipiv[j] = pv;
    if (a[pv + n * j] != 0.0) {
      if (pv != j)
        for (int k = 0; k < n; ++k) {
          const double t = a[j + n * k];
          a[j + n * k] = a[pv + n * k];
          a[pv + n * k] = t;
        }
      const double r = 1.0 / a[j + n * j];
      for (int i = j + 1; i < n; ++i) a[i + n * j] = a[i + n * j] * r;
    }
    for (int k = j + 1; k < n; ++k) {
      const double t = -a[j + n * k];
      for (int i = j + 1; i < n; ++i) a[i + n * k] = a[i + n * k] + a[i + n * j] * t;
    }
  }
  for (int m = 0; m < nrhs; ++m) {
    double *x = bm + n * m;
    for (int j = 0; j < n; ++j)
      if (ipiv[j] != j) {
        const double t = x[j];
        x[j] = x[ipiv[j]];
        x[ipiv[j]] = t;
      }
    for (int k = 0; k < n; ++k)
      if (x[k] != 0.0)
        for (int i = k + 1; i < n; ++i) x[i] = x[i] - x[k] * a[i + n * k];
    for (int k = n - 1; k >= 0; --k)
      if (x[k] != 0.0) {
        x[k] = x[k] / a[k + n * k];
        for (int i = 0; i < k; ++i) x[i] = x[i] - x[k] * a[i + n * k];
      }
  }
}

// update_bhb (src/update.f90:1301-1848), mean-flow equations.  One thread
// per interior cell: (I + ar omega dtau D) q = rhs over the snapshots (dtau =
// dtvol V of the row's snapshot), the five equations as five right-hand
// sides; qcopy (stage 1) receives qold.  qsrc null (no IRS, one level): the
// residual holds no time-spectral term and rhs = qold - ar res dtvol.  qsrc
// set (IRS or multigrid): the residual, smoothed, includes src_hb's
// qhb = omega V D q of the stage state qsrc, and rhs = qold + (qhb - res) ar
// dtvol with qhb recomputed from qsrc in src_bhb's order.  qsrc may be qout
// (the k-omega stage updates in place): a cell's values are all read first.
template <class BS>
__global__ void k_update_bhb(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                             const double *__restrict__ qold, double *qout, double *__restrict__ qcopy,
                             const double *__restrict__ dtv, const double *__restrict__ vol, double ar,
                             const double *qsrc) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni_ = b.im - 1, nj_ = b.jm - 1, nk_ = b.km - 1;
  const int64_t n = (int64_t)ni_ * nj_ * nk_;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni_) + 1; r /= ni_;
    const int j = (int)(r % nj_) + 1;
    const int k = (int)(r / nj_) + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP * 5];
    for (int si = 0; si < S; ++si) {
      const double dt = dtv[p1_idx(b, S, i, j, k, si)];
      const double dtau = dt * v;
      for (int sj = 0; sj < S; ++sj) a[si + S * sj] = (si == sj ? 1.0 : 0.0) + ar * P.omega * dtau * P.dhb[si * S + sj];
      for (int m = 0; m < 5; ++m) {
        const int64_t o = p3_var(b, npde, S, m + 1, si) + c;
        const double q0 = qold[o];
        if (qcopy) qcopy[o] = q0;
        if (qsrc) {
          double qhb = 0.0;
          for (int sj = 0; sj < S; ++sj)
            qhb = qhb + P.omega * v * P.dhb[si * S + sj] * qsrc[p3_var(b, npde, S, m + 1, sj) + c];
          x[si + S * m] = q0 + (qhb - res[o]) * ar * dt;
        } else {
          x[si + S * m] = q0 - ar * res[o] * dt;
        }
      }
    }
    hb_lu_solve(S, a, x, 5);
    for (int si = 0; si < S; ++si)
      for (int m = 0; m < 5; ++m) qout[p3_var(b, npde, S, m + 1, si) + c] = x[si + S * m];
  }
}

// resg_brms_hb partial sums with rkimp (src/cosa.f90:4629-4697): the
// residual plus omega D q V, one snapshot at a time, squared; 8 doubles per CTA
__global__ void k_rms_bhb_partial(DevBlock b, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                                  const double *__restrict__ q, const double *__restrict__ vol,
                                  double *__restrict__ part) {
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t ncell = (int64_t)ni * nj * nk;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)r + 1;
    const int64_t c = p3_cell(b, i, j, k);
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    for (int n = 0; n < S; ++n)
      for (int m = 0; m < npde; ++m) {
        double w = res[p3_var(b, npde, S, m + 1, n) + c];
        for (int s2 = 0; s2 < S; ++s2) w = w + P.omega * P.dhb[n * S + s2] * q[p3_var(b, npde, S, m + 1, s2) + c] * v;
        acc[m] += w * w;
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
