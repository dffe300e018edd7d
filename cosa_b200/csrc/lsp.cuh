// Low-speed preconditioning (lomach) of the B200 path, Euler and laminar
// flow (npde = 5), explicit stages:
//
//   k_lm_cutoff_pg   lm_bcutoff_pg: Weiss and Darmofal's pressure-gradient
//                    cut-off of every interior cell
//   k_lm_viscoff     lm_bviscoff: the viscous cut-off from the cell Reynolds
//                    and Mach numbers
//   k_rest3          rest3_b: volume-weighted restriction of a cut-off field
//   k_proflux        lm_cutoff + proflux_b of one face family (reference
//                    array contract: qr = qp, ql = qm of muscl)
//   k_lsp_faces      the preconditioned convective fluxes (MUSCL + proflux)
//                    and, viscous runs, the laminar viscous fluxes of all three
//                    families in one launch, one flux plane each
//   k_lsp_prec       blsp's preconditioner of every interior cell
//   k_precres        prec_bres: res <- P res with a given P
//   k_lsp_precres    blsp + prec_bres fused: P built in registers and applied
//
// The cut-offs live in the interior-cell layout of the reference
// (imax-1, jmax-1, kmax-1, 0:S-1) per block at off_m1 * S (DevBlock::om1).
#pragma once
#include "kom.cuh"

__device__ __forceinline__ int64_t m1_idx(const DevBlock &b, int S, int i, int j, int k, int n) {
  const int I = b.im - 1, J = b.jm - 1, K = b.km - 1;
  return b.om1 * S + (int64_t)n * I * J * K + (i - 1) + (int64_t)I * ((j - 1) + (int64_t)J * (k - 1));
}

// lm_bcutoff_pg (src/losp.f90:1112-1165), primitive state with halos
template <class BS>
__global__ void k_lm_cutoff_pg(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                               double *__restrict__ cut) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    const int64_t o1 = p3_var(b, npde, S, 1, n), o5 = p3_var(b, npde, S, 5, n);
    const int64_t c = p3_cell(b, i, j, k);
    const double rho = q[o1 + c], pc = q[o5 + c];
    const double a2 = P.gamma * pc / rho;
    const double *p5 = q + o5;
    double dpmax = 0.0;
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i + 1, j, k)] - pc));
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i, j + 1, k)] - pc));
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i, j, k + 1)] - pc));
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i - 1, j, k)] - pc));
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i, j - 1, k)] - pc));
    dpmax = fmax(dpmax, fabs(p5[p3_cell(b, i, j, k - 1)] - pc));
    cut[m1_idx(b, S, i, j, k, n)] = dpmax / rho / a2;
  }
}

// lm_bviscoff (src/losp.f90:1317-1414); the reference pairs the i-direction
// speed with the j-face area and the j-direction speed with the i-face area
template <class BS>
__global__ void k_lm_viscoff(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                             const double *__restrict__ si, const double *__restrict__ sj,
                             const double *__restrict__ sk, double *__restrict__ cut) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const double g = P.gamma, st = P.stemp, epsi = 1.0e-7, rm = P.reyno / P.machfs;
  KOM_CELL_LOOP
    const int nh = n * P.hbmove;
    const int64_t c = p3_cell(b, i, j, k);
    auto Q = [&](int v) { return q[p3_var(b, npde, S, v, n) + c]; };
    const double rho = Q(1), u = Q(2), v = Q(3), w = Q(4), p = Q(5);
    const double tc = g * p / rho, a = sqrt(tc);
    const double mu = (st + 1) / (tc + st) * pow(tc, 1.5);
    double sm[3][4], sp[3][4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      sm[0][m] = si[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[0][m] = si[p2_idx(b, S2, m + 1, i + 1, j, k, nh)];
      sm[1][m] = sj[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[1][m] = sj[p2_idx(b, S2, m + 1, i, j + 1, k, nh)];
      sm[2][m] = sk[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[2][m] = sk[p2_idx(b, S2, m + 1, i, j, k + 1, nh)];
    }
    double U[3], A[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double x = 0.5 * (sm[d][0] + sp[d][0]), y = 0.5 * (sm[d][1] + sp[d][1]), z = 0.5 * (sm[d][2] + sp[d][2]);
      U[d] = fmax(epsi, fabs(u * x + v * y + w * z));
      A[d] = (sm[d][3] + sp[d][3]) / 2;
    }
    const double dd[3] = {A[1], A[0], A[2]};  // dx (with ux), dy (with uy), dz (with uz)
    double cmax = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double re = rm * rho * U[d] * dd[d] / mu, ma = U[d] / a;
      const double cf = (ma * ma * (1 - re)) / (re * re + ma * ma * re * (1 - re));
      cmax = d == 0 ? cf : fmax(cmax, cf);
    }
    cut[m1_idx(b, S, i, j, k, n)] = cmax;
  }
}

// rest3_b (src/cosa.f90:3046-3088): one thread per coarse cell and snapshot
__global__ void k_rest3(DevBlock b1, DevBlock b2, int S, const double *__restrict__ c1, double *__restrict__ c2,
                        const double *__restrict__ v1, const double *__restrict__ v2) {
  const int ni = (b1.im - 1) / 2, nj = (b1.jm - 1) / 2, nk = (b1.km - 1) / 2;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i2 = (int)(r % ni) + 1; r /= ni;
    const int j2 = (int)(r % nj) + 1; r /= nj;
    const int k2 = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const int i1 = 2 * i2 - 1, j1 = 2 * j2 - 1, k1 = 2 * k2 - 1;
    auto V = [&](int a, int bb, int c) { return v1[p1_idx(b1, 1, a, bb, c, 0)]; };
    auto C1 = [&](int a, int bb, int c) { return c1[m1_idx(b1, S, a, bb, c, n)]; };
    const double s = V(i1, j1, k1) * C1(i1, j1, k1) + V(i1, j1 + 1, k1) * C1(i1, j1 + 1, k1) +
                     V(i1 + 1, j1, k1) * C1(i1 + 1, j1, k1) + V(i1 + 1, j1 + 1, k1) * C1(i1 + 1, j1 + 1, k1) +
                     V(i1, j1, k1 + 1) * C1(i1, j1, k1 + 1) + V(i1, j1 + 1, k1 + 1) * C1(i1, j1 + 1, k1 + 1) +
                     V(i1 + 1, j1, k1 + 1) * C1(i1 + 1, j1, k1 + 1) +
                     V(i1 + 1, j1 + 1, k1 + 1) * C1(i1 + 1, j1 + 1, k1 + 1);
    c2[m1_idx(b2, S, i2, j2, k2, n)] = s / v2[p1_idx(b2, 1, i2, j2, k2, 0)];
  }
}

// lm_cutoff_b[ijk] (src/losp.f90:1167-1288): face e of family d takes the
// larger cut-off of its two cells, the boundary cell's own on the block faces
__device__ __forceinline__ double lsp_face_cut(const double *__restrict__ cut, const DevBlock &b, int S, int d, int i,
                                               int j, int k, int n) {
  const int e = d == 1 ? i : (d == 2 ? j : k), mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  const int di = d == 1, dj = d == 2, dk = d == 3;
  if (e == 1) return cut[m1_idx(b, S, i, j, k, n)];
  if (e == mx) return cut[m1_idx(b, S, i - di, j - dj, k - dk, n)];
  return fmax(cut[m1_idx(b, S, i, j, k, n)], cut[m1_idx(b, S, i - di, j - dj, k - dk, n)]);
}

// the preconditioned eigenvalue moduli and wave factors of proflux_b with
// the entropy fix / cut-off of the mean-flow (turb = false) or turbulence set
struct LspWaves {
  double rm123, rm4, rm5, esse, erre;
};
__device__ __forceinline__ LspWaves lsp_waves(const cosa_params &P, bool turb, double theth, double ubn, double a2,
                                              double mp2s, double u, double v, double w) {
  const double tu = theth - ubn;
  const double sq = sqrt(tu * tu * ((1 - mp2s) * (1 - mp2s)) + 4 * a2 * mp2s);
  const double lp4 = 0.5 * (tu * (1 + mp2s) + sq), lp5 = 0.5 * (tu * (1 + mp2s) - sq);
  LspWaves W;
  W.rm123 = fabs(tu); W.rm4 = fabs(lp4); W.rm5 = fabs(lp5);
  if (turb ? P.efx_setup_t : P.efx_setup_f) {
    const double asos = 0.5 * sq;
    const int *fw = turb ? P.entfx_t_w : P.entfx_f_w;
    double rdelta = (turb ? P.cntrpy_t : P.cntrpy_f) *
                    (fw[0] * (turb ? P.entfxctf_t : P.entfxctf_f) + fw[1] * (sqrt(u * u + v * v + w * w) + asos) +
                     fw[2] * 0.2 * (fabs(theth) + asos + fabs(ubn)));
    rdelta = fmax(rdelta, 1.0e-12);
    const bool all = turb ? P.efx_all_t : P.efx_all_f;
    if (W.rm123 <= rdelta && all) W.rm123 = 0.5 * (W.rm123 * W.rm123 + rdelta * rdelta) / rdelta;
    if (W.rm4 <= rdelta) W.rm4 = 0.5 * (W.rm4 * W.rm4 + rdelta * rdelta) / rdelta;
    if (W.rm5 <= rdelta) W.rm5 = 0.5 * (W.rm5 * W.rm5 + rdelta * rdelta) / rdelta;
  }
  if (turb ? P.eig_limit_t : P.eig_limit_f) {
    const double cut = turb ? P.eig_cutoff_t : P.eig_cutoff_f;
    const bool all = turb ? P.eig_lim_all_t : P.eig_lim_all_f;
    if (W.rm123 <= cut) W.rm123 = cut;
    if (all && W.rm4 <= cut) W.rm4 = cut;
    if (all && W.rm5 <= cut) W.rm5 = cut;
  }
  W.esse = tu - lp4;
  W.erre = tu - lp5;
  return W;
}

// proflux_b, one face (src/flux.f90:480-823): qr / ql the primitive face
// states (npde variables), cpg / cvs the face cut-offs; F[0..npde-1]
__device__ __forceinline__ void proflux_face(const cosa_params &P, double eps2, int npde, double kx, double ky,
                                             double kz, double ds, double ubn, const double *qr, const double *ql,
                                             double cpg, double cvs, double *F) {
  const double g = P.gamma;
  const bool kom = npde > 5;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
  const double tker = kom ? qr[5] : 0.0, tkel = kom ? ql[5] : 0.0;
  const double thethr = ur * kx + vr * ky + wr * kz - ubn, thethl = ul * kx + vl * ky + wl * kz - ubn;
  const double h0r = g / (g - 1) * pr / rhor + (ur * ur + vr * vr + wr * wr) / 2 + tker;
  const double h0l = g / (g - 1) * pl / rhol + (ul * ul + vl * vl + wl * wl) / 2 + tkel;
  const double rh0r = rhor * h0r, rh0l = rhol * h0l;
  const double fr[5] = {rhor * thethr, rhor * ur * thethr + pr * kx, rhor * vr * thethr + pr * ky,
                        rhor * wr * thethr + pr * kz, rh0r * thethr + pr * ubn};
  const double fl[5] = {rhol * thethl, rhol * ul * thethl + pl * kx, rhol * vl * thethl + pl * ky,
                        rhol * wl * thethl + pl * kz, rh0l * thethl + pl * ubn};
  const double drho = rhor - rhol, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl;
  const double dtheth = thethr - thethl, dtke = tker - tkel;
  const double rhols = sqrt(rhol), rhors = sqrt(rhor);
  const double rho = rhols * rhors, denom = rhols + rhors;
  const double u = (rhols * ul + rhors * ur) / denom, v = (rhols * vl + rhors * vr) / denom;
  const double w = (rhols * wl + rhors * wr) / denom;
  const double theth = u * kx + v * ky + w * kz;
  const double h0 = (rhols * h0l + rhors * h0r) / denom;
  const double tke = (rhols * tkel + rhors * tker) / denom;
  const double q2 = u * u + v * v + w * w;
  const double a2 = (g - 1) * (h0 - q2 / 2 - tke);
  const double a = sqrt(a2);
  const double m2 = q2 / a2, ump2 = (P.uprv / a) * (P.uprv / a);
  const double mp2 = fmin(1.0, fmax(fmax(fmax(fmax(m2, ump2), cpg), cvs), eps2));
  const double mp2s = fmin(1.0, fmax(fmax(fmax(fmax(m2, cpg), cvs), (1 - P.mixpi) * ump2), eps2));
  const LspWaves W = lsp_waves(P, false, theth, ubn, a2, mp2s, u, v, w);
  const double esse = W.esse, erre = W.erre;
  const double al1 = (drho - dp / a2) * W.rm123, al2 = rho * W.rm123;
  const double al4 = (rho * erre / (a * (erre - esse)) * dtheth + dp / (a * (erre - esse))) * W.rm4;
  const double al5 = (rho * esse / (a * (erre - esse)) * dtheth + dp / (a * (erre - esse))) * W.rm5;
  double df[5];
  df[0] = al1 + (al4 * (-esse) + al5 * erre) / a / mp2;
  df[1] = al1 * u + al2 * (du - dtheth * kx) + a * kx * (al4 - al5) + u * (al5 * erre - al4 * esse) / a / mp2;
  df[2] = al1 * v + al2 * (dv - dtheth * ky) + a * ky * (al4 - al5) + v * (al5 * erre - al4 * esse) / a / mp2;
  df[3] = al1 * w + al2 * (dw - dtheth * kz) + a * kz * (al4 - al5) + w * (al5 * erre - al4 * esse) / a / mp2;
  const double ht = a2 / (g - 1) + q2 / 2 + tke;
  df[4] = al1 * (q2 / 2 + tke) + al2 * (u * du + v * dv + w * dw - theth * dtheth + dtke) + a * theth * (al4 - al5) +
          al4 * (-(esse * ht / mp2 / a)) + al5 * (erre * ht / mp2 / a);
#pragma unroll
  for (int m = 0; m < 5; ++m) F[m] = (fr[m] + fl[m] - df[m]) / 2 * ds;
  if (!kom) return;
  const double omer = qr[6], omel = ql[6];
  const double ome = (rhols * omel + rhors * omer) / denom, dome = omer - omel;
  const LspWaves T = lsp_waves(P, true, theth, ubn, a2, mp2s, u, v, w);
  const double bl1 = (drho - dp / a2) * T.rm123, bl2 = rho * T.rm123;
  const double bl4 = (rho * T.erre / (a * (T.erre - T.esse)) * dtheth + dp / (a * (T.erre - T.esse))) * T.rm4;
  const double bl5 = (rho * T.esse / (a * (T.erre - T.esse)) * dtheth + dp / (a * (T.erre - T.esse))) * T.rm5;
  const double dfk = tke * (bl1 - (bl4 * T.esse - bl5 * T.erre) / a / mp2) + bl2 * dtke;
  const double dfw = ome * (bl1 - (bl4 * T.esse - bl5 * T.erre) / a / mp2) + bl2 * dome;
  F[5] = (rhor * thethr * tker + rhol * thethl * tkel - dfk) / 2 * ds;
  F[6] = (rhor * thethr * omer + rhol * thethl * omel - dfw) / 2 * ds;
}

// lm_cutoff + proflux_b of face family d with the reference's arrays
template <class BS>
__global__ void k_proflux(BS bs_, int d, const cosa_params *__restrict__ Pp, int nl, const double *__restrict__ qr,
                          const double *__restrict__ ql, double *__restrict__ flux, const double *__restrict__ s,
                          const double *__restrict__ cpg, const double *__restrict__ cvs) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const double eps2 = P.epsp[nl - 1] * P.epsp[nl - 1];
  KOM_FACE_LOOP(d)
    const int64_t c = p3_cell(b, i, j, k);
    double vr[7], vl[7], F[7];
    for (int m = 0; m < npde; ++m) {
      vr[m] = qr[p3_var(b, npde, S, m + 1, n) + c];
      vl[m] = ql[p3_var(b, npde, S, m + 1, n) + c];
    }
    const int64_t e4 = p2_idx(b, 1, 1, i, j, k, 0);
    proflux_face(P, eps2, npde, s[e4], s[e4 + 1], s[e4 + 2], s[e4 + 3], 0.0, vr, vl,
                 lsp_face_cut(cpg, b, S, d, i, j, k, n), lsp_face_cut(cvs, b, S, d, i, j, k, n), F);
    for (int m = 0; m < npde; ++m) flux[f0_idx(b, npde, S, i, j, k, m + 1, n)] = F[m];
  }
}

// every face flux of the preconditioned stage in one launch: grid (x,
// block, 3 or 6), z = family - 1 for MUSCL + lm_cutoff + proflux, 3 +
// family - 1 for the laminar viscous fluxes (q_face / q_der / vflux_b), each
// into its own plane of rf (n0 npde S doubles per plane)
__global__ void __launch_bounds__(128, 3) k_lsp_faces(BlockList bs_, const cosa_params *__restrict__ Pp,
                                                      const int *__restrict__ bct, const double *__restrict__ q, int nl,
                                                      const double *__restrict__ si, const double *__restrict__ sj,
                                                      const double *__restrict__ sk, const double *__restrict__ cpg,
                                                      const double *__restrict__ cvs, const double *__restrict__ vm,
                                                      int64_t n0, double *__restrict__ rf) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, z = blockIdx.z, d = z % 3 + 1;
  const double *s = d == 1 ? si : (d == 2 ? sj : sk);
  double *F = rf + (int64_t)z * n0 * npde * S;
  if (z >= 3) {
    if (d == 1) rans_visc_faces<1, 5>(b, blockIdx.y, P, bct, q, nullptr, vm, n0, s, nullptr, F);
    else if (d == 2) rans_visc_faces<2, 5>(b, blockIdx.y, P, bct, q, nullptr, vm, n0, s, nullptr, F);
    else rans_visc_faces<3, 5>(b, blockIdx.y, P, bct, q, nullptr, vm, n0, s, nullptr, F);
    return;
  }
  const double eps2 = P.epsp[nl - 1] * P.epsp[nl - 1];
  KOM_FACE_LOOP(d)
    double vr[7], vl[7], f[7];
    rans_face_recon<false>(b, P, bct, q, d, nl, i, j, k, n, npde, vr, vl);
    const int64_t e4 = p2_idx(b, 1, 1, i, j, k, 0);
    proflux_face(P, eps2, npde, s[e4], s[e4 + 1], s[e4 + 2], s[e4 + 3], 0.0, vr, vl,
                 lsp_face_cut(cpg, b, S, d, i, j, k, n), lsp_face_cut(cvs, b, S, d, i, j, k, n), f);
    for (int m = 0; m < npde; ++m) F[f0_idx(b, npde, S, i, j, k, m + 1, n)] = f[m];
  }
}

// blsp (src/losp.f90:42-195): P of one cell from its conservative state qc,
// pm[(r-1)*npde + (c-1)] = prec(i,j,k,r,c)
__device__ __forceinline__ void lsp_prec_cell(const cosa_params &P, double eps2, int npde, const double *qc, double cpg,
                                              double cvs, double *pm) {
  const double g = P.gamma, gam1 = g - 1;
  const bool kom = npde > 5;
  const double rho = qc[0], u = qc[1] / rho, v = qc[2] / rho, w = qc[3] / rho;
  const double q2 = u * u + v * v + w * w, e0 = qc[4] / rho;
  const double tke = kom ? qc[5] / rho : 0.0;
  const double p = (g - 1) * (e0 - 0.5 * q2 - tke) * rho;
  const double a2 = g * p / rho, a = sqrt(a2);
  const double ump2 = (P.uprv / a) * (P.uprv / a);
  const double mp2 = fmin(1.0, fmax(fmax(fmax(fmax(q2 / a2, ump2), cpg), cvs), eps2));
  const double m1 = mp2 - 1;
  const double vel[3] = {u, v, w};
  for (int e = 0; e < npde * npde; ++e) pm[e] = 0.0;
  auto E = [&](int r, int c) -> double & { return pm[(r - 1) * npde + (c - 1)]; };
  E(1, 1) = gam1 * m1 * q2 / 2 / a2 + 1;
#pragma unroll
  for (int c = 2; c <= 4; ++c) E(1, c) = -(vel[c - 2] * m1 * gam1 / a2);
  E(1, 5) = m1 * gam1 / a2;
#pragma unroll
  for (int r = 2; r <= 4; ++r) {
    const double x = vel[r - 2];
    E(r, 1) = x * gam1 * m1 * q2 / 2 / a2;
#pragma unroll
    for (int c = 2; c <= 4; ++c)
      E(r, c) = r == c ? 1 - x * x * m1 * gam1 / a2 : -(vel[min(r, c) - 2] * vel[max(r, c) - 2] * m1 * gam1 / a2);
    E(r, 5) = x * m1 * gam1 / a2;
  }
  const double hq = 2 * a2 + gam1 * (q2 + 2 * tke);
  E(5, 1) = q2 * m1 * hq / 4 / a2;
#pragma unroll
  for (int c = 2; c <= 4; ++c) E(5, c) = -(vel[c - 2] * m1 * hq / 2 / a2);
  E(5, 5) = mp2 + gam1 * (q2 + 2 * tke) * m1 / 2 / a2;
  if (!kom) return;
  const double ome = qc[6] / rho;
  E(1, 6) = -(m1 * gam1 / a2);
#pragma unroll
  for (int r = 2; r <= 4; ++r) E(r, 6) = -(vel[r - 2] * m1 * gam1 / a2);
  E(5, 6) = 1 - mp2 - gam1 * (q2 + 2 * tke) * m1 / 2 / a2;
  const double tw[2] = {tke, ome};
#pragma unroll
  for (int r = 6; r <= 7; ++r) {
    const double t = tw[r - 6];
    E(r, 1) = t * gam1 * m1 * q2 / 2 / a2;
#pragma unroll
    for (int c = 2; c <= 4; ++c) E(r, c) = -(vel[c - 2] * t * m1 * gam1 / a2);
    E(r, 5) = t * m1 * gam1 / a2;
  }
  E(6, 6) = 1 - tke * m1 * gam1 / a2;
  E(7, 6) = -(ome * m1 * gam1 / a2);
  E(7, 7) = 1;
}

// blsp's preconditioner into the reference's prec array
// (imax-1, jmax-1, kmax-1, npde, npde, 0:S-1) per block at om1 npde^2 S
template <class BS>
__global__ void k_lsp_prec(BS bs_, const cosa_params *__restrict__ Pp, int nl, const double *__restrict__ q,
                           const double *__restrict__ cpg, const double *__restrict__ cvs, double *__restrict__ prec) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const double eps2 = P.epsp[nl - 1] * P.epsp[nl - 1];
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k), m = m1_idx(b, S, i, j, k, n);
    double qc[7], pm[49];
    for (int v = 0; v < npde; ++v) qc[v] = q[p3_var(b, npde, S, v + 1, n) + c];
    lsp_prec_cell(P, eps2, npde, qc, cpg[m], cvs[m], pm);
    const int64_t nc = (int64_t)ni * nj * nk, cl = m - b.om1 * S - (int64_t)n * nc;
    double *pb = prec + b.om1 * npde * npde * S;
    for (int r = 0; r < npde; ++r)
      for (int cc = 0; cc < npde; ++cc) pb[(((int64_t)n * npde + cc) * npde + r) * nc + cl] = pm[r * npde + cc];
  }
}

// prec_bres (src/cosa.f90:2470-2521): res <- prec res, columns summed in order
template <class BS>
__global__ void k_precres(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ res,
                          const double *__restrict__ prec) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k), nc = (int64_t)ni * nj * nk;
    const int64_t cl = m1_idx(b, S, i, j, k, n) - b.om1 * S - (int64_t)n * nc;
    const double *pb = prec + b.om1 * npde * npde * S;
    double r[7], w[7];
    for (int v = 0; v < npde; ++v) r[v] = res[p3_var(b, npde, S, v + 1, n) + c];
    for (int a = 0; a < npde; ++a) {
      double x = 0.0;
      for (int cc = 0; cc < npde; ++cc) x = x + pb[(((int64_t)n * npde + cc) * npde + a) * nc + cl] * r[cc];
      w[a] = x;
    }
    for (int v = 0; v < npde; ++v) res[p3_var(b, npde, S, v + 1, n) + c] = w[v];
  }
}

// lsp + precres of the stage: P built in registers from the conservative q
// and applied to res
template <class BS>
__global__ void k_lsp_precres(BS bs_, const cosa_params *__restrict__ Pp, int nl, const double *__restrict__ q,
                              const double *__restrict__ cpg, const double *__restrict__ cvs,
                              double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const double eps2 = P.epsp[nl - 1] * P.epsp[nl - 1];
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k), m = m1_idx(b, S, i, j, k, n);
    double qc[5], pm[25], r[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      qc[v] = q[p3_var(b, npde, S, v + 1, n) + c];
      r[v] = res[p3_var(b, npde, S, v + 1, n) + c];
    }
    lsp_prec_cell(P, eps2, 5, qc, cpg[m], cvs[m], pm);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      double x = 0.0;
#pragma unroll
      for (int cc = 0; cc < 5; ++cc) x = x + pm[a * 5 + cc] * r[cc];
      res[p3_var(b, npde, S, a + 1, n) + c] = x;
    }
  }
}
