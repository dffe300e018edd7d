// k-omega terms of the B200 path (Wilcox kom, BSL kom_bsl, SST kom_sst;
// viscous, fixed grid), with the reference's array contract (one kernel per
// routine, the level drivers in cosa_gpu.cu loop over blocks like the
// Fortran drivers).
//
//   k_qface_mut       q_face with calmut: face mut into flux(.,1)
//   k_rtst            b_rtst: Reynolds stresses on the faces
//   k_vflux_kom       vflux_b, k-omega branch + laminar terms
//   k_qder_c          q_der_c: cell-centred velocity differences
//   k_turprod         turprod_b: production, div u, delta+
//   k_srckw           srckw_b: k and omega sources into res
//   k_update_kom      update_b's point-implicit k / omega update
//   k_cut_scalar      cut_q on a scalar P3 array (cutman_mut)
//   k_rest4           rest4_b: volume-weighted restriction of a scalar field
//   k_lim_prod_mg     lim_prod_mg_b: production limiter before restriction
//   k_lim_res_ome     lim_res_ome_b: omega residual limiter (residual pass)
//   k_add_interior    add_array over the interior cells (multigrid forcing)
//   k_facedist        facedist_b: face wall distances (BSL/SST)
//   k_update_ttrm     update_ttrm_b: blended gamma, beta, cross diffusion
//   k_tur_vis_sst     tur_vis_sst_b: SST eddy viscosity (+ k_tur_vis_sst_halo)
//
// BSL/SST: ttrm is (-1:imax+1,...,3,0:S-1) per block at op3*3*S; the face
// distances are one F0 scalar per face family; k_srckw, k_update_kom and
// k_lim_res_ome read gamma, beta (and the cross diffusion) from ttrm when it
// is given, Wilcox's constants otherwise.
#pragma once
#include "visc.cuh"

// ---- per-routine kernels ---------------------------------------------------------------
// one thread per face (i,j,k) of family D and snapshot
#define KOM_FACE_LOOP(D)                                                                                    \
  const int ni = (D) == 1 ? b.im : b.im - 1, nj = (D) == 2 ? b.jm : b.jm - 1, nk = (D) == 3 ? b.km : b.km - 1; \
  const int64_t total = (int64_t)ni * nj * nk * S;                                                          \
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;                              \
       t += (int64_t)gridDim.x * blockDim.x) {                                                              \
    int64_t r_ = t;                                                                                         \
    const int i = (int)(r_ % ni) + 1; r_ /= ni;                                                             \
    const int j = (int)(r_ % nj) + 1; r_ /= nj;                                                             \
    const int k = (int)(r_ % nk) + 1;                                                                       \
    const int n = (int)(r_ / nk);

#define KOM_CELL_LOOP                                                                                       \
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;                                                    \
  const int64_t total = (int64_t)ni * nj * nk * S;                                                          \
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;                              \
       t += (int64_t)gridDim.x * blockDim.x) {                                                              \
    int64_t r_ = t;                                                                                         \
    const int i = (int)(r_ % ni) + 1; r_ /= ni;                                                             \
    const int j = (int)(r_ % nj) + 1; r_ /= nj;                                                             \
    const int k = (int)(r_ % nk) + 1;                                                                       \
    const int n = (int)(r_ / nk);

__device__ __forceinline__ int64_t p3s_idx(const DevBlock &b, int S, int i, int j, int k, int n) {
  return b.op3 * S + (int64_t)n * b.P3 + p3_cell(b, i, j, k);
}
// ttrm(i,j,k,c,n), c = 1..3
__device__ __forceinline__ int64_t ttrm_idx(const DevBlock &b, int S, int i, int j, int k, int c, int n) {
  return b.op3 * 3 * S + ((int64_t)n * 3 + (c - 1)) * b.P3 + p3_cell(b, i, j, k);
}

// the BSL/SST closure constants of input() (src/input.f90:2522-2539)
struct BlendPar {
  double sigk1, sigk2, sigw1, sigw2, b1, b2, g1, g2, a1;
};
__device__ __forceinline__ BlendPar make_blend(const cosa_params &P) {
  BlendPar c;
  const double bstr = 0.09;
  c.a1 = 0.31;
  c.sigk1 = P.kom_sst ? 0.85 : 0.5;
  c.sigk2 = 1.0;
  c.sigw1 = 0.5;
  c.b1 = 3.0 / 40.0;
  c.g1 = __dsub_rn(c.b1 / bstr, __dmul_rn(c.sigw1, P.kappa * P.kappa) / sqrt(bstr));
  c.sigw2 = 0.856;
  c.b2 = 0.0828;
  c.g2 = __dsub_rn(c.b2 / bstr, __dmul_rn(c.sigw2, P.kappa * P.kappa) / sqrt(bstr));
  return c;
}
// F1 (F2) as the reference writes tanh: (e^2a - 1) / (e^2a + 1)
__device__ __forceinline__ double tanh_ref(double a) {
  const double e = exp(2 * a);
  return (e - 1) / (e + 1);
}
// F1 of update_ttrm_b / vflux from rho, k, omega, mu, the k.omega gradient
// product and the wall distance; cdt out
__device__ __forceinline__ double blend_f1(const BlendPar &c, const cosa_params &P, double rho, double tke, double ome,
                                           double mu, double gradkw, double dist, double &cdt) {
  const double dd = dist + P.epst, d2 = dd * dd;
  double arg1 = fmax(sqrt(tke) / 0.09 / ome / dd, 500 * mu / rho / ome / d2 * P.machfs / P.reyno);
  cdt = 2 * rho * c.sigw2 / ome * gradkw;
  const double acdt = fmax(cdt, 1.0e-20);
  arg1 = fmin(arg1, 4 * rho * c.sigw2 * tke / acdt / d2);
  const double a2 = arg1 * arg1;
  arg1 = fmin(a2 * a2, 1.0e2);
  return tanh_ref(arg1);
}

// mut on the faces of family D into flux(.,1) (bq_face_* calmut part)
template <int D, class BS>
__global__ void k_qface_mut(BS bs_, int npde, int S, const double *__restrict__ mut, double *__restrict__ flux) {
  const DevBlock b = bs_.get();
  KOM_FACE_LOOP(D)
    const int di = D == 1, dj = D == 2, dk = D == 3;
    flux[f0_idx(b, npde, S, i, j, k, 1, n)] =
        (mut[p3s_idx(b, S, i - di, j - dj, k - dk, n)] + mut[p3s_idx(b, S, i, j, k, n)]) / 2;
  }
}
__global__ void k_qwall_mut(const DevBlock *__restrict__ blocks, const WallFace *__restrict__ walls, int nw, int d,
                            int npde, int S, const double *__restrict__ mut, double *__restrict__ flux) {
  const int64_t total = (int64_t)nw * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const WallFace w = walls[t % nw];
    if (w.d != d) continue;
    const int n = (int)(t / nw);
    const DevBlock b = blocks[w.blk];
    int pa[3] = {w.fi, w.fj, w.fk};
    pa[d - 1] = w.inrout == 1 ? 0 : (d == 1 ? b.im : (d == 2 ? b.jm : b.km));
    flux[f0_idx(b, npde, S, w.fi, w.fj, w.fk, 1, n)] = mut[p3s_idx(b, S, pa[0], pa[1], pa[2], n)];
  }
}

// b_rtst of one face (src/flux.f90:2846-2946): tau1(1..6) from the face
// density and k, the velocity gradients gr[var u,v,w][xi, eta, zeta], the
// face inverse metrics and the face mut
__device__ __forceinline__ void rtst_face(const cosa_params &P, double rho, double tke, const double gr[3][3],
                                          const double vmf[9], double mut, double tau[6]) {
  const double fact = 2.0 / 3.0, mr = P.machfs / P.reyno;
  double dv[3][3];  // dv[var][x, y, z]
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int c3 = 0; c3 < 3; ++c3) dv[m][c3] = gr[m][0] * vmf[c3] + gr[m][1] * vmf[3 + c3] + gr[m][2] * vmf[6 + c3];
  const double divv = (dv[0][0] + dv[1][1] + dv[2][2]) * P.turcmp;
  const double txx = 2 * mut * (dv[0][0] - divv / 3), txy = mut * (dv[0][1] + dv[1][0]);
  const double txz = mut * (dv[0][2] + dv[2][0]), tyy = 2 * mut * (dv[1][1] - divv / 3);
  const double tyz = mut * (dv[1][2] + dv[2][1]), tzz = 2 * mut * (dv[2][2] - divv / 3);
  tau[0] = mr * txx - fact * rho * tke;
  tau[1] = mr * txy;
  tau[2] = mr * txz;
  tau[3] = mr * tyy - fact * rho * tke;
  tau[4] = mr * tyz;
  tau[5] = mr * tzz - fact * rho * tke;
}

// vflux_b with kom on one face: the k-omega branch (Reynolds stresses, k
// and omega diffusion; the omega row keeps the reference's dk/dz) plus the
// laminar terms with the face mut in the heat flux.  qf primitive face state
// (7 variables), g[dir][var] its gradients, fd the face wall distance
// (BSL/SST sigma blending) or negative for Wilcox's constants; F[0] = 0
__device__ __forceinline__ void vflux_kom_face(const cosa_params &P, const ViscPar &V, const double qf[7],
                                               const double g[3][7], const double tau[6], const double vmf[9],
                                               double kx, double ky, double kz, double ds, double mut, double fd,
                                               double F[7]) {
  const double rho = qf[0], p = qf[4];
  const double tt = P.gamma * p / rho;
  const double mu = sutherland(tt, P.stemp);
  const double tkexi = g[0][5], tkeeta = g[1][5], tkezeta = g[2][5];
  const double omexi = g[0][6], omeeta = g[1][6], omezeta = g[2][6];
  const double dtkedx = tkexi * vmf[0] + tkeeta * vmf[3] + tkezeta * vmf[6];
  const double dtkedy = tkexi * vmf[1] + tkeeta * vmf[4] + tkezeta * vmf[7];
  const double dtkedz = tkexi * vmf[2] + tkeeta * vmf[5] + tkezeta * vmf[8];
  const double domedx = omexi * vmf[0] + omeeta * vmf[3] + omezeta * vmf[6];
  const double domedy = omexi * vmf[1] + omeeta * vmf[4] + omezeta * vmf[7];
  const double txx = tau[0], txy = tau[1], txz = tau[2], tyy = tau[3], tyz = tau[4], tzz = tau[5];
  double Fk[7];
  Fk[1] = -(txx * kx + txy * ky + txz * kz) * ds;
  Fk[2] = -(txy * kx + tyy * ky + tyz * kz) * ds;
  Fk[3] = -(txz * kx + tyz * ky + tzz * kz) * ds;
  double sigk = P.sigk, sigw = P.sigw;
  if (fd >= 0) {
    // BSL/SST (src/flux.f90:987-1061): sigma_k, sigma_omega blended by F1 of
    // the face state and the face's wall distance
    const BlendPar c = make_blend(P);
    const double domedz = omexi * vmf[2] + omeeta * vmf[5] + omezeta * vmf[8];
    double cdt;
    const double f1 = blend_f1(c, P, rho, qf[5], qf[6], mu, dtkedx * domedx + dtkedy * domedy + dtkedz * domedz, fd,
                               cdt);
    sigk = f1 * c.sigk1 + (1 - f1) * c.sigk2;
    sigw = f1 * c.sigw1 + (1 - f1) * c.sigw2;
  }
  const double ctke = (mu + sigk * mut) * P.machfs / P.reyno;
  const double come = (mu + sigw * mut) * P.machfs / P.reyno;
  Fk[4] = -ctke * (dtkedx * kx + dtkedy * ky + dtkedz * kz) * ds;
  Fk[5] = -ctke * (dtkedx * kx + dtkedy * ky + dtkedz * kz) * ds;
  Fk[6] = -come * (domedx * kx + domedy * ky + dtkedz * kz) * ds;
  double f5[5], g5[3][5], F5[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) { f5[m] = qf[m]; g5[0][m] = g[0][m]; g5[1][m] = g[1][m]; g5[2][m] = g[2][m]; }
  vflux_face(V, f5, g5, vmf, kx, ky, kz, ds, mut, F5);
  F[0] = 0.0;
#pragma unroll
  for (int m = 1; m < 5; ++m) F[m] = Fk[m] + F5[m];
  F[5] = Fk[5];
  F[6] = Fk[6];
}

// b_rtst (src/flux.f90:2846-2946): tau1(.,1..6) on the faces of family d
template <class BS>
__global__ void k_rtst(BS bs_, int d, const cosa_params *__restrict__ Pp, const double *__restrict__ qf,
                       const double *__restrict__ g0, const double *__restrict__ g1, const double *__restrict__ g2,
                       const double *__restrict__ vm, int64_t n0, const double *__restrict__ flux,
                       double *__restrict__ tau) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_FACE_LOOP(d)
    const int64_t c = p3_cell(b, i, j, k);
    auto Q = [&](const double *a, int v) { return a[p3_var(b, npde, S, v, n) + c]; };
    const double rho = Q(qf, 1), tke = Q(qf, 6), mut = flux[f0_idx(b, npde, S, i, j, k, 1, n)];
    double vmf[9];
    load_vm(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, d, i, j, k, vmf);
    double gr[3][3];  // gr[var u,v,w][xi, eta, zeta]
#pragma unroll
    for (int m = 0; m < 3; ++m) { gr[m][0] = Q(g0, m + 2); gr[m][1] = Q(g1, m + 2); gr[m][2] = Q(g2, m + 2); }
    double t6[6];
    rtst_face(P, rho, tke, gr, vmf, mut, t6);
#pragma unroll
    for (int m = 0; m < 6; ++m) tau[p3_var(b, npde, S, m + 1, n) + c] = t6[m];
  }
}

// vflux_b with kom: the k-omega branch (Reynolds stresses, k and omega
// diffusion; the omega row keeps the reference's dk/dz) followed by the
// laminar terms with the face mut of flux(.,1)
template <class BS>
__global__ void k_vflux_kom(BS bs_, int d, const cosa_params *__restrict__ Pp, const double *__restrict__ qf,
                            const double *__restrict__ g0, const double *__restrict__ g1,
                            const double *__restrict__ g2, const double *__restrict__ tau,
                            const double *__restrict__ vm, int64_t n0, const double *__restrict__ s,
                            double *__restrict__ flux, const double *__restrict__ fdist) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const ViscPar V = make_visc(P);
  KOM_FACE_LOOP(d)
    const int nh = n * P.hbmove;
    const int64_t c = p3_cell(b, i, j, k);
    auto Q = [&](const double *a, int v) { return a[p3_var(b, npde, S, v, n) + c]; };
    const int64_t e = p2_idx(b, S2, 1, i, j, k, nh);
    const double kx = s[e], ky = s[e + 1], kz = s[e + 2], ds = s[e + 3];
    double vmf[9];
    load_vm(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, d, i, j, k, vmf);
    const double mut = flux[f0_idx(b, npde, S, i, j, k, 1, n)];
    double f7[7], g[3][7], t6[6], F[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) { f7[m] = Q(qf, m + 1); g[0][m] = Q(g0, m + 1); g[1][m] = Q(g1, m + 1); g[2][m] = Q(g2, m + 1); }
#pragma unroll
    for (int m = 0; m < 6; ++m) t6[m] = Q(tau, m + 1);
    vflux_kom_face(P, V, f7, g, t6, vmf, kx, ky, kz, ds, mut, fdist ? fdist[f0_idx(b, 1, 1, i, j, k, 1, 0)] : -1.0, F);
#pragma unroll
    for (int m = 0; m < 7; ++m) flux[f0_idx(b, npde, S, i, j, k, m + 1, n)] = F[m];
  }
}

// q_der_c (src/flux.f90:2979-3130): velocity differences of the face
// values, and of k and omega under BSL/SST (vhi = 7)
template <int D, class BS>
__global__ void k_qder_c(BS bs_, int npde, int S, const double *__restrict__ qf, double *__restrict__ dc, int vhi) {
  const DevBlock b = bs_.get();
  KOM_CELL_LOOP
    const int di = D == 1, dj = D == 2, dk = D == 3;
    const int64_t c0 = p3_cell(b, i, j, k), c1 = p3_cell(b, i + di, j + dj, k + dk);
    for (int v = 2; v <= vhi; ++v) {
      if (v == 5) continue;
      const int64_t o = p3_var(b, npde, S, v, n);
      dc[o + c0] = qf[o + c1] - qf[o + c0];
    }
  }
}

// turprod_b (src/src.f90:40-177)
template <class BS>
__global__ void k_turprod(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ dx,
                          const double *__restrict__ de, const double *__restrict__ dz, const double *__restrict__ vm,
                          int64_t n0, double *__restrict__ prd, double *__restrict__ divvel,
                          double *__restrict__ delpls) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    // cell metrics: derivative m, component c from the two faces of family c+1
    double met[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      met[m][0] = (vm[vm_idx(b, n0, 1, m, 0, i + 1, j, k)] + vm[vm_idx(b, n0, 1, m, 0, i, j, k)]) / 2;
      met[m][1] = (vm[vm_idx(b, n0, 2, m, 1, i, j + 1, k)] + vm[vm_idx(b, n0, 2, m, 1, i, j, k)]) / 2;
      met[m][2] = (vm[vm_idx(b, n0, 3, m, 2, i, j, k + 1)] + vm[vm_idx(b, n0, 3, m, 2, i, j, k)]) / 2;
    }
    const int64_t c = p3_cell(b, i, j, k);
    double dv[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const int64_t o = p3_var(b, npde, S, v + 2, n) + c;
      const double a = dx[o], e = de[o], f = dz[o];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) dv[v][cc] = a * met[0][cc] + e * met[1][cc] + f * met[2][cc];
    }
    const double divv = (dv[0][0] + dv[1][1] + dv[2][2]) * P.turcmp;
    const double txx = dv[0][0], txy = (dv[0][1] + dv[1][0]) / 2, txz = (dv[0][2] + dv[2][0]) / 2;
    const double tyy = dv[1][1], tyz = (dv[1][2] + dv[2][1]) / 2, tzz = dv[2][2];
    const double prod = 2 * (txx * txx + tyy * tyy + tzz * tzz + 2 * (txy * txy + txz * txz + tyz * tyz) - divv * divv / 3);
    const int64_t o = p3s_idx(b, S, i, j, k, n);
    prd[o] = prod;
    divvel[o] = divv;
    delpls[o] = 2.0 / 3.0 * fmax(divv, 0.0);
  }
}

// srckw_b (src/src.f90:196-272)
template <class BS>
__global__ void k_srckw(BS bs_, const cosa_params *__restrict__ Pp, int nl, const double *__restrict__ q,
                        const double *__restrict__ mut, const double *__restrict__ prd,
                        const double *__restrict__ divvel, double *__restrict__ res, const double *__restrict__ vol,
                        const double *__restrict__ ttrm) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const double fact = 2.0 / 3.0, mor = P.machfs / P.reyno;
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    const double rho = q[p3_var(b, npde, S, 1, n) + c], tke = q[p3_var(b, npde, S, 6, n) + c];
    const double ome = q[p3_var(b, npde, S, 7, n) + c];
    const double mt = mut[o], divv = divvel[o];
    double prod = prd[o], prodw = prd[o];
    if (P.lim_prodtke && (nl == 1 || P.prd_all_lvls)) {
      const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
      if (mor * mt * prod > tstdis) {
        prod = tstdis / mor / mt;
        if (P.lim_prodomega) prodw = prod;
      }
    }
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    double *r6 = res + p3_var(b, npde, S, 6, n) + c, *r7 = res + p3_var(b, npde, S, 7, n) + c;
    *r6 = *r6 - v * (mor * mt * prod - fact * divv * rho * tke - P.bstrkw * rho * tke * ome);
    if (ttrm) {
      // srckw_sst_b (src/src.f90:306-378): blended gamma, beta and the cross diffusion
      const double cdif = ttrm[ttrm_idx(b, S, i, j, k, 1, n)], gav = ttrm[ttrm_idx(b, S, i, j, k, 2, n)];
      const double bav = ttrm[ttrm_idx(b, S, i, j, k, 3, n)];
      *r7 = *r7 - v * (gav * P.cmu * rho * prodw - gav * fact * divv * rho * ome - bav * rho * (ome * ome) + cdif);
    } else {
      *r7 = *r7 - v * (P.gkw * P.cmu * rho * prodw - P.gkw * fact * divv * rho * ome - P.bkw * rho * (ome * ome));
    }
  }
}

// update_b, explicit k-omega part (src/update.f90:601-640)
template <class BS>
__global__ void k_update_kom(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                             double *__restrict__ q, const double *__restrict__ qold, const double *__restrict__ vol,
                             const double *__restrict__ dtt, const double *__restrict__ delpls,
                             const double *__restrict__ prd, double ar, const double *__restrict__ ttrm) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
    const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    const int64_t i1 = p3_var(b, npde, S, 1, n) + c, i6 = p3_var(b, npde, S, 6, n) + c, i7 = p3_var(b, npde, S, 7, n) + c;
    const double rho = q[i1], ome = q[i7] / q[i1], tke = q[i6] / q[i1];
    const double dt = dtt[p1_idx(b, S, i, j, k, n)];
    const double dtau = dt * vol[p1_idx(b, 1, i, j, k, 0)];
    const double dp = delpls[o];
    double rhomega = (qold[i7] - ar * res[i7] * dt + ar * dtau * rho * ome * (gav * dp + 2 * bav * ome)) /
                     (1 + ar * dtau * (gav * dp + 2 * bav * ome));
    const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
    if (rhomega < rhomegamin) rhomega = rhomegamin;
    q[i7] = rhomega;
    const double drhomega = rhomega - rho * ome;
    q[i6] = (qold[i6] - ar * res[i6] * dt + ar * dtau * rho * tke * (dp + P.bstrkw * ome) -
             ar * dtau * P.bstrkw * tke * drhomega) /
            (1 + ar * dtau * (dp + P.bstrkw * ome));
  }
}

// cut_q on a scalar P3 array with S snapshots (cutman_mut, src/bc.f90:2713-2799)
__global__ void k_cut_scalar(const DevBlock *__restrict__ blocks, const HaloItem *__restrict__ items, int nitems,
                             int S, double *__restrict__ a) {
  const int64_t total = (int64_t)nitems * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const HaloItem it = items[t % nitems];
    const int n = (int)(t / nitems);
    const DevBlock db = blocks[it.dblk], sb = blocks[it.sblk];
    const int64_t bd = db.op3 * S + (int64_t)n * db.P3, bs = sb.op3 * S + (int64_t)n * sb.P3;
    // the cut of the reference's last write keeps each halo cell (host mask)
    if (it.mask & 1) a[bd + it.h1] = a[bs + it.c1];
    if (it.mask & 2) a[bd + it.h2] = a[bs + it.c2];
  }
}

// ---- k-omega multigrid (src/cosa.f90:2672-2755, 3122-3160; src/src.f90:708-745;
// src/update.f90:2585-2835) --------------------------------------------------------------
// rest4_b: coarse cell = volume-weighted mean of its 8 fine cells, the
// reference's summation order (one thread per coarse cell and snapshot)
__global__ void k_rest4(DevBlock b1, DevBlock b2, int S, const double *__restrict__ f1, double *__restrict__ f2,
                        const double *__restrict__ vol1, const double *__restrict__ vol2) {
  const int ni = b2.im - 1, nj = b2.jm - 1, nk = b2.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i2 = (int)(r % ni) + 1; r /= ni;
    const int j2 = (int)(r % nj) + 1; r /= nj;
    const int k2 = (int)(r % nk) + 1; r /= nk;
    const int n = (int)r;
    const int i1 = 2 * i2 - 1, j1 = 2 * j2 - 1, k1 = 2 * k2 - 1;
    const int di[8] = {0, 0, 1, 1, 0, 0, 1, 1}, dj[8] = {0, 1, 0, 1, 0, 1, 0, 1}, dk[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double w = vol1[p1_idx(b1, 1, i1 + di[m], j1 + dj[m], k1 + dk[m], 0)];
      const double a = f1[p3s_idx(b1, S, i1 + di[m], j1 + dj[m], k1 + dk[m], n)];
      s = m == 0 ? w * a : s + w * a;
    }
    f2[p3s_idx(b2, S, i2, j2, k2, n)] = s / vol2[p1_idx(b2, 1, i2, j2, k2, 0)];
  }
}

// lim_prod_mg_b: q conservative (tke, ome are rho k, rho omega), as the
// reference's residual pass leaves it
template <class BS>
__global__ void k_lim_prod_mg(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                              double *__restrict__ prd, const double *__restrict__ mut) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const double mor = P.machfs / P.reyno;
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    const double rho = q[p3_var(b, npde, S, 1, n) + c], tke = q[p3_var(b, npde, S, 6, n) + c];
    const double ome = q[p3_var(b, npde, S, 7, n) + c];
    const double mt = mut[o], prod = prd[o];
    const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
    if (mor * mt * prod > tstdis) prd[o] = tstdis / mor / mt;
  }
}

// lim_res_ome_b, explicit branch without low-speed preconditioning
// (ttrm = (0, gkw, bkw) for the Wilcox model)
template <class BS>
__global__ void k_lim_res_ome(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ res,
                              const double *__restrict__ q, const double *__restrict__ vol,
                              const double *__restrict__ dtt, const double *__restrict__ delpls,
                              const double *__restrict__ prd, double ar, const double *__restrict__ ttrm) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
    const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    const int64_t i1 = p3_var(b, npde, S, 1, n) + c, i7 = p3_var(b, npde, S, 7, n) + c;
    const double dt = dtt[p1_idx(b, S, i, j, k, n)];
    const double dtau = dt * vol[p1_idx(b, 1, i, j, k, 0)];
    const double rho = q[i1], ome = q[i7] / q[i1];
    if (P.rkimp && P.dualt) {
      // rkimp (src/update.f90:2785-2823): the physical-time term in the
      // denominator; the reference's den1 has no ar here
      const double den1 = 1 + dtau * (gav * delpls[o] + 2 * bav * ome);
      const double den2 = ar * (P.bdf1 ? 1.0 : 1.5) * dtau / P.dt;
      const double rhomega = q[i7] - ar * res[i7] * dt / (den1 + den2);
      const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
      if (rhomega < rhomegamin) res[i7] = ((den1 + den2) * (q[i7] - rhomegamin)) / dt / ar;
      continue;
    }
    const double den1 = 1 + ar * dtau * (gav * delpls[o] + 2 * bav * ome);
    const double rhomega = q[i7] - ar * res[i7] * dt / den1;
    const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
    if (rhomega < rhomegamin) res[i7] = den1 * (q[i7] - rhomegamin) / dt / ar;
  }
}

// add_array over the interior cells (off_l = -1, src/util.f90:137-222):
// v1 += fact v2 for all nvs = npde * S variable planes
template <class BS>
__global__ void k_add_interior(BS bs_, int nvs, double *__restrict__ v1, const double *__restrict__ v2,
                               double fact) {
  const DevBlock b = bs_.get();
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * nvs;
  const int64_t base = b.op3 * nvs;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int64_t o = base + r * b.P3 + p3_cell(b, i, j, k);
    v1[o] = v1[o] + v2[o] * fact;
  }
}

// ---- BSL / SST ---------------------------------------------------------------------------
// facedist_b (src/grid.f90:2833-2870): one thread per face of family D with
// interior tangential indices; the mean of the two cells' wall distances,
// the boundary cell's own on the block faces
template <int D>
__global__ void k_facedist(DevBlock b, const double *__restrict__ dist, double *__restrict__ fd) {
  const int S = 1;
  KOM_FACE_LOOP(D)
    (void)n;
    const int m = D == 1 ? i : (D == 2 ? j : k), mx = D == 1 ? b.im : (D == 2 ? b.jm : b.km);
    const int di = D == 1, dj = D == 2, dk = D == 3;
    double v;
    if (m == 1) v = dist[p1_idx(b, 1, i - di, j - dj, k - dk, 0)];
    else if (m == mx) v = dist[p1_idx(b, 1, i, j, k, 0)];
    else v = (dist[p1_idx(b, 1, i - di, j - dj, k - dk, 0)] + dist[p1_idx(b, 1, i, j, k, 0)]) / 2;
    fd[f0_idx(b, 1, 1, i, j, k, 1, 0)] = v;
  }
}

// the cell-centre inverse metrics of turprod_b / update_ttrm_b / tur_vis_sst_b:
// met[m][c] = d(xi_m)/d(x_c), averaged over the two faces of family c + 1
__device__ __forceinline__ void cell_met(const double *__restrict__ vm, const DevBlock &b, int64_t n0, int i, int j,
                                         int k, double met[3][3]) {
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    met[m][0] = (vm[vm_idx(b, n0, 1, m, 0, i + 1, j, k)] + vm[vm_idx(b, n0, 1, m, 0, i, j, k)]) / 2;
    met[m][1] = (vm[vm_idx(b, n0, 2, m, 1, i, j + 1, k)] + vm[vm_idx(b, n0, 2, m, 1, i, j, k)]) / 2;
    met[m][2] = (vm[vm_idx(b, n0, 3, m, 2, i, j, k + 1)] + vm[vm_idx(b, n0, 3, m, 2, i, j, k)]) / 2;
  }
}

// update_ttrm_b (src/update.f90:3036-3161) on the primitive state with the
// cell-centred k and omega differences; Wilcox: (0, gkw, bkw)
template <class BS>
__global__ void k_update_ttrm(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                              const double *__restrict__ dx, const double *__restrict__ de,
                              const double *__restrict__ dz, const double *__restrict__ vm, int64_t n0,
                              double *__restrict__ ttrm, const double *__restrict__ dist) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const BlendPar cb = make_blend(P);
  KOM_CELL_LOOP
    if (P.kom) {
      ttrm[ttrm_idx(b, S, i, j, k, 1, n)] = 0.0;
      ttrm[ttrm_idx(b, S, i, j, k, 2, n)] = P.gkw;
      ttrm[ttrm_idx(b, S, i, j, k, 3, n)] = P.bkw;
      continue;
    }
    const int64_t c = p3_cell(b, i, j, k);
    auto Q = [&](const double *a, int v) { return a[p3_var(b, npde, S, v, n) + c]; };
    const double rho = Q(q, 1), tke = Q(q, 6), ome = Q(q, 7), p = Q(q, 5);
    const double tt = P.gamma * p / rho;
    const double mu = sutherland(tt, P.stemp);
    double met[3][3];
    cell_met(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, i, j, k, met);
    const double tkexi = Q(dx, 6), tkeeta = Q(de, 6), tkezeta = Q(dz, 6);
    const double omexi = Q(dx, 7), omeeta = Q(de, 7), omezeta = Q(dz, 7);
    const double dtkedx = tkexi * met[0][0] + tkeeta * met[1][0] + tkezeta * met[2][0];
    const double dtkedy = tkexi * met[0][1] + tkeeta * met[1][1] + tkezeta * met[2][1];
    const double dtkedz = tkexi * met[0][2] + tkeeta * met[1][2] + tkezeta * met[2][2];
    const double domedx = omexi * met[0][0] + omeeta * met[1][0] + omezeta * met[2][0];
    const double domedy = omexi * met[0][1] + omeeta * met[1][1] + omezeta * met[2][1];
    const double domedz = omexi * met[0][2] + omeeta * met[1][2] + omezeta * met[2][2];
    double cdt;
    const double f1 = blend_f1(cb, P, rho, tke, ome, mu, dtkedx * domedx + dtkedy * domedy + dtkedz * domedz,
                               dist[p1_idx(b, 1, i, j, k, 0)], cdt);
    ttrm[ttrm_idx(b, S, i, j, k, 1, n)] = cdt * (1 - f1);
    ttrm[ttrm_idx(b, S, i, j, k, 2, n)] = f1 * cb.g1 + (1 - f1) * cb.g2;
    ttrm[ttrm_idx(b, S, i, j, k, 3, n)] = f1 * cb.b1 + (1 - f1) * cb.b2;
  }
}

// tur_vis_sst_b (src/update.f90:2375-2460), interior cells: mut = a1 rho k /
// max(a1 omega, sqrt(2 S) F2) of the conservative state with the stage's
// cell-centred velocity differences
template <class BS>
__global__ void k_tur_vis_sst(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                              double *__restrict__ mut, const double *__restrict__ dx,
                              const double *__restrict__ de, const double *__restrict__ dz,
                              const double *__restrict__ vm, int64_t n0, const double *__restrict__ dist) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const BlendPar cb = make_blend(P);
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k);
    auto Q = [&](const double *a, int v) { return a[p3_var(b, npde, S, v, n) + c]; };
    const double q1 = Q(q, 1), q2 = Q(q, 2), q3 = Q(q, 3), q4 = Q(q, 4);
    const double p = (P.gamma - 1) * (Q(q, 5) - (q2 * q2 + q3 * q3 + q4 * q4) / q1 / 2 - Q(q, 6));
    const double rho = q1, tke = Q(q, 6) / rho, ome = Q(q, 7) / rho;
    const double tt = P.gamma * p / rho;
    const double mu = sutherland(tt, P.stemp);
    double met[3][3];
    cell_met(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, i, j, k, met);
    double dv[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const double a = Q(dx, v + 2), e = Q(de, v + 2), f = Q(dz, v + 2);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) dv[v][cc] = a * met[0][cc] + e * met[1][cc] + f * met[2][cc];
    }
    const double sxx = dv[0][0], sxy = (dv[0][1] + dv[1][0]) / 2, sxz = (dv[0][2] + dv[2][0]) / 2;
    const double syy = dv[1][1], syz = (dv[1][2] + dv[2][1]) / 2, szz = dv[2][2];
    const double sn = sxx * sxx + syy * syy + szz * szz + 2 * (sxy * sxy + sxz * sxz + syz * syz);
    const double dd = dist[p1_idx(b, 1, i, j, k, 0)] + P.epst;
    double arg2 = fmax(2 * sqrt(tke) / 0.09 / ome / dd, 500 * mu / rho / ome / (dd * dd) * P.machfs / P.reyno);
    arg2 = fmin(arg2 * arg2, 1.0e2);
    const double f2 = tanh_ref(arg2);
    const double fact = sqrt(2 * sn);
    mut[p3s_idx(b, S, i, j, k, n)] = cb.a1 * rho * tke / fmax(cb.a1 * ome, fact * f2) * P.reyno / P.machfs;
  }
}
// the face halos of tur_vis_sst_b: mut of the adjacent interior cell, on the
// six faces over the interior tangential ranges (edges and corners left)
template <class BS>
__global__ void k_tur_vis_sst_halo(BS bs_, int S, double *__restrict__ mut) {
  const DevBlock b = bs_.get();
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t fi = (int64_t)nj * nk, fj = (int64_t)ni * nk, fk = (int64_t)ni * nj;
  const int64_t per = 2 * (fi + fj + fk), total = per * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(t / per);
    int64_t r = t % per;
    int i, j, k, si, sj, sk;
    if (r < 2 * fk) {
      const int side = (int)(r / fk); r %= fk;
      i = (int)(r % ni) + 1; j = (int)(r / ni) + 1; k = side ? b.km : 0;
      si = i; sj = j; sk = side ? b.km - 1 : 1;
    } else if ((r -= 2 * fk) < 2 * fj) {
      const int side = (int)(r / fj); r %= fj;
      i = (int)(r % ni) + 1; k = (int)(r / ni) + 1; j = side ? b.jm : 0;
      si = i; sj = side ? b.jm - 1 : 1; sk = k;
    } else {
      r -= 2 * fj;
      const int side = (int)(r / fi); r %= fi;
      j = (int)(r % nj) + 1; k = (int)(r / nj) + 1; i = side ? b.im : 0;
      si = side ? b.im - 1 : 1; sj = j; sk = k;
    }
    mut[p3s_idx(b, S, i, j, k, n)] = mut[p3s_idx(b, S, si, sj, sk, n)];
  }
}

// ---- fused faces of the k-omega stage ---------------------------------------------------
// the last strong-BC patch (row of bct) of block b whose face at position e
// (1 or mx) along d covers the tangential indices (t2, t3); -1 if none.  A
// later patch replaces an earlier one on a shared face, as the wall-face
// list of q_face / q_der keeps it.
__device__ __forceinline__ int strong_row(const DevBlock &b, const int *__restrict__ bct, int d, int e, int mx, int t2,
                                          int t3) {
  if (e != 1 && e != mx) return -1;
  int row = -1;
  for (int ib = 0; ib < b.nbcs; ++ib) {
    const int *rw = bct + b.obct + 10 * ib;
    if (rw[1] != d || !strong_bc(rw[0])) continue;
    if (e != (rw[2] == 1 ? 1 : mx)) continue;
    const int s2 = d == 1 ? rw[5] : rw[3], e2 = d == 1 ? rw[6] : rw[4];
    const int s3 = d == 3 ? rw[5] : rw[7], e3 = d == 3 ? rw[6] : rw[8];
    if (t2 >= s2 && t2 <= e2 && t3 >= s3 && t3 <= e3) row = ib;
  }
  return row;
}
// the inflow/outflow side (1 = min face, 2 = max face) of a strong-BC patch
// covering position e along d; 0 if none
__device__ __forceinline__ int strong_side(const DevBlock &b, const int *__restrict__ bct, int d, int e, int mx,
                                           int t2, int t3) {
  return strong_row(b, bct, d, e, mx, t2, t3) < 0 ? 0 : (e == 1 ? 1 : 2);
}

// muscl_b* (dq with the strong-BC doubling, limiter, first order on coarse
// levels / foturb, the strong-BC override) of variables 1..nv at face
// (i,j,k) of family d, snapshot n: vr = qp (cell side), vl = qm (minus side),
// as k_muscl_dq + k_muscl_face compute them
template <bool MIXED>
__device__ __forceinline__ void rans_face_recon(const DevBlock &b, const cosa_params &P, const int *__restrict__ bct,
                                                const double *__restrict__ q, int d, int nl, int i, int j, int k,
                                                int n, int nv, double *vr, double *vl) {
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int di = d == 1, dj = d == 2, dk = d == 3;
  const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  const int e = d == 1 ? i : (d == 2 ? j : k);
  const int t2 = d == 1 ? j : i, t3 = d == 3 ? j : k;
  const int64_t cm2 = p3_cell(b, i - 2 * di, j - 2 * dj, k - 2 * dk), cm = p3_cell(b, i - di, j - dj, k - dk);
  const int64_t c0 = p3_cell(b, i, j, k), cp = p3_cell(b, i + di, j + dj, k + dk);
  const bool first_all = nl >= P.nl_crs;
  // doubling of the differences at strong-BC faces (index e-1, e, e+1)
  const int side = strong_side(b, bct, d, e, mx, t2, t3);
  const bool dlo2 = strong_side(b, bct, d, e - 1, mx, t2, t3) != 0;
  const bool dmi2 = side != 0;
  const bool dhi2 = strong_side(b, bct, d, e + 1, mx, t2, t3) != 0;
#pragma unroll
  for (int v = 1; v <= 7; ++v) {
    if (v > nv) break;
    const int64_t base = p3_var(b, npde, S, v, n);
    const double qm2 = q[base + cm2], qm = q[base + cm], q0 = q[base + c0], qp = q[base + cp];
    const bool fo = first_all || (P.foturb && v >= 6);
    double a_ = 0.0, b_ = 0.0;
    if (!fo) {
      double dlo = qm - qm2, dmid = q0 - qm, dhi = qp - q0;
      if (dlo2) dlo = dlo * 2;
      if (dmi2) dmid = dmid * 2;
      if (dhi2) dhi = dhi * 2;
      const int ilim = v <= 5 ? P.ilimf : P.ilimt;
      const double eps = v <= 5 ? P.epslimf : P.epslimt;
      if (MIXED) {
        float fa, fb;
        limit_face_fast(ilim, (float)eps, (float)P.rkap, (float)dlo, (float)dmid, (float)dhi, fa, fb);
        a_ = fa; b_ = fb;
      } else {
        limit_face<double>(ilim, eps, P.rkap, dlo, dmid, dhi, a_, b_);
      }
    }
    double vp = fo ? q0 : q0 + a_, vm = fo ? qm : qm + b_;
    if (side) vp = vm = side == 1 ? qm : q0;  // q(0) at the min face, q(mx) at the max face
    vr[v - 1] = vp;
    vl[v - 1] = vm;
  }
}

// roflux_b's turbulence fluxes use h0 of the mean-flow loop's last face
// (src/flux.f90:312): both sides' h0 at face (imax, jmax-1, kmax-1) of the i
// family (and its j, k counterparts) per block, family and snapshot, into
// h0[((block * 3 + d - 1) * S + n) * 2 + side]
template <bool MIXED>
__global__ void k_rans_h0(const DevBlock *__restrict__ blocks, int nb, const cosa_params *__restrict__ Pp,
                          const int *__restrict__ bct, const double *__restrict__ q, int nl, double *__restrict__ h0) {
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1;
  const int64_t total = (int64_t)nb * 3 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int n = (int)(t % S), d = (int)((t / S) % 3) + 1, ib = (int)(t / (3 * S));
    const DevBlock b = blocks[ib];
    const int ic = d == 1 ? b.im : b.im - 1, jc = d == 2 ? b.jm : b.jm - 1, kc = d == 3 ? b.km : b.km - 1;
    double a7[7], b7[7];
    rans_face_recon<MIXED>(b, P, bct, q, d, nl, ic, jc, kc, n, 6, a7, b7);
    h0[t * 2] = face_h0(P.gamma, a7);
    h0[t * 2 + 1] = face_h0(P.gamma, b7);
  }
}

// muscl + roflux_b of the faces of family D of block b: the reconstructed
// states stay in registers, the seven convective face fluxes go to F
template <int D, bool MIXED>
__device__ __forceinline__ void rans_conv_faces(const DevBlock &b, const cosa_params &P, const int *__restrict__ bct,
                                                const double *__restrict__ q, int nl, const double *__restrict__ s,
                                                const double *__restrict__ h0b, double *__restrict__ F,
                                                const double *__restrict__ fv = nullptr) {
  const PhysPar ph = make_phys(P);
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  KOM_FACE_LOOP(D)
    double vr[7], vl[7], f[5];
    rans_face_recon<MIXED>(b, P, bct, q, D, nl, i, j, k, n, npde, vr, vl);
    const int nh = n * P.hbmove;
    const int64_t e4 = p2_idx(b, S2, 1, i, j, k, nh);
    const double kx = s[e4], ky = s[e4 + 1], kz = s[e4 + 2], ds = s[e4 + 3];
    // the face speed of a moving grid (roflux_b, src/flux.f90:110-113, 262-264)
    const double ubn = fv ? fv[(e4 >> 2) * 3] * kx + fv[(e4 >> 2) * 3 + 1] * ky + fv[(e4 >> 2) * 3 + 2] * kz : 0.0;
    if (MIXED) roe_flux_mixed_tke(ph, kx, ky, kz, ds, vr, vl, vr[5], vl[5], f, ubn);
    else roe_flux_fp64(ph, kx, ky, kz, ds, vr, vl, vr[5], vl[5], f, ubn);
#pragma unroll
    for (int m = 0; m < 5; ++m) F[f0_idx(b, npde, S, i, j, k, m + 1, n)] = f[m];
    double fk, fw;
    roe_turb(P, kx, ky, kz, ds, vr, vl, h0b[2 * n], h0b[2 * n + 1], fk, fw, ubn);
    F[f0_idx(b, npde, S, i, j, k, 6, n)] = fk;
    F[f0_idx(b, npde, S, i, j, k, 7, n)] = fw;
  }
}

// q_face (+ calmut) / q_der / b_rtst / vflux_b of the faces of family D of
// block ib: the face state and gradients of the bulk loops, or on strong-BC
// faces the one-sided wall formulas with the halo mut (src/flux.f90:1848-1962,
// 2846-2946, 947-1180); the NV viscous face fluxes go to F.  NV = 7: k-omega
// (Reynolds stresses, k and omega diffusion); NV = 5: laminar flow (mut null)
template <int D, int NV = 7>
__device__ __forceinline__ void rans_visc_faces(const DevBlock &b, int ib, const cosa_params &P,
                                                const int *__restrict__ bct, const double *__restrict__ q,
                                                const double *__restrict__ mut, const double *__restrict__ vm,
                                                int64_t n0, const double *__restrict__ s,
                                                const double *__restrict__ fdist, double *__restrict__ F) {
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const ViscPar V = make_visc(P);
  constexpr int di = D == 1, dj = D == 2, dk = D == 3;
  const int mx = D == 1 ? b.im : (D == 2 ? b.jm : b.km);
  KOM_FACE_LOOP(D)
    const QView Q = qview(b, q, S, n, npde);
    const int e = D == 1 ? i : (D == 2 ? j : k);
    const int row = strong_row(b, bct, D, e, mx, D == 1 ? j : i, D == 3 ? j : k);
    double qf[NV], g[3][NV], mf = 0.0;
    if (row < 0) {
      face_interior<D, NV>(Q, i, j, k, qf, g);
      if (NV == 7) mf = (mut[p3s_idx(b, S, i - di, j - dj, k - dk, n)] + mut[p3s_idx(b, S, i, j, k, n)]) / 2;
    } else {
      const int *rw = bct + b.obct + 10 * row;
      WallFace w;
      w.blk = ib; w.d = D; w.inrout = rw[2];
      w.fi = i; w.fj = j; w.fk = k;
      w.lo[0] = rw[3]; w.lo[1] = rw[5]; w.lo[2] = rw[7];
      w.hi[0] = rw[4]; w.hi[1] = rw[6]; w.hi[2] = rw[8];
      face_wall<NV>(Q, w, mx, qf, g);
      const int a = e == 1 ? 0 : mx;
      if (NV == 7) mf = mut[p3s_idx(b, S, D == 1 ? a : i, D == 2 ? a : j, D == 3 ? a : k, n)];
    }
    double vmf[9];
    load_vm(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, D, i, j, k, vmf);
    const int64_t e4 = p2_idx(b, 2 * P.nharms * P.hbmove + 1, 1, i, j, k, n * P.hbmove);
    double Fv[NV];
    if constexpr (NV == 7) {
      double gr[3][3], t6[6];
#pragma unroll
      for (int m = 0; m < 3; ++m) { gr[m][0] = g[0][m + 1]; gr[m][1] = g[1][m + 1]; gr[m][2] = g[2][m + 1]; }
      rtst_face(P, qf[0], qf[5], gr, vmf, mf, t6);
      vflux_kom_face(P, V, qf, g, t6, vmf, s[e4], s[e4 + 1], s[e4 + 2], s[e4 + 3], mf,
                     fdist ? fdist[f0_idx(b, 1, 1, i, j, k, 1, 0)] : -1.0, Fv);
    } else {
      vflux_face(V, qf, g, vmf, s[e4], s[e4 + 1], s[e4 + 2], s[e4 + 3], 0.0, Fv);
    }
#pragma unroll
    for (int m = 0; m < NV; ++m) F[f0_idx(b, npde, S, i, j, k, m + 1, n)] = Fv[m];
  }
}

// every face flux of the k-omega stage in one launch: grid (x, block, 6),
// z = family - 1 for the convective fluxes (muscl + roflux) and 3 + family - 1
// for the viscous ones, each into its own plane of rf (n0 npde S doubles per
// plane); fd holds the three families' face wall distances (BSL/SST) or is null
template <bool MIXED>
__global__ void __launch_bounds__(128, 3) k_rans_faces(BlockList bs_, const cosa_params *__restrict__ Pp,
                                                       const int *__restrict__ bct, const double *__restrict__ q,
                                                       int nl, const double *__restrict__ si,
                                                       const double *__restrict__ sj, const double *__restrict__ sk,
                                                       const double *__restrict__ h0, const double *__restrict__ mut,
                                                       const double *__restrict__ vm, int64_t n0,
                                                       const double *__restrict__ fd, double *__restrict__ rf,
                                                       FaceVel fvel = FaceVel{{nullptr, nullptr, nullptr}}) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, z = blockIdx.z, d = z % 3 + 1;
  const double *s = d == 1 ? si : (d == 2 ? sj : sk);
  double *F = rf + (int64_t)z * n0 * P.npde * S;
  if (z < 3) {
    const double *h0b = h0 + ((int64_t)blockIdx.y * 3 + (d - 1)) * S * 2;
    const double *fv = fvel.f[d - 1];
    if (d == 1) rans_conv_faces<1, MIXED>(b, P, bct, q, nl, s, h0b, F, fv);
    else if (d == 2) rans_conv_faces<2, MIXED>(b, P, bct, q, nl, s, h0b, F, fv);
    else rans_conv_faces<3, MIXED>(b, P, bct, q, nl, s, h0b, F, fv);
  } else {
    const double *fdd = fd ? fd + (int64_t)(d - 1) * n0 : nullptr;
    if (d == 1) rans_visc_faces<1>(b, blockIdx.y, P, bct, q, mut, vm, n0, s, fdd, F);
    else if (d == 2) rans_visc_faces<2>(b, blockIdx.y, P, bct, q, mut, vm, n0, s, fdd, F);
    else rans_visc_faces<3>(b, blockIdx.y, P, bct, q, mut, vm, n0, s, fdd, F);
  }
}

// bresid of the three families on the summed convective + viscous face
// fluxes of k_rans_faces (visc = 0: the convective ones alone), families in
// the reference's order (src/cosa.f90:1149-1200)
__global__ void k_rans_resid(BlockList bs_, const cosa_params *__restrict__ Pp, int64_t n0,
                             const double *__restrict__ rf, double *__restrict__ res, int visc = 1) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int64_t plane = n0 * npde * S;
  KOM_CELL_LOOP
    const int64_t c = p3_cell(b, i, j, k);
    for (int v = 1; v <= npde; ++v) {
      const int64_t o = p3_var(b, npde, S, v, n) + c;
      double x = res[o];
#pragma unroll
      for (int d = 1; d <= 3; ++d) {
        const int64_t fp = f0_idx(b, npde, S, i + (d == 1), j + (d == 2), k + (d == 3), v, n);
        const int64_t fm = f0_idx(b, npde, S, i, j, k, v, n);
        const double *Fc = rf + (d - 1) * plane, *Fv = rf + (d + 2) * plane;
        if (visc) x = x + (Fc[fp] + Fv[fp]) - (Fc[fm] + Fv[fm]);
        else x = x + Fc[fp] - Fc[fm];
      }
      res[o] = x;
    }
  }
}

// update_b of the k-omega stage in one pass (src/update.f90:568-640): the
// point-implicit rho omega / rho k of k_update_kom, the mean-flow update
// q = q^n - ar R dt/V, and with ifixq the floors of fixq_b
template <class BS>
__global__ void k_update_rans(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ res,
                              double *__restrict__ q, const double *__restrict__ qold,
                              const double *__restrict__ vol, const double *__restrict__ dtt,
                              const double *__restrict__ dtv, const double *__restrict__ delpls,
                              const double *__restrict__ prd, double ar, const double *__restrict__ ttrm) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  KOM_CELL_LOOP
    const double gav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 2, n)] : P.gkw;
    const double bav = ttrm ? ttrm[ttrm_idx(b, S, i, j, k, 3, n)] : P.bkw;
    const int64_t c = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    const int64_t i1 = p3_var(b, npde, S, 1, n) + c, i6 = p3_var(b, npde, S, 6, n) + c, i7 = p3_var(b, npde, S, 7, n) + c;
    const double rho = q[i1], ome = q[i7] / q[i1], tke = q[i6] / q[i1];
    const double dt = dtt[p1_idx(b, S, i, j, k, n)];
    const double dtau = dt * vol[p1_idx(b, 1, i, j, k, 0)];
    const double dp = delpls[o];
    double rhomega = (qold[i7] - ar * res[i7] * dt + ar * dtau * rho * ome * (gav * dp + 2 * bav * ome)) /
                     (1 + ar * dtau * (gav * dp + 2 * bav * ome));
    const double rhomegamin = gav * P.cmu * rho * sqrt(prd[o]);
    if (rhomega < rhomegamin) rhomega = rhomegamin;
    const double drhomega = rhomega - rho * ome;
    double rk = (qold[i6] - ar * res[i6] * dt + ar * dtau * rho * tke * (dp + P.bstrkw * ome) -
                 ar * dtau * P.bstrkw * tke * drhomega) /
                (1 + ar * dtau * (dp + P.bstrkw * ome));
    const double dm = dtv[p1_idx(b, S, i, j, k, n)];
    double rho1 = rho;
#pragma unroll
    for (int m = 1; m <= 5; ++m) {
      const int64_t om = p3_var(b, npde, S, m, n) + c;
      const double v = qold[om] - ar * res[om] * dm;
      q[om] = v;
      if (m == 1) rho1 = v;
    }
    if (P.ifixq) {
      // fixq_b (src/update.f90:2216-2269) on the updated cell
      if (rk / rho1 < P.qmin[5]) rk = rho1 * P.qmin[5];
      if (rhomega / rho1 < P.qmin[6]) rhomega = rho1 * P.qmin[6];
    }
    q[i6] = rk;
    q[i7] = rhomega;
  }
}

// the cell side of the k-omega stage in one pass over the cells
// (src/cosa.f90:1878-1901): q_face + q_der_c of the three families (the
// differences still written to dx, dy, dz), turprod_b on the levels that
// compute production (else the restricted prd and div u are read), under
// BSL/SST update_ttrm_b, and srckw_b / srckw_sst_b into res; the state is
// primitive
template <bool BLEND>
__global__ void k_rans_cellsrc(BlockList bs_, const cosa_params *__restrict__ Pp, int nl, const int *__restrict__ bct,
                               const double *__restrict__ q, double *__restrict__ dx, double *__restrict__ dy,
                               double *__restrict__ dz, const double *__restrict__ vm, int64_t n0,
                               const double *__restrict__ mut, const double *__restrict__ dist,
                               const double *__restrict__ vol, double *__restrict__ prd, double *__restrict__ divvel,
                               double *__restrict__ delpls, double *__restrict__ ttrm, double *__restrict__ res) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  constexpr int vhi = BLEND ? 7 : 4;
  const bool own_prod = nl == 1 || P.prd_all_lvls;
  const double fact = 2.0 / 3.0, mor = P.machfs / P.reyno;
  KOM_CELL_LOOP
    const int64_t c0 = p3_cell(b, i, j, k), o = p3s_idx(b, S, i, j, k, n);
    // dc[d][v - 2]: differences of u, v, w (and k, omega) across the cell
    double dc[3][6];
#pragma unroll
    for (int d = 1; d <= 3; ++d) {
      const int di = d == 1, dj = d == 2, dk = d == 3;
      const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
      const int e = d == 1 ? i : (d == 2 ? j : k);
      const int t2 = d == 1 ? j : i, t3 = d == 3 ? j : k;
      const bool wlo = strong_row(b, bct, d, e, mx, t2, t3) >= 0;
      const bool whi = strong_row(b, bct, d, e + 1, mx, t2, t3) >= 0;
      const int64_t cm = p3_cell(b, i - di, j - dj, k - dk), cp = p3_cell(b, i + di, j + dj, k + dk);
      double *dd = d == 1 ? dx : (d == 2 ? dy : dz);
#pragma unroll
      for (int v = 2; v <= vhi; ++v) {
        if (v == 5) continue;
        const int64_t ov = p3_var(b, npde, S, v, n);
        const double qm = q[ov + cm], qc = q[ov + c0], qp = q[ov + cp];
        const double flo = wlo ? qm : (qm + qc) / 2;
        const double fhi = whi ? qp : (qc + qp) / 2;
        dc[d - 1][v - 2] = fhi - flo;
        dd[ov + c0] = dc[d - 1][v - 2];
      }
    }
    double met[3][3];
    if (own_prod || BLEND) cell_met(vm + (int64_t)(n * P.hbmove) * 27 * n0, b, n0, i, j, k, met);
    double prod, divv;
    if (own_prod) {
      // turprod_b (src/src.f90:40-177)
      double dv[3][3];
#pragma unroll
      for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) dv[v][cc] = dc[0][v] * met[0][cc] + dc[1][v] * met[1][cc] + dc[2][v] * met[2][cc];
      divv = (dv[0][0] + dv[1][1] + dv[2][2]) * P.turcmp;
      const double txx = dv[0][0], txy = (dv[0][1] + dv[1][0]) / 2, txz = (dv[0][2] + dv[2][0]) / 2;
      const double tyy = dv[1][1], tyz = (dv[1][2] + dv[2][1]) / 2, tzz = dv[2][2];
      prod = 2 * (txx * txx + tyy * tyy + tzz * tzz + 2 * (txy * txy + txz * txz + tyz * tyz) - divv * divv / 3);
      prd[o] = prod;
      divvel[o] = divv;
      delpls[o] = 2.0 / 3.0 * fmax(divv, 0.0);
    } else {
      prod = prd[o];
      divv = divvel[o];
    }
    auto Q = [&](int v) { return q[p3_var(b, npde, S, v, n) + c0]; };
    const double rho = Q(1), tke = Q(6), ome = Q(7);
    double cdif = 0.0, gav = P.gkw, bav = P.bkw;
    if (BLEND) {
      // update_ttrm_b (src/update.f90:3036-3161)
      const BlendPar cb = make_blend(P);
      const double tt = P.gamma * Q(5) / rho;
      const double mu = sutherland(tt, P.stemp);
      const double tkexi = dc[0][4], tkeeta = dc[1][4], tkezeta = dc[2][4];
      const double omexi = dc[0][5], omeeta = dc[1][5], omezeta = dc[2][5];
      const double dtkedx = tkexi * met[0][0] + tkeeta * met[1][0] + tkezeta * met[2][0];
      const double dtkedy = tkexi * met[0][1] + tkeeta * met[1][1] + tkezeta * met[2][1];
      const double dtkedz = tkexi * met[0][2] + tkeeta * met[1][2] + tkezeta * met[2][2];
      const double domedx = omexi * met[0][0] + omeeta * met[1][0] + omezeta * met[2][0];
      const double domedy = omexi * met[0][1] + omeeta * met[1][1] + omezeta * met[2][1];
      const double domedz = omexi * met[0][2] + omeeta * met[1][2] + omezeta * met[2][2];
      double cdt;
      const double f1 = blend_f1(cb, P, rho, tke, ome, mu, dtkedx * domedx + dtkedy * domedy + dtkedz * domedz,
                                 dist[p1_idx(b, 1, i, j, k, 0)], cdt);
      cdif = cdt * (1 - f1);
      gav = f1 * cb.g1 + (1 - f1) * cb.g2;
      bav = f1 * cb.b1 + (1 - f1) * cb.b2;
      ttrm[ttrm_idx(b, S, i, j, k, 1, n)] = cdif;
      ttrm[ttrm_idx(b, S, i, j, k, 2, n)] = gav;
      ttrm[ttrm_idx(b, S, i, j, k, 3, n)] = bav;
    }
    // srckw_b / srckw_sst_b (src/src.f90:196-378)
    const double mt = mut[o];
    double prodk = prod, prodw = prod;
    if (P.lim_prodtke && own_prod) {
      const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
      if (mor * mt * prodk > tstdis) {
        prodk = tstdis / mor / mt;
        if (P.lim_prodomega) prodw = prodk;
      }
    }
    const double v = vol[p1_idx(b, 1, i, j, k, 0)];
    double *r6 = res + p3_var(b, npde, S, 6, n) + c0, *r7 = res + p3_var(b, npde, S, 7, n) + c0;
    *r6 = *r6 - v * (mor * mt * prodk - fact * divv * rho * tke - P.bstrkw * rho * tke * ome);
    if (BLEND)
      *r7 = *r7 - v * (gav * P.cmu * rho * prodw - gav * fact * divv * rho * ome - bav * rho * (ome * ome) + cdif);
    else
      *r7 = *r7 - v * (P.gkw * P.cmu * rho * prodw - P.gkw * fact * divv * rho * ome - P.bkw * rho * (ome * ome));
  }
}
