// Laminar viscous terms of the B200 path (viscous = .true., no turbulence
// model, fixed grid).
//
// Set-up (once per level, src/cosa.f90:300-322):
//   k_coordex / k_volex      ghost nodes repeat the boundary nodes, face-halo
//                            volumes repeat the first cell (cordex_b, volex_b)
//   k_copy_list              cut_x / cut_v: node and volume halos copied from
//                            the neighbour block, one item per halo entry,
//                            host-deduplicated to the reference's last writer
//   k_vmetrix                the nine inverse metrics of every face, products
//                            rounded separately as the reference's compiler
//                            does, so the metrics match the oracle bit for bit
// Per stage (the viscous part of src/cosa.f90:1797-1876):
//   k_prim                   primitive copy of the stage state (interior
//                            converted, halos copied) for the face stencils
//   k_edges                  q_edges on that copy (mg.cuh)
//   k_dt_ns                  lambdab/eig_ns + bdeltat with viscous lambdas
//   k_vface                  face state, face gradients and viscous flux of
//                            every face of the three families in one launch
//   k_vwall                  the same on strong-boundary faces with the
//                            one-sided wall formulas, overwriting k_vface
//   k_vdiv                   flux balance of each cell; the fused stage
//                            kernel adds it to the convective residual
// Per-routine kernels with the reference's array contract (q_face, q_der,
// vflux, lambda/deltat) use the same device functions.
#pragma once
#include "kernels_ref.cuh"

// one halo entry of cut_x (grid nodes, P2 offsets without lmet) or cut_v
// (volumes, P1 offsets): a[dst] = a[src]
struct CopyItem {
  int64_t dst, src;
};

// one strong-boundary face of q_face / q_der (bq_face_*, bq_der_*)
struct WallFace {
  int blk, d, inrout;
  int fi, fj, fk;     // face index (1-based, family d)
  int lo[3], hi[3];   // the patch's index ranges (directions 1..3)
};

__host__ __device__ __forceinline__ int64_t g2_idx(const DevBlock &b, int i, int j, int k) {
  return b.op2 + i + (int64_t)(b.im + 2) * (j + (int64_t)(b.jm + 2) * k);
}
// array (d, m) of the face inverse metrics: derivatives of xi (m=0), eta (1),
// zeta (2) on the faces of family d; (3, im, jm, km) per block at of0*3
__host__ __device__ __forceinline__ int64_t vm_idx(const DevBlock &b, int64_t n0, int d, int m, int c, int i, int j,
                                                   int k) {
  return ((int64_t)((d - 1) * 3 + m) * 3) * n0 + b.of0 * 3 +
         ((i - 1) + (int64_t)b.im * ((j - 1) + (int64_t)b.jm * (k - 1))) * 3 + c;
}

// ---- cordex_b (src/grid.f90:29-80) -------------------------------------------------
__global__ void k_coordex(DevBlock b, double *__restrict__ x, double *__restrict__ y, double *__restrict__ z) {
  const int im = b.im, jm = b.jm, km = b.km;
  const int64_t nj_ = (int64_t)im * km, ni_ = (int64_t)jm * km, nk_ = (int64_t)im * jm;
  const int64_t total = 2 * (nj_ + ni_ + nk_);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    int gi, gj, gk, si, sj, sk;
    if (r < 2 * nj_) {
      const int side = (int)(r / nj_); r %= nj_;
      gi = si = (int)(r % im) + 1; gk = sk = (int)(r / im) + 1;
      gj = side ? jm + 1 : 0; sj = side ? jm : 1;
    } else if ((r -= 2 * nj_) < 2 * ni_) {
      const int side = (int)(r / ni_); r %= ni_;
      gj = sj = (int)(r % jm) + 1; gk = sk = (int)(r / jm) + 1;
      gi = side ? im + 1 : 0; si = side ? im : 1;
    } else {
      r -= 2 * ni_;
      const int side = (int)(r / nk_); r %= nk_;
      gi = si = (int)(r % im) + 1; gj = sj = (int)(r / im) + 1;
      gk = side ? km + 1 : 0; sk = side ? km : 1;
    }
    const int64_t d = g2_idx(b, gi, gj, gk), s = g2_idx(b, si, sj, sk);
    x[d] = x[s]; y[d] = y[s]; z[d] = z[s];
  }
}

// ---- volex_b (src/grid.f90:110-136) ------------------------------------------------
__global__ void k_volex(DevBlock b, double *__restrict__ vol) {
  const int im = b.im, jm = b.jm, km = b.km;
  const int64_t nj_ = (int64_t)(im - 1) * (km - 1), ni_ = (int64_t)(jm - 1) * (km - 1);
  const int64_t nk_ = (int64_t)(im - 1) * (jm - 1);
  const int64_t total = 2 * (nj_ + ni_ + nk_);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    int gi, gj, gk, si, sj, sk;
    if (r < 2 * nj_) {
      const int side = (int)(r / nj_); r %= nj_;
      gi = si = (int)(r % (im - 1)) + 1; gk = sk = (int)(r / (im - 1)) + 1;
      gj = side ? jm : 0; sj = side ? jm - 1 : 1;
    } else if ((r -= 2 * nj_) < 2 * ni_) {
      const int side = (int)(r / ni_); r %= ni_;
      gj = sj = (int)(r % (jm - 1)) + 1; gk = sk = (int)(r / (jm - 1)) + 1;
      gi = side ? im : 0; si = side ? im - 1 : 1;
    } else {
      r -= 2 * ni_;
      const int side = (int)(r / nk_); r %= nk_;
      gi = si = (int)(r % (im - 1)) + 1; gj = sj = (int)(r / (im - 1)) + 1;
      gk = side ? km : 0; sk = side ? km - 1 : 1;
    }
    vol[p1_idx(b, 1, gi, gj, gk, 0)] = vol[p1_idx(b, 1, si, sj, sk, 0)];
  }
}

// ---- cut_x / cut_v in-process branches (src/grid.f90:242-523, 612-700) -------------
// sources are interior entries of the neighbour block, never written here
__global__ void k_copy_list(const CopyItem *__restrict__ items, int n, double *__restrict__ a,
                            double *__restrict__ b2, double *__restrict__ b3) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const CopyItem it = items[t];
    a[it.dst] = a[it.src];
    if (b2) b2[it.dst] = b2[it.src];
    if (b3) b3[it.dst] = b3[it.src];
  }
}

// ---- vmetrix_b (src/grid.f90:3150-3582) --------------------------------------------
// The derivative of the coordinates along the face normal is the mean of
// central differences at the face's four nodes (doubled where the ghost node
// repeats its node: one-sided at a physical boundary); along each tangent it
// is the mean of the two node differences of the face's edges.  The inverse
// metrics are the cofactors divided by the mean volume of the two cells.
__global__ void k_vmetrix(DevBlock b, int d, const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, const double *__restrict__ vol, double *__restrict__ vm,
                          int64_t n0) {
  const int im = b.im, jm = b.jm, km = b.km;
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const int64_t total = (int64_t)ni * nj * nk;
  const int mx = d == 1 ? im : (d == 2 ? jm : km);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1;
    const int k = (int)(r / nj) + 1;
    const int p[3] = {i, j, k};
    const int pos = p[d - 1];
    double g[3][3];  // g[dir][xyz]: coordinate derivative along dir
#pragma unroll
    for (int dir = 1; dir <= 3; ++dir) {
      const int e0 = dir == 1, e1 = dir == 2, e2 = dir == 3;
      if (dir == d) {
        // corners in the reference's order
        int cr[4][3];
        if (d == 1) { cr[0][0] = 0; cr[0][1] = 0; cr[0][2] = 0; cr[1][0] = 0; cr[1][1] = 1; cr[1][2] = 0;
                      cr[2][0] = 0; cr[2][1] = 1; cr[2][2] = 1; cr[3][0] = 0; cr[3][1] = 0; cr[3][2] = 1; }
        else if (d == 2) { cr[0][0] = 0; cr[0][1] = 0; cr[0][2] = 0; cr[1][0] = 0; cr[1][1] = 0; cr[1][2] = 1;
                           cr[2][0] = 1; cr[2][1] = 0; cr[2][2] = 1; cr[3][0] = 1; cr[3][1] = 0; cr[3][2] = 0; }
        else { cr[0][0] = 0; cr[0][1] = 0; cr[0][2] = 0; cr[1][0] = 1; cr[1][1] = 0; cr[1][2] = 0;
               cr[2][0] = 1; cr[2][1] = 1; cr[2][2] = 0; cr[3][0] = 0; cr[3][1] = 1; cr[3][2] = 0; }
        double v[4][3];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int a0 = i + cr[m][0], a1 = j + cr[m][1], a2 = k + cr[m][2];
          const int64_t hp = g2_idx(b, a0 + e0, a1 + e1, a2 + e2), hm = g2_idx(b, a0 - e0, a1 - e1, a2 - e2);
          v[m][0] = (x[hp] - x[hm]) / 2;
          v[m][1] = (y[hp] - y[hm]) / 2;
          v[m][2] = (z[hp] - z[hm]) / 2;
          if (pos == 1 || pos == mx) {
            const int64_t gh = pos == 1 ? hm : hp, c0 = g2_idx(b, a0, a1, a2);
            const double dx = x[gh] - x[c0], dy = y[gh] - y[c0], dz = z[gh] - z[c0];
            const double dist = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
            if (dist < 1.0e-14) { v[m][0] = 2 * v[m][0]; v[m][1] = 2 * v[m][1]; v[m][2] = 2 * v[m][2]; }
          }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) g[dir - 1][c] = (v[0][c] + v[1][c] + v[2][c] + v[3][c]) / 4;
      } else {
        const int other = 6 - d - dir;
        const int o0 = other == 1, o1 = other == 2, o2 = other == 3;
        const int64_t a0 = g2_idx(b, i, j, k), a1 = g2_idx(b, i + e0, j + e1, k + e2);
        const int64_t b0 = g2_idx(b, i + o0, j + o1, k + o2), b1 = g2_idx(b, i + o0 + e0, j + o1 + e1, k + o2 + e2);
        g[dir - 1][0] = ((x[a1] - x[a0]) + (x[b1] - x[b0])) / 2;
        g[dir - 1][1] = ((y[a1] - y[a0]) + (y[b1] - y[b0])) / 2;
        g[dir - 1][2] = ((z[a1] - z[a0]) + (z[b1] - z[b0])) / 2;
      }
    }
    const int di = d == 1, dj = d == 2, dk = d == 3;
    const double vv = (vol[p1_idx(b, 1, i - di, j - dj, k - dk, 0)] + vol[p1_idx(b, 1, i, j, k, 0)]) / 2;
    const double x_xi = g[0][0], y_xi = g[0][1], z_xi = g[0][2];
    const double x_eta = g[1][0], y_eta = g[1][1], z_eta = g[1][2];
    const double x_zeta = g[2][0], y_zeta = g[2][1], z_zeta = g[2][2];
    auto cof = [](double a, double b_, double c, double e) { return __dsub_rn(__dmul_rn(a, b_), __dmul_rn(c, e)); };
    double out[9];
    out[0] = cof(z_zeta, y_eta, z_eta, y_zeta) / vv;
    out[1] = cof(x_zeta, z_eta, x_eta, z_zeta) / vv;
    out[2] = cof(y_zeta, x_eta, y_eta, x_zeta) / vv;
    out[3] = cof(z_xi, y_zeta, z_zeta, y_xi) / vv;
    out[4] = cof(x_xi, z_zeta, x_zeta, z_xi) / vv;
    out[5] = cof(y_xi, x_zeta, y_zeta, x_xi) / vv;
    out[6] = cof(z_eta, y_xi, z_xi, y_eta) / vv;
    out[7] = cof(x_eta, z_xi, x_xi, z_eta) / vv;
    out[8] = cof(y_eta, x_xi, y_xi, x_eta) / vv;
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int c = 0; c < 3; ++c) vm[vm_idx(b, n0, d, m, c, i, j, k)] = out[m * 3 + c];
  }
}

// ---- face state and gradients ------------------------------------------------------
// primitive state of one block and snapshot: variable m at q[m*P3 + cell]
struct QView {
  const double *q;
  int64_t P3;
  int I3, J3;
  __device__ __forceinline__ double operator()(int i, int j, int k, int m) const {
    return q[m * P3 + (i + 1) + (int64_t)I3 * ((j + 1) + (int64_t)J3 * (k + 1))];
  }
};
__device__ __forceinline__ QView qview(const DevBlock &b, const double *q, int S, int n, int npde = 5) {
  QView v;
  v.q = q + p3_var(b, npde, S, 1, n);
  v.P3 = b.P3; v.I3 = b.I3; v.J3 = b.J3;
  return v;
}

// bq_face_* / bq_der_* bulk loops (src/flux.f90:1848-1880, 2029-2070, 2210-2250,
// 2432-2450): face (i,j,k) of family D between cells c-e_D and c
template <int D, int NV = 5>
__device__ __forceinline__ void face_interior(const QView &Q, int i, int j, int k, double qf[NV], double g[3][NV]) {
  constexpr int di = D == 1, dj = D == 2, dk = D == 3;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const double c = Q(i, j, k, m), cm = Q(i - di, j - dj, k - dk, m);
    qf[m] = (cm + c) / 2;
    g[D - 1][m] = c - cm;
#pragma unroll
    for (int t = 1; t <= 3; ++t) {
      if (t == D) continue;
      const int ti = t == 1, tj = t == 2, tk = t == 3;
      const double q2 = (cm + c + Q(i + ti, j + tj, k + tk, m) + Q(i - di + ti, j - dj + tj, k - dk + tk, m)) / 4;
      const double q1 = (Q(i - di - ti, j - dj - tj, k - dk - tk, m) + Q(i - ti, j - tj, k - tk, m) + c + cm) / 4;
      g[t - 1][m] = q2 - q1;
    }
  }
}

// the strong-boundary corrections (src/flux.f90:1896-1962 and the j, k
// counterparts; 2466-2488): face state = the halo (wall) value, three-point
// one-sided normal derivative, tangential derivatives along the halo line,
// one-sided at the ends of the patch
template <int NV = 5>
__device__ __forceinline__ void face_wall(const QView &Q, const WallFace &w, int mx, double qf[NV], double g[3][NV]) {
  const int d = w.d;
  const bool lo = w.inrout == 1;
  const int aux = lo ? 0 : mx, in1 = lo ? 1 : mx - 1, in2 = lo ? 2 : mx - 2;
  const double sgnm = lo ? 1.0 : -1.0;
  int pa[3] = {w.fi, w.fj, w.fk};
  int p1[3] = {w.fi, w.fj, w.fk};
  int p2[3] = {w.fi, w.fj, w.fk};
  pa[d - 1] = aux; p1[d - 1] = in1; p2[d - 1] = in2;
  const int fpos[3] = {w.fi, w.fj, w.fk};
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const double qa = Q(pa[0], pa[1], pa[2], m);
    qf[m] = qa;
    g[d - 1][m] = sgnm / 3 * (-qa * 8 + Q(p1[0], p1[1], p1[2], m) * 9 - Q(p2[0], p2[1], p2[2], m));
#pragma unroll
    for (int t = 1; t <= 3; ++t) {
      if (t == d) continue;
      const int ti = t == 1, tj = t == 2, tk = t == 3;
      const int pos = fpos[t - 1];
      double q2, q1;
      if (pos == w.lo[t - 1]) {
        const double qp = Q(pa[0] + ti, pa[1] + tj, pa[2] + tk, m);
        q2 = (qa + qp) / 2; q1 = (qa * 3 - qp) / 2;
      } else if (pos == w.hi[t - 1]) {
        const double qm = Q(pa[0] - ti, pa[1] - tj, pa[2] - tk, m);
        q2 = (qa * 3 - qm) / 2; q1 = (qa + qm) / 2;
      } else {
        const double qp = Q(pa[0] + ti, pa[1] + tj, pa[2] + tk, m);
        const double qm = Q(pa[0] - ti, pa[1] - tj, pa[2] - tk, m);
        q2 = (qa + qp) / 2; q1 = (qm + qa) / 2;
      }
      g[t - 1][m] = q2 - q1;
    }
  }
}

// ---- vflux_b, laminar branch (src/flux.f90:1073-1180) ------------------------------
struct ViscPar {
  double g, stemp, mr, pranl, prant;
};
__host__ __device__ __forceinline__ ViscPar make_visc(const cosa_params &P) {
  ViscPar v;
  v.g = P.gamma; v.stemp = P.stemp; v.mr = P.machfs / P.reyno; v.pranl = P.pranl; v.prant = P.prant;
  return v;
}
// Sutherland's law in the reference's non-dimensional form, t^1.5 = t sqrt(t)
__device__ __forceinline__ double sutherland(double t, double stemp) { return (stemp + 1) / (t + stemp) * (t * sqrt(t)); }

// viscous flux of one face: qf primitive face state, g[dir][var] the
// gradients along xi, eta, zeta, vmf[m*3+c] the face's inverse metrics,
// (kx, ky, kz, ds) the face normal and area; the energy row keeps the
// reference's (u txy + v tyy + w tyz) kz term
__device__ __forceinline__ void vflux_face(const ViscPar &V, const double qf[5], const double g[3][5],
                                           const double vmf[9], double kx, double ky, double kz, double ds, double mut,
                                           double F[5]) {
  const double rho = qf[0], u = qf[1], v = qf[2], w = qf[3], p = qf[4];
  const double t = V.g * p / rho;
  const double mu = sutherland(t, V.stemp);
  const double xix = vmf[0], xiy = vmf[1], xiz = vmf[2];
  const double etax = vmf[3], etay = vmf[4], etaz = vmf[5];
  const double zetax = vmf[6], zetay = vmf[7], zetaz = vmf[8];
  const double txi = t * (g[0][4] / p - g[0][0] / rho);
  const double teta = t * (g[1][4] / p - g[1][0] / rho);
  const double tzeta = t * (g[2][4] / p - g[2][0] / rho);
  const double dudx = g[0][1] * xix + g[1][1] * etax + g[2][1] * zetax;
  const double dudy = g[0][1] * xiy + g[1][1] * etay + g[2][1] * zetay;
  const double dudz = g[0][1] * xiz + g[1][1] * etaz + g[2][1] * zetaz;
  const double dvdx = g[0][2] * xix + g[1][2] * etax + g[2][2] * zetax;
  const double dvdy = g[0][2] * xiy + g[1][2] * etay + g[2][2] * zetay;
  const double dvdz = g[0][2] * xiz + g[1][2] * etaz + g[2][2] * zetaz;
  const double dwdx = g[0][3] * xix + g[1][3] * etax + g[2][3] * zetax;
  const double dwdy = g[0][3] * xiy + g[1][3] * etay + g[2][3] * zetay;
  const double dwdz = g[0][3] * xiz + g[1][3] * etaz + g[2][3] * zetaz;
  const double dtdx = txi * xix + teta * etax + tzeta * zetax;
  const double dtdy = txi * xiy + teta * etay + tzeta * zetay;
  const double dtdz = txi * xiz + teta * etaz + tzeta * zetaz;
  const double divv = dudx + dvdy + dwdz;
  const double txx = V.mr * 2 * mu * (dudx - divv / 3);
  const double txy = V.mr * mu * (dudy + dvdx);
  const double txz = V.mr * mu * (dudz + dwdx);
  const double tyy = V.mr * 2 * mu * (dvdy - divv / 3);
  const double tyz = V.mr * mu * (dvdz + dwdy);
  const double tzz = V.mr * 2 * mu * (dwdz - divv / 3);
  const double cq = V.mr * (mu / V.pranl + mut / V.prant) / (V.g - 1);
  const double qx = -(cq * dtdx), qy = -(cq * dtdy), qz = -(cq * dtdz);
  F[0] = 0.0;
  F[1] = -((txx * kx + txy * ky + txz * kz) * ds);
  F[2] = -((txy * kx + tyy * ky + tyz * kz) * ds);
  F[3] = -((txz * kx + tyz * ky + tzz * kz) * ds);
  F[4] = -(((u * txx + v * txy + w * txz) * kx + (u * txy + v * tyy + w * tyz) * ky + (u * txy + v * tyy + w * tyz) * kz) *
           ds) + (qx * kx + qy * ky + qz * kz) * ds;
}

__device__ __forceinline__ void load_vm(const double *__restrict__ vm, const DevBlock &b, int64_t n0, int d, int i,
                                        int j, int k, double vmf[9]) {
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) vmf[m * 3 + c] = vm[vm_idx(b, n0, d, m, c, i, j, k)];
}

// ---- per-stage kernels of the fused viscous path -------------------------------------
// primitive copy of a stage state (interior conservative, halos primitive)
__global__ void k_prim(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                       const double *__restrict__ q, double *__restrict__ qp, int *status = nullptr) {
  int st = 0;
  const DevBlock b = blocks[blockIdx.y];
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1;
  const int64_t total = b.P3 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t % b.P3;
    const int n = (int)(t / b.P3);
    const int i = (int)(c % b.I3) - 1, j = (int)((c / b.I3) % b.J3) - 1, k = (int)(c / ((int64_t)b.I3 * b.J3)) - 1;
    const int64_t base = p3_var(b, 5, S, 1, n) + c;
    double v[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) v[m] = q[base + m * b.P3];
    if (i >= 1 && i <= b.im - 1 && j >= 1 && j <= b.jm - 1 && k >= 1 && k <= b.km - 1) {
      c2p5_nr(P.gamma, v);
      // bprtest on the interior (src/cosa.f90:1000-1040)
      if (v[4] <= P.qmin[4]) st |= COSA_ERR_NEG_P;
      else if (v[0] <= P.qmin[0]) st |= COSA_ERR_NEG_RHO;
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) qp[base + m * b.P3] = v[m];
  }
  if (st && status) atomicOr(status, st);
}

// viscous flux of every face: grid (x, nblocks, 3 families)
template <int D>
__device__ __forceinline__ void vface_one(const DevBlock &b, const ViscPar &V, const QView &Q,
                                          const double *__restrict__ s, int S2, const double *__restrict__ vm,
                                          int64_t n0, int i, int j, int k, int nh, double *__restrict__ F) {
  double qf[5], g[3][5], vmf[9], F5[5];
  face_interior<D>(Q, i, j, k, qf, g);
  load_vm(vm + (int64_t)nh * 27 * n0, b, n0, D, i, j, k, vmf);  // inverse metrics of node snapshot nh
  const int64_t e = p2_idx(b, S2, 1, i, j, k, nh);
  const double2 a = __ldg(reinterpret_cast<const double2 *>(s + e));
  const double2 c = __ldg(reinterpret_cast<const double2 *>(s + e + 2));
  vflux_face(V, qf, g, vmf, a.x, a.y, c.x, c.y, 0.0, F5);
#pragma unroll
  for (int m = 0; m < 5; ++m) F[m] = F5[m];
}

__global__ void k_vface(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                        const double *__restrict__ qp, const double *__restrict__ si, const double *__restrict__ sj,
                        const double *__restrict__ sk, const double *__restrict__ vm, int64_t n0,
                        double *__restrict__ fv) {
  const DevBlock b = blocks[blockIdx.y];
  const int d = blockIdx.z + 1;
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const ViscPar V = make_visc(P);
  const int ni = d == 1 ? b.im : b.im - 1, nj = d == 2 ? b.jm : b.jm - 1, nk = d == 3 ? b.km : b.km - 1;
  const int64_t nf = (int64_t)ni * nj * nk, total = nf * S;
  const double *s = d == 1 ? si : (d == 2 ? sj : sk);
  double *F = fv + (int64_t)(d - 1) * n0 * 5 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk), nh = n * P.hbmove;
    const QView Q = qview(b, qp, S, n);
    double out[5];
    if (d == 1) vface_one<1>(b, V, Q, s, S2, vm, n0, i, j, k, nh, out);
    else if (d == 2) vface_one<2>(b, V, Q, s, S2, vm, n0, i, j, k, nh, out);
    else vface_one<3>(b, V, Q, s, S2, vm, n0, i, j, k, nh, out);
#pragma unroll
    for (int m = 0; m < 5; ++m) F[f0_idx(b, 5, S, i, j, k, m + 1, n)] = out[m];
  }
}

// strong-boundary faces (overwrite k_vface's values there)
__global__ void k_vwall(const DevBlock *__restrict__ blocks, const WallFace *__restrict__ walls, int nw,
                        const cosa_params *__restrict__ Pp, const double *__restrict__ qp,
                        const double *__restrict__ si, const double *__restrict__ sj, const double *__restrict__ sk,
                        const double *__restrict__ vm, int64_t n0, double *__restrict__ fv) {
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const ViscPar V = make_visc(P);
  const int64_t total = (int64_t)nw * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const WallFace w = walls[t % nw];
    const int n = (int)(t / nw), nh = n * P.hbmove;
    const DevBlock b = blocks[w.blk];
    const QView Q = qview(b, qp, S, n);
    const int mx = w.d == 1 ? b.im : (w.d == 2 ? b.jm : b.km);
    double qf[5], g[3][5], vmf[9], F[5];
    face_wall(Q, w, mx, qf, g);
    load_vm(vm + (int64_t)nh * 27 * n0, b, n0, w.d, w.fi, w.fj, w.fk, vmf);
    const double *s = w.d == 1 ? si : (w.d == 2 ? sj : sk);
    const int64_t e = p2_idx(b, S2, 1, w.fi, w.fj, w.fk, nh);
    vflux_face(V, qf, g, vmf, s[e], s[e + 1], s[e + 2], s[e + 3], 0.0, F);
    double *Fd = fv + (int64_t)(w.d - 1) * n0 * 5 * S;
#pragma unroll
    for (int m = 0; m < 5; ++m) Fd[f0_idx(b, 5, S, w.fi, w.fj, w.fk, m + 1, n)] = F[m];
  }
}

// flux balance of each cell, summed like bresid (src/cosa.f90:1149-1200)
__global__ void k_vdiv(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                       const double *__restrict__ fv, int64_t n0, double *__restrict__ vres) {
  const DevBlock b = blocks[blockIdx.y];
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  const double *Fi = fv, *Fj = fv + n0 * 5 * S, *Fk = fv + 2 * n0 * 5 * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const int64_t cell = p3_cell(b, i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double x = Fi[f0_idx(b, 5, S, i + 1, j, k, m + 1, n)] - Fi[f0_idx(b, 5, S, i, j, k, m + 1, n)];
      x = x + Fj[f0_idx(b, 5, S, i, j + 1, k, m + 1, n)] - Fj[f0_idx(b, 5, S, i, j, k, m + 1, n)];
      x = x + Fk[f0_idx(b, 5, S, i, j, k + 1, m + 1, n)] - Fk[f0_idx(b, 5, S, i, j, k, m + 1, n)];
      vres[p3_var(b, 5, S, m + 1, n) + cell] = x;
    }
  }
}

// ---- lambdab viscous branch + eig_ns + bdeltat (src/cosa.f90:1349-1423,
// 4239-4297, 4831-5010) ---------------------------------------------------------------
// convective and viscous spectral radii of cell (i,j,k); the + neighbour's
// temperature uses the - neighbour's density, as the reference does
__device__ __forceinline__ void eig_ns_cell(const DevBlock &b, const cosa_params &P, const QView &Q,
                                            const double *__restrict__ si, const double *__restrict__ sj,
                                            const double *__restrict__ sk, int S2, int nh, double volc, int i, int j,
                                            int k, double lam[3], double lamv[3], const double *mut = nullptr,
                                            int S = 1, int n = 0, double lsp_cut = -1.0, double lsp_eps2 = 0.0,
                                            const double *gv = nullptr) {
  const double g = P.gamma, st = P.stemp;
  double qc[5], sm[3][4], sp[3][4];
#pragma unroll
  for (int m = 0; m < 5; ++m) qc[m] = Q(i, j, k, m);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    sm[0][m] = si[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[0][m] = si[p2_idx(b, S2, m + 1, i + 1, j, k, nh)];
    sm[1][m] = sj[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[1][m] = sj[p2_idx(b, S2, m + 1, i, j + 1, k, nh)];
    sm[2][m] = sk[p2_idx(b, S2, m + 1, i, j, k, nh)]; sp[2][m] = sk[p2_idx(b, S2, m + 1, i, j, k + 1, nh)];
  }
  if (lsp_cut >= 0)  // eig_ns_p: the preconditioned convective radii (src/cosa.f90:4374-4460)
    eig_eul_p(g, P.uprv, lsp_eps2, lsp_cut, qc, sm[0], sp[0], sm[1], sp[1], sm[2], sp[2], lam[0], lam[1], lam[2]);
  else
    eig_eul(g, qc, sm[0], sp[0], sm[1], sp[1], sm[2], sp[2], lam[0], lam[1], lam[2], gv);
  const double rho = qc[0];
  const double mu = sutherland(g * qc[4] / rho, st);
  auto MUT = [&](int a, int c, int e) { return mut ? mut[b.op3 * S + (int64_t)n * b.P3 + p3_cell(b, a, c, e)] : 0.0; };
  const double mutc = MUT(i, j, k);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int a = d == 0, c = d == 1, e = d == 2;
    const double rhom = Q(i - a, j - c, k - e, 0);
    const double tm = g * Q(i - a, j - c, k - e, 4) / rhom;
    const double tp = g * Q(i + a, j + c, k + e, 4) / rhom;
    const double mum = sutherland(tm, st), mup = sutherland(tp, st);
    const double mud = (mum + 2 * mu + mup) / 4;
    const double mutd = (MUT(i - a, j - c, k - e) + 2 * mutc + MUT(i + a, j + c, k + e)) / 4;
    const double area = (sm[d][3] + sp[d][3]) / 2;
    lamv[d] = P.cdff * area * area * g * P.machfs / P.reyno * (mud / P.pranl + mutd / P.prant) / (rho * volc);
  }
}

// IRS coefficients of bdeltat for ratio rat (rat: mean flow, ratt: k-omega),
// with the viscous floor c1/4 lamv / sum(lam) for irsop 5 and 6
__device__ __forceinline__ void irs_coef_ns(int irsop, double rat, double psirs, const double lam[3],
                                            const double lamv[3], double &bx, double &by, double &bz) {
  const double c1 = 40.0;
  bx = by = bz = 0.0;
  if (irsop < 2 || irsop == 4) return;
  irs_beta(irsop, rat, psirs, lam[0], lam[1], lam[2], bx, by, bz);
  const double sl = lam[0] + lam[1] + lam[2];
  if (irsop == 5) {
    bx = fmax(bx, c1 / 4 * lamv[0] / sl); by = fmax(by, c1 / 4 * lamv[1] / sl); bz = fmax(bz, c1 / 4 * lamv[2] / sl);
  } else if (irsop == 6) {
    bx = fmax(bx, 0.25 * c1 * lamv[0] / sl); by = fmax(by, 0.25 * c1 * lamv[1] / sl);
    bz = fmax(bz, 0.25 * c1 * lamv[2] / sl);
  }
}

__device__ __forceinline__ void deltat_ns_cell(const cosa_params &P, const double lam[3], const double lamv[3],
                                               double &dt, double &bx, double &by, double &bz) {
  if (P.irsop == 5 || P.irsop == 6) dt = P.cfl / (lam[0] + lam[1] + lam[2]);
  else dt = P.cfl / (lam[0] + lam[1] + lam[2] + lamv[0] + lamv[1] + lamv[2]);
  irs_coef_ns(P.irsop, P.rat, P.psirs, lam, lamv, bx, by, bz);
}

// time step (and IRS coefficients) of the fused viscous path, from the
// primitive stage copy
__global__ void k_dt_ns(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                        const double *__restrict__ qp, const double *__restrict__ si, const double *__restrict__ sj,
                        const double *__restrict__ sk, const double *__restrict__ vol, double *__restrict__ dtv,
                        double *bx, double *by, double *bz, const double *__restrict__ cvx = nullptr,
                        const double *__restrict__ cvy = nullptr, const double *__restrict__ cvz = nullptr) {
  // cv*: the cell grid velocities of a moving grid (node layout, per snapshot)
  const DevBlock b = blocks[blockIdx.y];
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk), nh = n * P.hbmove;
    const QView Q = qview(b, qp, S, n);
    double lam[3], lamv[3], gv[3];
    if (cvx) {
      const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
      const int64_t gi = b.op2 * S2 + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k);
      gv[0] = cvx[gi]; gv[1] = cvy[gi]; gv[2] = cvz[gi];
    }
    eig_ns_cell(b, P, Q, si, sj, sk, S2, nh, vol[p1_idx(b, 1, i, j, k, 0)], i, j, k, lam, lamv, nullptr, 1, 0, -1.0,
                0.0, cvx ? gv : nullptr);
    double dt, a, c, e;
    deltat_ns_cell(P, lam, lamv, dt, a, c, e);
    const int64_t o = p1_idx(b, S, i, j, k, n);
    dtv[o] = dt;
    if (bx) { bx[o] = a; by[o] = c; bz[o] = e; }
  }
}

// ---- per-routine kernels (reference array contract) ----------------------------------
// lambda with viscous = .true.: lam(.,1:3) convective, lamv(.,1:3) viscous
template <class BS>
__global__ void k_lambda_ns(BS bs_, const cosa_params *__restrict__ Pp, const double *__restrict__ q,
                            const double *__restrict__ si, const double *__restrict__ sj,
                            const double *__restrict__ sk, const double *__restrict__ vol,
                            const double *__restrict__ mut, double *__restrict__ lam, double *__restrict__ lamv,
                            const double *__restrict__ cpg = nullptr, const double *__restrict__ cvs = nullptr,
                            int nl = 1, const double *__restrict__ cvx = nullptr,
                            const double *__restrict__ cvy = nullptr, const double *__restrict__ cvz = nullptr) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk), nh = n * P.hbmove;
    const QView Q = qview(b, q, S, n, npde);
    double l[3], lv[3];
    double cut = -1.0;
    if (cpg) {
      const int64_t m = b.om1 * S + (int64_t)n * ni * nj * nk + (i - 1) + (int64_t)ni * ((j - 1) + (int64_t)nj * (k - 1));
      cut = fmax(cpg[m], cvs[m]);
    }
    double gv[3];
    if (cvx) {
      // cell grid velocity of a moving grid (node-array layout, snapshot nh)
      const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
      const int64_t gi = b.op2 * S2 + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k);
      gv[0] = cvx[gi]; gv[1] = cvy[gi]; gv[2] = cvz[gi];
    }
    eig_ns_cell(b, P, Q, si, sj, sk, S2, nh, vol[p1_idx(b, 1, i, j, k, 0)], i, j, k, l, lv, mut, S, n, cut,
                P.epsp[nl - 1] * P.epsp[nl - 1], cvx ? gv : nullptr);
    const int64_t c = p3_cell(b, i, j, k);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      lam[p3_var(b, npde, S, m + 1, n) + c] = l[m];
      lamv[p3_var(b, npde, S, m + 1, n) + c] = lv[m];
    }
  }
}

template <class BS>
__global__ void k_deltat_ns(BS bs_, const cosa_params *__restrict__ Pp, double *__restrict__ dtv,
                            const double *__restrict__ lam, const double *__restrict__ lamv, double *bx, double *by,
                            double *bz, double *dtt, double *tbx, double *tby, double *tbz) {
  const DevBlock b = bs_.get();
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const int64_t c = p3_cell(b, i, j, k);
    double l[3], lv[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      l[m] = lam[p3_var(b, npde, S, m + 1, n) + c];
      lv[m] = lamv[p3_var(b, npde, S, m + 1, n) + c];
    }
    double dt, a, e, f;
    deltat_ns_cell(P, l, lv, dt, a, e, f);
    const int64_t o = p1_idx(b, S, i, j, k, n);
    dtv[o] = dt;
    if (bx && P.irsop >= 2 && P.irsop != 4) { bx[o] = a; by[o] = e; bz[o] = f; }
    // k-omega: dtvolt = cflt/cfl dtvol and the turbulence coefficients with ratt
    if (dtt) dtt[o] = P.cflt / P.cfl * dt;
    if (tbx && P.irsop >= 2 && P.irsop != 4) {
      irs_coef_ns(P.irsop, P.ratt, P.psirs, l, lv, a, e, f);
      tbx[o] = a; tby[o] = e; tbz[o] = f;
    }
  }
}

// q_face / q_der bulk loops with the reference's P3 outputs
template <int D, int NV, class BS>
__global__ void k_qface_qder(BS bs_, int S, const double *__restrict__ q, double *__restrict__ qf,
                             double *__restrict__ g0, double *__restrict__ g1, double *__restrict__ g2) {
  const DevBlock b = bs_.get();
  const int ni = D == 1 ? b.im : b.im - 1, nj = D == 2 ? b.jm : b.jm - 1, nk = D == 3 ? b.km : b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const QView Q = qview(b, q, S, n, NV);
    double f[NV], g[3][NV];
    face_interior<D, NV>(Q, i, j, k, f, g);
    const int64_t c = p3_cell(b, i, j, k);
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const int64_t o = p3_var(b, NV, S, m + 1, n) + c;
      if (qf) qf[o] = f[m];
      if (g0) { g0[o] = g[0][m]; g1[o] = g[1][m]; g2[o] = g[2][m]; }
    }
  }
}

template <int NV>
__global__ void k_qwall(const DevBlock *__restrict__ blocks, const WallFace *__restrict__ walls, int nw, int d, int S,
                        const double *__restrict__ q, double *__restrict__ qf, double *__restrict__ g0,
                        double *__restrict__ g1, double *__restrict__ g2) {
  const int64_t total = (int64_t)nw * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const WallFace w = walls[t % nw];
    if (w.d != d) continue;
    const int n = (int)(t / nw);
    const DevBlock b = blocks[w.blk];
    const QView Q = qview(b, q, S, n, NV);
    const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
    double f[NV], g[3][NV];
    face_wall<NV>(Q, w, mx, f, g);
    const int64_t c = p3_cell(b, w.fi, w.fj, w.fk);
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const int64_t o = p3_var(b, NV, S, m + 1, n) + c;
      if (qf) qf[o] = f[m];
      if (g0) { g0[o] = g[0][m]; g1[o] = g[1][m]; g2[o] = g[2][m]; }
    }
  }
}

// vflux with the reference's arrays (qf, dq* in P3, flux in F0)
__global__ void k_vflux_ref(DevBlock b, int d, const cosa_params *__restrict__ Pp, const double *__restrict__ qf,
                            const double *__restrict__ g0, const double *__restrict__ g1,
                            const double *__restrict__ g2, const double *__restrict__ vm, int64_t n0,
                            const double *__restrict__ s, double *__restrict__ flux) {
  const cosa_params &P = *Pp;
  const int S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const ViscPar V = make_visc(P);
  const int ni = d == 1 ? b.im : b.im - 1, nj = d == 2 ? b.jm : b.jm - 1, nk = d == 3 ? b.km : b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk), nh = n * P.hbmove;
    const int64_t c = p3_cell(b, i, j, k);
    double f[5], g[3][5], vmf[9], F[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const int64_t o = p3_var(b, 5, S, m + 1, n) + c;
      f[m] = qf[o]; g[0][m] = g0[o]; g[1][m] = g1[o]; g[2][m] = g2[o];
    }
    load_vm(vm + (int64_t)nh * 27 * n0, b, n0, d, i, j, k, vmf);
    const int64_t e = p2_idx(b, S2, 1, i, j, k, nh);
    vflux_face(V, f, g, vmf, s[e], s[e + 1], s[e + 2], s[e + 3], 0.0, F);
#pragma unroll
    for (int m = 0; m < 5; ++m) flux[f0_idx(b, 5, S, i, j, k, m + 1, n)] = F[m];
  }
}
