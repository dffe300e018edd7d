// Pointwise physics of COSA's explicit residual path as device functions.
//
// Every function restates a Fortran routine (cited) with the same operation
// order and parenthesisation, so an FP64 build differs from the reference
// only by FMA contraction.  The variants used by the fused stage kernel
// (limit_face_nr, roe_flux_euler, c2p5_nr) take the reciprocals and
// reciprocal square roots on their dependency chains from rcp_nr / rsqrt_nr
// below: results differ from the IEEE division and square root by at most a
// couple of ulp, far inside the parity bound, and each chain gets shorter.
// The MIXED variants keep the FP64 state and take the slopes and the Roe
// dissipation in FP32 on FP64 differences.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

struct PhysPar {
  double g, gm1, g_gm1;       // gamma, gamma-1, gamma/(gamma-1)
  double rkap, epslimf, epslimt;
  int ilimf, ilimt;
  int efx_setup_f, efx_all_f, eig_limit_f, eig_lim_all_f;
  double cntrpy_f, entfxctf_f, eig_cutoff_f;
  double w1, w2, w3;          // entfx_f_w(1:3) as reals
};

__host__ __device__ __forceinline__ PhysPar make_phys(const cosa_params &P) {
  PhysPar q;
  q.g = P.gamma; q.gm1 = P.gamma - 1; q.g_gm1 = P.gamma / (P.gamma - 1);
  q.rkap = P.rkap; q.epslimf = P.epslimf; q.epslimt = P.epslimt;
  q.ilimf = P.ilimf; q.ilimt = P.ilimt;
  q.efx_setup_f = P.efx_setup_f; q.efx_all_f = P.efx_all_f;
  q.eig_limit_f = P.eig_limit_f; q.eig_lim_all_f = P.eig_lim_all_f;
  q.cntrpy_f = P.cntrpy_f; q.entfxctf_f = P.entfxctf_f; q.eig_cutoff_f = P.eig_cutoff_f;
  q.w1 = P.entfx_f_w[0]; q.w2 = P.entfx_f_w[1]; q.w3 = P.entfx_f_w[2];
  return q;
}

// ---- Newton-Raphson reciprocal and reciprocal square root -------------------------
// Seeds from the PTX approximations rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64
// (relative error around 2^-22), then two Newton-Raphson steps each:
//   1/x:        r <- r + r (1 - x r)              (error e -> e^2)
//   1/sqrt(x):  y <- y (3/2 - (x/2) y^2)          (error e -> 3 e^2 / 2)
// which leaves only the rounding of the last operations (a few ulp at most).
// Inputs are positive normal numbers here (densities, speeds of sound squared,
// sums of squares plus a positive epsilon); no zero, denormal or infinity
// handling is needed or done.
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double h = 0.5 * x;
  y = y * fma(-h * y, y, 1.5);
  return y * fma(-h * y, y, 1.5);
}

// ---- cons2prim_b / prim2cons_b cell formulas (src/update.f90:2135-2188, 1875-2084)
// q[0..4] = (rho, rho u, rho v, rho w, rho E) -> (rho, u, v, w, p); Euler
__device__ __forceinline__ void c2p5(double g, double *q) {
  const double rho = q[0];
  const double u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
  q[1] = u; q[2] = v; q[3] = w;
  q[4] = (g - 1) * (q[4] - rho * (u * u + v * v + w * w) / 2);
}
// c2p5 with one reciprocal of rho (fused stage kernels); every rounding is
// pinned with explicit intrinsics, so the result does not depend on how the
// compiler contracts it in each kernel that inlines it
__device__ __forceinline__ void c2p5_nr(double g, double *q) {
  const double rho = q[0], ri = rcp_nr(rho);
  const double u = __dmul_rn(q[1], ri), v = __dmul_rn(q[2], ri), w = __dmul_rn(q[3], ri);
  q[1] = u; q[2] = v; q[3] = w;
  const double q2 = __fma_rn(w, w, __fma_rn(v, v, __dmul_rn(u, u)));
  q[4] = __dmul_rn(g - 1, __fma_rn(-__dmul_rn(rho, q2), 0.5, q[4]));
}
// with k-omega: q[5] = rho k, q[6] = rho omega (divided by rho as well)
__device__ __forceinline__ void c2p7(double g, double *q) {
  const double rho = q[0];
  const double u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
  const double tke = q[5] / rho;
  q[1] = u; q[2] = v; q[3] = w; q[5] = tke; q[6] = q[6] / rho;
  q[4] = (g - 1) * (q[4] - rho * (u * u + v * v + w * w) / 2 - rho * tke);
}
__device__ __forceinline__ void p2c(double g, double *q, int npde) {
  const double tke = npde > 5 ? q[5] : 0.0;
  const double rho = q[0];
  for (int v = 1; v < npde; ++v)
    if (v != 4) q[v] = q[v] * rho;
  const double ru = q[1], rv = q[2], rw = q[3], p = q[4];
  double e = p / (g - 1) + (ru * ru + rv * rv + rw * rw) / 2 / rho;
  if (npde > 5) e = e + rho * tke;
  q[4] = e;
}

// ---- limiters limit_i/j/k (src/flux.f90:3472-3888) -----------------------------
// For face f of a line: dlo = dq(f-1), dmid = dq(f), dhi = dq(f+1).
// dqp(f) depends on (dq(f), dq(f+1)), dqm(f) on (dq(f-1), dq(f)).
template <typename T>
__device__ __forceinline__ void limit_face(int ilim, T eps, T rkap, T dlo, T dmid, T dhi, T &dqp, T &dqm) {
  if (ilim == 1) {
    T s = (2 * dhi * dmid + eps) / (dhi * dhi + dmid * dmid + eps);
    T rkp = 1 + rkap * s, rkm = 1 - rkap * s;
    dqp = -s * (rkp * dmid + rkm * dhi) / 4;
    s = (2 * dmid * dlo + eps) / (dmid * dmid + dlo * dlo + eps);
    rkp = 1 + rkap * s; rkm = 1 - rkap * s;
    dqm = s * (rkm * dlo + rkp * dmid) / 4;
  } else if (ilim == 0) {
    const T rkp = 1 + rkap, rkm = 1 - rkap;
    dqp = -(rkp * dmid + rkm * dhi) / 4;
    dqm = (rkm * dlo + rkp * dmid) / 4;
  } else if (ilim == 2) {
    const T rkp = 1 + rkap, rkm = 1 - rkap;
    const T bb = (T(3) - rkap) / (T(1) - rkap);
    // pair (d0,d1) = (dq(f), dq(f+1)) gives dqp(f)
    T d0 = dmid, d1 = dhi;
    T dqmx = (copysign(T(1), d0) + copysign(T(1), d1)) / 2 * fmin(fabs(d0), fabs(d1) * bb);
    T dqpx = (copysign(T(1), d1) + copysign(T(1), d0)) / 2 * fmin(fabs(d1), fabs(d0) * bb);
    dqp = -(rkp * dqmx + rkm * dqpx) / 4;
    // pair (dq(f-1), dq(f)) gives dqm(f)
    d0 = dlo; d1 = dmid;
    dqmx = (copysign(T(1), d0) + copysign(T(1), d1)) / 2 * fmin(fabs(d0), fabs(d1) * bb);
    dqpx = (copysign(T(1), d1) + copysign(T(1), d0)) / 2 * fmin(fabs(d1), fabs(d0) * bb);
    dqm = (rkm * dqmx + rkp * dqpx) / 4;
  } else if (ilim == 3) {
    const T epsq = eps * eps;
    T d1 = dhi, d2 = dmid;
    T dqpx = (d2 * (d1 * d1 + 2 * epsq) + d1 * (2 * (d2 * d2) + epsq)) /
             (2 * (d2 * d2) - d2 * d1 + 2 * (d1 * d1) + 3 * epsq);
    dqp = -dqpx / 2;
    d1 = dmid; d2 = dlo;
    T dqmx = (d1 * (d2 * d2 + 2 * epsq) + d2 * (2 * (d1 * d1) + epsq)) /
             (2 * (d1 * d1) - d1 * d2 + 2 * (d2 * d2) + 3 * epsq);
    dqm = dqmx / 2;
  } else {  // ilim == 4
    const T epsq = eps * eps;
    T d1 = dhi, d2 = dmid;
    T dqpx = (d1 * (d2 * d2 + epsq) + d2 * (d1 * d1 + epsq)) / (d1 * d1 + d2 * d2 + 2 * epsq);
    dqp = -dqpx / 2;
    d1 = dmid; d2 = dlo;
    T dqmx = (d1 * (d2 * d2 + epsq) + d2 * (d1 * d1 + epsq)) / (d1 * d1 + d2 * d2 + 2 * epsq);
    dqm = dqmx / 2;
  }
}

// The limiter of one cell from its two slopes a = dq(c), b = dq(c+1):
// dqp(c), the offset to its lower face (limit_face's dqp with dmid = a,
// dhi = b), and dqm(c+1), the offset to its upper face (limit_face's dqm with
// dlo = a, dmid = b), in FP64 for the fused stage kernels.  The sensor's
// division is a Newton-Raphson reciprocal; every rounding is pinned with
// explicit intrinsics (fixed contraction), so the tile kernel (two cells per
// face) and the line-marching face kernel (one cell at a time) give the same
// bits.  ilim 1, 2 and 4 share their sensor between dqp and dqm, as the
// reference's two expressions coincide (src/flux.f90:3561-3604).
__device__ __forceinline__ double lim3_nr(double x, double y, double epsq) {
  // (x (y^2 + 2 e) + y (2 x^2 + e)) / (2 x^2 - x y + 2 y^2 + 3 e), limit_i ilim 3
  const double xx = __dmul_rn(x, x), yy = __dmul_rn(y, y);
  const double num = __fma_rn(y, __fma_rn(2.0, xx, epsq), __dmul_rn(x, __fma_rn(2.0, epsq, yy)));
  const double den = __fma_rn(3.0, epsq, __fma_rn(2.0, yy, __fma_rn(-x, y, __dmul_rn(2.0, xx))));
  return __ddiv_rn(num, den);
}
__device__ __forceinline__ void limit_cell64(int ilim, double eps, double rkap, double a, double b, double &dqp,
                                             double &dqm) {
  if (ilim == 1) {
    const double num = __fma_rn(__dmul_rn(2.0, b), a, eps);
    const double den = __dadd_rn(__fma_rn(b, b, __dmul_rn(a, a)), eps);
    const double s = __dmul_rn(num, rcp_nr(den));
    const double rkp = __fma_rn(rkap, s, 1.0), rkm = __fma_rn(-rkap, s, 1.0);
    dqp = __dmul_rn(__dmul_rn(-s, __fma_rn(rkp, a, __dmul_rn(rkm, b))), 0.25);
    dqm = __dmul_rn(__dmul_rn(s, __fma_rn(rkm, a, __dmul_rn(rkp, b))), 0.25);
  } else if (ilim == 0) {
    const double rkp = 1 + rkap, rkm = 1 - rkap;
    dqp = __dmul_rn(-__fma_rn(rkp, a, __dmul_rn(rkm, b)), 0.25);
    dqm = __dmul_rn(__fma_rn(rkm, a, __dmul_rn(rkp, b)), 0.25);
  } else if (ilim == 2) {
    const double rkp = 1 + rkap, rkm = 1 - rkap;
    const double bb = (3.0 - rkap) / (1.0 - rkap);
    const double sg = (copysign(1.0, a) + copysign(1.0, b)) * 0.5;  // -1, 0 or 1: exact
    const double dqmx = sg * fmin(fabs(a), __dmul_rn(fabs(b), bb));
    const double dqpx = sg * fmin(fabs(b), __dmul_rn(fabs(a), bb));
    dqp = __dmul_rn(-__fma_rn(rkp, dqmx, __dmul_rn(rkm, dqpx)), 0.25);
    dqm = __dmul_rn(__fma_rn(rkm, dqmx, __dmul_rn(rkp, dqpx)), 0.25);
  } else if (ilim == 3) {
    const double epsq = __dmul_rn(eps, eps);
    dqp = -0.5 * lim3_nr(a, b, epsq);
    dqm = 0.5 * lim3_nr(b, a, epsq);
  } else {  // ilim == 4
    const double epsq = __dmul_rn(eps, eps);
    const double num = __fma_rn(a, __fma_rn(b, b, epsq), __dmul_rn(b, __fma_rn(a, a, epsq)));
    const double den = __fma_rn(2.0, epsq, __fma_rn(a, a, __dmul_rn(b, b)));
    const double x = __ddiv_rn(num, den);
    dqp = -0.5 * x;
    dqm = 0.5 * x;
  }
}

// limit_face on the fused stage kernels' arithmetic: the two cells' halves
// of limit_cell64 (dqp from cell f, dqm from cell f-1)
__device__ __forceinline__ void limit_face_nr(int ilim, double eps, double rkap, double dlo, double dmid, double dhi,
                                              double &dqp, double &dqm) {
  double unused;
  limit_cell64(ilim, eps, rkap, dmid, dhi, dqp, unused);
  limit_cell64(ilim, eps, rkap, dlo, dmid, unused, dqm);
}

// FP32 limiter of the mixed path: limit_face's algebra with fast division
__device__ __forceinline__ void limit_face_fast(int ilim, float eps, float rkap, float dlo, float dmid, float dhi,
                                                float &dqp, float &dqm) {
  if (ilim == 1) {
    float s = __fdividef(2.0f * dhi * dmid + eps, dhi * dhi + dmid * dmid + eps);
    dqp = -s * ((1.0f + rkap * s) * dmid + (1.0f - rkap * s) * dhi) * 0.25f;
    s = __fdividef(2.0f * dmid * dlo + eps, dmid * dmid + dlo * dlo + eps);
    dqm = s * ((1.0f - rkap * s) * dlo + (1.0f + rkap * s) * dmid) * 0.25f;
  } else {
    limit_face<float>(ilim, eps, rkap, dlo, dmid, dhi, dqp, dqm);
  }
}

// ---- roflux_b mean-flow face flux (src/flux.f90:45-238), fixed grid ---------------
// qr/ql: primitive right/left states (rho,u,v,w,p); tker/tkel: TKE (0 for Euler)
// ubn: the face's normal grid speed on moving grids (src/flux.f90:110-113)
__device__ __forceinline__ void roe_flux_fp64(const PhysPar &P, double kx, double ky, double kz, double ds,
                                              const double *qr, const double *ql, double tker, double tkel,
                                              double *flux, double ubn = 0.0) {
  const double g = P.g;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
  const double unr = ur * kx + vr * ky + wr * kz - ubn;
  const double q2r = ur * ur + vr * vr + wr * wr;
  const double h0r = g / (g - 1) * pr / rhor + q2r / 2 + tker;
  const double rh0r = rhor * h0r;
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
  const double unl = ul * kx + vl * ky + wl * kz - ubn;
  const double q2l = ul * ul + vl * vl + wl * wl;
  const double h0l = g / (g - 1) * pl / rhol + q2l / 2 + tkel;
  const double rh0l = rhol * h0l;
  const double drho = rhor - rhol, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl;
  const double dun = unr - unl, dtke = tker - tkel;
  const double rhols = sqrt(rhol), rhors = sqrt(rhor);
  const double rho = rhols * rhors, denom = rhols + rhors;
  const double u = (rhols * ul + rhors * ur) / denom;
  const double v = (rhols * vl + rhors * vr) / denom;
  const double w = (rhols * wl + rhors * wr) / denom;
  const double un = u * kx + v * ky + w * kz;
  const double h0 = (rhols * h0l + rhors * h0r) / denom;
  const double tke = (rhols * tkel + rhors * tker) / denom;
  const double q2 = u * u + v * v + w * w;
  const double a2 = (g - 1) * (h0 - q2 / 2 - tke);
  const double a = sqrt(a2);
  double rm123 = fabs(un - ubn), rm4 = fabs(un + a - ubn), rm5 = fabs(un - a - ubn);
  if (P.efx_setup_f) {
    double rdelta = P.cntrpy_f * (P.w1 * P.entfxctf_f + P.w2 * (sqrt(u * u + v * v + w * w) + a) +
                                  P.w3 * 0.2 * (fabs(un) + a + fabs(ubn)));
    rdelta = fmax(rdelta, 1.0e-12);
    if (rm123 <= rdelta && P.efx_all_f) rm123 = 0.5 * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5 * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5 * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_f) {
    if (rm123 <= P.eig_cutoff_f) rm123 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm4 <= P.eig_cutoff_f) rm4 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm5 <= P.eig_cutoff_f) rm5 = P.eig_cutoff_f;
  }
  const double dpa2 = dp / a2, rdua = rho * dun / a;
  const double al1 = rm123 * (drho - dpa2);
  const double al2 = rm123 * rho;
  const double al3 = rm4 * (dpa2 + rdua) / 2;
  const double al4 = rm5 * (dpa2 - rdua) / 2;
  const double df1 = al1 + al3 + al4;
  const double df2 = al1 * u + al2 * (du - dun * kx) + al3 * (u + a * kx) + al4 * (u - a * kx);
  const double df3 = al1 * v + al2 * (dv - dun * ky) + al3 * (v + a * ky) + al4 * (v - a * ky);
  const double df4 = al1 * w + al2 * (dw - dun * kz) + al3 * (w + a * kz) + al4 * (w - a * kz);
  const double df5 = al1 * (q2 / 2 + tke) + al2 * (u * du + v * dv + w * dw - un * dun + dtke) +
                     al3 * (h0 + a * un) + al4 * (h0 - a * un);
  const double fr1 = rhor * unr, fl1 = rhol * unl;
  const double fr2 = (rhor * ur * unr + pr * kx), fl2 = (rhol * ul * unl + pl * kx);
  const double fr3 = (rhor * vr * unr + pr * ky), fl3 = (rhol * vl * unl + pl * ky);
  const double fr4 = (rhor * wr * unr + pr * kz), fl4 = (rhol * wl * unl + pl * kz);
  const double fr5 = (rh0r * unr + pr * ubn), fl5 = (rh0l * unl + pl * ubn);
  flux[0] = (fr1 + fl1 - df1) / 2 * ds;
  flux[1] = (fr2 + fl2 - df2) / 2 * ds;
  flux[2] = (fr3 + fl3 - df3) / 2 * ds;
  flux[3] = (fr4 + fl4 - df4) / 2 * ds;
  flux[4] = (fr5 + fl5 - df5) / 2 * ds;
}

// Euler face flux for the fused stage: roflux_b's algebra with the TKE terms
// (zero for Euler) dropped; sqrt(rho), 1/rho, the Roe-average weights, the
// speed of sound and its inverse come from rsqrt_nr / rcp_nr instead of
// separate square roots and divisions (last-bit differences).  MV: moving
// face with normal grid speed ubn (src/flux.f90:110-113, 122-189): the normal
// velocities relative to the face, the energy flux's p ubn and the shifted
// eigenvalues; the fixed-grid instantiation has none of these terms.
template <bool MV = false>
__device__ __forceinline__ void roe_flux_euler(const PhysPar &P, double kx, double ky, double kz, double ds,
                                               const double *qr, const double *ql, double *flux,
                                               double ubn = 0.0) {
  const double g_gm1 = P.g_gm1, gm1 = P.gm1;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
  const double unr = MV ? ur * kx + vr * ky + wr * kz - ubn : ur * kx + vr * ky + wr * kz;
  const double q2r = ur * ur + vr * vr + wr * wr;
  const double rsr = rsqrt_nr(rhor);  // 1/sqrt(rho_R): sqrt(rho_R) and 1/rho_R from it
  const double h0r = g_gm1 * pr * (rsr * rsr) + q2r / 2;
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
  const double unl = MV ? ul * kx + vl * ky + wl * kz - ubn : ul * kx + vl * ky + wl * kz;
  const double q2l = ul * ul + vl * vl + wl * wl;
  const double rsl = rsqrt_nr(rhol);
  const double h0l = g_gm1 * pl * (rsl * rsl) + q2l / 2;
  const double drho = rhor - rhol, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl;
  const double dun = unr - unl;
  const double rhols = rhol * rsl, rhors = rhor * rsr;
  const double rho = rhols * rhors;
  const double rden = rcp_nr(rhols + rhors);
  const double u = (rhols * ul + rhors * ur) * rden;
  const double v = (rhols * vl + rhors * vr) * rden;
  const double w = (rhols * wl + rhors * wr) * rden;
  const double un = u * kx + v * ky + w * kz;
  const double h0 = (rhols * h0l + rhors * h0r) * rden;
  const double q2 = u * u + v * v + w * w;
  const double a2 = gm1 * (h0 - q2 / 2);
  const double ra = rsqrt_nr(a2);  // 1/a
  const double a = a2 * ra;
  double rm123 = MV ? fabs(un - ubn) : fabs(un), rm4 = MV ? fabs(un + a - ubn) : fabs(un + a);
  double rm5 = MV ? fabs(un - a - ubn) : fabs(un - a);
  if (P.efx_setup_f) {
    double rdelta = P.cntrpy_f * (P.w1 * P.entfxctf_f + P.w2 * (sqrt(q2) + a) +
                                  P.w3 * 0.2 * (MV ? fabs(un) + a + fabs(ubn) : fabs(un) + a));
    rdelta = fmax(rdelta, 1.0e-12);
    if (rm123 <= rdelta && P.efx_all_f) rm123 = 0.5 * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5 * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5 * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_f) {
    if (rm123 <= P.eig_cutoff_f) rm123 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm4 <= P.eig_cutoff_f) rm4 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm5 <= P.eig_cutoff_f) rm5 = P.eig_cutoff_f;
  }
  const double dpa2 = dp * (ra * ra), rdua = rho * dun * ra;
  const double al1 = rm123 * (drho - dpa2);
  const double al2 = rm123 * rho;
  const double al3 = rm4 * (dpa2 + rdua) / 2;
  const double al4 = rm5 * (dpa2 - rdua) / 2;
  const double df1 = al1 + al3 + al4;
  const double df2 = al1 * u + al2 * (du - dun * kx) + al3 * (u + a * kx) + al4 * (u - a * kx);
  const double df3 = al1 * v + al2 * (dv - dun * ky) + al3 * (v + a * ky) + al4 * (v - a * ky);
  const double df4 = al1 * w + al2 * (dw - dun * kz) + al3 * (w + a * kz) + al4 * (w - a * kz);
  const double df5 = al1 * (q2 / 2) + al2 * (u * du + v * dv + w * dw - un * dun) + al3 * (h0 + a * un) +
                     al4 * (h0 - a * un);
  const double hds = ds / 2;
  flux[0] = (rhor * unr + rhol * unl - df1) * hds;
  flux[1] = ((rhor * ur * unr + pr * kx) + (rhol * ul * unl + pl * kx) - df2) * hds;
  flux[2] = ((rhor * vr * unr + pr * ky) + (rhol * vl * unl + pl * ky) - df3) * hds;
  flux[3] = ((rhor * wr * unr + pr * kz) + (rhol * wl * unl + pl * kz) - df4) * hds;
  if (MV) flux[4] = ((rhor * h0r * unr + pr * ubn) + (rhol * h0l * unl + pl * ubn) - df5) * hds;
  else flux[4] = (rhor * h0r * unr + rhol * h0l * unl - df5) * hds;
}

// Mixed precision: the central part (fr + fl) in FP64 from the FP64 face
// states, the Roe dissipation df in FP32 from FP32 copies of the states and
// of their FP64 differences.  Same algebra as roe_flux_fp64.
__device__ __forceinline__ void roe_flux_mixed(const PhysPar &P, double kx, double ky, double kz, double ds,
                                               const double *qr, const double *ql, double *flux) {
  const double g = P.g;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
  const double unr = ur * kx + vr * ky + wr * kz;
  const double unl = ul * kx + vl * ky + wl * kz;
  const double q2r = ur * ur + vr * vr + wr * wr;
  const double q2l = ul * ul + vl * vl + wl * wl;
  const double h0r = P.g_gm1 * pr * rcp_nr(rhor) + q2r / 2;
  const double h0l = P.g_gm1 * pl * rcp_nr(rhol) + q2l / 2;
  // FP32 dissipation on FP64 differences
  const float fkx = (float)kx, fky = (float)ky, fkz = (float)kz;
  const float drho = (float)(rhor - rhol), dp = (float)(pr - pl);
  const float du = (float)(ur - ul), dv = (float)(vr - vl), dw = (float)(wr - wl);
  const float dun = (float)(unr - unl);
  const float frl = (float)rhol, frr = (float)rhor;
  const float rhols = frl * rsqrtf(frl), rhors = frr * rsqrtf(frr);
  const float rho = rhols * rhors;
  const float rden = __fdividef(1.0f, rhols + rhors);
  const float u = (rhols * (float)ul + rhors * (float)ur) * rden;
  const float v = (rhols * (float)vl + rhors * (float)vr) * rden;
  const float w = (rhols * (float)wl + rhors * (float)wr) * rden;
  const float un = u * fkx + v * fky + w * fkz;
  const float h0 = (rhols * (float)h0l + rhors * (float)h0r) * rden;
  const float q2 = u * u + v * v + w * w;
  const float a2 = (float)(g - 1) * (h0 - q2 * 0.5f);
  const float ria = rsqrtf(a2);
  const float a = a2 * ria;
  float rm123 = fabsf(un), rm4 = fabsf(un + a), rm5 = fabsf(un - a);
  if (P.efx_setup_f) {
    float rdelta = (float)P.cntrpy_f * ((float)P.w1 * (float)P.entfxctf_f + (float)P.w2 * (sqrtf(q2) + a) +
                                        (float)P.w3 * 0.2f * (fabsf(un) + a));
    rdelta = fmaxf(rdelta, 1.0e-12f);
    if (rm123 <= rdelta && P.efx_all_f) rm123 = 0.5f * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5f * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5f * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_f) {
    const float c = (float)P.eig_cutoff_f;
    if (rm123 <= c) rm123 = c;
    if (P.eig_lim_all_f && rm4 <= c) rm4 = c;
    if (P.eig_lim_all_f && rm5 <= c) rm5 = c;
  }
  const float ia2 = ria * ria;
  const float dpa2 = dp * ia2, rdua = rho * dun * ria;
  const float al1 = rm123 * (drho - dpa2);
  const float al2 = rm123 * rho;
  const float al3 = rm4 * (dpa2 + rdua) * 0.5f;
  const float al4 = rm5 * (dpa2 - rdua) * 0.5f;
  const float df1 = al1 + al3 + al4;
  const float df2 = al1 * u + al2 * (du - dun * fkx) + al3 * (u + a * fkx) + al4 * (u - a * fkx);
  const float df3 = al1 * v + al2 * (dv - dun * fky) + al3 * (v + a * fky) + al4 * (v - a * fky);
  const float df4 = al1 * w + al2 * (dw - dun * fkz) + al3 * (w + a * fkz) + al4 * (w - a * fkz);
  const float df5 = al1 * (q2 * 0.5f) + al2 * (u * du + v * dv + w * dw - un * dun) + al3 * (h0 + a * un) +
                    al4 * (h0 - a * un);
  const double hds = 0.5 * ds;
  flux[0] = (rhor * unr + rhol * unl - (double)df1) * hds;
  flux[1] = ((rhor * ur * unr + pr * kx) + (rhol * ul * unl + pl * kx) - (double)df2) * hds;
  flux[2] = ((rhor * vr * unr + pr * ky) + (rhol * vl * unl + pl * ky) - (double)df3) * hds;
  flux[3] = ((rhor * wr * unr + pr * kz) + (rhol * wl * unl + pl * kz) - (double)df4) * hds;
  flux[4] = (rhor * h0r * unr + rhol * h0l * unl - (double)df5) * hds;
}

// roflux_b's mean-flow flux with the turbulent kinetic energy terms
// (roe_flux_fp64's algebra) in mixed precision: central part in FP64, the
// Roe dissipation in FP32 from FP32 copies of the states and of their FP64
// differences (the k-omega path's counterpart of roe_flux_mixed).
__device__ __forceinline__ void roe_flux_mixed_tke(const PhysPar &P, double kx, double ky, double kz, double ds,
                                                   const double *qr, const double *ql, double tker, double tkel,
                                                   double *flux, double ubn = 0.0) {
  // ubn: the face's normal grid speed on moving grids (src/flux.f90:110-113),
  // FP64 in the central flux, FP32 in the dissipation like the rest of it
  const double g = P.g;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4];
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4];
  const double unr = ur * kx + vr * ky + wr * kz - ubn;
  const double unl = ul * kx + vl * ky + wl * kz - ubn;
  const double q2r = ur * ur + vr * vr + wr * wr;
  const double q2l = ul * ul + vl * vl + wl * wl;
  const double h0r = g / (g - 1) * pr / rhor + q2r / 2 + tker;
  const double h0l = g / (g - 1) * pl / rhol + q2l / 2 + tkel;
  const float fkx = (float)kx, fky = (float)ky, fkz = (float)kz;
  const float drho = (float)(rhor - rhol), dp = (float)(pr - pl);
  const float du = (float)(ur - ul), dv = (float)(vr - vl), dw = (float)(wr - wl);
  const float dun = (float)(unr - unl), dtke = (float)(tker - tkel);
  const float frl = (float)rhol, frr = (float)rhor;
  const float rhols = sqrtf(frl), rhors = sqrtf(frr);
  const float rho = rhols * rhors;
  const float rden = 1.0f / (rhols + rhors);
  const float u = (rhols * (float)ul + rhors * (float)ur) * rden;
  const float v = (rhols * (float)vl + rhors * (float)vr) * rden;
  const float w = (rhols * (float)wl + rhors * (float)wr) * rden;
  const float un = u * fkx + v * fky + w * fkz;
  const float h0 = (rhols * (float)h0l + rhors * (float)h0r) * rden;
  const float tke = (rhols * (float)tkel + rhors * (float)tker) * rden;
  const float q2 = u * u + v * v + w * w;
  const float a2 = (float)(g - 1) * (h0 - q2 * 0.5f - tke);
  const float a = sqrtf(a2);
  const float fubn = (float)ubn;
  float rm123 = fabsf(un - fubn), rm4 = fabsf(un + a - fubn), rm5 = fabsf(un - a - fubn);
  if (P.efx_setup_f) {
    float rdelta = (float)P.cntrpy_f * ((float)P.w1 * (float)P.entfxctf_f + (float)P.w2 * (sqrtf(q2) + a) +
                                        (float)P.w3 * 0.2f * (fabsf(un) + a + fabsf(fubn)));
    rdelta = fmaxf(rdelta, 1.0e-12f);
    if (rm123 <= rdelta && P.efx_all_f) rm123 = 0.5f * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5f * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5f * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_f) {
    const float c = (float)P.eig_cutoff_f;
    if (rm123 <= c) rm123 = c;
    if (P.eig_lim_all_f && rm4 <= c) rm4 = c;
    if (P.eig_lim_all_f && rm5 <= c) rm5 = c;
  }
  const float dpa2 = dp / a2, rdua = rho * dun / a;
  const float al1 = rm123 * (drho - dpa2);
  const float al2 = rm123 * rho;
  const float al3 = rm4 * (dpa2 + rdua) * 0.5f;
  const float al4 = rm5 * (dpa2 - rdua) * 0.5f;
  const float df1 = al1 + al3 + al4;
  const float df2 = al1 * u + al2 * (du - dun * fkx) + al3 * (u + a * fkx) + al4 * (u - a * fkx);
  const float df3 = al1 * v + al2 * (dv - dun * fky) + al3 * (v + a * fky) + al4 * (v - a * fky);
  const float df4 = al1 * w + al2 * (dw - dun * fkz) + al3 * (w + a * fkz) + al4 * (w - a * fkz);
  const float df5 = al1 * (q2 * 0.5f + tke) + al2 * (u * du + v * dv + w * dw - un * dun + dtke) +
                    al3 * (h0 + a * un) + al4 * (h0 - a * un);
  flux[0] = (rhor * unr + rhol * unl - (double)df1) / 2 * ds;
  flux[1] = ((rhor * ur * unr + pr * kx) + (rhol * ul * unl + pl * kx) - (double)df2) / 2 * ds;
  flux[2] = ((rhor * vr * unr + pr * ky) + (rhol * vl * unl + pl * ky) - (double)df3) / 2 * ds;
  flux[3] = ((rhor * wr * unr + pr * kz) + (rhol * wl * unl + pl * kz) - (double)df4) / 2 * ds;
  flux[4] = (rhor * h0r * unr + pr * ubn + rhol * h0l * unl + pl * ubn - (double)df5) / 2 * ds;
}

// ---- eig_eul (src/cosa.f90:4183-4233); gv: the cell's grid velocity on
// moving grids (src/cosa.f90:4225-4229), null on fixed grids ----------------------------
__device__ __forceinline__ void eig_eul(double g, const double *qc, const double *sim, const double *sip,
                                        const double *sjm, const double *sjp, const double *skm,
                                        const double *skp, double &lami, double &lamj, double &lamk,
                                        const double *gv = nullptr) {
  const double rho = qc[0], p = qc[4];
  double u = qc[1], v = qc[2], w = qc[3];
  if (gv) { u = u - gv[0]; v = v - gv[1]; w = w - gv[2]; }
  const double a = sqrt(g * p / rho);
  const double xix = 0.5 * (sim[0] * sim[3] + sip[0] * sip[3]);
  const double xiy = 0.5 * (sim[1] * sim[3] + sip[1] * sip[3]);
  const double xiz = 0.5 * (sim[2] * sim[3] + sip[2] * sip[3]);
  const double etax = 0.5 * (sjm[0] * sjm[3] + sjp[0] * sjp[3]);
  const double etay = 0.5 * (sjm[1] * sjm[3] + sjp[1] * sjp[3]);
  const double etaz = 0.5 * (sjm[2] * sjm[3] + sjp[2] * sjp[3]);
  const double zetax = 0.5 * (skm[0] * skm[3] + skp[0] * skp[3]);
  const double zetay = 0.5 * (skm[1] * skm[3] + skp[1] * skp[3]);
  const double zetaz = 0.5 * (skm[2] * skm[3] + skp[2] * skp[3]);
  const double axi = (sim[3] + sip[3]) / 2;
  const double aeta = (sjm[3] + sjp[3]) / 2;
  const double azeta = (skm[3] + skp[3]) / 2;
  lami = fabs(u * xix + v * xiy + w * xiz) + a * axi;
  lamj = fabs(u * etax + v * etay + w * etaz) + a * aeta;
  lamk = fabs(u * zetax + v * zetay + w * zetaz) + a * azeta;
}

// eig_eul_p (src/cosa.f90:4300-4372): the convective spectral radii of the
// low-speed preconditioned system, with the preconditioned Mach number
// mp2 = min(max(M^2, (uprv/a)^2, cutoff, epsp(nl)^2), 1)
__device__ __forceinline__ void eig_eul_p(double g, double uprv, double eps2, double cutoff, const double *qc,
                                          const double *sim, const double *sip, const double *sjm,
                                          const double *sjp, const double *skm, const double *skp, double &lami,
                                          double &lamj, double &lamk) {
  const double rho = qc[0], p = qc[4], u = qc[1], v = qc[2], w = qc[3];
  const double a = sqrt(g * p / rho);
  const double q2 = u * u + v * v + w * w, a2 = a * a;
  const double ump2 = (uprv / a) * (uprv / a);
  const double mp2 = fmin(fmax(fmax(fmax(q2 / a2, ump2), cutoff), eps2), 1.0);
  const double xix = 0.5 * (sim[0] * sim[3] + sip[0] * sip[3]);
  const double xiy = 0.5 * (sim[1] * sim[3] + sip[1] * sip[3]);
  const double xiz = 0.5 * (sim[2] * sim[3] + sip[2] * sip[3]);
  const double etax = 0.5 * (sjm[0] * sjm[3] + sjp[0] * sjp[3]);
  const double etay = 0.5 * (sjm[1] * sjm[3] + sjp[1] * sjp[3]);
  const double etaz = 0.5 * (sjm[2] * sjm[3] + sjp[2] * sjp[3]);
  const double zetax = 0.5 * (skm[0] * skm[3] + skp[0] * skp[3]);
  const double zetay = 0.5 * (skm[1] * skm[3] + skp[1] * skp[3]);
  const double zetaz = 0.5 * (skm[2] * skm[3] + skp[2] * skp[3]);
  const double axi = (sim[3] + sip[3]) / 2, aeta = (sjm[3] + sjp[3]) / 2, azeta = (skm[3] + skp[3]) / 2;
  const double ui = u * xix + v * xiy + w * xiz, uj = u * etax + v * etay + w * etaz;
  const double uk = u * zetax + v * zetay + w * zetaz;
  const double m1 = (1 - mp2) * (1 - mp2);
  lami = ((1 + mp2) * fabs(ui) + sqrt(ui * ui * m1 + 4 * a2 * mp2 * (axi * axi))) / 2;
  lamj = ((1 + mp2) * fabs(uj) + sqrt(uj * uj * m1 + 4 * a2 * mp2 * (aeta * aeta))) / 2;
  lamk = ((1 + mp2) * fabs(uk) + sqrt(uk * uk * m1 + 4 * a2 * mp2 * (azeta * azeta))) / 2;
}

// ---- boundary conditions (src/bc.f90) --------------------------------------------
// Each BC maps the primitive interior values next to the face (c1 = first
// interior cell, c2 = second) and the face normal to the two halo layers
// (h1 = first halo, h2 = second).  Returned mask: bit0 h1 set, bit1 h2 set.
struct BcPar {
  double g, rhoinf, ainf, pinf, sinf;
  double qfst[5];
  double t0, p0, sx, sy, sz;
  double pout1, pout3;
  double tkefar, omefar, qmin6, qmin7;
  int npde;
  // low-speed preconditioning: lomach, mixpi, uprv and epsp(nl)^2 of the level
  int lomach, mixpi;
  double uprv, eps2;
};

__device__ __forceinline__ BcPar make_bcpar(const cosa_params &P, int nl = 1) {
  BcPar b;
  b.g = P.gamma; b.rhoinf = P.rhoinf; b.ainf = P.ainf; b.pinf = P.pinf;
  b.sinf = P.pinf / pow(P.rhoinf, P.gamma);
  b.qfst[0] = P.rhoinf;
  b.qfst[1] = P.machfs * cos(P.alpha) * cos(P.beta);
  b.qfst[2] = P.machfs * sin(P.alpha) * cos(P.beta);
  b.qfst[3] = P.machfs * sin(P.beta);
  b.qfst[4] = P.pinf;
  b.t0 = P.inlet_t0; b.p0 = P.inlet_p0;
  b.sx = P.inlet_dir[0]; b.sy = P.inlet_dir[1]; b.sz = P.inlet_dir[2];
  b.pout1 = P.outlet_p[0]; b.pout3 = P.outlet_p[2];
  b.tkefar = P.tkefar; b.omefar = P.omefar; b.qmin6 = P.qmin[5]; b.qmin7 = P.qmin[6];
  b.npde = P.npde;
  b.lomach = P.lomach; b.mixpi = P.mixpi; b.uprv = P.uprv;
  b.eps2 = P.epsp[nl - 1] * P.epsp[nl - 1];
  return b;
}

// bc_sym (src/bc.f90:2595-2710)
__device__ __forceinline__ int bc_sym(int idir, int npde, const double *c1, const double *c2, double *h1, double *h2) {
  for (int v = 0; v < npde; ++v) {
    const double s = (v == idir) ? -1.0 : 1.0;
    h1[v] = s * c1[v];
    h2[v] = s * c2[v];
  }
  return 3;
}
// bc_extrapol (src/bc.f90:2494-2592)
__device__ __forceinline__ int bc_extrapol(int npde, const double *c1, double *h1, double *h2) {
  for (int v = 0; v < npde; ++v) { h1[v] = c1[v]; h2[v] = c1[v]; }
  return 3;
}
// bc_walinv_14 (src/bc.f90:1457-1675), fixed grid; n = face metric at ibcm
// wv: the wall face's velocity on moving grids (src/bc.f90:1567-1614), null on
// fixed grids
__device__ __forceinline__ int bc_walinv(int npde, double nx, double ny, double nz, const double *c1,
                                         const double *c2, double *h1, double *h2, const double *wv = nullptr) {
  const double rhow = (3 * c1[0] - c2[0]) / 2, uw = (3 * c1[1] - c2[1]) / 2;
  const double vw = (3 * c1[2] - c2[2]) / 2, ww = (3 * c1[3] - c2[3]) / 2, pw = (3 * c1[4] - c2[4]) / 2;
  const double un1 = c1[1] * nx + c1[2] * ny + c1[3] * nz;
  const double un2 = c2[1] * nx + c2[2] * ny + c2[3] * nz;
  double unw = (3 * un1 - un2) / 2;
  if (wv) unw = unw - (wv[0] * nx + wv[1] * ny + wv[2] * nz);
  h1[0] = rhow; h1[1] = uw - unw * nx; h1[2] = vw - unw * ny; h1[3] = ww - unw * nz; h1[4] = pw;
  if (npde > 5) { h1[5] = c1[5]; h1[6] = c1[6]; }
  for (int v = 0; v < npde; ++v) h2[v] = h1[v];
  return 3;
}
// bc_insub (src/bc.f90:875-1175): subsonic inlet, Newton on the normal
// velocity; n already multiplied by sgnm.  Returns mask, sets *err on a
// Newton iteration count of 10 (the reference stops there).
__device__ __forceinline__ int bc_insub(const BcPar &B, double nx, double ny, double nz, const double *c1,
                                        const double *c2, double *h1, double *h2, int *err) {
  const double g = B.g;
  const double rho1 = c1[0], rho2 = c2[0];
  const double un1 = c1[1] * nx + c1[2] * ny + c1[3] * nz;
  const double un2 = c2[1] * nx + c2[2] * ny + c2[3] * nz;
  const double p1 = c1[4], p2 = c2[4];
  double rc1 = sqrt(g * p1 * rho1);
  double rc2 = sqrt(g * p2 * rho2);
  if (B.lomach) {
    // the preconditioned outgoing characteristic (src/bc.f90:1032-1056)
    auto rc_lsp = [&](const double *c, double un) {
      const double q2 = c[1] * c[1] + c[2] * c[2] + c[3] * c[3], a2 = g * c[4] / c[0], a = sqrt(a2);
      const double ump2 = (B.uprv / a) * (B.uprv / a);
      const double mp2 = fmin(fmax(fmax(q2 / a2, ump2), B.eps2), 1.0);
      const double lp3 = 0.5 * (un * (1. + mp2) + sqrt(un * un * ((1. - mp2) * (1. - mp2)) + 4. * a2 * mp2));
      return -(c[0] * (un - lp3));
    };
    rc1 = rc_lsp(c1, un1);
    rc2 = rc_lsp(c2, un2);
  }
  const double rcun1 = rc1 * un1, rcun2 = rc2 * un2;
  const double h0inl = 1 / (g - 1) * B.t0;
  const double dot = B.sx * nx + B.sy * ny + B.sz * nz;
  const double con1 = 0.5 / (h0inl * (dot * dot));
  const double con2 = 2 * con1 * g / (g - 1);
  for (int icell = 1; icell <= 2; ++icell) {
    double p, un, rc, rcun;
    if (icell == 1) {
      p = 2 * p1 - p2; un = 2 * un1 - un2; rc = 2 * rc1 - rc2; rcun = 2 * rcun1 - rcun2;
    } else {
      p = 3 * p1 - 2 * p2; un = 3 * un1 - 2 * un2; rc = 3 * rc1 - 2 * rc2; rcun = 3 * rcun1 - 2 * rcun2;
    }
    const double con3 = p - rcun;
    double dun = 1.0;
    int count = 0;
    while (fabs(dun) > 1.0e-10) {
      count = count + 1;
      if (count == 10) { *err = 1; break; }
      const double par = 1.0 - con1 * (un * un);
      p = B.p0 * pow(par, g / (g - 1));
      const double f = p - rc * un - con3;
      const double fp = -con2 * un * p / par - rc;
      dun = -f / fp;
      un = un + dun;
    }
    p = +rc * un + con3;
    const double modv = un / dot;
    double *h = icell == 1 ? h1 : h2;
    h[0] = g * p / ((g - 1) * (h0inl - 0.5 * (modv * modv)));
    h[1] = modv * B.sx; h[2] = modv * B.sy; h[3] = modv * B.sz; h[4] = p;
    if (B.npde > 5) { h[5] = B.tkefar; h[6] = B.omefar; }
  }
  return 3;
}
// bc_outsub (src/bc.f90:1178-1455): static-pressure outlet
__device__ __forceinline__ int bc_outsub(const BcPar &B, const double *c1, const double *c2, double *h1, double *h2) {
  const double g = B.g;
  const int npde = B.npde;
  const bool kom = npde > 5;
  double qc1[7], qc2[7];
  const double tke1 = kom ? c1[5] : 0.0, tke2 = kom ? c2[5] : 0.0;
  qc1[0] = c1[0]; qc2[0] = c2[0];
  for (int v = 1; v < npde; ++v)
    if (v != 4) { qc1[v] = c1[v] * c1[0]; qc2[v] = c2[v] * c2[0]; }
  {
    const double rho = qc1[0], ru = qc1[1], rv = qc1[2], rw = qc1[3];
    qc1[4] = c1[4] / (g - 1) + (ru * ru + rv * rv + rw * rw) / 2 / rho + rho * tke1;
  }
  {
    const double rho = qc2[0], ru = qc2[1], rv = qc2[2], rw = qc2[3];
    qc2[4] = c2[4] / (g - 1) + (ru * ru + rv * rv + rw * rw) / 2 / rho + rho * tke2;
  }
  double a[7], b[7];  // conservative halo values
  for (int v = 0; v < npde; ++v)
    if (v != 4) a[v] = 2 * qc1[v] - qc2[v];
  double rhotke0 = 0.0;
  if (kom) {
    a[5] = fmax(a[5], a[0] * B.qmin6);
    a[6] = fmax(a[6], a[0] * B.qmin7);
    rhotke0 = a[5];
  }
  a[4] = B.pout1 / (g - 1) + (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) / 2 / a[0] + rhotke0;
  for (int v = 0; v < npde; ++v)
    if (v != 4) b[v] = 3 * qc1[v] - 2 * qc2[v];
  double rhotke2 = 0.0, rhotke1 = 0.0, rhotkem1 = 0.0;
  if (kom) {
    b[5] = fmax(b[5], b[0] * B.qmin6);
    b[6] = fmax(b[6], b[0] * B.qmin7);
    rhotke2 = qc2[5]; rhotke1 = qc1[5]; rhotkem1 = b[5];
  }
  const double rhol = (3 * qc1[0] - qc2[0]) / 2;
  const double rhor = (3 * a[0] - b[0]) / 2;
  const double pp1 = (g - 1) * (qc1[4] - rhotke1 - (qc1[1] * qc1[1] + qc1[2] * qc1[2] + qc1[3] * qc1[3]) / 2 / qc1[0]);
  const double pp2 = (g - 1) * (qc2[4] - rhotke2 - (qc2[1] * qc2[1] + qc2[2] * qc2[2] + qc2[3] * qc2[3]) / 2 / qc2[0]);
  const double pl = (3 * pp1 - pp2) / 2;
  const double pr = (B.pout3 * (sqrt(rhol) + sqrt(rhor)) - pl * sqrt(rhol)) / sqrt(rhor);
  const double pm1 = 3 * B.pout1 - 2 * pr;
  b[4] = pm1 / (g - 1) + (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]) / 2 / b[0] + rhotkem1;
  for (int v = 1; v < npde; ++v)
    if (v != 4) { a[v] = a[v] / a[0]; b[v] = b[v] / b[0]; }
  const double tk1 = kom ? a[5] : 0.0, tk2 = kom ? b[5] : 0.0;
  {
    const double r1 = a[0], u1 = a[1], v1 = a[2], w1 = a[3], e1 = a[4];
    a[4] = (g - 1) * (e1 - r1 * (u1 * u1 + v1 * v1 + w1 * w1) / 2 - r1 * tk1);
  }
  {
    const double r2 = b[0], u2 = b[1], v2 = b[2], w2 = b[3], e2 = b[4];
    b[4] = (g - 1) * (e2 - r2 * (u2 * u2 + v2 * v2 + w2 * w2) / 2 - r2 * tk2);
  }
  for (int v = 0; v < npde; ++v) { h1[v] = a[v]; h2[v] = b[v]; }
  return 3;
}
// bc_far0 (src/bc.f90:124-483): Riemann-invariant far field, aircraft free
// stream; s = face normal times sgnm
__device__ __forceinline__ int bc_far0(const BcPar &B, double sx, double sy, double sz, const double *c1,
                                       double *h1, double *h2) {
  if (B.lomach) {
    // low-speed preconditioning: both layers frozen at the free stream (src/bc.f90:264-276, 409-414)
    for (int v = 0; v < 5; ++v) h1[v] = B.qfst[v];
    if (B.npde > 5) { h1[5] = B.tkefar; h1[6] = B.omefar; }
    for (int v = 0; v < B.npde; ++v) h2[v] = h1[v];
    return 3;
  }
  const double g = B.g;
  const double qext = c1[1] * sx + c1[2] * sy + c1[3] * sz;
  const double qinf = B.qfst[1] * sx + B.qfst[2] * sy + B.qfst[3] * sz;
  const double rhoext = c1[0], pext = c1[4];
  const double aext = sqrt(g * pext / rhoext);
  const double rext = qext + 2 * aext / (g - 1);
  const double rinf = qinf - 2 * B.ainf / (g - 1);
  const double qdotn = (rext + rinf) / 2;
  const double a = (g - 1) * (rext - rinf) / 4;
  const double mach = qdotn / a;
  const double sext = pext / pow(rhoext, g);
  int mask = 0;
  if (qdotn <= 0.0) {
    if (fabs(mach) >= 1.0) {
      for (int v = 0; v < 5; ++v) h1[v] = B.qfst[v];
    } else {
      const double rhobc = pow(a * a / (g * B.sinf), 1.0 / (g - 1));
      const double p = rhobc * a * a / g;
      h1[0] = rhobc;
      h1[1] = B.qfst[1] + (qdotn - qinf) * sx;
      h1[2] = B.qfst[2] + (qdotn - qinf) * sy;
      h1[3] = B.qfst[3] + (qdotn - qinf) * sz;
      h1[4] = p;
    }
    mask = 3;
    if (B.npde > 5) { h1[5] = B.tkefar; h1[6] = B.omefar; }
  } else if (qdotn > 0.0) {
    if (fabs(mach) >= 1.0) {
      for (int v = 0; v < 5; ++v) h1[v] = c1[v];
    } else {
      const double rhobc = pow(a * a / (g * sext), 1.0 / (g - 1));
      const double p = rhobc * a * a / g;
      h1[0] = rhobc;
      h1[1] = c1[1] + (qdotn - qext) * sx;
      h1[2] = c1[2] + (qdotn - qext) * sy;
      h1[3] = c1[3] + (qdotn - qext) * sz;
      h1[4] = p;
    }
    mask = 3;
    if (B.npde > 5) { h1[5] = c1[5]; h1[6] = c1[6]; }
  }
  for (int v = 0; v < B.npde; ++v) h2[v] = h1[v];
  return mask;
}

// bc_walvis_15, laminar part on a fixed grid (src/bc.f90:2144-2300): no-slip
// wall; wall pressure extrapolated linearly from the first two cells, wall
// density from cell 1 along the isentrope; both halo layers take the wall state
// bc_far1 (src/bc.f90:486-870), aircraft free stream, no low-speed
// preconditioning: boundary normal velocity and pressure from the mean of
// the interior and free-stream states plus the acoustic jump, density from
// the isentrope of the upwind side; s = face normal times sgnm
__device__ __forceinline__ int bc_far1(const BcPar &B, double sx, double sy, double sz, const double *c1,
                                       double *h1, double *h2) {
  const double g = B.g;
  const double qext = c1[1] * sx + c1[2] * sy + c1[3] * sz;
  const double qinf = B.qfst[1] * sx + B.qfst[2] * sy + B.qfst[3] * sz;
  const double pext = c1[4], pinf = B.qfst[4], rhoext = c1[0];
  const double a = sqrt(g * pext / rhoext);
  double unb = (qext + qinf) / 2 + (pext - pinf) / (2 * rhoext * a);
  double pb = (pext + pinf) / 2 + rhoext * a * (qext - qinf) / 2;
  if (B.lomach) {
    // preconditioned characteristics with the artificial sound speed apr
    // (src/bc.f90:638-667)
    const double q2 = c1[1] * c1[1] + c1[2] * c1[2] + c1[3] * c1[3];
    const double a2 = g * pext / rhoext, al = sqrt(a2), un = qext;
    const double m2 = q2 / a2, ump2 = (B.uprv / al) * (B.uprv / al);
    const double mp2s = fmin(1.0, fmax(fmax(m2, (1 - B.mixpi) * ump2), B.eps2));
    const double am = (1 - mp2s) / 2;
    const double apr = sqrt(am * am * (un * un) + a2 * mp2s);
    unb = (qext + qinf) / 2 + (pext - pinf) / (2 * rhoext * apr) + (qext - qinf) / 2 * am * un / apr;
    pb = (pext + pinf) / 2 + rhoext * mp2s * a2 / apr * (qext - qinf) / 2 - (pext - pinf) / 2 * am * un / apr;
  }
  const double mach = unb / a;
  int mask = 0;
  if (unb <= 0.0) {
    if (fabs(mach) >= 1.0) {
      for (int v = 0; v < 5; ++v) h1[v] = B.qfst[v];
    } else {
      h1[0] = B.qfst[0] * pow(pb / pinf, 1 / g);
      h1[1] = B.qfst[1] + (unb - qinf) * sx;
      h1[2] = B.qfst[2] + (unb - qinf) * sy;
      h1[3] = B.qfst[3] + (unb - qinf) * sz;
      h1[4] = pb;
    }
    mask = 3;
    if (B.npde > 5) { h1[5] = B.tkefar; h1[6] = B.omefar; }
  } else if (unb > 0.0) {
    if (fabs(mach) >= 1.0) {
      for (int v = 0; v < 5; ++v) h1[v] = c1[v];
    } else {
      h1[0] = c1[0] * pow(pb / pext, 1 / g);
      h1[1] = c1[1] + (unb - qext) * sx;
      h1[2] = c1[2] + (unb - qext) * sy;
      h1[3] = c1[3] + (unb - qext) * sz;
      h1[4] = pb;
    }
    mask = 3;
    if (B.npde > 5) { h1[5] = c1[5]; h1[6] = c1[6]; }
  }
  for (int v = 0; v < B.npde; ++v) h2[v] = h1[v];
  return mask;
}

// wv: the wall face's velocity on moving grids (src/bc.f90:2256-2283), null
// on fixed grids
__device__ __forceinline__ int bc_walvis(double g, const double *c1, const double *c2, double *h1, double *h2,
                                         const double *wv = nullptr) {
  const double p1 = c1[4], p2 = c2[4];
  const double pw = 0.5 * (3 * p1 - p2);
  h1[0] = pow(pw / p1, 1 / g) * c1[0];
  h1[1] = wv ? wv[0] : 0.0; h1[2] = wv ? wv[1] : 0.0; h1[3] = wv ? wv[2] : 0.0;
  h1[4] = pw;
  for (int v = 0; v < 5; ++v) h2[v] = h1[v];
  return 3;
}

// ---- roflux_b turbulence fluxes ----------------------------------------------------
// Upwinded rho k u_n and rho omega u_n with the mean-flow wave strengths and
// the turbulence entropy-fix settings.  h0l/h0r are the values the
// mean-flow loop left behind, those of the block's last face (ic,jc,kc) of
// the snapshot (the reference does not recompute them in this loop).
__device__ __forceinline__ void roe_turb(const cosa_params &P, double kx, double ky, double kz, double ds,
                                         const double *qr, const double *ql, double h0r_last, double h0l_last,
                                         double &fk, double &fw, double ubn = 0.0) {
  const double g = P.gamma;
  const double rhor = qr[0], ur = qr[1], vr = qr[2], wr = qr[3], pr = qr[4], tker = qr[5], omer = qr[6];
  const double rhol = ql[0], ul = ql[1], vl = ql[2], wl = ql[3], pl = ql[4], tkel = ql[5], omel = ql[6];
  const double unr = ur * kx + vr * ky + wr * kz - ubn, unl = ul * kx + vl * ky + wl * kz - ubn;
  const double frk = rhor * unr * tker, frw = rhor * unr * omer;
  const double flk = rhol * unl * tkel, flw = rhol * unl * omel;
  const double drho = rhor - rhol, dp = pr - pl, dun = unr - unl, dtke = tker - tkel, dome = omer - omel;
  const double rhols = sqrt(rhol), rhors = sqrt(rhor);
  const double rho = rhols * rhors, denom = rhols + rhors;
  const double u = (rhols * ul + rhors * ur) / denom, v = (rhols * vl + rhors * vr) / denom;
  const double w = (rhols * wl + rhors * wr) / denom;
  const double un = u * kx + v * ky + w * kz;
  const double h0 = (rhols * h0l_last + rhors * h0r_last) / denom;
  const double tke = (rhols * tkel + rhors * tker) / denom, ome = (rhols * omel + rhors * omer) / denom;
  const double q2 = u * u + v * v + w * w;
  const double a2 = (g - 1) * (h0 - q2 / 2 - tke);
  const double a = sqrt(a2);
  double rm123 = fabs(un - ubn), rm4 = fabs(un + a - ubn), rm5 = fabs(un - a - ubn);
  if (P.efx_setup_t) {
    double rdelta = P.cntrpy_t * (P.entfx_t_w[0] * P.entfxctf_t + P.entfx_t_w[1] * (sqrt(q2) + a) +
                                  P.entfx_t_w[2] * 0.2 * (fabs(un) + a + fabs(ubn)));
    rdelta = fmax(rdelta, 1.0e-12);
    if (rm123 <= rdelta && P.efx_all_t) rm123 = 0.5 * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5 * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5 * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_t) {
    if (rm123 <= P.eig_cutoff_t) rm123 = P.eig_cutoff_t;
    if (P.eig_lim_all_t && rm4 <= P.eig_cutoff_t) rm4 = P.eig_cutoff_t;
    if (P.eig_lim_all_t && rm5 <= P.eig_cutoff_t) rm5 = P.eig_cutoff_t;
  }
  const double al1 = rm123 * (drho - dp / a2), al2 = rm123 * rho;
  const double al3 = rm4 * (dp / a2 + rho * dun / a) / 2, al4 = rm5 * (dp / a2 - rho * dun / a) / 2;
  const double dfk = (al1 + al3 + al4) * tke + al2 * dtke;
  const double dfw = (al1 + al3 + al4) * ome + al2 * dome;
  fk = (frk + flk - dfk) / 2 * ds;
  fw = (frw + flw - dfw) / 2 * ds;
}

// h0 of a face state (rho, u, v, w, p, k)
__device__ __forceinline__ double face_h0(double g, const double *q) {
  return g / (g - 1) * q[4] / q[0] + (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / 2 + q[5];
}

// ---- bc_walvis_15, k-omega part (src/bc.f90:2309-2470) ---------------------------
// h1 holds the wall state (laminar part already applied), c1 the first
// cell; d = wall distance of the first cell, (nx, ny, nz) the face normal
__device__ __forceinline__ void bc_walvis_kom(const cosa_params &P, double nx, double ny, double nz, double d,
                                              const double *c1, double *h1, double *h2,
                                              const double *wv = nullptr) {
  const double small = 1.0e-12, smasq = 1.0e-24, mor = P.machfs / P.reyno;
  const double rhow = h1[0], pw = h1[4];
  const double tw = pw * P.gamma / rhow;
  const double muw = (P.stemp + 1) / (tw + P.stemp) * pow(tw, 1.5);
  double omew;
  if (P.wallwilc) {
    // the first cell's velocity relative to a moving wall face (src/bc.f90:2346-2394)
    const double uc = wv ? c1[1] - wv[0] : c1[1], vc = wv ? c1[2] - wv[1] : c1[2], wc = wv ? c1[3] - wv[2] : c1[3];
    const double uorth = nx * uc + ny * vc + nz * wc;
    const double a = uc - uorth * nx, b = vc - uorth * ny, c = wc - uorth * nz;
    const double upar = sqrt(a * a + b * b + c * c);
    const double dupardn = upar / (d + small);
    const double tauw = muw * fabs(dupardn);
    const double rkrpls = P.roughk > 0.0 ? fmax(1.0, sqrt(rhow * tauw / mor) * P.roughk / muw) : 1.0;
    const double sr = rkrpls >= 25.0 ? 100.0 / rkrpls : 2500.0 / (rkrpls * rkrpls);
    omew = fabs(dupardn) * sr;
  } else {
    omew = 60.0 * muw / (P.bkw * rhow * (d * d) + smasq) * P.machfs / P.reyno;
  }
  h1[5] = 0.0; h1[6] = omew;
  h2[5] = h1[5]; h2[6] = h1[6];
}

__device__ __forceinline__ bool strong_bc(int t) {
  return t == 13 || t == 14 || t / 100 == 15 || t == 22 || t == 23 || t == 92 || t == 93 || t == 5;
}
