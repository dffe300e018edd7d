// Line-marching convective face kernel of the face-split stage schedule.
//
// Every face of a line (fixed transverse cell, family d) needs the limited
// MUSCL states of its two cells; the limiter of cell c depends only on its
// two slopes dq(c) = q(c) - q(c-1) and dq(c+1), and gives both the state of
// c on its lower face (dqp(c), for face c) and on its upper face (dqm(c+1),
// for face c+1) from one sensor (limit_i/j/k, src/flux.f90:3472-3888, where
// the two sensors of a cell are the same expression).  So a thread that
// walks a line evaluates each cell's sensor once instead of twice and loads
// each cell once instead of four times:
//
//   d = 2, 3   lanes along i (coalesced), each thread marches along j or k
//              over a segment of faces, carrying two cells, one slope and
//              the pending dqm;
//   d = 1      lanes along i as well: lane l owns cell c = i0 - 1 + l, gets
//              the neighbouring cells through L1, and passes its dqm(c+1) to
//              lane l + 1 with a warp shuffle; lanes 1..31 compute faces
//              i0 .. i0 + 30.
//
// The stage input holds conservative interior cells and primitive halo
// cells (k_halo); interior cells are converted on load (c2p5_nr) with the
// positivity test of bprtest, so no primitive copy of the state is made.
// The viscous path, which needs that copy anyway, reads it instead.
//
// FP64: the same device functions and operation order as k_faces (bit for
// bit).  MIXED: slopes are FP64 differences rounded to FP32, the limiter
// and the whole Roe flux run in FP32, and the flux enters FP64 as
//     F = ds * ( g(q_L cell) + [ (Dg_L + Dg_R)/2 - |A| dq / 2 ] )
// with g(q) = f(q).n the unit-normal flux of the left cell's FP64 state and
// Dg_X = g(q_X) - g(q_L cell) the exact change of g to the FP32 face state
// X, expanded so that every FP32 term is proportional to the differences:
// the FP32 rounding error scales with the local jumps, not with the state.
#pragma once
#include "split.cuh"

// one warp's share of a face family: d = 1: rows j = ta .. ta + nf - 1 at
// k = tb, lanes cells i0 - 1 + lane; d = 2: lanes i = i0 + lane, k = tb, faces
// j = f0 .. f0 + nf - 1; d = 3: lanes i = i0 + lane, j = tb, faces k = f0 ..
// f0 + nf - 1
struct FaceTask {
  int blk, d, n, i0, ta, tb, f0, nf;
};

// FP32 limiter of one cell (the mixed path's counterpart of limit_cell64):
// from the slopes a = dq(c), b = dq(c+1), dqp(c) and dqm(c+1), limit_face's
// algebra with fast division; ilim 1, 2 and 4 share their sensor
__device__ __forceinline__ void limit_cell32(int ilim, float eps, float rkap, float a, float b, float &dqp,
                                             float &dqm) {
  if (ilim == 1) {
    const float s = __fdividef(2.0f * b * a + eps, b * b + a * a + eps);
    const float rkp = 1.0f + rkap * s, rkm = 1.0f - rkap * s;
    dqp = -s * (rkp * a + rkm * b) * 0.25f;
    dqm = s * (rkm * a + rkp * b) * 0.25f;
  } else if (ilim == 0) {
    const float rkp = 1.0f + rkap, rkm = 1.0f - rkap;
    dqp = -(rkp * a + rkm * b) * 0.25f;
    dqm = (rkm * a + rkp * b) * 0.25f;
  } else if (ilim == 2) {
    const float rkp = 1.0f + rkap, rkm = 1.0f - rkap;
    const float bb = (3.0f - rkap) / (1.0f - rkap);
    const float sg = (copysignf(1.0f, a) + copysignf(1.0f, b)) * 0.5f;
    const float dqmx = sg * fminf(fabsf(a), fabsf(b) * bb);
    const float dqpx = sg * fminf(fabsf(b), fabsf(a) * bb);
    dqp = -(rkp * dqmx + rkm * dqpx) * 0.25f;
    dqm = (rkm * dqmx + rkp * dqpx) * 0.25f;
  } else if (ilim == 3) {
    const float epsq = eps * eps;
    dqp = -0.5f * __fdividef(a * (b * b + 2.0f * epsq) + b * (2.0f * (a * a) + epsq),
                             2.0f * (a * a) - a * b + 2.0f * (b * b) + 3.0f * epsq);
    dqm = 0.5f * __fdividef(b * (a * a + 2.0f * epsq) + a * (2.0f * (b * b) + epsq),
                            2.0f * (b * b) - b * a + 2.0f * (a * a) + 3.0f * epsq);
  } else {  // ilim == 4
    const float epsq = eps * eps;
    const float x = __fdividef(b * (a * a + epsq) + a * (b * b + epsq), b * b + a * a + 2.0f * epsq);
    dqp = -0.5f * x;
    dqm = 0.5f * x;
  }
}

// g(q) . n of a primitive state (rho, u, v, w, p) in FP64: the unit-normal
// Euler flux roflux_b builds from each face state (src/flux.f90:119-136)
// (MV: relative to a face moving with normal speed ubn, src/flux.f90:122-148)
template <bool MV>
__device__ __forceinline__ void unit_flux64(double g_gm1, double kx, double ky, double kz, const double *q, double *g,
                                            double ubn) {
  const double un = MV ? q[1] * kx + q[2] * ky + q[3] * kz - ubn : q[1] * kx + q[2] * ky + q[3] * kz;
  const double ru = q[0] * un;
  const double e = g_gm1 * q[4] + q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / 2;
  g[0] = ru;
  g[1] = ru * q[1] + q[4] * kx;
  g[2] = ru * q[2] + q[4] * ky;
  g[3] = ru * q[3] + q[4] * kz;
  g[4] = MV ? e * un + q[4] * ubn : e * un;
}

// base quantities of the FP32 expansions for the left cell: the state, its
// q^2 and E = G p + rho q^2 / 2 (rho h0)
struct Base32 {
  float r, u, v, w, p, q2, e;
};
__device__ __forceinline__ Base32 make_base32(float g_gm1, const float *b) {
  Base32 o;
  o.r = b[0]; o.u = b[1]; o.v = b[2]; o.w = b[3]; o.p = b[4];
  o.q2 = o.u * o.u + o.v * o.v + o.w * o.w;
  o.e = g_gm1 * o.p + 0.5f * o.r * o.q2;
  return o;
}

// Dg = g(base + d) - g(base) for the unit normal (kx, ky, kz), exactly
// rearranged so every term carries a factor of the difference d:
//   D(rho U)     = drho U + rho' dU
//   D(rho u U)   = D(rho U) u' + rho U du          (+ dp kx)
//   D(E)         = G dp + (drho q'^2 + rho (q'^2 - q^2)) / 2
//   D(E U)       = D(E) U' + E dU
// with primes for base + d and U = u.n
// (U is the normal velocity relative to the face; MV adds the change of the
// energy flux's p ubn term)
template <bool MV>
__device__ __forceinline__ void delta_flux32(float g_gm1, const Base32 &B, float U, float rU, float kx, float ky,
                                             float kz, const float *d, float *dg, float ubn) {
  const float dU = d[1] * kx + d[2] * ky + d[3] * kz;
  const float r1 = B.r + d[0], U1 = U + dU;
  const float u1 = B.u + d[1], v1 = B.v + d[2], w1 = B.w + d[3];
  const float drU = d[0] * U + r1 * dU;
  dg[0] = drU;
  dg[1] = drU * u1 + rU * d[1] + d[4] * kx;
  dg[2] = drU * v1 + rU * d[2] + d[4] * ky;
  dg[3] = drU * w1 + rU * d[3] + d[4] * kz;
  const float dq2 = d[1] * (B.u + u1) + d[2] * (B.v + v1) + d[3] * (B.w + w1);
  const float de = g_gm1 * d[4] + 0.5f * (d[0] * (B.q2 + dq2) + B.r * dq2);
  dg[4] = MV ? de * U1 + B.e * dU + d[4] * ubn : de * U1 + B.e * dU;
}

// Roe dissipation |A| (qR - qL) of roflux_b (src/flux.f90:137-230) in FP32
// from the FP32 face states and their jump dq (computed from differences)
template <bool MV>
__device__ __forceinline__ void roe_diss32(const PhysPar &P, float g, float g_gm1, float kx, float ky, float kz,
                                           const float *qr, const float *ql, const float *dq, float *df, float ubn) {
  const float rsr = rsqrtf(qr[0]), rsl = rsqrtf(ql[0]);
  const float h0r = g_gm1 * qr[4] * (rsr * rsr) + 0.5f * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
  const float h0l = g_gm1 * ql[4] * (rsl * rsl) + 0.5f * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
  const float rhols = ql[0] * rsl, rhors = qr[0] * rsr;
  const float rho = rhols * rhors;
  const float rden = __fdividef(1.0f, rhols + rhors);
  const float u = (rhols * ql[1] + rhors * qr[1]) * rden;
  const float v = (rhols * ql[2] + rhors * qr[2]) * rden;
  const float w = (rhols * ql[3] + rhors * qr[3]) * rden;
  const float un = u * kx + v * ky + w * kz;
  const float h0 = (rhols * h0l + rhors * h0r) * rden;
  const float q2 = u * u + v * v + w * w;
  const float a2 = (g - 1.0f) * (h0 - 0.5f * q2);
  const float ria = rsqrtf(a2);
  const float a = a2 * ria;
  const float drho = dq[0], du = dq[1], dv = dq[2], dw = dq[3], dp = dq[4];
  const float dun = du * kx + dv * ky + dw * kz;
  const float unr = MV ? un - ubn : un;  // normal velocity relative to the face
  float rm123 = fabsf(unr), rm4 = fabsf(unr + a), rm5 = fabsf(unr - a);
  if (P.efx_setup_f) {
    float rdelta = (float)P.cntrpy_f * ((float)P.w1 * (float)P.entfxctf_f + (float)P.w2 * (sqrtf(q2) + a) +
                                        (float)P.w3 * 0.2f * (fabsf(un) + a + (MV ? fabsf(ubn) : 0.0f)));
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
  const float dpa2 = dp * (ria * ria), rdua = rho * dun * ria;
  const float al1 = rm123 * (drho - dpa2);
  const float al2 = rm123 * rho;
  const float al3 = rm4 * (dpa2 + rdua) * 0.5f;
  const float al4 = rm5 * (dpa2 - rdua) * 0.5f;
  df[0] = al1 + al3 + al4;
  df[1] = al1 * u + al2 * (du - dun * kx) + al3 * (u + a * kx) + al4 * (u - a * kx);
  df[2] = al1 * v + al2 * (dv - dun * ky) + al3 * (v + a * ky) + al4 * (v - a * ky);
  df[3] = al1 * w + al2 * (dw - dun * kz) + al3 * (w + a * kz) + al4 * (w - a * kz);
  df[4] = al1 * (q2 * 0.5f) + al2 * (u * du + v * dv + w * dw - un * dun) + al3 * (h0 + a * un) +
          al4 * (h0 - a * un);
}

// mixed-precision face flux between cells L (FP64 state qL64, FP32 copy bL)
// and R (FP32 copy bR): dqL / dqR the FP32 offsets of the face states from
// their cells, dLR = (float)(qR64 - qL64)
template <bool MV>
__device__ __forceinline__ void face_flux_mixed(const PhysPar &P, float g, float g_gm1, const double *met,
                                                const double *qL64, const float *bL, const float *bR,
                                                const float *dLR, const float *dqL, const float *dqR,
                                                double *F, double ubn = 0.0) {
  const double kx = met[0], ky = met[1], kz = met[2], ds = met[3];
  const float fkx = (float)kx, fky = (float)ky, fkz = (float)kz, fub = (float)ubn;
  double g64[5];
  unit_flux64<MV>(P.g_gm1, kx, ky, kz, qL64, g64, ubn);
  const Base32 B = make_base32(g_gm1, bL);
  const float U = MV ? B.u * fkx + B.v * fky + B.w * fkz - fub : B.u * fkx + B.v * fky + B.w * fkz;
  const float rU = B.r * U;
  float dLs[5], dRs[5], ql[5], qr[5], jump[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    dLs[m] = dqL[m];              // face state L - cell L
    dRs[m] = dLR[m] + dqR[m];     // face state R - cell L
    ql[m] = bL[m] + dqL[m];
    qr[m] = bR[m] + dqR[m];
    jump[m] = dRs[m] - dLs[m];    // face state R - face state L
  }
  float dgl[5], dgr[5], df[5];
  delta_flux32<MV>(g_gm1, B, U, rU, fkx, fky, fkz, dLs, dgl, fub);
  delta_flux32<MV>(g_gm1, B, U, rU, fkx, fky, fkz, dRs, dgr, fub);
  roe_diss32<MV>(P, g, g_gm1, fkx, fky, fkz, qr, ql, jump, df, fub);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    const float t = 0.5f * (dgl[m] + dgr[m] - df[m]);
    F[m] = (g64[m] + (double)t) * ds;
  }
}

// per-slope doubling on strong-boundary faces (muscl_b*, src/flux.f90:1318-1406)
__device__ __forceinline__ bool dbl_at(int s, int mx, bool slo, bool shi) {
  return (s == 1 && slo) || (s == mx && shi);
}

// scheme constants of k_faces_line, passed by value: kernel parameters sit in
// the constant bank, where FP64 instructions read them as operands instead
// of holding them in registers across the marching loop
struct LinePar {
  PhysPar ph;
  double gamma, qmin_rho, qmin_p;
  int S, S2, hbmove;
};
inline LinePar make_line_par(const cosa_params &P) {
  LinePar o;
  o.ph = make_phys(P);
  o.gamma = P.gamma; o.qmin_rho = P.qmin[0]; o.qmin_p = P.qmin[4];
  o.S = 2 * P.nharms + 1; o.S2 = 2 * P.nharms * P.hbmove + 1; o.hbmove = P.hbmove;
  return o;
}

// state of cell c of a face line: conservative interior cells are converted
// (with bprtest's positivity test), halo cells are primitive already
template <bool CONV>
__device__ __forceinline__ void conv_cell(bool interior, const LinePar &LP, int &st, double *v) {
  if (CONV && interior) {
    c2p5_nr(LP.gamma, v);
    if (v[4] <= LP.qmin_p) st |= COSA_ERR_NEG_P;
    else if (v[0] <= LP.qmin_rho) st |= COSA_ERR_NEG_RHO;
  }
}
__device__ __forceinline__ void raw_cell(const double *__restrict__ p, int64_t P3, double *v) {
#pragma unroll
  for (int m = 0; m < 5; ++m) v[m] = __ldg(p + m * P3);
}
template <bool CONV>
__device__ __forceinline__ void load_cell(const double *__restrict__ p, int64_t P3, bool interior, const LinePar &LP,
                                          int &st, double *v) {
  raw_cell(p, P3, v);
  conv_cell<CONV>(interior, LP, st, v);
}

// the two FP64 face states of a face from its cells L, R and the offsets
// dqm (of L) and dqp (of R); first order takes the cells; the strong-boundary
// overrides (rare: the first and last face of a line) take one cell for both
__device__ __forceinline__ void face_states64(bool fo, bool ovr_lo, bool ovr_hi, const double *qL, const double *qR,
                                              const double *dqm, const double *dqp, double *ql, double *qr) {
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    if (fo) { qr[m] = qR[m]; ql[m] = qL[m]; }
    else { qr[m] = __dadd_rn(qR[m], dqp[m]); ql[m] = __dadd_rn(qL[m], dqm[m]); }
  }
  if (ovr_lo | ovr_hi) {
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const double v = ovr_lo ? qL[m] : qR[m];
      qr[m] = v; ql[m] = v;
    }
  }
}
// the mixed path's offsets of the face states from their cells (dqL from
// cell L, dqR from cell R) with the overrides; dlr = q_R - q_L
__device__ __forceinline__ void face_offsets32(bool ovr_lo, bool ovr_hi, const float *dlr, const float *dqm,
                                               const float *dqp, float *dqL, float *dqR) {
#pragma unroll
  for (int m = 0; m < 5; ++m) { dqL[m] = dqm[m]; dqR[m] = dqp[m]; }
  if (ovr_lo | ovr_hi) {
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      if (ovr_lo) { dqL[m] = 0.0f; dqR[m] = -dlr[m]; }  // both states = cell L
      else { dqL[m] = dlr[m]; dqR[m] = 0.0f; }          // both states = cell R
    }
  }
}
__device__ __forceinline__ void ld_met(const double *__restrict__ sp, double *m4) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(sp));
  const double2 c = __ldg(reinterpret_cast<const double2 *>(sp + 2));
  m4[0] = a.x; m4[1] = a.y; m4[2] = c.x; m4[3] = c.y;
}

// Grid: one CTA of 128 threads per 4 tasks (warp w takes task 4 blockIdx.x + w).
// q: the stage input (CONV) or its primitive copy; face fluxes of family d
// into cf + (d-1) n0 5 S (F0 layout per family).  IFAM: the tasks are i-face
// tasks (d = 1), else marching tasks (d = 2, 3); separate instantiations keep
// the register allocation of each to its own code.  The next row's (IFAM) or
// the next step's cells and face metrics are loaded one step ahead, and all
// addresses advance by constant strides.
// normal speed of face e (its metric record index p2_idx / 4) of family d:
// sijk(5)*kx + sijk(6)*ky + sijk(7)*kz, roflux_b's order (src/flux.f90:110-113)
__device__ __forceinline__ double face_ubn(const double *__restrict__ fv, int64_t rec, double kx, double ky,
                                           double kz) {
  const double *v = fv + rec * 3;
  return __ldg(v) * kx + __ldg(v + 1) * ky + __ldg(v + 2) * kz;
}

#ifndef COSA_LINE_MINB64
#define COSA_LINE_MINB64 3  // resident CTAs per SM the FP64 instantiations are compiled for
#endif
template <bool MIXED, bool CONV, bool IFAM, bool MV = false>
__global__ void __launch_bounds__(128, MIXED ? 4 : COSA_LINE_MINB64)
k_faces_line(const DevBlock *__restrict__ blocks, const FaceTask *__restrict__ tasks, int ntasks,
             const LinePar LP, const double *__restrict__ q, const double *__restrict__ si,
             const double *__restrict__ sj, const double *__restrict__ sk, const uint8_t *__restrict__ strong,
             const StrongMap *__restrict__ smap, int first_order, int64_t n0, double *__restrict__ cf,
             int *status, FaceVel FV = FaceVel{{nullptr, nullptr, nullptr}}) {
  const int wid = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (wid >= ntasks) return;
  const FaceTask T = tasks[wid];
  const DevBlock b = blocks[T.blk];
  const PhysPar &ph = LP.ph;
  const float g32 = (float)ph.g, gg32 = (float)ph.g_gm1, eps32 = (float)ph.epslimf, rk32 = (float)ph.rkap;
  const int S = LP.S, S2 = LP.S2;
  const int d = T.d, n = T.n, nh = n * LP.hbmove;
  const double *s = d == 1 ? si : (d == 2 ? sj : sk);
  double *F0 = cf + (int64_t)(d - 1) * n0 * 5 * S;
  const StrongMap sm = smap[T.blk];
  const int mx = d == 1 ? b.im : (d == 2 ? b.jm : b.km);
  const double *qv = q + p3_var(b, 5, S, 1, n);
  const int64_t fv = (int64_t)b.im * b.jm * b.km;  // variable stride of the F0 face arrays
  const bool fo = first_order != 0;
  int st = 0;

  if (IFAM) {
    // lane l: cell c = i0 - 1 + l of rows j = ta .., k = tb; faces c for lanes
    // 1..31.  Lanes past the line (c > mx) read cell mx's stencil and store nothing.
    const int k = T.tb, c = T.i0 - 1 + lane, cl = min(c, mx);
    const bool face = lane >= 1 && c >= 1 && c <= mx;
    const bool in_m = cl - 1 >= 1 && cl - 1 <= mx - 1, in_0 = cl >= 1 && cl <= mx - 1,
               in_p = cl + 1 >= 1 && cl + 1 <= mx - 1;
    const double *pc = qv + p3_cell(b, cl, T.ta, k);
    const double *sp = s + p2_idx(b, S2, 1, cl, T.ta, k, nh);
    const double *vp = MV ? FV.f[0] + p2_idx(b, S2, 1, cl, T.ta, k, nh) / 4 * 3 : nullptr;
    double *Fp = F0 + f0_idx(b, 5, S, max(cl, 1), T.ta, k, 1, n);  // lane 0 stores nothing
    const int64_t qrow = b.I3, mrow = (int64_t)(b.im + 2) * 4, frow = b.im;
    double A[3][5], met[4];
    raw_cell(pc - 1, b.P3, A[0]); raw_cell(pc, b.P3, A[1]); raw_cell(pc + 1, b.P3, A[2]);
    ld_met(sp, met);
    for (int row = 0; row < T.nf; ++row) {
      const int j = T.ta + row;
      conv_cell<CONV>(in_m, LP, st, A[0]);
      conv_cell<CONV>(in_0, LP, st, A[1]);
      conv_cell<CONV>(in_p, LP, st, A[2]);
      // the next row (the last row reloads itself: in bounds, unused)
      const int64_t nx = row + 1 < T.nf ? 1 : 0;
      double B[3][5], metn[4];
      raw_cell(pc + nx * qrow - 1, b.P3, B[0]); raw_cell(pc + nx * qrow, b.P3, B[1]);
      raw_cell(pc + nx * qrow + 1, b.P3, B[2]);
      ld_met(sp + nx * mrow, metn);
      const bool slo = strong_at(strong, sm, 0, 0, j, k), shi = strong_at(strong, sm, 0, 1, j, k);
      const bool dlo = dbl_at(c, mx, slo, shi), dhi = dbl_at(c + 1, mx, slo, shi);
      const bool ovr_lo = c == 1 && slo, ovr_hi = c == mx && shi;
      double Fv[5];
      if (!MIXED) {
        double dqp[5], dqmn[5], dqm[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          double a = A[1][m] - A[0][m], bb = A[2][m] - A[1][m];
          if (dlo) a = (A[1][m] - A[0][m]) * 2;
          if (dhi) bb = (A[2][m] - A[1][m]) * 2;
          if (!fo) limit_cell64(ph.ilimf, ph.epslimf, ph.rkap, a, bb, dqp[m], dqmn[m]);
          else { dqp[m] = 0.0; dqmn[m] = 0.0; }
          dqm[m] = __shfl_up_sync(0xffffffffu, dqmn[m], 1);
        }
        double qr[5], ql[5];
        face_states64(fo, ovr_lo, ovr_hi, A[0], A[1], dqm, dqp, ql, qr);
        if (face) {
          const double ubn = MV ? face_ubn(vp, 0, met[0], met[1], met[2]) : 0.0;
          roe_flux_euler<MV>(ph, met[0], met[1], met[2], met[3], qr, ql, Fv, ubn);
        }
      } else {
        float dqp[5], dqmn[5], dqm[5], b0[5], bm1[5], dlr[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          const float a = (float)(A[1][m] - A[0][m]), bb = (float)(A[2][m] - A[1][m]);
          dlr[m] = a;
          b0[m] = (float)A[1][m];
          bm1[m] = (float)A[0][m];
          if (!fo) limit_cell32(ph.ilimf, eps32, rk32, dlo ? a * 2.0f : a, dhi ? bb * 2.0f : bb, dqp[m], dqmn[m]);
          else { dqp[m] = 0.0f; dqmn[m] = 0.0f; }
          dqm[m] = __shfl_up_sync(0xffffffffu, dqmn[m], 1);
        }
        float dqL[5], dqR[5];
        face_offsets32(ovr_lo, ovr_hi, dlr, dqm, dqp, dqL, dqR);
        if (face) {
          const double ubn = MV ? face_ubn(vp, 0, met[0], met[1], met[2]) : 0.0;
          face_flux_mixed<MV>(ph, g32, gg32, met, A[0], bm1, b0, dlr, dqL, dqR, Fv, ubn);
        }
      }
      if (face) {
#pragma unroll
        for (int m = 0; m < 5; ++m) Fp[m * fv] = Fv[m];
      }
#pragma unroll
      for (int m = 0; m < 5; ++m) { A[0][m] = B[0][m]; A[1][m] = B[1][m]; A[2][m] = B[2][m]; }
#pragma unroll
      for (int m = 0; m < 4; ++m) met[m] = metn[m];
      pc += qrow; sp += mrow; Fp += frow;
      if (MV) vp += mrow / 4 * 3;
    }
  } else {
    // lanes along i; march along d over faces f0 .. f0 + nf - 1
    const int i = T.i0 + lane;
    if (i <= b.im - 1) {
      const int tb = T.tb;
      // transverse cell indices of the line for strong_at: (i, k) for d = 2, (i, j) for d = 3
      const bool slo = strong_at(strong, sm, d - 1, 0, i, tb), shi = strong_at(strong, sm, d - 1, 1, i, tb);
      const int64_t step = d == 2 ? (int64_t)b.I3 : (int64_t)b.I3 * b.J3;
      const int64_t mstep = d == 2 ? (int64_t)(b.im + 2) * 4 : (int64_t)(b.im + 2) * (b.jm + 2) * 4;
      const int64_t fstep = d == 2 ? (int64_t)b.im : (int64_t)b.im * b.jm;
      const int f0 = T.f0, f1 = T.f0 + T.nf;
      const double *p = qv + (d == 2 ? p3_cell(b, i, f0 - 2, tb) : p3_cell(b, i, tb, f0 - 2));
      const double *sp = s + (d == 2 ? p2_idx(b, S2, 1, i, f0, tb, nh) : p2_idx(b, S2, 1, i, tb, f0, nh));
      double *Fp = F0 + (d == 2 ? f0_idx(b, 5, S, i, f0, tb, 1, n) : f0_idx(b, 5, S, i, tb, f0, 1, n));
      const double *vp = MV ? FV.f[d - 1] + (sp - s) / 4 * 3 : nullptr;  // face velocity of face f0
      auto inner = [&](int cc) { return cc >= 1 && cc <= mx - 1; };
      double qa[5], qb[5], qc[5];
      load_cell<CONV>(p, b.P3, inner(f0 - 2), LP, st, qa);
      load_cell<CONV>(p + step, b.P3, inner(f0 - 1), LP, st, qb);
      load_cell<CONV>(p + 2 * step, b.P3, inner(f0), LP, st, qc);
      // cell f + 1 and the metrics of face f + 1 are loaded one step ahead
      // (the cell converted when its step comes): step f reads cell
      // min(f + 2, mx + 1) (the last halo layer) and face f + 1 <= mx + 1
      double qn[5], met[4];
      raw_cell(p + 3 * step, b.P3, qn);
      ld_met(sp, met);
      p += 4 * step;
      sp += mstep;
      // carried: qb = cell f-1, qc = cell f, dqm(f) (the slopes are taken
      // again from the cells: fewer live registers)
      if (!MIXED) {
        double dqm[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          double a = qb[m] - qa[m], bb = qc[m] - qb[m];
          if (dbl_at(f0 - 1, mx, slo, shi)) a = (qb[m] - qa[m]) * 2;
          if (dbl_at(f0, mx, slo, shi)) bb = (qc[m] - qb[m]) * 2;
          double unused;
          if (!fo) limit_cell64(ph.ilimf, ph.epslimf, ph.rkap, a, bb, unused, dqm[m]);
          else dqm[m] = 0.0;
        }
        for (int f = f0; f < f1; ++f) {
          conv_cell<CONV>(inner(f + 1), LP, st, qn);
          double qx[5], metn[4];
          raw_cell(f + 2 <= mx + 1 ? p : p - step, b.P3, qx);
          ld_met(sp, metn);
          p += step;
          sp += mstep;
          const bool dl = dbl_at(f, mx, slo, shi), dh = dbl_at(f + 1, mx, slo, shi);
          const bool ovr_lo = f == 1 && slo, ovr_hi = f == mx && shi;
          double dqp[5], dqmn[5];
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            double a = qc[m] - qb[m], bb = qn[m] - qc[m];
            if (dl) a = (qc[m] - qb[m]) * 2;
            if (dh) bb = (qn[m] - qc[m]) * 2;
            if (!fo) limit_cell64(ph.ilimf, ph.epslimf, ph.rkap, a, bb, dqp[m], dqmn[m]);
            else { dqp[m] = 0.0; dqmn[m] = 0.0; }
          }
          double qr[5], ql[5], Fv[5];
          face_states64(fo, ovr_lo, ovr_hi, qb, qc, dqm, dqp, ql, qr);
          const double ubn = MV ? face_ubn(vp, 0, met[0], met[1], met[2]) : 0.0;
          roe_flux_euler<MV>(ph, met[0], met[1], met[2], met[3], qr, ql, Fv, ubn);
          if (MV) vp += mstep / 4 * 3;
#pragma unroll
          for (int m = 0; m < 5; ++m) Fp[m * fv] = Fv[m];
          Fp += fstep;
#pragma unroll
          for (int m = 0; m < 5; ++m) { qb[m] = qc[m]; qc[m] = qn[m]; qn[m] = qx[m]; dqm[m] = dqmn[m]; }
#pragma unroll
          for (int m = 0; m < 4; ++m) met[m] = metn[m];
        }
      } else {
        float sB[5], dqm[5], fb[5], fc[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          const float a = (float)(qb[m] - qa[m]), bb = (float)(qc[m] - qb[m]);
          sB[m] = bb;
          fb[m] = (float)qb[m]; fc[m] = (float)qc[m];
          float unused;
          if (!fo)
            limit_cell32(ph.ilimf, eps32, rk32, dbl_at(f0 - 1, mx, slo, shi) ? a * 2.0f : a,
                         dbl_at(f0, mx, slo, shi) ? bb * 2.0f : bb, unused, dqm[m]);
          else dqm[m] = 0.0f;
        }
        for (int f = f0; f < f1; ++f) {
          conv_cell<CONV>(inner(f + 1), LP, st, qn);
          double qx[5], metn[4];
          raw_cell(f + 2 <= mx + 1 ? p : p - step, b.P3, qx);
          ld_met(sp, metn);
          p += step;
          sp += mstep;
          const bool dl = dbl_at(f, mx, slo, shi), dh = dbl_at(f + 1, mx, slo, shi);
          const bool ovr_lo = f == 1 && slo, ovr_hi = f == mx && shi;
          float dqp[5], dqmn[5], bbv[5];
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            const float bb = (float)(qn[m] - qc[m]);
            bbv[m] = bb;
            if (!fo) limit_cell32(ph.ilimf, eps32, rk32, dl ? sB[m] * 2.0f : sB[m], dh ? bb * 2.0f : bb, dqp[m],
                                  dqmn[m]);
            else { dqp[m] = 0.0f; dqmn[m] = 0.0f; }
          }
          // sB = (float)(q(f) - q(f-1)), undoubled
          float dqL[5], dqR[5];
          face_offsets32(ovr_lo, ovr_hi, sB, dqm, dqp, dqL, dqR);
          double Fv[5];
          const double ubn = MV ? face_ubn(vp, 0, met[0], met[1], met[2]) : 0.0;
          face_flux_mixed<MV>(ph, g32, gg32, met, qb, fb, fc, sB, dqL, dqR, Fv, ubn);
          if (MV) vp += mstep / 4 * 3;
#pragma unroll
          for (int m = 0; m < 5; ++m) Fp[m * fv] = Fv[m];
          Fp += fstep;
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            qb[m] = qc[m]; qc[m] = qn[m]; qn[m] = qx[m];
            fb[m] = fc[m]; fc[m] = (float)qc[m];
            sB[m] = bbv[m];
            dqm[m] = dqmn[m];
          }
#pragma unroll
          for (int m = 0; m < 4; ++m) met[m] = metn[m];
        }
      }
    }
  }
  if (st && status) atomicOr(status, st);
}
