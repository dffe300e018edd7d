// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of COSA's explicit residual-and-update hot path
// (LANCASTER-CFD/COSA, Fortran 90), used by tests/ as the parity checker
// and by bench.py's cpu_baseline / --impl reference leg as the timed CPU
// implementation.  Nothing in the product (cosa_b200/) links or calls it.
//
// COSA itself cannot be compiled here (no Fortran compiler; it also needs
// CGNS, TecIO and LAPACK), so this file restates the reference routines
// loop for loop, keeping their operation order and parenthesisation so
// that an FP64 build with -ffp-contract=off reproduces the reference's
// rounding.  Each function cites the Fortran it follows.  The reference
// ships no tests, inputs or golden vectors for this path, so the only
// pins are the known-answer tests in tests/test_oracle_kat.py (Roe
// consistency, free-stream preservation, conservation, symmetry, limiter
// hand values) -- "parity unpinned" against a running reference.
//
// Array layout is the reference's: column-major, i fastest, per-block
// arrays concatenated with the setoffs() offsets (src/input.f90:5502-5585).

#include "../include/cosa_gpu.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Level {
  int nb = 0, npde = 5, S = 1, lmet = 4, dim5h = 1;
  // moving grids (harmonic balance of a pitching body): face velocities of
  // the three families (3 components per face, the reference's sijk(5:7),
  // P2 x dim5h layout) and cell-centred grid velocities (the node arrays
  // xdot, ydot, zdot after vert2cell_g); null on fixed grids
  const double *fv[3] = {nullptr, nullptr, nullptr};
  const double *cv[3] = {nullptr, nullptr, nullptr};
  std::vector<int> im, jm, km, nbcs;
  std::vector<int64_t> op3, op2, op1, of0, om1, obct;
  std::vector<int> bct;   // 10 * sum(nbcs)
  int ncuts = 0;
  std::vector<int> cut;   // 21 * ncuts
  int64_t n3 = 0, n2 = 0, n1 = 0, n0 = 0, nm1 = 0;
};

// cyc / krd tables of input() (src/input.f90:2409-2410), 1-based
inline int cyc(int idir, int m) {
  static const int t[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};
  return t[idir - 1][m - 1];
}
inline int krd(int a, int b) { return a == b ? 1 : 0; }

// ---- per-block views -------------------------------------------------------
struct B3 {  // (-1:im+1,-1:jm+1,-1:km+1, npde, 0:S-1)
  double *p; int I, J, K; int64_t P; int npde;
  B3(double *base, const Level &L, int b)
      : I(L.im[b] + 3), J(L.jm[b] + 3), K(L.km[b] + 3), npde(L.npde) {
    P = (int64_t)I * J * K;
    p = base + L.op3[b] * L.npde * L.S;
  }
  inline double &operator()(int i, int j, int k, int v, int n) const {
    return p[((int64_t)n * npde + (v - 1)) * P + (i + 1) + (int64_t)I * ((j + 1) + (int64_t)J * (k + 1))];
  }
};
struct B3s {  // scalar P3 (-1:im+1,...,0:S-1) (mut, pr)
  double *p; int I, J, K; int64_t P;
  B3s(double *base, const Level &L, int b) : I(L.im[b] + 3), J(L.jm[b] + 3), K(L.km[b] + 3) {
    P = (int64_t)I * J * K;
    p = base + L.op3[b] * L.S;
  }
  inline double &operator()(int i, int j, int k, int n) const {
    return p[(int64_t)n * P + (i + 1) + (int64_t)I * ((j + 1) + (int64_t)J * (k + 1))];
  }
};
struct B2 {  // (lmet, 0:im+1, 0:jm+1, 0:km+1, 0:dim5h-1)
  const double *p; int I, J, K, lmet; int64_t P;
  B2(const double *base, const Level &L, int b)
      : I(L.im[b] + 2), J(L.jm[b] + 2), K(L.km[b] + 2), lmet(L.lmet) {
    P = (int64_t)I * J * K;
    p = base + L.op2[b] * L.lmet * L.dim5h;
  }
  inline double operator()(int c, int i, int j, int k, int nh) const {
    return p[((int64_t)nh * P + i + (int64_t)I * (j + (int64_t)J * k)) * lmet + (c - 1)];
  }
};
struct B2w {  // writable metric view
  double *p; int I, J, K, lmet; int64_t P;
  B2w(double *base, const Level &L, int b)
      : I(L.im[b] + 2), J(L.jm[b] + 2), K(L.km[b] + 2), lmet(L.lmet) {
    P = (int64_t)I * J * K;
    p = base + L.op2[b] * L.lmet * L.dim5h;
  }
  inline double &operator()(int c, int i, int j, int k, int nh) const {
    return p[((int64_t)nh * P + i + (int64_t)I * (j + (int64_t)J * k)) * lmet + (c - 1)];
  }
};
struct BG {  // grid (0:im+1, 0:jm+1, 0:km+1)
  const double *p; int I, J;
  BG(const double *base, const Level &L, int b) : I(L.im[b] + 2), J(L.jm[b] + 2) {
    p = base + L.op2[b];
  }
  inline double operator()(int i, int j, int k) const {
    return p[i + (int64_t)I * (j + (int64_t)J * k)];
  }
};
struct BGs {  // node array of snapshot nh: (0:im+1, 0:jm+1, 0:km+1, 0:dim5h-1)
  double *p; int I, J;
  BGs(const double *base, const Level &L, int b, int nh) : I(L.im[b] + 2), J(L.jm[b] + 2) {
    p = const_cast<double *>(base) + L.op2[b] * L.dim5h + (int64_t)nh * I * J * (L.km[b] + 2);
  }
  inline double &operator()(int i, int j, int k) const { return p[i + (int64_t)I * (j + (int64_t)J * k)]; }
};
struct BFv {  // face velocities (3, 0:im+1, 0:jm+1, 0:km+1, 0:dim5h-1)
  double *p; int I, J, K; int64_t P;
  BFv(const double *base, const Level &L, int b)
      : I(L.im[b] + 2), J(L.jm[b] + 2), K(L.km[b] + 2) {
    P = (int64_t)I * J * K;
    p = const_cast<double *>(base) + L.op2[b] * 3 * L.dim5h;
  }
  inline double &operator()(int c, int i, int j, int k, int nh) const {
    return p[((int64_t)nh * P + i + (int64_t)I * (j + (int64_t)J * k)) * 3 + (c - 1)];
  }
};
// face velocity . unit normal of face (i,j,k) of family d, snapshot nh, in
// roflux_b's order: sijk(5)*kx + sijk(6)*ky + sijk(7)*kz (src/flux.f90:110-113)
inline double face_ubn(const Level &L, int b, int d, int i, int j, int k, int nh, double kx, double ky, double kz) {
  if (!L.fv[d - 1]) return 0.0;
  BFv f(L.fv[d - 1], L, b);
  return f(1, i, j, k, nh) * kx + f(2, i, j, k, nh) * ky + f(3, i, j, k, nh) * kz;
}

struct B1 {  // (0:im, 0:jm, 0:km [, 0:S-1])
  double *p; int I, J, K; int64_t P;
  B1(double *base, const Level &L, int b, int nsnap)
      : I(L.im[b] + 1), J(L.jm[b] + 1), K(L.km[b] + 1) {
    P = (int64_t)I * J * K;
    p = base + L.op1[b] * nsnap;
  }
  inline double &operator()(int i, int j, int k, int n = 0) const {
    return p[(int64_t)n * P + i + (int64_t)I * (j + (int64_t)J * k)];
  }
};
struct B0 {  // flux (im, jm, km, npde, 0:S-1), 1-based
  double *p; int I, J, K, npde; int64_t P;
  B0(double *base, const Level &L, int b) : I(L.im[b]), J(L.jm[b]), K(L.km[b]), npde(L.npde) {
    P = (int64_t)I * J * K;
    p = base + L.of0[b] * L.npde * L.S;
  }
  inline double &operator()(int i, int j, int k, int v, int n) const {
    return p[((int64_t)n * npde + (v - 1)) * P + (i - 1) + (int64_t)I * ((j - 1) + (int64_t)J * (k - 1))];
  }
};

inline bool is_kom(const cosa_params &p) { return p.kom || p.kom_bsl || p.kom_sst; }
inline bool is_blend(const cosa_params &p) { return p.kom_bsl || p.kom_sst; }

struct B3t {  // ttrm (-1:im+1,-1:jm+1,-1:km+1, 3, 0:S-1)
  double *p; int I, J; int64_t P;
  B3t(double *base, const Level &L, int b) : I(L.im[b] + 3), J(L.jm[b] + 3) {
    P = (int64_t)I * J * (L.km[b] + 3);
    p = base + L.op3[b] * 3 * L.S;
  }
  inline double &operator()(int i, int j, int k, int c, int n) const {
    return p[((int64_t)n * 3 + (c - 1)) * P + (i + 1) + (int64_t)I * ((j + 1) + (int64_t)J * (k + 1))];
  }
};
struct B0s {  // face distance (im, jm, km), 1-based
  double *p; int I, J;
  B0s(double *base, const Level &L, int b) : I(L.im[b]), J(L.jm[b]) { p = base + L.of0[b]; }
  inline double &operator()(int i, int j, int k) const {
    return p[(i - 1) + (int64_t)I * ((j - 1) + (int64_t)J * (k - 1))];
  }
};

// the BSL/SST closure constants of input() (src/input.f90:2522-2539)
struct Blend {
  double sigk1, sigk2, sigw1, sigw2, b1, b2, bstr, g1, g2, a1;
};
inline Blend blend_of(const cosa_params &P) {
  Blend c;
  c.bstr = 0.09;
  c.a1 = 0.31;
  c.sigk1 = P.kom_sst ? 0.85 : 0.5;
  c.sigk2 = 1.0;
  c.sigw1 = 0.5;
  c.b1 = 3.0 / 40.0;
  c.g1 = c.b1 / c.bstr - c.sigw1 * (P.kappa * P.kappa) / std::sqrt(c.bstr);
  c.sigw2 = 0.856;
  c.b2 = 0.0828;
  c.g2 = c.b2 / c.bstr - c.sigw2 * (P.kappa * P.kappa) / std::sqrt(c.bstr);
  return c;
}
// x**4 and the blending tanh as the reference writes them
inline double pow4(double x) { const double x2 = x * x; return x2 * x2; }
inline double tanh_ref(double a) { return (std::exp(2 * a) - 1) / (std::exp(2 * a) + 1); }

// ---- cons2prim_b (src/update.f90:2135-2188) --------------------------------
#include "lsp_oracle.inc"

void cons2prim_b(const Level &L, int b, double *qa, int xtnd, const cosa_params &P) {
  B3 q(qa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int is = 1 - xtnd, ie = im - 1 + xtnd, js = 1 - xtnd, je = jm - 1 + xtnd;
  const int ks = 1 - xtnd, ke = km - 1 + xtnd;
  const double g = P.gamma;
  const bool kom = is_kom(P);
  for (int n = 0; n < L.S; ++n)
    for (int k = ks; k <= ke; ++k)
      for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
          double rho = q(i, j, k, 1, n);
          for (int v = 2; v <= L.npde; ++v)
            if (v != 5) q(i, j, k, v, n) = q(i, j, k, v, n) / rho;
          double tke = kom ? q(i, j, k, 6, n) : 0.0;
          double u = q(i, j, k, 2, n), vv = q(i, j, k, 3, n), w = q(i, j, k, 4, n);
          double rhoe = q(i, j, k, 5, n);
          q(i, j, k, 5, n) = (g - 1) * (rhoe - rho * (u * u + vv * vv + w * w) / 2 - rho * tke);
        }
}

// ---- prim2cons_b (src/update.f90:1875-2084): interior + face halos ---------
inline void p2c_cell(B3 &q, int i, int j, int k, int n, int npde, double g, bool kom) {
  double tke = kom ? q(i, j, k, 6, n) : 0.0;
  double rho = q(i, j, k, 1, n);
  for (int v = 2; v <= npde; ++v)
    if (v != 5) q(i, j, k, v, n) = q(i, j, k, v, n) * rho;
  double rhou = q(i, j, k, 2, n), rhov = q(i, j, k, 3, n), rhow = q(i, j, k, 4, n);
  double p = q(i, j, k, 5, n);
  q(i, j, k, 5, n) = p / (g - 1) + (rhou * rhou + rhov * rhov + rhow * rhow) / 2 / rho + rho * tke;
}
void prim2cons_b(const Level &L, int b, double *qa, const cosa_params &P) {
  B3 q(qa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const double g = P.gamma;
  const bool kom = is_kom(P);
  for (int n = 0; n < L.S; ++n) {
    for (int k = 1; k <= km - 1; ++k)
      for (int j = 1; j <= jm - 1; ++j)
        for (int i = -1; i <= im + 1; ++i) p2c_cell(q, i, j, k, n, L.npde, g, kom);
    for (int k = 1; k <= km - 1; ++k)
      for (int j : {-1, 0, jm, jm + 1})
        for (int i = 1; i <= im - 1; ++i) p2c_cell(q, i, j, k, n, L.npde, g, kom);
    for (int k : {-1, 0, km, km + 1})
      for (int j = 1; j <= jm - 1; ++j)
        for (int i = 1; i <= im - 1; ++i) p2c_cell(q, i, j, k, n, L.npde, g, kom);
  }
}

// ---- boundary conditions (src/bc.f90) --------------------------------------
struct Patch {
  int bctyp, idir, inrout, istrt[4], iend[4];  // 1-based index arrays
  int ijk[4];
  int ic1, ic2, ic3;
  int blk = 0;  // block of the patch (0-based)
};
inline Patch patch_of(const int *t, int im, int jm, int km) {
  Patch pa;
  pa.bctyp = t[0]; pa.idir = t[1]; pa.inrout = t[2];
  pa.istrt[1] = t[3]; pa.iend[1] = t[4];
  pa.istrt[2] = t[5]; pa.iend[2] = t[6];
  pa.istrt[3] = t[7]; pa.iend[3] = t[8];
  pa.ijk[1] = im; pa.ijk[2] = jm; pa.ijk[3] = km;
  pa.ic1 = cyc(pa.idir, 1); pa.ic2 = cyc(pa.idir, 2); pa.ic3 = cyc(pa.idir, 3);
  return pa;
}
// index (i,j,k) of the point at normal position `nrm` and tangential (i2,i3)
inline void pidx(const Patch &pa, int nrm, int i2, int i3, int &i, int &j, int &k) {
  i = nrm * krd(pa.ic1, 1) + i2 * krd(pa.ic2, 1) + i3 * krd(pa.ic3, 1);
  j = nrm * krd(pa.ic1, 2) + i2 * krd(pa.ic2, 2) + i3 * krd(pa.ic3, 2);
  k = nrm * krd(pa.ic1, 3) + i2 * krd(pa.ic2, 3) + i3 * krd(pa.ic3, 3);
}

// bc_sym (src/bc.f90:2595-2710)
void bc_sym(const Patch &pa, B3 &q, const Level &L) {
  int ibcpt, ibcpt2, ibcn, ibcn2;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcn2 = 2; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcn2 = ibcpt - 2; }
  int isym[8];
  for (int v = 1; v <= L.npde; ++v) isym[v] = 1;
  isym[pa.idir + 1] = -1;
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, a2, b2, c2, an, bn, cn, an2, bn2, cn2;
          pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
          pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcn2, i2, i3, an2, bn2, cn2);
          q(a, bb, c, v, n) = isym[v] * q(an, bn, cn, v, n);
          q(a2, b2, c2, v, n) = isym[v] * q(an2, bn2, cn2, v, n);
        }
}

// bc_extrapol (src/bc.f90:2494-2592)
void bc_extrapol(const Patch &pa, B3 &q, const Level &L) {
  int ibcpt, ibcpt2, ibcn;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; }
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, a2, b2, c2, an, bn, cn;
          pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
          pidx(pa, ibcn, i2, i3, an, bn, cn);
          q(a, bb, c, v, n) = q(an, bn, cn, v, n);
          q(a2, b2, c2, v, n) = q(an, bn, cn, v, n);
        }
}

inline void face_normal(const Patch &pa, const B2 &si, const B2 &sj, const B2 &sk, int a,
                        int bb, int c, int nh, double &nx, double &ny, double &nz) {
  const B2 &s = pa.idir == 1 ? si : (pa.idir == 2 ? sj : sk);
  nx = s(1, a, bb, c, nh); ny = s(2, a, bb, c, nh); nz = s(3, a, bb, c, nh);
}

// bc_walinv_14 (src/bc.f90:1457-1675), fixed grid
void bc_walinv_14(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk,
                  const Level &L, const cosa_params &P) {
  int ibcpt, ibcpt2, ibcn, ibcn2, ibcm;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcn2 = 2; ibcm = 1; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcn2 = ibcpt - 2; ibcm = ibcpt; }
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int a, bb, c, a2, b2, c2, an, bn, cn, an2, bn2, cn2, am, bm, cm;
        pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
        pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcn2, i2, i3, an2, bn2, cn2);
        pidx(pa, ibcm, i2, i3, am, bm, cm);
        double nx, ny, nz;
        face_normal(pa, si, sj, sk, am, bm, cm, nh, nx, ny, nz);
        double rho1 = q(an, bn, cn, 1, n), u1 = q(an, bn, cn, 2, n), v1 = q(an, bn, cn, 3, n);
        double w1 = q(an, bn, cn, 4, n), p1 = q(an, bn, cn, 5, n);
        double rho2 = q(an2, bn2, cn2, 1, n), u2 = q(an2, bn2, cn2, 2, n), v2 = q(an2, bn2, cn2, 3, n);
        double w2 = q(an2, bn2, cn2, 4, n), p2 = q(an2, bn2, cn2, 5, n);
        double rhow = (3 * rho1 - rho2) / 2, uw = (3 * u1 - u2) / 2, vw = (3 * v1 - v2) / 2;
        double ww = (3 * w1 - w2) / 2, pw = (3 * p1 - p2) / 2;
        double un1 = u1 * nx + v1 * ny + w1 * nz;
        double un2 = u2 * nx + v2 * ny + w2 * nz;
        double unw = (3 * un1 - un2) / 2;
        if (P.moving && L.fv[pa.idir - 1]) {
          // wall face velocity (src/bc.f90:1567-1614)
          BFv f(L.fv[pa.idir - 1], L, pa.blk);
          unw = unw - (f(1, am, bm, cm, nh) * nx + f(2, am, bm, cm, nh) * ny + f(3, am, bm, cm, nh) * nz);
        }
        q(a, bb, c, 1, n) = rhow;
        q(a, bb, c, 2, n) = uw - unw * nx;
        q(a, bb, c, 3, n) = vw - unw * ny;
        q(a, bb, c, 4, n) = ww - unw * nz;
        q(a, bb, c, 5, n) = pw;
        for (int v = 1; v <= 5; ++v) q(a2, b2, c2, v, n) = q(a, bb, c, v, n);
        if (is_kom(P)) {
          q(a, bb, c, 6, n) = q(an, bn, cn, 6, n);
          q(a, bb, c, 7, n) = q(an, bn, cn, 7, n);
          q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n);
          q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
        }
      }
  }
}

// bc_insub (src/bc.f90:875-1175); total state and direction are parameters
// whose defaults are the reference's hard-wired values.
int bc_insub(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk,
             const Level &L, const cosa_params &P, int nl = 1) {
  int status = 0;
  int ibcpt, ibcpt2, ibcn, ibcn2, ibcm;
  double sgnm;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcn2 = 2; ibcm = 1; sgnm = 1.0; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcn2 = ibcpt - 2; ibcm = ibcpt; sgnm = -1.0; }
  const double g = P.gamma;
  for (int icell = 1; icell <= 2; ++icell)
    for (int n = 0; n < L.S; ++n) {
      const int nh = n * P.hbmove;
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, a2, b2, c2, an, bn, cn, an2, bn2, cn2, am, bm, cm;
          pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
          pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcn2, i2, i3, an2, bn2, cn2);
          pidx(pa, ibcm, i2, i3, am, bm, cm);
          double nx, ny, nz;
          face_normal(pa, si, sj, sk, am, bm, cm, nh, nx, ny, nz);
          nx = sgnm * nx; ny = sgnm * ny; nz = sgnm * nz;
          double rho1 = q(an, bn, cn, 1, n), rho2 = q(an2, bn2, cn2, 1, n);
          double u1 = q(an, bn, cn, 2, n), u2 = q(an2, bn2, cn2, 2, n);
          double v1 = q(an, bn, cn, 3, n), v2 = q(an2, bn2, cn2, 3, n);
          double w1 = q(an, bn, cn, 4, n), w2 = q(an2, bn2, cn2, 4, n);
          double p1 = q(an, bn, cn, 5, n), p2 = q(an2, bn2, cn2, 5, n);
          double un1 = u1 * nx + v1 * ny + w1 * nz;
          double un2 = u2 * nx + v2 * ny + w2 * nz;
          double rc1 = std::sqrt(g * p1 * rho1);
          double rc2 = std::sqrt(g * p2 * rho2);
          if (P.lomach) {
            // the preconditioned outgoing characteristic (src/bc.f90:1032-1056)
            auto rc_lsp = [&](double rho_, double u_, double v_, double w_, double p_, double un_) {
              const double q2 = u_ * u_ + v_ * v_ + w_ * w_, a2 = g * p_ / rho_, a = std::sqrt(a2);
              const double ump2 = (P.uprv / a) * (P.uprv / a);
              const double mp2 = std::min(std::max(std::max(q2 / a2, ump2), lsp_eps2(P, nl)), 1.0);
              const double lp3 = 0.5 * (un_ * (1. + mp2) + std::sqrt(un_ * un_ * ((1. - mp2) * (1. - mp2)) + 4. * a2 * mp2));
              const double esse = un_ - lp3;
              return -(rho_ * esse);
            };
            rc1 = rc_lsp(rho1, u1, v1, w1, p1, un1);
            rc2 = rc_lsp(rho2, u2, v2, w2, p2, un2);
          }
          double rcun1 = rc1 * un1, rcun2 = rc2 * un2;
          double p, un, rc, rcun;
          if (icell == 1) {
            p = 2 * p1 - p2; un = 2 * un1 - un2; rc = 2 * rc1 - rc2; rcun = 2 * rcun1 - rcun2;
          } else {
            p = 3 * p1 - 2 * p2; un = 3 * un1 - 2 * un2; rc = 3 * rc1 - 2 * rc2; rcun = 3 * rcun1 - 2 * rcun2;
          }
          double t0 = P.inlet_t0, p0 = P.inlet_p0;
          double h0inl = 1 / (g - 1) * t0;
          double sx = P.inlet_dir[0], sy = P.inlet_dir[1], sz = P.inlet_dir[2];
          double dot = sx * nx + sy * ny + sz * nz;
          double con1 = 0.5 / (h0inl * (dot * dot));
          double con2 = 2 * con1 * g / (g - 1);
          double con3 = p - rcun;
          double dun = 1.0;
          int count = 0;
          while (std::fabs(dun) > 1.0e-10) {
            count = count + 1;
            if (count == 10) { status |= COSA_ERR_INFLOW; break; }
            double par = 1.0 - con1 * (un * un);
            p = p0 * std::pow(par, g / (g - 1));
            double f = p - rc * un - con3;
            double fp = -con2 * un * p / par - rc;
            dun = -f / fp;
            un = un + dun;
          }
          p = +rc * un + con3;
          double modv = un / dot;
          double u = modv * sx, v = modv * sy, w = modv * sz;
          double rho = g * p / ((g - 1) * (h0inl - 0.5 * (modv * modv)));
          if (icell == 1) {
            q(a, bb, c, 1, n) = rho; q(a, bb, c, 2, n) = u; q(a, bb, c, 3, n) = v;
            q(a, bb, c, 4, n) = w; q(a, bb, c, 5, n) = p;
          } else {
            q(a2, b2, c2, 1, n) = rho; q(a2, b2, c2, 2, n) = u; q(a2, b2, c2, 3, n) = v;
            q(a2, b2, c2, 4, n) = w; q(a2, b2, c2, 5, n) = p;
          }
        }
    }
  if (is_kom(P))
    for (int n = 0; n < L.S; ++n)
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, a2, b2, c2;
          pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
          q(a, bb, c, 6, n) = P.tkefar; q(a, bb, c, 7, n) = P.omefar;
          q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n); q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
        }
  return status;
}

// bc_outsub (src/bc.f90:1178-1455); pressures are parameters whose defaults
// are the reference's hard-wired 0.714285714285714.
void bc_outsub(const Patch &pa, B3 &q, const Level &L, const cosa_params &P) {
  int ibcpt, ibcpt2, ibcn, ibcn2;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcn2 = 2; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcn2 = ibcpt - 2; }
  const double g = P.gamma;
  const bool kom = is_kom(P);
  const int npde = L.npde;
  for (int n = 0; n < L.S; ++n)
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int a, bb, c, a2, b2, c2, an, bn, cn, an2, bn2, cn2;
        pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
        pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcn2, i2, i3, an2, bn2, cn2);
        const double pout1 = P.outlet_p[0], pout3 = P.outlet_p[2];
        double tke[3], pp[3], qc[8][3];
        tke[1] = kom ? q(an, bn, cn, 6, n) : 0.0;
        tke[2] = kom ? q(an2, bn2, cn2, 6, n) : 0.0;
        for (int v = 1; v <= npde; ++v) {
          if (v == 1) { qc[v][1] = q(an, bn, cn, v, n); qc[v][2] = q(an2, bn2, cn2, v, n); }
          else if (v == 5) { pp[1] = q(an, bn, cn, v, n); pp[2] = q(an2, bn2, cn2, v, n); }
          else {
            qc[v][1] = q(an, bn, cn, v, n) * q(an, bn, cn, 1, n);
            qc[v][2] = q(an2, bn2, cn2, v, n) * q(an2, bn2, cn2, 1, n);
          }
        }
        for (int ic = 1; ic <= 2; ++ic) {
          double rho = qc[1][ic], rhou = qc[2][ic], rhov = qc[3][ic], rhow = qc[4][ic];
          qc[5][ic] = pp[ic] / (g - 1) + (rhou * rhou + rhov * rhov + rhow * rhow) / 2 / rho + rho * tke[ic];
        }
        for (int v = 1; v <= npde; ++v)
          if (v != 5) q(a, bb, c, v, n) = 2 * qc[v][1] - qc[v][2];
        double rhotke0 = 0.0;
        if (kom) {
          q(a, bb, c, 6, n) = std::max(q(a, bb, c, 6, n), q(a, bb, c, 1, n) * P.qmin[5]);
          q(a, bb, c, 7, n) = std::max(q(a, bb, c, 7, n), q(a, bb, c, 1, n) * P.qmin[6]);
          rhotke0 = q(a, bb, c, 6, n);
        }
        q(a, bb, c, 5, n) = pout1 / (g - 1) +
                            (q(a, bb, c, 2, n) * q(a, bb, c, 2, n) + q(a, bb, c, 3, n) * q(a, bb, c, 3, n) +
                             q(a, bb, c, 4, n) * q(a, bb, c, 4, n)) / 2 / q(a, bb, c, 1, n) + rhotke0;
        for (int v = 1; v <= npde; ++v)
          if (v != 5) q(a2, b2, c2, v, n) = 3 * qc[v][1] - 2 * qc[v][2];
        double rhotke2 = 0.0, rhotke1 = 0.0, rhotkem1 = 0.0;
        if (kom) {
          q(a2, b2, c2, 6, n) = std::max(q(a2, b2, c2, 6, n), q(a2, b2, c2, 1, n) * P.qmin[5]);
          q(a2, b2, c2, 7, n) = std::max(q(a2, b2, c2, 7, n), q(a2, b2, c2, 1, n) * P.qmin[6]);
          rhotke2 = qc[6][2]; rhotke1 = qc[6][1]; rhotkem1 = q(a2, b2, c2, 6, n);
        }
        double rhol = (3 * qc[1][1] - qc[1][2]) / 2;
        double rhor = (3 * q(a, bb, c, 1, n) - q(a2, b2, c2, 1, n)) / 2;
        double p1 = (g - 1) * (qc[5][1] - rhotke1 -
                               (qc[2][1] * qc[2][1] + qc[3][1] * qc[3][1] + qc[4][1] * qc[4][1]) / 2 / qc[1][1]);
        double p2 = (g - 1) * (qc[5][2] - rhotke2 -
                               (qc[2][2] * qc[2][2] + qc[3][2] * qc[3][2] + qc[4][2] * qc[4][2]) / 2 / qc[1][2]);
        double pl = (3 * p1 - p2) / 2;
        double pr = (pout3 * (std::sqrt(rhol) + std::sqrt(rhor)) - pl * std::sqrt(rhol)) / std::sqrt(rhor);
        double pm1 = 3 * pout1 - 2 * pr;
        q(a2, b2, c2, 5, n) = pm1 / (g - 1) +
                              (q(a2, b2, c2, 2, n) * q(a2, b2, c2, 2, n) + q(a2, b2, c2, 3, n) * q(a2, b2, c2, 3, n) +
                               q(a2, b2, c2, 4, n) * q(a2, b2, c2, 4, n)) / 2 / q(a2, b2, c2, 1, n) + rhotkem1;
        for (int v = 2; v <= npde; ++v)
          if (v != 5) {
            q(a, bb, c, v, n) = q(a, bb, c, v, n) / q(a, bb, c, 1, n);
            q(a2, b2, c2, v, n) = q(a2, b2, c2, v, n) / q(a2, b2, c2, 1, n);
          }
        double tk1 = kom ? q(a, bb, c, 6, n) : 0.0, tk2 = kom ? q(a2, b2, c2, 6, n) : 0.0;
        double r1 = q(a, bb, c, 1, n), r2 = q(a2, b2, c2, 1, n);
        double uu1 = q(a, bb, c, 2, n), uu2 = q(a2, b2, c2, 2, n);
        double vv1 = q(a, bb, c, 3, n), vv2 = q(a2, b2, c2, 3, n);
        double ww1 = q(a, bb, c, 4, n), ww2 = q(a2, b2, c2, 4, n);
        double e1 = q(a, bb, c, 5, n), e2 = q(a2, b2, c2, 5, n);
        q(a, bb, c, 5, n) = (g - 1) * (e1 - r1 * (uu1 * uu1 + vv1 * vv1 + ww1 * ww1) / 2 - r1 * tk1);
        q(a2, b2, c2, 5, n) = (g - 1) * (e2 - r2 * (uu2 * uu2 + vv2 * vv2 + ww2 * ww2) / 2 - r2 * tk2);
      }
}

// bc_far0 (src/bc.f90:124-483), fixed grid, aircraft free stream
void bc_far0(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk,
             const Level &L, const cosa_params &P) {
  if (P.lomach) {
    // low-speed preconditioning: both halo layers frozen at the free stream
    // (src/bc.f90:264-276, 409-414)
    int ibcpt, ibcpt2;
    if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; }
    else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; }
    const double qf[6] = {0.0, P.rhoinf, P.machfs * std::cos(P.alpha) * std::cos(P.beta),
                          P.machfs * std::sin(P.alpha) * std::cos(P.beta), P.machfs * std::sin(P.beta), P.pinf};
    for (int n = 0; n < L.S; ++n)
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, a2, b2, c2;
          pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
          for (int v = 1; v <= 5; ++v) { q(a, bb, c, v, n) = qf[v]; q(a2, b2, c2, v, n) = q(a, bb, c, v, n); }
          if (is_kom(P)) {
            q(a, bb, c, 6, n) = P.tkefar; q(a, bb, c, 7, n) = P.omefar;
            q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n); q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
          }
        }
    return;
  }
  int ibcpt, ibcpt2, ibcn, ibcm;
  double sgnm;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcm = 1; sgnm = -1.0; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcm = ibcpt; sgnm = 1.0; }
  const double g = P.gamma;
  double qfst[6];
  qfst[1] = P.rhoinf;
  qfst[2] = P.machfs * std::cos(P.alpha) * std::cos(P.beta);
  qfst[3] = P.machfs * std::sin(P.alpha) * std::cos(P.beta);
  qfst[4] = P.machfs * std::sin(P.beta);
  qfst[5] = P.pinf;
  const double sinf = P.pinf / std::pow(P.rhoinf, g);
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int a, bb, c, a2, b2, c2, an, bn, cn, am, bm, cm;
        pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
        pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcm, i2, i3, am, bm, cm);
        double sx, sy, sz;
        face_normal(pa, si, sj, sk, am, bm, cm, nh, sx, sy, sz);
        sx = sx * sgnm; sy = sy * sgnm; sz = sz * sgnm;
        double qext = q(an, bn, cn, 2, n) * sx + q(an, bn, cn, 3, n) * sy + q(an, bn, cn, 4, n) * sz;
        double qinf = qfst[2] * sx + qfst[3] * sy + qfst[4] * sz;
        double rhoext = q(an, bn, cn, 1, n), pext = q(an, bn, cn, 5, n);
        double aext = std::sqrt(g * pext / rhoext);
        double rext = qext + 2 * aext / (g - 1);
        double rinf = qinf - 2 * P.ainf / (g - 1);
        double qdotn = (rext + rinf) / 2;
        double a_ = (g - 1) * (rext - rinf) / 4;
        double mach = qdotn / a_;
        double sext = pext / std::pow(rhoext, g);
        double out[6];
        bool set = true;
        if (qdotn <= 0.0) {
          if (std::fabs(mach) >= 1.0) {
            for (int v = 1; v <= 5; ++v) out[v] = qfst[v];
          } else {
            double rhobc = std::pow(a_ * a_ / (g * sinf), 1.0 / (g - 1));
            double p = rhobc * a_ * a_ / g;
            out[1] = rhobc;
            out[2] = qfst[2] + (qdotn - qinf) * sx;
            out[3] = qfst[3] + (qdotn - qinf) * sy;
            out[4] = qfst[4] + (qdotn - qinf) * sz;
            out[5] = p;
          }
        } else if (qdotn > 0.0) {
          if (std::fabs(mach) >= 1.0) {
            for (int v = 1; v <= 5; ++v) out[v] = q(an, bn, cn, v, n);
          } else {
            double rhobc = std::pow(a_ * a_ / (g * sext), 1.0 / (g - 1));
            double p = rhobc * a_ * a_ / g;
            out[1] = rhobc;
            out[2] = q(an, bn, cn, 2, n) + (qdotn - qext) * sx;
            out[3] = q(an, bn, cn, 3, n) + (qdotn - qext) * sy;
            out[4] = q(an, bn, cn, 4, n) + (qdotn - qext) * sz;
            out[5] = p;
          }
        } else {
          set = false;  // NaN qdotn: the reference leaves the halo untouched
        }
        if (set)
          for (int v = 1; v <= 5; ++v) { q(a, bb, c, v, n) = out[v]; q(a2, b2, c2, v, n) = out[v]; }
        if (is_kom(P)) {
          if (qdotn <= 0.0) {
            q(a, bb, c, 6, n) = P.tkefar; q(a, bb, c, 7, n) = P.omefar;
          } else if (qdotn > 0.0) {
            q(a, bb, c, 6, n) = q(an, bn, cn, 6, n); q(a, bb, c, 7, n) = q(an, bn, cn, 7, n);
          }
          q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n); q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
        }
      }
  }
}

// bc_far1 (src/bc.f90:486-870), fixed grid, aircraft free stream, without
// low-speed preconditioning: the boundary normal velocity and pressure from
// the average of the interior and free-stream states plus the acoustic
// jump, the density from the isentrope of the upwind side
void bc_far1(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk,
             const Level &L, const cosa_params &P, int nl = 1) {
  int ibcpt, ibcpt2, ibcn, ibcm;
  double sgnm;
  if (pa.inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcm = 1; sgnm = -1.0; }
  else { ibcpt = pa.ijk[pa.idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcm = ibcpt; sgnm = 1.0; }
  const double g = P.gamma;
  double qfst[6];
  qfst[1] = P.rhoinf;
  qfst[2] = P.machfs * std::cos(P.alpha) * std::cos(P.beta);
  qfst[3] = P.machfs * std::sin(P.alpha) * std::cos(P.beta);
  qfst[4] = P.machfs * std::sin(P.beta);
  qfst[5] = P.pinf;
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int a, bb, c, a2, b2, c2, an, bn, cn, am, bm, cm;
        pidx(pa, ibcpt, i2, i3, a, bb, c); pidx(pa, ibcpt2, i2, i3, a2, b2, c2);
        pidx(pa, ibcn, i2, i3, an, bn, cn); pidx(pa, ibcm, i2, i3, am, bm, cm);
        double sx, sy, sz;
        face_normal(pa, si, sj, sk, am, bm, cm, nh, sx, sy, sz);
        sx = sx * sgnm; sy = sy * sgnm; sz = sz * sgnm;
        const double qext = q(an, bn, cn, 2, n) * sx + q(an, bn, cn, 3, n) * sy + q(an, bn, cn, 4, n) * sz;
        const double qinf = qfst[2] * sx + qfst[3] * sy + qfst[4] * sz;
        const double pext = q(an, bn, cn, 5, n), pinf = qfst[5];
        const double rhoext = q(an, bn, cn, 1, n);
        const double a_ = std::sqrt(g * pext / rhoext);
        double unb = (qext + qinf) / 2 + (pext - pinf) / (2 * rhoext * a_);
        double pb = (pext + pinf) / 2 + rhoext * a_ * (qext - qinf) / 2;
        if (P.lomach) {
          // preconditioned characteristics with the artificial sound speed
          // apr (src/bc.f90:638-667)
          const double u1 = q(an, bn, cn, 2, n), v1 = q(an, bn, cn, 3, n), w1 = q(an, bn, cn, 4, n);
          const double q2 = u1 * u1 + v1 * v1 + w1 * w1;
          const double a2 = g * pext / rhoext, a = std::sqrt(a2), un = qext;
          const double m2 = q2 / a2, ump2 = (P.uprv / a) * (P.uprv / a);
          const double mp2s = std::min(1.0, std::max(std::max(m2, (1 - P.mixpi) * ump2), lsp_eps2(P, nl)));
          const double am = (1 - mp2s) / 2;
          const double apr = std::sqrt(am * am * (un * un) + a2 * mp2s);
          unb = (qext + qinf) / 2 + (pext - pinf) / (2 * rhoext * apr) + (qext - qinf) / 2 * am * un / apr;
          pb = (pext + pinf) / 2 + rhoext * mp2s * a2 / apr * (qext - qinf) / 2 - (pext - pinf) / 2 * am * un / apr;
        }
        const double mach = unb / a_;
        double out[6];
        bool set = true;
        if (unb <= 0.0) {
          if (std::fabs(mach) >= 1.0) {
            for (int v = 1; v <= 5; ++v) out[v] = qfst[v];
          } else {
            out[1] = qfst[1] * std::pow(pb / pinf, 1 / g);
            out[2] = qfst[2] + (unb - qinf) * sx;
            out[3] = qfst[3] + (unb - qinf) * sy;
            out[4] = qfst[4] + (unb - qinf) * sz;
            out[5] = pb;
          }
        } else if (unb > 0.0) {
          if (std::fabs(mach) >= 1.0) {
            for (int v = 1; v <= 5; ++v) out[v] = q(an, bn, cn, v, n);
          } else {
            out[1] = q(an, bn, cn, 1, n) * std::pow(pb / pext, 1 / g);
            out[2] = q(an, bn, cn, 2, n) + (unb - qext) * sx;
            out[3] = q(an, bn, cn, 3, n) + (unb - qext) * sy;
            out[4] = q(an, bn, cn, 4, n) + (unb - qext) * sz;
            out[5] = pb;
          }
        } else {
          set = false;  // NaN unb: the reference leaves the halo untouched
        }
        if (set)
          for (int v = 1; v <= 5; ++v) { q(a, bb, c, v, n) = out[v]; q(a2, b2, c2, v, n) = out[v]; }
        if (is_kom(P)) {
          // second pass of the reference, same unb (src/bc.f90:800-860)
          if (unb <= 0.0) {
            q(a, bb, c, 6, n) = P.tkefar; q(a, bb, c, 7, n) = P.omefar;
            q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n); q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
          } else if (unb > 0.0) {
            q(a, bb, c, 6, n) = q(an, bn, cn, 6, n); q(a, bb, c, 7, n) = q(an, bn, cn, 7, n);
            q(a2, b2, c2, 6, n) = q(a, bb, c, 6, n); q(a2, b2, c2, 7, n) = q(a, bb, c, 7, n);
          }
        }
      }
  }
}

void bc_walvis_15(const Patch &pa, B3 &q, const Level &L, const cosa_params &P);
void bc_walvis_15_kom(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk, const double *dista,
                      const Level &L, int b, const cosa_params &P);

// bbc dispatch (src/bc.f90:35-121): patches in table order; dist (wall
// distance, P1) is read by the k-omega wall
int bc_level(const Level &L, double *qa, const double *si, const double *sj, const double *sk,
             const cosa_params &P, const double *dist = nullptr, int nl = 1) {
  int status = 0;
#pragma omp parallel for reduction(| : status) schedule(dynamic)
  for (int b = 0; b < L.nb; ++b) {
    B3 q(qa, L, b);
    B2 vi(si, L, b), vj(sj, L, b), vk(sk, L, b);
    const int *t = L.bct.data() + L.obct[b];
    for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
      Patch pa = patch_of(t + 10 * ibc, L.im[b], L.jm[b], L.km[b]);
      pa.blk = b;
      switch (pa.bctyp) {
        case 80: bc_sym(pa, q, L); break;
        case 4: bc_extrapol(pa, q, L); break;
        case 30: bc_far0(pa, q, vi, vj, vk, L, P); break;
        case 31: bc_far1(pa, q, vi, vj, vk, L, P, nl); break;
        case 14: bc_walinv_14(pa, q, vi, vj, vk, L, P); break;
        case 21: status |= bc_insub(pa, q, vi, vj, vk, L, P, nl); break;
        case 91: bc_outsub(pa, q, L, P); break;
        default:
          if (pa.bctyp / 100 == 15 && (!is_kom(P) || dist)) {
            bc_walvis_15(pa, q, L, P);
            if (is_kom(P)) bc_walvis_15_kom(pa, q, vi, vj, vk, dist, L, b, P);
          } else if (pa.bctyp / 100 == 15) {
            status |= COSA_ERR_UNSUPPORTED;
          }
          break;
      }
    }
  }
  return status;
}

// ---- cut_q, in-process branch (src/bc.f90:1894-2141) -----------------------
void cutman_q_level(const Level &L, double *qa, int nvar_override = 0) {
  const int nv = nvar_override ? nvar_override : L.npde;
  for (int icut = 0; icut < L.ncuts; ++icut) {
    const int *c = L.cut.data() + 21 * icut;
    const int b1 = c[0] - 1, b2 = c[9] - 1;
    B3 q1(qa, L, b1), q2(qa, L, b2);
    int ijk1[4] = {0, L.im[b1], L.jm[b1], L.km[b1]};
    int ijk2[4] = {0, L.im[b2], L.jm[b2], L.km[b2]};
    int idir1 = c[1], inout1 = c[2], idir2 = c[10], inout2 = c[11];
    int istr1[4] = {0, c[3], c[5], c[7]}, iend1[4] = {0, c[4], c[6], c[8]};
    int istr2[4] = {0, c[12], c[14], c[16]}, iend2[4] = {0, c[13], c[15], c[17]};
    int iord[4] = {0, c[18], c[19], c[20]};
    (void)idir2;
    int ibcpt, ibcinc, inr, inrinc;
    if (inout1 == 1) { ibcpt = 0; ibcinc = -1; } else { ibcpt = ijk1[idir1]; ibcinc = 1; }
    if (inout2 == 1) { inr = 1; inrinc = 1; } else { inr = ijk2[idir2] - 1; inrinc = -1; }
    int len[4], isgn1[4], isgn2[4];
    for (int l = 1; l <= 3; ++l) {
      len[l] = std::abs(iend1[l] - istr1[l]);
      isgn1[l] = iend1[l] > istr1[l] ? 1 : -1;
      isgn2[l] = iend2[l] > istr2[l] ? 1 : -1;
    }
    int ic1 = cyc(idir1, 1), ic2 = cyc(idir1, 2), ic3 = cyc(idir1, 3);
    int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
    for (int i3 = 0; i3 <= len[ic3]; ++i3)
      for (int i2 = 0; i2 <= len[ic2]; ++i2) {
        int a2_ = istr1[ic2] + isgn1[ic2] * i2, a3_ = istr1[ic3] + isgn1[ic3] * i3;
        int ii1 = ibcpt * krd(ic1, 1) + a2_ * krd(ic2, 1) + a3_ * krd(ic3, 1);
        int jj1 = ibcpt * krd(ic1, 2) + a2_ * krd(ic2, 2) + a3_ * krd(ic3, 2);
        int kk1 = ibcpt * krd(ic1, 3) + a2_ * krd(ic2, 3) + a3_ * krd(ic3, 3);
        int ii2 = ii1 + ibcinc * krd(ic1, 1), jj2 = jj1 + ibcinc * krd(ic1, 2), kk2 = kk1 + ibcinc * krd(ic1, 3);
        int b2_ = istr2[jc2] + isgn2[jc2] * i2, b3_ = istr2[jc3] + isgn2[jc3] * i3;
        int in1 = inr * krd(jc1, 1) + b2_ * krd(jc2, 1) + b3_ * krd(jc3, 1);
        int jn1 = inr * krd(jc1, 2) + b2_ * krd(jc2, 2) + b3_ * krd(jc3, 2);
        int kn1 = inr * krd(jc1, 3) + b2_ * krd(jc2, 3) + b3_ * krd(jc3, 3);
        int in2 = in1 + inrinc * krd(jc1, 1), jn2 = jn1 + inrinc * krd(jc1, 2), kn2 = kn1 + inrinc * krd(jc1, 3);
        for (int n = 0; n < L.S; ++n)
          for (int v = 1; v <= nv; ++v) {
            q1(ii1, jj1, kk1, v, n) = q2(in1, jn1, kn1, v, n);
            q1(ii2, jj2, kk2, v, n) = q2(in2, jn2, kn2, v, n);
          }
      }
  }
}

// ---- prtest (src/cosa.f90:960-1120) -----------------------------------------
int prtest_level(const Level &L, const double *qa, const cosa_params &P) {
  int status = 0;
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b);
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = -1; i <= L.im[b] + 1; ++i) {
            double rho = q(i, j, k, 1, n), pr = q(i, j, k, 5, n);
            if (pr <= P.qmin[4]) status |= COSA_ERR_NEG_P;
            else if (rho <= P.qmin[0]) status |= COSA_ERR_NEG_RHO;
          }
  }
  return status;
}

// ---- lambdab + eig_eul (src/cosa.f90:1248-1330, 4183-4233), inviscid -------
// preconditioned spectral radii of eig_eul_p / eig_ns_p (src/cosa.f90:4300-
// 4460): the convective lambdas of the low-speed preconditioned system
inline void lsp_lambdas(const cosa_params &P, int nl, double u, double v, double w, double a, double cutoff,
                        double xix, double xiy, double xiz, double etax, double etay, double etaz, double zetax,
                        double zetay, double zetaz, double axi, double aeta, double azeta, double *lam) {
  const double q2 = u * u + v * v + w * w, a2 = a * a;
  const double ump2 = (P.uprv / a) * (P.uprv / a);
  const double mp2 = std::min(std::max(std::max(std::max(q2 / a2, ump2), cutoff), lsp_eps2(P, nl)), 1.0);
  const double ui = u * xix + v * xiy + w * xiz, uj = u * etax + v * etay + w * etaz;
  const double uk = u * zetax + v * zetay + w * zetaz;
  lam[0] = ((1 + mp2) * std::fabs(ui) + std::sqrt(ui * ui * ((1 - mp2) * (1 - mp2)) + 4 * a2 * mp2 * (axi * axi))) / 2;
  lam[1] = ((1 + mp2) * std::fabs(uj) + std::sqrt(uj * uj * ((1 - mp2) * (1 - mp2)) + 4 * a2 * mp2 * (aeta * aeta))) / 2;
  lam[2] =
      ((1 + mp2) * std::fabs(uk) + std::sqrt(uk * uk * ((1 - mp2) * (1 - mp2)) + 4 * a2 * mp2 * (azeta * azeta))) / 2;
}

// lambdab (src/cosa.f90:1309-1590), inviscid; with low-speed
// preconditioning (cpg, cvs: the level's cut-offs, nl its index) eig_eul_p
void lambda_level(const Level &L, const double *qa, const double *si, const double *sj,
                  const double *sk, double *lam, const cosa_params &P, const double *cpga = nullptr,
                  const double *cvsa = nullptr, int nl = 1) {
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b), lm(lam, L, b);
    B2 vi(si, L, b), vj(sj, L, b), vk(sk, L, b);
    const double g = P.gamma;
    for (int n = 0; n < L.S; ++n) {
      const int nh = n * P.hbmove;
#pragma omp parallel for schedule(static)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            double rho = q(i, j, k, 1, n), u = q(i, j, k, 2, n), v = q(i, j, k, 3, n);
            double w = q(i, j, k, 4, n), p = q(i, j, k, 5, n);
            double a = std::sqrt(g * p / rho);
            double sim[5], sip[5], sjm[5], sjp[5], skm[5], skp[5];
            for (int c = 1; c <= 4; ++c) {
              sim[c] = vi(c, i, j, k, nh); sip[c] = vi(c, i + 1, j, k, nh);
              sjm[c] = vj(c, i, j, k, nh); sjp[c] = vj(c, i, j + 1, k, nh);
              skm[c] = vk(c, i, j, k, nh); skp[c] = vk(c, i, j, k + 1, nh);
            }
            double xix = 0.5 * (sim[1] * sim[4] + sip[1] * sip[4]);
            double xiy = 0.5 * (sim[2] * sim[4] + sip[2] * sip[4]);
            double xiz = 0.5 * (sim[3] * sim[4] + sip[3] * sip[4]);
            double etax = 0.5 * (sjm[1] * sjm[4] + sjp[1] * sjp[4]);
            double etay = 0.5 * (sjm[2] * sjm[4] + sjp[2] * sjp[4]);
            double etaz = 0.5 * (sjm[3] * sjm[4] + sjp[3] * sjp[4]);
            double zetax = 0.5 * (skm[1] * skm[4] + skp[1] * skp[4]);
            double zetay = 0.5 * (skm[2] * skm[4] + skp[2] * skp[4]);
            double zetaz = 0.5 * (skm[3] * skm[4] + skp[3] * skp[4]);
            double axi = (sim[4] + sip[4]) / 2;
            double aeta = (sjm[4] + sjp[4]) / 2;
            double azeta = (skm[4] + skp[4]) / 2;
            if (P.moving && L.cv[0]) {
              // eig_eul: velocity relative to the cell's grid velocity (src/cosa.f90:4225-4229)
              u = u - BGs(L.cv[0], L, b, nh)(i, j, k);
              v = v - BGs(L.cv[1], L, b, nh)(i, j, k);
              w = w - BGs(L.cv[2], L, b, nh)(i, j, k);
            }
            if (P.lomach && cpga) {
              B1m cpg(const_cast<double *>(cpga), L, b), cvs(const_cast<double *>(cvsa), L, b);
              double l3[3];
              lsp_lambdas(P, nl, u, v, w, a, std::max(cpg(i, j, k, n), cvs(i, j, k, n)), xix, xiy, xiz, etax, etay,
                          etaz, zetax, zetay, zetaz, axi, aeta, azeta, l3);
              for (int c = 0; c < 3; ++c) lm(i, j, k, c + 1, n) = l3[c];
              continue;
            }
            lm(i, j, k, 1, n) = std::fabs(u * xix + v * xiy + w * xiz) + a * axi;
            lm(i, j, k, 2, n) = std::fabs(u * etax + v * etay + w * etaz) + a * aeta;
            lm(i, j, k, 3, n) = std::fabs(u * zetax + v * zetay + w * zetaz) + a * azeta;
          }
    }
  }
}

// ---- bdeltat (src/cosa.f90:4733-5203), inviscid, no CFL ramping ------------
void deltat_level(const Level &L, double *dtv, const double *lam, double *bx_, double *by_,
                  double *bz_, const cosa_params &P) {
  const double zeta = 0.4, c1 = 40.0;
  (void)c1;
  for (int b = 0; b < L.nb; ++b) {
    B3 lm(const_cast<double *>(lam), L, b);
    B1 dt(dtv, L, b, L.S);
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i)
            dt(i, j, k, n) = P.cfl / (lm(i, j, k, 1, n) + lm(i, j, k, 2, n) + lm(i, j, k, 3, n));
    if (P.irsop == 0 || !bx_) continue;
    B1 bx(bx_, L, b, L.S), by(by_, L, b, L.S), bz(bz_, L, b, L.S);
    const double rat = P.rat, psirs = P.psirs;
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            double lami = lm(i, j, k, 1, n), lamj = lm(i, j, k, 2, n), lamk = lm(i, j, k, 3, n);
            if (P.irsop == 2 || P.irsop == 5) {
              double phixi = 1 + std::pow(lamj / lami, zeta) + std::pow(lamk / lami, zeta);
              double phieta = 1 + std::pow(lami / lamj, zeta) + std::pow(lamk / lamj, zeta);
              double phizeta = 1 + std::pow(lami / lamk, zeta) + std::pow(lamj / lamk, zeta);
              double t;
              t = (rat * lami * phixi / (lami + lamj + lamk));
              bx(i, j, k, n) = std::max(0.0, (t * t - 1) / 4);
              t = (rat * lamj * phieta / (lami + lamj + lamk));
              by(i, j, k, n) = std::max(0.0, (t * t - 1) / 4);
              t = (rat * lamk * phizeta / (lami + lamj + lamk));
              bz(i, j, k, n) = std::max(0.0, (t * t - 1) / 4);
            } else if (P.irsop == 3 || P.irsop == 6) {
              double rji = lamj / lami, rki = lamk / lami, rij = lami / lamj;
              double rkj = lamk / lamj, rik = lami / lamk, rjk = lamj / lamk;
              double t;
              t = rat / (1 + psirs * (rji + rki));
              bx(i, j, k, n) = std::max(0.0, 0.25 * (t * t - 1));
              t = rat / (1 + psirs * (rij + rkj));
              by(i, j, k, n) = std::max(0.0, 0.25 * (t * t - 1));
              t = rat / (1 + psirs * (rik + rjk));
              bz(i, j, k, n) = std::max(0.0, 0.25 * (t * t - 1));
            }
          }
  }
}

// ---- limiters limit_i/j/k (src/flux.f90:3472-3888) -------------------------
// The three directions are the same loops with the stencil along `d`; the
// helpers below take the line accessor dq(., m) = dq at offset m along d.
struct Line {
  B3 *a; int d;
  inline double &at(int i, int j, int k, int m, int v, int n) const {
    return d == 1 ? (*a)(i + m, j, k, v, n) : (d == 2 ? (*a)(i, j + m, k, v, n) : (*a)(i, j, k + m, v, n));
  }
};

void limit_dir(B3 &dq, B3 &dqp, B3 &dqm, int d, double epslim, double rkap, int vs, int ve,
               int ilim, int im, int jm, int km, int S) {
  // loop ranges per direction: along d, faces 1..max (ilim 0/1) or 0..max (2..4)
  Line Lq{&dq, d}, Lp{&dqp, d}, Lm{&dqm, d};
  int lo[4] = {0, 1, 1, 1}, hi[4] = {0, im - 1, jm - 1, km - 1};
  const int nmax = d == 1 ? im : (d == 2 ? jm : km);
  for (int n = 0; n < S; ++n)
    for (int v = vs; v <= ve; ++v) {
      int l0[4], h0[4];
      for (int e = 1; e <= 3; ++e) { l0[e] = lo[e]; h0[e] = hi[e]; }
      l0[d] = (ilim <= 1) ? 1 : 0;
      h0[d] = nmax;
      for (int k = l0[3]; k <= h0[3]; ++k)
        for (int j = l0[2]; j <= h0[2]; ++j)
          for (int i = l0[1]; i <= h0[1]; ++i) {
            if (ilim == 0) {
              double rkp = 1 + rkap, rkm = 1 - rkap;
              Lp.at(i, j, k, 0, v, n) = -(rkp * Lq.at(i, j, k, 0, v, n) + rkm * Lq.at(i, j, k, 1, v, n)) / 4;
              Lm.at(i, j, k, 0, v, n) = (rkm * Lq.at(i, j, k, -1, v, n) + rkp * Lq.at(i, j, k, 0, v, n)) / 4;
            } else if (ilim == 1) {
              double d0 = Lq.at(i, j, k, 0, v, n), dp1 = Lq.at(i, j, k, 1, v, n), dm1 = Lq.at(i, j, k, -1, v, n);
              double s = (2 * dp1 * d0 + epslim) / (dp1 * dp1 + d0 * d0 + epslim);
              double rkp = 1 + rkap * s, rkm = 1 - rkap * s;
              Lp.at(i, j, k, 0, v, n) = -s * (rkp * d0 + rkm * dp1) / 4;
              s = (2 * d0 * dm1 + epslim) / (d0 * d0 + dm1 * dm1 + epslim);
              rkp = 1 + rkap * s; rkm = 1 - rkap * s;
              Lm.at(i, j, k, 0, v, n) = s * (rkm * dm1 + rkp * d0) / 4;
            } else if (ilim == 2) {
              double rkp = 1 + rkap, rkm = 1 - rkap;
              double bb = (3.0 - rkap) / (1.0 - rkap);
              double d0 = Lq.at(i, j, k, 0, v, n), d1 = Lq.at(i, j, k, 1, v, n);
              double dqmx = (std::copysign(1.0, d0) + std::copysign(1.0, d1)) / 2 *
                            std::min(std::fabs(d0), std::fabs(d1) * bb);
              double dqpx = (std::copysign(1.0, d1) + std::copysign(1.0, d0)) / 2 *
                            std::min(std::fabs(d1), std::fabs(d0) * bb);
              Lp.at(i, j, k, 0, v, n) = -(rkp * dqmx + rkm * dqpx) / 4;
              Lm.at(i, j, k, 1, v, n) = (rkm * dqmx + rkp * dqpx) / 4;
            } else if (ilim == 3) {
              double epsq = epslim * epslim;
              double d1 = Lq.at(i, j, k, 1, v, n), d2 = Lq.at(i, j, k, 0, v, n);
              double dqmx = (d1 * (d2 * d2 + 2 * epsq) + d2 * (2 * (d1 * d1) + epsq)) /
                            (2 * (d1 * d1) - d1 * d2 + 2 * (d2 * d2) + 3 * epsq);
              double dqpx = (d2 * (d1 * d1 + 2 * epsq) + d1 * (2 * (d2 * d2) + epsq)) /
                            (2 * (d2 * d2) - d2 * d1 + 2 * (d1 * d1) + 3 * epsq);
              Lp.at(i, j, k, 0, v, n) = -dqpx / 2;
              Lm.at(i, j, k, 1, v, n) = dqmx / 2;
            } else if (ilim == 4) {
              double epsq = epslim * epslim;
              double d1 = Lq.at(i, j, k, 1, v, n), d2 = Lq.at(i, j, k, 0, v, n);
              double dqmx = (d1 * (d2 * d2 + epsq) + d2 * (d1 * d1 + epsq)) / (d1 * d1 + d2 * d2 + 2 * epsq);
              double dqpx = dqmx;
              Lp.at(i, j, k, 0, v, n) = -dqpx / 2;
              Lm.at(i, j, k, 1, v, n) = dqmx / 2;
            }
          }
    }
}

inline bool strong_bc(int t) {
  return t == 13 || t == 14 || t / 100 == 15 || t == 22 || t == 23 || t == 92 || t == 93 || t == 5;
}

// ---- muscl_bi/bj/bk (src/flux.f90:1221-1810) ------------------------------
void muscl_b(const Level &L, int b, int d, int nl, double *qa, double *qpa, double *qma,
             double *dqa, double *dqpa, double *dqma, const cosa_params &P) {
  B3 q(qa, L, b), qp(qpa, L, b), qm(qma, L, b), dq(dqa, L, b), dqp(dqpa, L, b), dqm(dqma, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b], npde = L.npde, S = L.S;
  int fo_beg = 0, fo_end = -1, so_beg = 1, so_end = npde;
  bool dofirst = false, doscnd = true;
  if (nl >= P.nl_crs) { fo_beg = 1; fo_end = npde; so_beg = 0; so_end = -1; dofirst = true; doscnd = false; }
  else if (P.foturb) { fo_beg = 6; fo_end = npde; so_beg = 1; so_end = 5; dofirst = true; doscnd = true; }
  // face ranges: along d 1..max, others 1..max-1
  int flo[4] = {0, 1, 1, 1}, fhi[4] = {0, im - 1, jm - 1, km - 1};
  fhi[d] = d == 1 ? im : (d == 2 ? jm : km);
  auto off = [&](int e) { return e == d ? 1 : 0; };
  if (dofirst)
    for (int n = 0; n < S; ++n)
      for (int v = fo_beg; v <= fo_end; ++v)
        for (int k = flo[3]; k <= fhi[3]; ++k)
          for (int j = flo[2]; j <= fhi[2]; ++j)
            for (int i = flo[1]; i <= fhi[1]; ++i) {
              qp(i, j, k, v, n) = q(i, j, k, v, n);
              qm(i, j, k, v, n) = q(i - off(1), j - off(2), k - off(3), v, n);
            }
  const int *t = L.bct.data() + L.obct[b];
  if (doscnd) {
    int dlo[4] = {0, 1, 1, 1}, dhi[4] = {0, im - 1, jm - 1, km - 1};
    dlo[d] = 0;
    dhi[d] = (d == 1 ? im : (d == 2 ? jm : km)) + 1;
    for (int n = 0; n < S; ++n)
      for (int v = so_beg; v <= so_end; ++v)
        for (int k = dlo[3]; k <= dhi[3]; ++k)
          for (int j = dlo[2]; j <= dhi[2]; ++j)
            for (int i = dlo[1]; i <= dhi[1]; ++i)
              dq(i, j, k, v, n) = q(i, j, k, v, n) - q(i - off(1), j - off(2), k - off(3), v, n);
    for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
      const int *r = t + 10 * ibc;
      if (r[1] != d || !strong_bc(r[0])) continue;
      int bcpt = r[2] == 1 ? 1 : (d == 1 ? im : (d == 2 ? jm : km));
      int s[4] = {0, r[3], r[5], r[7]}, e[4] = {0, r[4], r[6], r[8]};
      s[d] = e[d] = bcpt;
      for (int n = 0; n < S; ++n)
        for (int v = so_beg; v <= so_end; ++v)
          for (int k = s[3]; k <= e[3]; ++k)
            for (int j = s[2]; j <= e[2]; ++j)
              for (int i = s[1]; i <= e[1]; ++i)
                dq(i, j, k, v, n) = (q(i, j, k, v, n) - q(i - off(1), j - off(2), k - off(3), v, n)) * 2;
    }
    limit_dir(dq, dqp, dqm, d, P.epslimf, P.rkap, 1, 5, P.ilimf, im, jm, km, S);
    limit_dir(dq, dqp, dqm, d, P.epslimt, P.rkap, 6, npde, P.ilimt, im, jm, km, S);
    for (int n = 0; n < S; ++n)
      for (int v = so_beg; v <= so_end; ++v)
        for (int k = flo[3]; k <= fhi[3]; ++k)
          for (int j = flo[2]; j <= fhi[2]; ++j)
            for (int i = flo[1]; i <= fhi[1]; ++i) {
              qp(i, j, k, v, n) = q(i, j, k, v, n) + dqp(i, j, k, v, n);
              qm(i, j, k, v, n) = q(i - off(1), j - off(2), k - off(3), v, n) + dqm(i, j, k, v, n);
            }
  }
  for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
    const int *r = t + 10 * ibc;
    if (r[1] != d || !strong_bc(r[0])) continue;
    const int mx = d == 1 ? im : (d == 2 ? jm : km);
    int qpm = r[2] == 1 ? 1 : mx, bcpt = r[2] == 1 ? 0 : mx;
    int s[4] = {0, r[3], r[5], r[7]}, e[4] = {0, r[4], r[6], r[8]};
    s[d] = e[d] = 0;
    for (int n = 0; n < S; ++n)
      for (int v = 1; v <= npde; ++v)
        for (int k = s[3]; k <= e[3]; ++k)
          for (int j = s[2]; j <= e[2]; ++j)
            for (int i = s[1]; i <= e[1]; ++i) {
              int a = i, bb = j, c = k, a2 = i, b2 = j, c2 = k;
              if (d == 1) { a = qpm; a2 = bcpt; } else if (d == 2) { bb = qpm; b2 = bcpt; } else { c = qpm; c2 = bcpt; }
              qp(a, bb, c, v, n) = q(a2, b2, c2, v, n);
              qm(a, bb, c, v, n) = q(a2, b2, c2, v, n);
            }
  }
}

// ---- roflux_b mean-flow part (src/flux.f90:45-238) --------------------------
struct RoeOut { double f[6]; };
inline void roe_face(const cosa_params &P, double kx, double ky, double kz, double ds, double ubn,
                     const double *qr, const double *ql, double tker, double tkel, double *flux) {
  const double g = P.gamma;
  double rhor = qr[1], ur = qr[2], vr = qr[3], wr = qr[4], pr = qr[5];
  double unr = ur * kx + vr * ky + wr * kz - ubn;
  double q2r = ur * ur + vr * vr + wr * wr;
  double h0r = g / (g - 1) * pr / rhor + q2r / 2 + tker;
  double rh0r = rhor * h0r;
  double fr[6], fl[6], df[6];
  fr[1] = rhor * unr;
  fr[2] = (rhor * ur * unr + pr * kx);
  fr[3] = (rhor * vr * unr + pr * ky);
  fr[4] = (rhor * wr * unr + pr * kz);
  fr[5] = (rh0r * unr + pr * ubn);
  double rhol = ql[1], ul = ql[2], vl = ql[3], wl = ql[4], pl = ql[5];
  double unl = ul * kx + vl * ky + wl * kz - ubn;
  double q2l = ul * ul + vl * vl + wl * wl;
  double h0l = g / (g - 1) * pl / rhol + q2l / 2 + tkel;
  double rh0l = rhol * h0l;
  fl[1] = rhol * unl;
  fl[2] = (rhol * ul * unl + pl * kx);
  fl[3] = (rhol * vl * unl + pl * ky);
  fl[4] = (rhol * wl * unl + pl * kz);
  fl[5] = (rh0l * unl + pl * ubn);
  double drho = rhor - rhol, dp = pr - pl, du = ur - ul, dv = vr - vl, dw = wr - wl;
  double dun = unr - unl, dtke = tker - tkel;
  double rhols = std::sqrt(rhol), rhors = std::sqrt(rhor);
  double rho = rhols * rhors, denom = rhols + rhors;
  double u = (rhols * ul + rhors * ur) / denom;
  double v = (rhols * vl + rhors * vr) / denom;
  double w = (rhols * wl + rhors * wr) / denom;
  double un = u * kx + v * ky + w * kz;
  double h0 = (rhols * h0l + rhors * h0r) / denom;
  double tke = (rhols * tkel + rhors * tker) / denom;
  double q2 = u * u + v * v + w * w;
  double a2 = (g - 1) * (h0 - q2 / 2 - tke);
  double a = std::sqrt(a2);
  double rm123 = std::fabs(un - ubn), rm4 = std::fabs(un + a - ubn), rm5 = std::fabs(un - a - ubn);
  if (P.efx_setup_f) {
    double rdelta = P.cntrpy_f * (P.entfx_f_w[0] * P.entfxctf_f +
                                  P.entfx_f_w[1] * (std::sqrt(u * u + v * v + w * w) + a) +
                                  P.entfx_f_w[2] * 0.2 * (std::fabs(un) + a + std::fabs(ubn)));
    rdelta = std::max(rdelta, 1.0e-12);
    if (rm123 <= rdelta && P.efx_all_f) rm123 = 0.5 * (rm123 * rm123 + rdelta * rdelta) / rdelta;
    if (rm4 <= rdelta) rm4 = 0.5 * (rm4 * rm4 + rdelta * rdelta) / rdelta;
    if (rm5 <= rdelta) rm5 = 0.5 * (rm5 * rm5 + rdelta * rdelta) / rdelta;
  }
  if (P.eig_limit_f) {
    if (rm123 <= P.eig_cutoff_f) rm123 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm4 <= P.eig_cutoff_f) rm4 = P.eig_cutoff_f;
    if (P.eig_lim_all_f && rm5 <= P.eig_cutoff_f) rm5 = P.eig_cutoff_f;
  }
  double al1 = rm123 * (drho - dp / a2);
  double al2 = rm123 * rho;
  double al3 = rm4 * (dp / a2 + rho * dun / a) / 2;
  double al4 = rm5 * (dp / a2 - rho * dun / a) / 2;
  df[1] = al1 + al3 + al4;
  df[2] = al1 * u + al2 * (du - dun * kx) + al3 * (u + a * kx) + al4 * (u - a * kx);
  df[3] = al1 * v + al2 * (dv - dun * ky) + al3 * (v + a * ky) + al4 * (v - a * ky);
  df[4] = al1 * w + al2 * (dw - dun * kz) + al3 * (w + a * kz) + al4 * (w - a * kz);
  df[5] = al1 * (q2 / 2 + tke) + al2 * (u * du + v * dv + w * dw - un * dun + dtke) +
          al3 * (h0 + a * un) + al4 * (h0 - a * un);
  for (int m = 1; m <= 5; ++m) flux[m] = (fr[m] + fl[m] - df[m]) / 2 * ds;
}

// roflux_b, turbulence fluxes (src/flux.f90:249-380): upwinded rho k u_n and
// rho omega u_n with the mean-flow wave strengths.  The Roe-averaged total
// enthalpy uses h0l/h0r as the mean-flow loop left them, i.e. those of the
// block's last face (ic,jc,kc) of the snapshot: the reference does not
// recompute them in this loop, and the restatement keeps that.
void roflux_turb(const Level &L, int b, int d, B3 &qr, B3 &ql, B0 &flux, const B2 &s, const cosa_params &P, int n,
                 int ic, int jc, int kc) {
  const double g = P.gamma;
  const int nh = n * P.hbmove;
  double h0r_last, h0l_last;
  {
    const double ur = qr(ic, jc, kc, 2, n), vr = qr(ic, jc, kc, 3, n), wr = qr(ic, jc, kc, 4, n);
    const double ul = ql(ic, jc, kc, 2, n), vl = ql(ic, jc, kc, 3, n), wl = ql(ic, jc, kc, 4, n);
    h0r_last = g / (g - 1) * qr(ic, jc, kc, 5, n) / qr(ic, jc, kc, 1, n) + (ur * ur + vr * vr + wr * wr) / 2 +
               qr(ic, jc, kc, 6, n);
    h0l_last = g / (g - 1) * ql(ic, jc, kc, 5, n) / ql(ic, jc, kc, 1, n) + (ul * ul + vl * vl + wl * wl) / 2 +
               ql(ic, jc, kc, 6, n);
  }
  for (int k = 1; k <= kc; ++k)
    for (int j = 1; j <= jc; ++j)
      for (int i = 1; i <= ic; ++i) {
        const double kx = s(1, i, j, k, nh), ky = s(2, i, j, k, nh), kz = s(3, i, j, k, nh), ds = s(4, i, j, k, nh);
        const double ubn = P.moving ? face_ubn(L, b, d, i, j, k, nh, kx, ky, kz) : 0.0;
        const double rhor = qr(i, j, k, 1, n), ur = qr(i, j, k, 2, n), vr = qr(i, j, k, 3, n), wr = qr(i, j, k, 4, n);
        const double pr = qr(i, j, k, 5, n), omer = qr(i, j, k, 7, n), tker = qr(i, j, k, 6, n);
        const double unr = ur * kx + vr * ky + wr * kz - ubn;
        const double frk = rhor * unr * tker, frw = rhor * unr * omer;
        const double rhol = ql(i, j, k, 1, n), ul = ql(i, j, k, 2, n), vl = ql(i, j, k, 3, n), wl = ql(i, j, k, 4, n);
        const double pl = ql(i, j, k, 5, n), omel = ql(i, j, k, 7, n), tkel = ql(i, j, k, 6, n);
        const double unl = ul * kx + vl * ky + wl * kz - ubn;
        const double flk = rhol * unl * tkel, flw = rhol * unl * omel;
        const double drho = rhor - rhol, dp = pr - pl, dun = unr - unl, dtke = tker - tkel, dome = omer - omel;
        const double rhols = std::sqrt(rhol), rhors = std::sqrt(rhor);
        const double rho = rhols * rhors, denom = rhols + rhors;
        const double u = (rhols * ul + rhors * ur) / denom, v = (rhols * vl + rhors * vr) / denom;
        const double w = (rhols * wl + rhors * wr) / denom;
        const double un = u * kx + v * ky + w * kz;
        const double h0 = (rhols * h0l_last + rhors * h0r_last) / denom;
        const double tke = (rhols * tkel + rhors * tker) / denom, ome = (rhols * omel + rhors * omer) / denom;
        const double q2 = u * u + v * v + w * w;
        const double a2 = (g - 1) * (h0 - q2 / 2 - tke);
        const double a = std::sqrt(a2);
        double rm123 = std::fabs(un - ubn), rm4 = std::fabs(un + a - ubn), rm5 = std::fabs(un - a - ubn);
        if (P.efx_setup_t) {
          double rdelta = P.cntrpy_t * (P.entfx_t_w[0] * P.entfxctf_t + P.entfx_t_w[1] * (std::sqrt(q2) + a) +
                                        P.entfx_t_w[2] * 0.2 * (std::fabs(un) + a + std::fabs(ubn)));
          rdelta = std::max(rdelta, 1.0e-12);
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
        flux(i, j, k, 6, n) = (frk + flk - dfk) / 2 * ds;
        flux(i, j, k, 7, n) = (frw + flw - dfw) / 2 * ds;
      }
}

void roflux_b(const Level &L, int b, int d, double *qra, double *qla, double *fa, const double *sijk,
              const cosa_params &P) {
  B3 qr(qra, L, b), ql(qla, L, b);
  B0 flux(fa, L, b);
  B2 s(sijk, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  int ic = d == 1 ? im : im - 1, jc = d == 2 ? jm : jm - 1, kc = d == 3 ? km : km - 1;
  const bool kom = is_kom(P);
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= kc; ++k)
      for (int j = 1; j <= jc; ++j)
        for (int i = 1; i <= ic; ++i) {
          double kx = s(1, i, j, k, nh), ky = s(2, i, j, k, nh), kz = s(3, i, j, k, nh), ds = s(4, i, j, k, nh);
          double vr[6], vl[6], f[6];
          for (int v = 1; v <= 5; ++v) { vr[v] = qr(i, j, k, v, n); vl[v] = ql(i, j, k, v, n); }
          double tker = kom ? qr(i, j, k, 6, n) : 0.0, tkel = kom ? ql(i, j, k, 6, n) : 0.0;
          const double ubn = P.moving ? face_ubn(L, b, d, i, j, k, nh, kx, ky, kz) : 0.0;
          roe_face(P, kx, ky, kz, ds, ubn, vr, vl, tker, tkel, f);
          for (int v = 1; v <= 5; ++v) flux(i, j, k, v, n) = f[v];
        }
    if (kom) roflux_turb(L, b, d, qr, ql, flux, s, P, n, ic, jc, kc);
  }
}

// ---- bresid (src/cosa.f90:1149-1211) ----------------------------------------
void resid_b(const Level &L, int b, int d, double *fa, double *ra) {
  B0 flux(fa, L, b);
  B3 res(ra, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int oi = d == 1, oj = d == 2, ok = d == 3;
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 1; i <= im - 1; ++i)
            res(i, j, k, v, n) = res(i, j, k, v, n) + flux(i + oi, j + oj, k + ok, v, n) - flux(i, j, k, v, n);
}


// ---- update_b explicit, non-k-omega (src/update.f90:568-640) ---------------
void update_b(const Level &L, int b, double *ra, double *qa, double *qoa, double *dta, double ar) {
  B3 res(ra, L, b), q(qa, L, b), qold(qoa, L, b);
  B1 dt(dta, L, b, L.S);
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= 5; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i)
            q(i, j, k, v, n) = qold(i, j, k, v, n) - ar * res(i, j, k, v, n) * dt(i, j, k, n);
}


// ---- implicit residual smoothing (src/cosa.f90:2035-2443, 5206-5773) -------
// tridi (src/cosa.f90:2418-2443): Thomas algorithm, x overwritten by the solution
void tridi(const double *a, const double *b, const double *c, double *x, int dim) {
  std::vector<double> r(dim + 1), t(dim + 1);
  if (dim == 1) { x[0] = x[0] / b[0]; return; }
  r[0] = c[0] / b[0];
  t[0] = x[0] / b[0];
  for (int j = 1; j < dim - 1; ++j) {
    r[j] = c[j] / (b[j] - r[j - 1] * a[j]);
    t[j] = (x[j] - t[j - 1] * a[j]) / (b[j] - r[j - 1] * a[j]);
  }
  t[dim - 1] = (x[dim - 1] - t[dim - 2] * a[dim - 1]) / (b[dim - 1] - r[dim - 2] * a[dim - 1]);
  x[dim - 1] = t[dim - 1];
  for (int j = dim - 2; j >= 0; --j) x[j] = t[j] - x[j + 1] * r[j];
}

// one direction of cirs_b / ccirs_b for variables vs..ve: line solves with
// coefficient eps (irsop 1) or beta(i,j,k) (irsop >= 2); for the cut
// variant (rhs_src = ores for d = 1) the boundary rows take eps * halo.
void irs_dir(const Level &L, int b, int d, double *ra, const double *rhs_src, const double *beta_a,
             double epsc, int vs, int ve, bool with_halo) {
  B3 res(ra, L, b);
  B3 src(const_cast<double *>(rhs_src ? rhs_src : ra), L, b);
  const int im = L.im[b] - 1, jm = L.jm[b] - 1, km = L.km[b] - 1;
  const int len = d == 1 ? im : (d == 2 ? jm : km);
  const int n2 = d == 1 ? jm : im, n3 = d == 3 ? jm : km;
  std::vector<double> A(len), Bv(len), Cv(len), X(len);
  for (int n = 0; n < L.S; ++n)
    for (int v = vs; v <= ve; ++v)
      for (int t3 = 1; t3 <= n3; ++t3)
        for (int t2 = 1; t2 <= n2; ++t2) {
          auto at = [&](int m, int &i, int &j, int &k) {
            if (d == 1) { i = m; j = t2; k = t3; }
            else if (d == 2) { i = t2; j = m; k = t3; }
            else { i = t2; j = t3; k = m; }
          };
          for (int m = 1; m <= len; ++m) {
            int i, j, k;
            at(m, i, j, k);
            double e = epsc;
            if (beta_a) { B1 bt(const_cast<double *>(beta_a), L, b, L.S); e = bt(i, j, k, n); }
            A[m - 1] = m == 1 ? 0 : -e;
            Bv[m - 1] = 1 + 2 * e;
            Cv[m - 1] = m == len ? 0 : -e;
            X[m - 1] = src(i, j, k, v, n);
            if (with_halo && m == 1) {
              int hi, hj, hk; at(0, hi, hj, hk);
              X[0] = src(i, j, k, v, n) + e * res(hi, hj, hk, v, n);
            }
            if (with_halo && m == len) {
              int hi, hj, hk; at(len + 1, hi, hj, hk);
              X[len - 1] = src(i, j, k, v, n) + e * res(hi, hj, hk, v, n);
            }
          }
          tridi(A.data(), Bv.data(), Cv.data(), X.data(), len);
          for (int m = 1; m <= len; ++m) {
            int i, j, k;
            at(m, i, j, k);
            res(i, j, k, v, n) = X[m - 1];
          }
        }
}

// scalef_b / scaleb_b (src/cosa.f90:5652-5773): res *= or /= dtvol (dtvolt for k-omega)
void scale_res(const Level &L, double *ra, const double *dtv, const double *dtvt, bool forward, const cosa_params &P) {
  for (int b = 0; b < L.nb; ++b) {
    B3 res(ra, L, b);
    B1 dt(const_cast<double *>(dtv), L, b, L.S);
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v) {
        const bool turb = v >= 6;
        if (turb && !dtvt) continue;
        B1 dtt(const_cast<double *>(turb ? dtvt : dtv), L, b, L.S);
        for (int k = 1; k <= L.km[b] - 1; ++k)
          for (int j = 1; j <= L.jm[b] - 1; ++j)
            for (int i = 1; i <= L.im[b] - 1; ++i)
              res(i, j, k, v, n) = forward ? res(i, j, k, v, n) * dtt(i, j, k, n) : res(i, j, k, v, n) / dtt(i, j, k, n);
      }
  }
}

// cirs (cutcirs = 0) and the ccirs loop (cutcirs = 1) of smooth()
// (src/cosa.f90:1977-1998)
void irs_level(const Level &L, double *res, const double *dtv, const double *dtvt, const double *bx,
               const double *by, const double *bz, const double *tbx, const double *tby, const double *tbz,
               const cosa_params &P) {
  const double epsc = 0.25 * (P.rat * P.rat - 1.0);
  const bool kom = is_kom(P);
  const double *bet[4] = {nullptr, bx, by, bz}, *tbet[4] = {nullptr, tbx, tby, tbz};
  auto sweep3 = [&](double *r, const double *ores, bool with_halo) {
    for (int b = 0; b < L.nb; ++b)
      for (int d = 1; d <= 3; ++d) {
        const double *src = (d == 1) ? ores : nullptr;
        if (P.irsop == 1) {
          irs_dir(L, b, d, r, src, nullptr, epsc, 1, L.npde, with_halo);
        } else {
          irs_dir(L, b, d, r, src, bet[d], 0.0, 1, 5, with_halo);
          if (kom) irs_dir(L, b, d, r, src, tbet[d], 0.0, 6, L.npde, with_halo);
        }
      }
  };
  if (P.cutcirs == 0) {
    scale_res(L, res, dtv, kom ? dtvt : nullptr, true, P);
    // cirs_b does i, j, k per block with the residual itself as right-hand side
    for (int b = 0; b < L.nb; ++b)
      for (int d = 1; d <= 3; ++d) {
        if (P.irsop == 1) irs_dir(L, b, d, res, nullptr, nullptr, epsc, 1, L.npde, false);
        else {
          irs_dir(L, b, d, res, nullptr, bet[d], 0.0, 1, 5, false);
          if (kom) irs_dir(L, b, d, res, nullptr, tbet[d], 0.0, 6, L.npde, false);
        }
      }
    scale_res(L, res, dtv, kom ? dtvt : nullptr, false, P);
  } else {
    scale_res(L, res, dtv, kom ? dtvt : nullptr, true, P);
    // work1 = res over 0..imax (copy_array extent 1)
    std::vector<double> ores(res, res + L.n3 * L.npde * L.S);
    for (int its = 0; its < 2; ++its) {
      cutman_q_level(L, res);
      sweep3(res, ores.data(), true);
    }
    scale_res(L, res, dtv, kom ? dtvt : nullptr, false, P);
  }
}

// ---- src_bhb (src/src.f90:556-613): res(n) += omega V sum_m D(n,m) q(m) --------
void src_hb_level(const Level &L, const double *qa, const double *va, double *ra, const cosa_params &P) {
  const int S = L.S;
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b), res(ra, L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            double qhb[COSA_MAX_SNAP];
            for (int ni = 0; ni < S; ++ni) qhb[ni] = 0.0;
            for (int ni = 0; ni < S; ++ni)
              for (int nj = 0; nj < S; ++nj)
                qhb[ni] = qhb[ni] + P.omega * vol(i, j, k) * P.dhb[ni * S + nj] * q(i, j, k, v, nj);
            for (int ni = 0; ni < S; ++ni) res(i, j, k, v, ni) = res(i, j, k, v, ni) + qhb[ni];
          }
  }
}

// resg_rms_hb / resg_brms_hb (src/cosa.f90:4584-4697), explicit branch
void resg_rms_hb_level(const Level &L, double *ra, double *out) {
  double acc[10] = {0};
  int64_t ncell = 0;
  for (int b = 0; b < L.nb; ++b) {
    B3 res(ra, L, b);
    double rb[10] = {0};
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int k = 1; k <= L.km[b] - 1; ++k)
          for (int j = 1; j <= L.jm[b] - 1; ++j)
            for (int i = 1; i <= L.im[b] - 1; ++i) rb[v] = rb[v] + res(i, j, k, v, n) * res(i, j, k, v, n);
    for (int v = 1; v <= L.npde; ++v) rb[L.npde + 1] = rb[L.npde + 1] + rb[v];
    for (int v = 1; v <= L.npde + 1; ++v) acc[v] = acc[v] + rb[v];
    ncell += (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
  }
  for (int v = 1; v <= L.npde; ++v) out[v - 1] = std::sqrt(acc[v] / ncell / L.S);
  out[L.npde] = std::sqrt(acc[L.npde + 1] / ncell / L.S / L.npde);
}

// resg_brms_hb with rkimp, no IRS and one level (src/cosa.f90:4629-4697):
// the harmonic-balance term omega D q V is added to the residual, one
// snapshot nj at a time, before the squares are summed
void resg_rms_hbimp_level(const Level &L, const double *ra, const double *qa, const double *va, const cosa_params &P,
                          double *out) {
  const int S = L.S;
  double acc[10] = {0};
  int64_t ncell = 0;
  for (int b = 0; b < L.nb; ++b) {
    B3 res(const_cast<double *>(ra), L, b), q(const_cast<double *>(qa), L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    double rb[10] = {0};
    for (int n = 0; n < S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int k = 1; k <= L.km[b] - 1; ++k)
          for (int j = 1; j <= L.jm[b] - 1; ++j)
            for (int i = 1; i <= L.im[b] - 1; ++i) {
              double w = res(i, j, k, v, n);
              for (int nj = 0; nj < S; ++nj) w = w + P.omega * P.dhb[n * S + nj] * q(i, j, k, v, nj) * vol(i, j, k);
              rb[v] = rb[v] + w * w;
            }
    for (int v = 1; v <= L.npde; ++v) rb[L.npde + 1] = rb[L.npde + 1] + rb[v];
    for (int v = 1; v <= L.npde + 1; ++v) acc[v] = acc[v] + rb[v];
    ncell += (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
  }
  for (int v = 1; v <= L.npde; ++v) out[v - 1] = std::sqrt(acc[v] / ncell / S);
  out[L.npde] = std::sqrt(acc[L.npde + 1] / ncell / S / L.npde);
}

// LU factorisation with partial pivoting of an n x n matrix (column-major,
// a[i + n*j]) and the solve for nrhs right-hand sides (b[i + n*m]), in the
// order of LAPACK's unblocked DGETF2 (pivot = first largest |a(i,j)|, whole
// rows swapped, column scaled by the pivot's reciprocal, rank-1 update) and
// DGETRS 'N' (row interchanges, unit-lower then upper triangular solves);
// DGETRF's recursive variant may round differently.
void lu_solve(int n, double *a, double *bm, int nrhs) {
  int ipiv[COSA_MAX_SNAP];
  for (int j = 0; j < n; ++j) {
    int pv = j;
    double amax = std::fabs(a[j + n * j]);
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(a[i + n * j]) > amax) { amax = std::fabs(a[i + n * j]); pv = i; }
    ipiv[j] = pv;
    if (a[pv + n * j] != 0.0) {
      if (pv != j)
        for (int k = 0; k < n; ++k) std::swap(a[j + n * k], a[pv + n * k]);
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
      if (ipiv[j] != j) std::swap(x[j], x[ipiv[j]]);
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

// update_bhb, rkimp, mean-flow equations: per cell the snapshots are coupled
// through (I + ar omega dtau D) q = rhs, dtau = dtvol V of the row's snapshot.
// Without IRS on one level (src/update.f90:1564-1604) the residual holds no
// time-spectral term and rhs = qold - ar res dtvol.  With IRS or multigrid
// (src/update.f90:1771-1836) src_hb has added qhb = omega V D q to the
// residual before the smoothing (src/cosa.f90:1918-1922) and
// rhs = qold + (qhb - res) ar dtvol, qhb recomputed here from the same q in
// src_bhb's order (src/src.f90:556-600)
void update_bhb_b(const Level &L, int b, const double *ra, double *qa, const double *qoa, const double *dta,
                  const double *va, double ar, const cosa_params &P, bool src_in_res) {
  const int S = L.S;
  B3 res(const_cast<double *>(ra), L, b), q(qa, L, b), qold(const_cast<double *>(qoa), L, b);
  B1 dtv(const_cast<double *>(dta), L, b, S), vol(const_cast<double *>(va), L, b, 1);
  for (int k = 1; k <= L.km[b] - 1; ++k)
    for (int j = 1; j <= L.jm[b] - 1; ++j)
      for (int i = 1; i <= L.im[b] - 1; ++i) {
        double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP * 5];
        for (int ni = 0; ni < S; ++ni) {
          const double dtau = dtv(i, j, k, ni) * vol(i, j, k);
          for (int nj = 0; nj < S; ++nj)
            a[ni + S * nj] = (ni == nj ? 1.0 : 0.0) + ar * P.omega * dtau * P.dhb[ni * S + nj];
        }
        for (int ni = 0; ni < S; ++ni)
          for (int m = 0; m < 5; ++m) {
            if (src_in_res) {
              double qhb = 0.0;
              for (int nj = 0; nj < S; ++nj)
                qhb = qhb + P.omega * vol(i, j, k) * P.dhb[ni * S + nj] * q(i, j, k, m + 1, nj);
              x[ni + S * m] = qold(i, j, k, m + 1, ni) + (qhb - res(i, j, k, m + 1, ni)) * ar * dtv(i, j, k, ni);
            } else {
              x[ni + S * m] = qold(i, j, k, m + 1, ni) - ar * res(i, j, k, m + 1, ni) * dtv(i, j, k, ni);
            }
          }
        lu_solve(S, a, x, 5);
        for (int ni = 0; ni < S; ++ni)
          for (int m = 0; m < 5; ++m) q(i, j, k, m + 1, ni) = x[ni + S * m];
      }
}

// update_bhb's k-omega part with rkimp (src/update.f90:1427-1560 without IRS
// on one level, 1633-1768 with IRS or multigrid): per cell the snapshots of
// rho omega, then of rho k, coupled through (I (1 + ar dtau a_n) + ar omega
// dtau D) x = rhs with the point-implicit destruction a_n; rho omega floored
// by gav cmu rho sqrt(prd); the k equation takes omega before the update
// and the change of rho omega.  Runs before update_bhb_b (variables 1..5).
void update_bhb_kom_b(const Level &L, int b, const double *ra, double *qa, const double *qoa, const double *va,
                      const double *dtta, const double *dpla, const double *prda, double ar, const cosa_params &P,
                      const double *ttrma, bool src_in_res) {
  const int S = L.S;
  B3 res(const_cast<double *>(ra), L, b), q(qa, L, b), qold(const_cast<double *>(qoa), L, b);
  B1 dtt(const_cast<double *>(dtta), L, b, S), vol(const_cast<double *>(va), L, b, 1);
  B3s dpl(const_cast<double *>(dpla), L, b), prd(const_cast<double *>(prda), L, b);
  for (int k = 1; k <= L.km[b] - 1; ++k)
    for (int j = 1; j <= L.jm[b] - 1; ++j)
      for (int i = 1; i <= L.im[b] - 1; ++i) {
        auto gav_of = [&](int n) { return ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 2, n) : P.gkw; };
        auto bav_of = [&](int n) { return ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 3, n) : P.bkw; };
        auto hbsrc = [&](int v, int ni) {  // src_bhb's term of variable v, snapshot ni
          double qhb = 0.0;
          for (int nj = 0; nj < S; ++nj) qhb = qhb + P.omega * vol(i, j, k) * P.dhb[ni * S + nj] * q(i, j, k, v, nj);
          return qhb;
        };
        double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP], w7[COSA_MAX_SNAP], dw[COSA_MAX_SNAP];
        // rho omega
        for (int ni = 0; ni < S; ++ni) {
          const double gav = gav_of(ni), bav = bav_of(ni);
          const double ome = q(i, j, k, 7, ni) / q(i, j, k, 1, ni);
          const double dtau = dtt(i, j, k, ni) * vol(i, j, k);
          const double dps = dpl(i, j, k, ni);
          if (src_in_res)
            x[ni] = qold(i, j, k, 7, ni) + ar * dtt(i, j, k, ni) * (hbsrc(7, ni) - res(i, j, k, 7, ni)) +
                    ar * dtau * q(i, j, k, 7, ni) * (gav * dps + 2 * bav * ome);
          else
            x[ni] = qold(i, j, k, 7, ni) - ar * res(i, j, k, 7, ni) * dtt(i, j, k, ni) +
                    ar * dtau * q(i, j, k, 7, ni) * (gav * dps + 2 * bav * ome);
          w7[ni] = q(i, j, k, 7, ni);
          for (int nj = 0; nj < S; ++nj)
            a[ni + S * nj] = (ni == nj ? 1.0 : 0.0) * (1 + ar * dtau * (gav * dps + 2 * bav * ome)) +
                             ar * P.omega * dtau * P.dhb[ni * S + nj];
        }
        // the k right-hand sides read rho k and the src_bhb terms before any update
        double xk[COSA_MAX_SNAP], qk[COSA_MAX_SNAP], sk[COSA_MAX_SNAP];
        for (int ni = 0; ni < S; ++ni) {
          qk[ni] = q(i, j, k, 6, ni);
          sk[ni] = src_in_res ? hbsrc(6, ni) : 0.0;
        }
        lu_solve(S, a, x, 1);
        for (int ni = 0; ni < S; ++ni) {
          const double rho = q(i, j, k, 1, ni);
          const double rhomegamin = gav_of(ni) * P.cmu * rho * std::sqrt(prd(i, j, k, ni));
          if (x[ni] < rhomegamin) x[ni] = rhomegamin;
          q(i, j, k, 7, ni) = x[ni];
          dw[ni] = q(i, j, k, 7, ni) - w7[ni];
        }
        // rho k
        for (int ni = 0; ni < S; ++ni) {
          const double rho = q(i, j, k, 1, ni);
          const double ome = w7[ni] / q(i, j, k, 1, ni);
          const double dtau = dtt(i, j, k, ni) * vol(i, j, k);
          const double dps = dpl(i, j, k, ni);
          if (src_in_res)
            xk[ni] = (qold(i, j, k, 6, ni) + ar * dtt(i, j, k, ni) * (sk[ni] - res(i, j, k, 6, ni)) +
                      ar * dtau * qk[ni] * (dps + P.bstrkw * ome - P.bstrkw * dw[ni] / rho));
          else
            xk[ni] = (qold(i, j, k, 6, ni) - ar * res(i, j, k, 6, ni) * dtt(i, j, k, ni) +
                      ar * dtau * qk[ni] * (dps + P.bstrkw * ome - P.bstrkw * dw[ni] / rho));
          for (int nj = 0; nj < S; ++nj)
            a[ni + S * nj] = (ni == nj ? 1.0 : 0.0) * (1 + ar * dtau * (dps + P.bstrkw * ome)) +
                             ar * P.omega * dtau * P.dhb[ni * S + nj];
        }
        lu_solve(S, a, xk, 1);
        for (int ni = 0; ni < S; ++ni) q(i, j, k, 6, ni) = xk[ni];
      }
}

// lim_res_ome_bhb (src/update.f90:2836-2999), without low-speed
// preconditioning: the omega residual of the residual pass limited so that
// rho omega cannot go below its floor; explicit per snapshot, with rkimp
// through the snapshot-coupled system (I (1 + dtau a_n) + omega dtau D)
void lim_res_ome_bhb_b(const Level &L, int b, double *ra, const double *qa, const double *qoa, const double *va,
                       const double *dtta, const double *dpla, const double *prda, const cosa_params &P,
                       const double *ttrma) {
  const int S = L.S;
  B3 res(ra, L, b), q(const_cast<double *>(qa), L, b), qold(const_cast<double *>(qoa), L, b);
  B1 dtt(const_cast<double *>(dtta), L, b, S), vol(const_cast<double *>(va), L, b, 1);
  B3s dpl(const_cast<double *>(dpla), L, b), prd(const_cast<double *>(prda), L, b);
  for (int k = 1; k <= L.km[b] - 1; ++k)
    for (int j = 1; j <= L.jm[b] - 1; ++j)
      for (int i = 1; i <= L.im[b] - 1; ++i) {
        auto gav_of = [&](int n) { return ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 2, n) : P.gkw; };
        auto bav_of = [&](int n) { return ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 3, n) : P.bkw; };
        if (!P.rkimp) {
          for (int n = 0; n < S; ++n) {
            const double gav = gav_of(n), bav = bav_of(n);
            const double rho = q(i, j, k, 1, n), ome = q(i, j, k, 7, n) / q(i, j, k, 1, n);
            const double dtau = dtt(i, j, k, n) * vol(i, j, k);
            const double rhomega = qold(i, j, k, 7, n) -
                                   res(i, j, k, 7, n) * dtt(i, j, k, n) / (1 + dtau * (gav * dpl(i, j, k, n) + 2 * bav * ome));
            const double rhomegamin = gav * P.cmu * rho * std::sqrt(prd(i, j, k, n));
            res(i, j, k, 7, n) = res(i, j, k, 7, n) - (1 + dtau * (gav * dpl(i, j, k, n) + 2 * bav * ome)) *
                                                          std::max(0.0, (rhomegamin - rhomega) / dtt(i, j, k, n));
          }
          continue;
        }
        double a[COSA_MAX_SNAP * COSA_MAX_SNAP], x[COSA_MAX_SNAP];
        for (int ni = 0; ni < S; ++ni) {
          const double gav = gav_of(ni), bav = bav_of(ni);
          const double dtau = dtt(i, j, k, ni) * vol(i, j, k);
          const double ome = q(i, j, k, 7, ni) / q(i, j, k, 1, ni);
          const double dps = dpl(i, j, k, ni);
          for (int nj = 0; nj < S; ++nj)
            a[ni + S * nj] = (ni == nj ? 1.0 : 0.0) * (1 + dtau * (gav * dps + 2 * bav * ome)) +
                             P.omega * dtau * P.dhb[ni * S + nj];
          x[ni] = res(i, j, k, 7, ni) * dtt(i, j, k, ni);
        }
        lu_solve(S, a, x, 1);
        for (int n = 0; n < S; ++n) {
          const double rho = q(i, j, k, 1, n);
          const double rhomegamin = gav_of(n) * P.cmu * rho * std::sqrt(prd(i, j, k, n));
          const double rhomeganew = qold(i, j, k, 7, n) - x[n];
          res(i, j, k, 7, n) = res(i, j, k, 7, n) - std::max(0.0, (rhomegamin - rhomeganew)) / dtt(i, j, k, n);
        }
      }
}

// ---- dual time stepping (src/src.f90:381-527; src/update.f90:568-740;
// src/cosa.f90:4503-4560) ---------------------------------------------------------
// src_uns_b: res += 3/2 q V / dt (BDF2), q V / dt on a first-order first step
void src_uns_level(const Level &L, const double *qa, const double *va, double *ra, const cosa_params &P) {
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b), res(ra, L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            if (P.bdf1) res(i, j, k, v, 0) = res(i, j, k, v, 0) + q(i, j, k, v, 0) * vol(i, j, k) / P.dt;
            else res(i, j, k, v, 0) = res(i, j, k, v, 0) + 3 * q(i, j, k, v, 0) * vol(i, j, k) / 2 / P.dt;
          }
  }
}
// rhs_uns_b: rhs = q1 V / dt, or (2 q1 - q2 / 2) V / dt (q1 = q^n, q2 = q^(n-1))
void rhs_uns_level(const Level &L, double *rha, const double *q1a, const double *q2a, const double *va,
                   const cosa_params &P) {
  for (int b = 0; b < L.nb; ++b) {
    B3 rhs(rha, L, b), q1(const_cast<double *>(q1a), L, b), q2(const_cast<double *>(q2a), L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            if (P.bdf1) rhs(i, j, k, v, 0) = q1(i, j, k, v, 0) * vol(i, j, k) / P.dt;
            else rhs(i, j, k, v, 0) = (2 * q1(i, j, k, v, 0) - q2(i, j, k, v, 0) / 2) * vol(i, j, k) / P.dt;
          }
  }
}
// resg_brms with rkimp, no IRS, one level: the physical-time term fact q V /
// dt added back to res - rhs
void resg_rms_dualimp_level(const Level &L, const double *ra, const double *rha, const double *qa, const double *va,
                            const cosa_params &P, double *out) {
  const double fact = P.bdf1 ? 1.0 : 1.5;
  double acc[10] = {0};
  int64_t ncell = 0;
  for (int b = 0; b < L.nb; ++b) {
    B3 res(const_cast<double *>(ra), L, b), rhs(const_cast<double *>(rha), L, b), q(const_cast<double *>(qa), L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    double rb[10] = {0};
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            const double t = fact * q(i, j, k, v, 0) * vol(i, j, k) / P.dt + res(i, j, k, v, 0) - rhs(i, j, k, v, 0);
            rb[v] = rb[v] + t * t;
          }
    for (int v = 1; v <= L.npde; ++v) rb[L.npde + 1] = rb[L.npde + 1] + rb[v];
    for (int v = 1; v <= L.npde + 1; ++v) acc[v] = acc[v] + rb[v];
    ncell += (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
  }
  for (int v = 1; v <= L.npde; ++v) out[v - 1] = std::sqrt(acc[v] / ncell);
  out[L.npde] = std::sqrt(acc[L.npde + 1] / ncell / L.npde);
}
// update_b with rkimp (src/update.f90:650-738): the physical-time term
// implicit.  Without IRS on one level the residual holds no physical-time
// term; with IRS or multigrid src_uns added it and it is taken out again.
void update_dual_b(const Level &L, int b, const double *ra, double *qa, const double *qoa, const double *dta,
                   const double *va, double ar, const cosa_params &P, bool src_in_res) {
  B3 res(const_cast<double *>(ra), L, b), q(qa, L, b), qold(const_cast<double *>(qoa), L, b);
  B1 dtv(const_cast<double *>(dta), L, b, 1), vol(const_cast<double *>(va), L, b, 1);
  const double fact = P.bdf1 ? 1.0 : 1.5;
  for (int v = 1; v <= 5; ++v)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double den = 1 + fact * ar * dtv(i, j, k) * vol(i, j, k) / P.dt;
          if (src_in_res)
            q(i, j, k, v, 0) = (qold(i, j, k, v, 0) -
                                ar * dtv(i, j, k) * (-fact * vol(i, j, k) / P.dt * q(i, j, k, v, 0) + res(i, j, k, v, 0))) /
                               den;
          else
            q(i, j, k, v, 0) = (qold(i, j, k, v, 0) - ar * res(i, j, k, v, 0) * dtv(i, j, k)) / den;
        }
}
// the k-omega part of update_b with rkimp (src/update.f90:655-732)
void update_kom_dual_b(const Level &L, int b, const double *ra, double *qa, const double *qoa, const double *va,
                       const double *dtta, const double *dpla, const double *prda, double ar, const cosa_params &P,
                       const double *ttrma, bool src_in_res) {
  B3 res(const_cast<double *>(ra), L, b), q(qa, L, b), qold(const_cast<double *>(qoa), L, b);
  B1 vol(const_cast<double *>(va), L, b, 1), dtt(const_cast<double *>(dtta), L, b, 1);
  B3s dpl(const_cast<double *>(dpla), L, b), prd(const_cast<double *>(prda), L, b);
  const double fact = P.bdf1 ? 1.0 : 1.5;
  for (int k = 1; k <= L.km[b] - 1; ++k)
    for (int j = 1; j <= L.jm[b] - 1; ++j)
      for (int i = 1; i <= L.im[b] - 1; ++i) {
        const double gav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 2, 0) : P.gkw;
        const double bav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 3, 0) : P.bkw;
        const double rho = q(i, j, k, 1, 0);
        const double ome = q(i, j, k, 7, 0) / q(i, j, k, 1, 0);
        const double dtau = dtt(i, j, k) * vol(i, j, k);
        const double dp = dpl(i, j, k, 0);
        double rhomega;
        if (src_in_res)
          rhomega = (qold(i, j, k, 7, 0) + ar * fact * dtau / P.dt * q(i, j, k, 7, 0) -
                     ar * res(i, j, k, 7, 0) * dtt(i, j, k) + ar * dtau * q(i, j, k, 7, 0) * (gav * dp + 2 * bav * ome)) /
                    (1 + ar * dtau * (gav * dp + 2 * bav * ome) + ar * fact * dtau / P.dt);
        else
          rhomega = (qold(i, j, k, 7, 0) - ar * res(i, j, k, 7, 0) * dtt(i, j, k) +
                     ar * dtau * q(i, j, k, 7, 0) * (gav * dp + 2 * bav * ome)) /
                    (1 + ar * dtau * (gav * dp + 2 * bav * ome) + fact * ar * dtau / P.dt);
        const double rhomegamin = gav * P.cmu * rho * std::sqrt(prd(i, j, k, 0));
        if (rhomega < rhomegamin) rhomega = rhomegamin;
        q(i, j, k, 7, 0) = rhomega;
        const double drhomega = q(i, j, k, 7, 0) - rho * ome;
        if (src_in_res)
          q(i, j, k, 6, 0) = (qold(i, j, k, 6, 0) + ar * fact * dtau / P.dt * q(i, j, k, 6, 0) -
                              ar * res(i, j, k, 6, 0) * dtt(i, j, k) +
                              ar * dtau * q(i, j, k, 6, 0) * (dp + P.bstrkw * ome - P.bstrkw * drhomega / rho)) /
                             (1 + ar * dtau * (dp + P.bstrkw * ome) + ar * fact * dtau / P.dt);
        else
          q(i, j, k, 6, 0) = (qold(i, j, k, 6, 0) - ar * res(i, j, k, 6, 0) * dtt(i, j, k) +
                              ar * dtau * q(i, j, k, 6, 0) * (dp + P.bstrkw * ome - P.bstrkw * drhomega / rho)) /
                             (1 + ar * dtau * (dp + P.bstrkw * ome) + ar * fact * dtau / P.dt);
      }
}
// src_uns enters the residual unless rkimp without IRS on one level
inline bool dual_src_in_res(const cosa_params &P) { return P.dualt && (!P.rkimp || P.irsop > 0 || P.nlevel > 1); }

// ---- resg_brms (src/cosa.f90:4503-4582), explicit steady branch ------------
void resg_rms_level(const Level &L, double *ra, double *rha, double *out) {
  double acc[10] = {0};
  int64_t ncell = 0;
  for (int b = 0; b < L.nb; ++b) {
    B3 res(ra, L, b), rhs(rha ? rha : ra, L, b);
    double rb[10] = {0};
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            // rkuns has no rhs (src/cosa.f90:4562-4571)
            double t = rha ? res(i, j, k, v, 0) - rhs(i, j, k, v, 0) : res(i, j, k, v, 0);
            rb[v] = rb[v] + t * t;
          }
    for (int v = 1; v <= L.npde; ++v) rb[L.npde + 1] = rb[L.npde + 1] + rb[v];
    for (int v = 1; v <= L.npde + 1; ++v) acc[v] = acc[v] + rb[v];
    ncell += (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
  }
  for (int v = 1; v <= L.npde; ++v) out[v - 1] = std::sqrt(acc[v] / ncell);
  out[L.npde] = std::sqrt(acc[L.npde + 1] / ncell / L.npde);
}

void zero_res(const Level &L, double *ra) {
  for (int b = 0; b < L.nb; ++b) {
    B3 r(ra, L, b);
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int k = 0; k <= L.km[b]; ++k)
          for (int j = 0; j <= L.jm[b]; ++j)
            for (int i = 0; i <= L.im[b]; ++i) r(i, j, k, v, n) = 0.0;
  }
}

void copy_interior(const Level &L, double *dst, const double *src) {
  for (int b = 0; b < L.nb; ++b) {
    B3 d(dst, L, b), s(const_cast<double *>(src), L, b);
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int k = 1; k <= L.km[b] - 1; ++k)
          for (int j = 1; j <= L.jm[b] - 1; ++j)
            for (int i = 1; i <= L.im[b] - 1; ++i) d(i, j, k, v, n) = s(i, j, k, v, n);
  }
}

// ---- imetrix_b / bvols (src/grid.f90:847-1010, 2160-2230), fixed grid -------
void imetrix_b(const Level &L, int b, const double *xa, const double *ya, const double *za,
               double *sia, double *sja, double *ska) {
  // one set of metrics per grid snapshot (dim5h = 2 nharms hbmove + 1)
  for (int n = 0; n < L.dim5h; ++n) {
  BGs x(xa, L, b, n), y(ya, L, b, n), z(za, L, b, n);
  B2w si(sia, L, b), sj(sja, L, b), sk(ska, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  for (int k = 1; k <= km - 1; ++k)
    for (int j = 1; j <= jm - 1; ++j)
      for (int i = 1; i <= im; ++i) {
        double a1 = ((y(i, j + 1, k + 1) - y(i, j, k)) * (z(i, j, k + 1) - z(i, j + 1, k)) -
                     (z(i, j + 1, k + 1) - z(i, j, k)) * (y(i, j, k + 1) - y(i, j + 1, k))) / 2;
        double a2 = ((z(i, j + 1, k + 1) - z(i, j, k)) * (x(i, j, k + 1) - x(i, j + 1, k)) -
                     (x(i, j + 1, k + 1) - x(i, j, k)) * (z(i, j, k + 1) - z(i, j + 1, k))) / 2;
        double a3 = ((x(i, j + 1, k + 1) - x(i, j, k)) * (y(i, j, k + 1) - y(i, j + 1, k)) -
                     (y(i, j + 1, k + 1) - y(i, j, k)) * (x(i, j, k + 1) - x(i, j + 1, k))) / 2;
        double a4 = std::sqrt(a1 * a1 + a2 * a2 + a3 * a3);
        si(1, i, j, k, n) = a1 / a4; si(2, i, j, k, n) = a2 / a4; si(3, i, j, k, n) = a3 / a4; si(4, i, j, k, n) = a4;
      }
  for (int k = 1; k <= km - 1; ++k)
    for (int i = 1; i <= im - 1; ++i)
      for (int j = 1; j <= jm; ++j) {
        double a1 = ((z(i + 1, j, k + 1) - z(i, j, k)) * (y(i, j, k + 1) - y(i + 1, j, k)) -
                     (y(i + 1, j, k + 1) - y(i, j, k)) * (z(i, j, k + 1) - z(i + 1, j, k))) / 2;
        double a2 = ((x(i + 1, j, k + 1) - x(i, j, k)) * (z(i, j, k + 1) - z(i + 1, j, k)) -
                     (z(i + 1, j, k + 1) - z(i, j, k)) * (x(i, j, k + 1) - x(i + 1, j, k))) / 2;
        double a3 = ((y(i + 1, j, k + 1) - y(i, j, k)) * (x(i, j, k + 1) - x(i + 1, j, k)) -
                     (x(i + 1, j, k + 1) - x(i, j, k)) * (y(i, j, k + 1) - y(i + 1, j, k))) / 2;
        double a4 = std::sqrt(a1 * a1 + a2 * a2 + a3 * a3);
        sj(1, i, j, k, n) = a1 / a4; sj(2, i, j, k, n) = a2 / a4; sj(3, i, j, k, n) = a3 / a4; sj(4, i, j, k, n) = a4;
      }
  for (int j = 1; j <= jm - 1; ++j)
    for (int i = 1; i <= im - 1; ++i)
      for (int k = 1; k <= km; ++k) {
        double a1 = ((y(i + 1, j + 1, k) - y(i, j, k)) * (z(i, j + 1, k) - z(i + 1, j, k)) -
                     (z(i + 1, j + 1, k) - z(i, j, k)) * (y(i, j + 1, k) - y(i + 1, j, k))) / 2;
        double a2 = ((z(i + 1, j + 1, k) - z(i, j, k)) * (x(i, j + 1, k) - x(i + 1, j, k)) -
                     (x(i + 1, j + 1, k) - x(i, j, k)) * (z(i, j + 1, k) - z(i + 1, j, k))) / 2;
        double a3 = ((x(i + 1, j + 1, k) - x(i, j, k)) * (y(i, j + 1, k) - y(i + 1, j, k)) -
                     (y(i + 1, j + 1, k) - y(i, j, k)) * (x(i, j + 1, k) - x(i + 1, j, k))) / 2;
        double a4 = std::sqrt(a1 * a1 + a2 * a2 + a3 * a3);
        sk(1, i, j, k, n) = a1 / a4; sk(2, i, j, k, n) = a2 / a4; sk(3, i, j, k, n) = a3 / a4; sk(4, i, j, k, n) = a4;
      }
  }
}

// ---- moving grids: rigid pitching (src/grid.f90:1783-1966) ------------------
// movegrid_b + pitch: node positions and velocities of every snapshot n from
// the reference grid x0 and the per-node displacement scales dx, dy (P1
// arrays, nodes 1..imax), theta(n) = dtheta0 sin(omegas t_n).  The reference
// moves nodes 1..imax; the ghost nodes 0 and imax+1 are rotated rigidly here as
// well (the forces read them as moment arms).  The branch for |dx| or |dy| <=
// 1e-4 keeps the reference's y0 (not y0 - yh) in its rotation terms.
void pitch_b(const Level &L, int b, const double *x0a, const double *y0a, const double *z0a, const double *dxa,
             const double *dya, const double *dza, double *xa, double *ya, double *za, double *xda, double *yda,
             double *zda, const cosa_params &P, const double *zeit, const double *dth) {
  BG x0(x0a, L, b), y0(y0a, L, b), z0(z0a, L, b);
  B1 dx(const_cast<double *>(dxa), L, b, 1), dy(const_cast<double *>(dya), L, b, 1);
  (void)dza;
  const double xh = P.xh, yh = P.yh, dtheta0 = P.dtheta0, omegas = P.omegas;
  for (int n = 0; n < L.dim5h; ++n) {
    BGs x(xa, L, b, n), y(ya, L, b, n), z(za, L, b, n), xd(xda, L, b, n), yd(yda, L, b, n), zd(zda, L, b, n);
    const double dtheta = dth[n], c = std::cos(dtheta), sn = std::sin(dtheta);
    const double cw = std::cos(omegas * zeit[n]);
    for (int k = 0; k <= L.km[b] + 1; ++k)
      for (int i = 0; i <= L.im[b] + 1; ++i)
        for (int j = 0; j <= L.jm[b] + 1; ++j) {
          z(i, j, k) = z0(i, j, k);
          zd(i, j, k) = 0.0;
          // ghost nodes (index 0 or imax+1, read by the forces' moment arm)
          // rotate rigidly: unit displacement scales
          const bool ghost = i == 0 || j == 0 || k == 0 || i > L.im[b] || j > L.jm[b] || k > L.km[b];
          const double X0 = x0(i, j, k), Y0 = y0(i, j, k);
          const double DX = ghost ? 1.0 : dx(i, j, k), DY = ghost ? 1.0 : dy(i, j, k);
          if (std::fabs(DX) > 1e-4 && std::fabs(DY) > 1e-4) {
            const double d1 = ((X0 - xh) * (c - 1) - (Y0 - yh) * sn) / DX;
            const double d2 = ((X0 - xh) * sn + (Y0 - yh) * (c - 1)) / DY;
            x(i, j, k) = X0 + d1 * DX;
            y(i, j, k) = Y0 + d2 * DY;
            const double v1 = (-(X0 - xh) * sn - (Y0 - yh) * c) * dtheta0 * cw / DX;
            const double v2 = ((X0 - xh) * c - (Y0 - yh) * sn) * dtheta0 * cw / DY;
            xd(i, j, k) = omegas * v1 * DX;
            yd(i, j, k) = omegas * v2 * DY;
          } else {
            const double d1 = ((X0 - xh) * (c - 1.0) - Y0 * sn);
            const double d2 = ((X0 - xh) * sn + Y0 * (c - 1.0));
            x(i, j, k) = X0 + d1;
            y(i, j, k) = Y0 + d2;
            const double v1 = dtheta0 * cw * (-(X0 - xh) * sn - Y0 * c);
            const double v2 = dtheta0 * cw * ((X0 - xh) * c - Y0 * sn);
            xd(i, j, k) = omegas * v1;
            yd(i, j, k) = omegas * v2;
          }
        }
  }
}

// imetrix_b, moving part (src/grid.f90:1024-1062): the velocity of each face
// midpoint as the mean of its four nodes' velocities
void face_vel_b(const Level &L, int b, const double *xda, const double *yda, const double *zda, double *fia,
                double *fja, double *fka) {
  BFv fi(fia, L, b), fj(fja, L, b), fk(fka, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  for (int n = 0; n < L.dim5h; ++n) {
    BGs xd(xda, L, b, n), yd(yda, L, b, n), zd(zda, L, b, n);
    const BGs *v[3] = {&xd, &yd, &zd};
    for (int c = 0; c < 3; ++c) {
      const BGs &a = *v[c];
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 1; i <= im; ++i)
            fi(c + 1, i, j, k, n) = (a(i, j + 1, k + 1) + a(i, j + 1, k) + a(i, j, k + 1) + a(i, j, k)) / 4;
      for (int k = 1; k <= km - 1; ++k)
        for (int i = 1; i <= im - 1; ++i)
          for (int j = 1; j <= jm; ++j)
            fj(c + 1, i, j, k, n) = (a(i + 1, j, k + 1) + a(i + 1, j, k) + a(i, j, k + 1) + a(i, j, k)) / 4;
      for (int j = 1; j <= jm - 1; ++j)
        for (int i = 1; i <= im - 1; ++i)
          for (int k = 1; k <= km; ++k)
            fk(c + 1, i, j, k, n) = (a(i + 1, j + 1, k) + a(i + 1, j, k) + a(i, j + 1, k) + a(i, j, k)) / 4;
    }
  }
}

// vert2cell_bg (src/output.f90:3276-3480): node values -> cell values in
// place (cells 0..imax: the block's vertices, edges and bounding faces take
// the nearest boundary nodes, interior cells the mean of their 8 nodes)
void vert2cell_b(const Level &L, int b, double *wa) {
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  for (int n = 0; n < L.dim5h; ++n) {
    BGs x(wa, L, b, n);
    const int64_t np = (int64_t)(im + 2) * (jm + 2) * (km + 2);
    std::vector<double> w(x.p, x.p + np);
    auto W = [&](int i, int j, int k) { return w[i + (int64_t)(im + 2) * (j + (int64_t)(jm + 2) * k)]; };
    auto bnd = [](int i, int m) { return i == 0 ? 1 : m; };
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          const bool bi = i == 0 || i == im, bj = j == 0 || j == jm, bk = k == 0 || k == km;
          const int i1 = bnd(i, im), j1 = bnd(j, jm), k1 = bnd(k, km);
          double v;
          if (bi && bj && bk) v = W(i1, j1, k1);
          else if (bj && bk) v = (W(i, j1, k1) + W(i + 1, j1, k1)) / 2;
          else if (bi && bk) v = (W(i1, j, k1) + W(i1, j + 1, k1)) / 2;
          else if (bi && bj) v = (W(i1, j1, k) + W(i1, j1, k + 1)) / 2;
          else if (bk) v = (W(i, j, k1) + W(i + 1, j, k1) + W(i, j + 1, k1) + W(i + 1, j + 1, k1)) / 4;
          else if (bj) v = (W(i, j1, k) + W(i + 1, j1, k) + W(i, j1, k + 1) + W(i + 1, j1, k + 1)) / 4;
          else if (bi) v = (W(i1, j, k) + W(i1, j, k + 1) + W(i1, j + 1, k) + W(i1, j + 1, k + 1)) / 4;
          else
            v = (W(i, j, k) + W(i + 1, j, k) + W(i, j + 1, k) + W(i + 1, j + 1, k) + W(i, j, k + 1) +
                 W(i + 1, j, k + 1) + W(i, j + 1, k + 1) + W(i + 1, j + 1, k + 1)) / 8;
          x(i, j, k) = v;
        }
  }
}

void bvols(const Level &L, int b, const double *xa, const double *ya, const double *za, double *va) {
  // the volumes of the first grid snapshot (rigid motions keep them)
  BGs x(xa, L, b, 0), y(ya, L, b, 0), z(za, L, b, 0);
  B1 vol(va, L, b, 1);
  for (int k = 1; k <= L.km[b] - 1; ++k)
    for (int j = 1; j <= L.jm[b] - 1; ++j)
      for (int i = 1; i <= L.im[b] - 1; ++i) {
        double si1 = ((y(i, j + 1, k + 1) - y(i, j, k)) * (z(i, j, k + 1) - z(i, j + 1, k)) -
                      (z(i, j + 1, k + 1) - z(i, j, k)) * (y(i, j, k + 1) - y(i, j + 1, k))) / 2;
        double sj1 = ((z(i + 1, j, k + 1) - z(i, j, k)) * (y(i, j, k + 1) - y(i + 1, j, k)) -
                      (y(i + 1, j, k + 1) - y(i, j, k)) * (z(i, j, k + 1) - z(i + 1, j, k))) / 2;
        double sk1 = ((y(i + 1, j + 1, k) - y(i, j, k)) * (z(i, j + 1, k) - z(i + 1, j, k)) -
                      (z(i + 1, j + 1, k) - z(i, j, k)) * (y(i, j + 1, k) - y(i + 1, j, k))) / 2;
        double dx = (si1 + sj1 + sk1) * (x(i + 1, j + 1, k + 1) - x(i, j, k));
        double si2 = ((z(i, j + 1, k + 1) - z(i, j, k)) * (x(i, j, k + 1) - x(i, j + 1, k)) -
                      (x(i, j + 1, k + 1) - x(i, j, k)) * (z(i, j, k + 1) - z(i, j + 1, k))) / 2;
        double sj2 = ((x(i + 1, j, k + 1) - x(i, j, k)) * (z(i, j, k + 1) - z(i + 1, j, k)) -
                      (z(i + 1, j, k + 1) - z(i, j, k)) * (x(i, j, k + 1) - x(i + 1, j, k))) / 2;
        double sk2 = ((z(i + 1, j + 1, k) - z(i, j, k)) * (x(i, j + 1, k) - x(i + 1, j, k)) -
                      (x(i + 1, j + 1, k) - x(i, j, k)) * (z(i, j + 1, k) - z(i + 1, j, k))) / 2;
        double dy = (si2 + sj2 + sk2) * (y(i + 1, j + 1, k + 1) - y(i, j, k));
        double si3 = ((x(i, j + 1, k + 1) - x(i, j, k)) * (y(i, j, k + 1) - y(i, j + 1, k)) -
                      (y(i, j + 1, k + 1) - y(i, j, k)) * (x(i, j, k + 1) - x(i, j + 1, k))) / 2;
        double sj3 = ((y(i + 1, j, k + 1) - y(i, j, k)) * (x(i, j, k + 1) - x(i + 1, j, k)) -
                      (x(i + 1, j, k + 1) - x(i, j, k)) * (y(i, j, k + 1) - y(i + 1, j, k))) / 2;
        double sk3 = ((x(i + 1, j + 1, k) - x(i, j, k)) * (y(i, j + 1, k) - y(i + 1, j, k)) -
                      (y(i + 1, j + 1, k) - y(i, j, k)) * (x(i, j + 1, k) - x(i + 1, j, k))) / 2;
        double dz = (si3 + sj3 + sk3) * (z(i + 1, j + 1, k + 1) - z(i, j, k));
        vol(i, j, k) = (dx + dy + dz) / 3;
      }
}

// ---- multigrid transfers ---------------------------------------------------
// rest1_b (src/cosa.f90:2788-2833): volume-weighted restriction of the
// solution onto the coarse interior cells
void rest1_b(const Level &L1, const Level &L2, int b, const double *q1a, double *q2a, const double *v1a,
             const double *v2a) {
  B3 q1(const_cast<double *>(q1a), L1, b), q2(q2a, L2, b);
  B1 v1(const_cast<double *>(v1a), L1, b, 1), v2(const_cast<double *>(v2a), L2, b, 1);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  for (int n = 0; n < L1.S; ++n)
    for (int k1 = 1; k1 <= km1 - 2; k1 += 2)
      for (int j1 = 1; j1 <= jm1 - 2; j1 += 2)
        for (int i1 = 1; i1 <= im1 - 2; i1 += 2) {
          const int i2 = 1 + i1 / 2, j2 = 1 + j1 / 2, k2 = 1 + k1 / 2;
          for (int v = 1; v <= L1.npde; ++v)
            q2(i2, j2, k2, v, n) =
                (v1(i1, j1, k1) * q1(i1, j1, k1, v, n) + v1(i1, j1 + 1, k1) * q1(i1, j1 + 1, k1, v, n) +
                 v1(i1 + 1, j1, k1) * q1(i1 + 1, j1, k1, v, n) + v1(i1 + 1, j1 + 1, k1) * q1(i1 + 1, j1 + 1, k1, v, n) +
                 v1(i1, j1, k1 + 1) * q1(i1, j1, k1 + 1, v, n) + v1(i1, j1 + 1, k1 + 1) * q1(i1, j1 + 1, k1 + 1, v, n) +
                 v1(i1 + 1, j1, k1 + 1) * q1(i1 + 1, j1, k1 + 1, v, n) +
                 v1(i1 + 1, j1 + 1, k1 + 1) * q1(i1 + 1, j1 + 1, k1 + 1, v, n)) /
                v2(i2, j2, k2);
        }
}

// rest2_lo_b (src/cosa.f90:2955-3012): rhs2 = -(sum of the 8 fine residuals)
void rest2_lo_b(const Level &L1, const Level &L2, int b, double *rhs2a, const double *res1a) {
  B3 r1(const_cast<double *>(res1a), L1, b), rhs2(rhs2a, L2, b);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  for (int n = 0; n < L1.S; ++n)
    for (int v = 1; v <= L1.npde; ++v)
      for (int k1 = 1; k1 <= km1 - 2; k1 += 2)
        for (int j1 = 1; j1 <= jm1 - 2; j1 += 2)
          for (int i1 = 1; i1 <= im1 - 2; i1 += 2) {
            const int i2 = 1 + i1 / 2, j2 = 1 + j1 / 2, k2 = 1 + k1 / 2;
            rhs2(i2, j2, k2, v, n) =
                -(r1(i1, j1, k1, v, n) + r1(i1, j1 + 1, k1, v, n) + r1(i1 + 1, j1, k1, v, n) +
                  r1(i1 + 1, j1 + 1, k1, v, n) + r1(i1, j1, k1 + 1, v, n) + r1(i1, j1 + 1, k1 + 1, v, n) +
                  r1(i1 + 1, j1, k1 + 1, v, n) + r1(i1 + 1, j1 + 1, k1 + 1, v, n));
          }
}

// rest2_ho_b (src/cosa.f90:2871-2954): rhs2 = -(27 x the 8 fine cells of the
// coarse cell + 9 x their 24 face neighbours + 3 x the 24 edge neighbours +
// the 8 corner neighbours) / 64, in the reference's summation order
void rest2_ho_b(const Level &L1, const Level &L2, int b, double *rhs2a, const double *res1a) {
  B3 r(const_cast<double *>(res1a), L1, b), rhs2(rhs2a, L2, b);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  for (int n = 0; n < L1.S; ++n)
    for (int v = 1; v <= L1.npde; ++v)
      for (int k1 = 1; k1 <= km1 - 2; k1 += 2)
        for (int j1 = 1; j1 <= jm1 - 2; j1 += 2)
          for (int i1 = 1; i1 <= im1 - 2; i1 += 2) {
            const int i2 = 1 + i1 / 2, j2 = 1 + j1 / 2, k2 = 1 + k1 / 2;
            const int i = i1, j = j1, k = k1;
            const double c27 = r(i, j, k, v, n) + r(i, j + 1, k, v, n) + r(i + 1, j, k, v, n) +
                               r(i + 1, j + 1, k, v, n) + r(i, j, k + 1, v, n) + r(i, j + 1, k + 1, v, n) +
                               r(i + 1, j, k + 1, v, n) + r(i + 1, j + 1, k + 1, v, n);
            const double c9 = r(i - 1, j, k, v, n) + r(i - 1, j + 1, k, v, n) + r(i + 2, j, k, v, n) +
                              r(i + 2, j + 1, k, v, n) + r(i - 1, j, k + 1, v, n) + r(i - 1, j + 1, k + 1, v, n) +
                              r(i + 2, j, k + 1, v, n) + r(i + 2, j + 1, k + 1, v, n) + r(i, j - 1, k, v, n) +
                              r(i + 1, j - 1, k, v, n) + r(i, j + 2, k, v, n) + r(i + 1, j + 2, k, v, n) +
                              r(i, j - 1, k + 1, v, n) + r(i + 1, j - 1, k + 1, v, n) + r(i, j + 2, k + 1, v, n) +
                              r(i + 1, j + 2, k + 1, v, n) + r(i, j, k - 1, v, n) + r(i, j + 1, k - 1, v, n) +
                              r(i, j, k + 2, v, n) + r(i, j + 1, k + 2, v, n) + r(i + 1, j, k - 1, v, n) +
                              r(i + 1, j + 1, k - 1, v, n) + r(i + 1, j, k + 2, v, n) + r(i + 1, j + 1, k + 2, v, n);
            const double c3 = r(i, j - 1, k - 1, v, n) + r(i + 1, j - 1, k - 1, v, n) + r(i, j + 2, k - 1, v, n) +
                              r(i + 1, j + 2, k - 1, v, n) + r(i - 1, j, k - 1, v, n) + r(i - 1, j + 1, k - 1, v, n) +
                              r(i + 2, j, k - 1, v, n) + r(i + 2, j + 1, k - 1, v, n) + r(i, j - 1, k + 2, v, n) +
                              r(i + 1, j - 1, k + 2, v, n) + r(i, j + 2, k + 2, v, n) + r(i + 1, j + 2, k + 2, v, n) +
                              r(i - 1, j, k + 2, v, n) + r(i - 1, j + 1, k + 2, v, n) + r(i + 2, j, k + 2, v, n) +
                              r(i + 2, j + 1, k + 2, v, n) + r(i - 1, j - 1, k, v, n) + r(i - 1, j - 1, k + 1, v, n) +
                              r(i - 1, j + 2, k, v, n) + r(i - 1, j + 2, k + 1, v, n) + r(i + 2, j - 1, k, v, n) +
                              r(i + 2, j - 1, k + 1, v, n) + r(i + 2, j + 2, k, v, n) + r(i + 2, j + 2, k + 1, v, n);
            const double c1 = r(i - 1, j - 1, k - 1, v, n) + r(i + 2, j - 1, k - 1, v, n) +
                              r(i - 1, j + 2, k - 1, v, n) + r(i + 2, j + 2, k - 1, v, n) +
                              r(i - 1, j - 1, k + 2, v, n) + r(i + 2, j - 1, k + 2, v, n) +
                              r(i - 1, j + 2, k + 2, v, n) + r(i + 2, j + 2, k + 2, v, n);
            rhs2(i2, j2, k2, v, n) = -(27 * c27 + 9 * c9 + 3 * c3 + c1) / 64;
          }
}

// bc_res / bbc_res / bc_res_bnd (src/bc.f90:2802-2995): at every patch the
// first halo layer = pm * first interior cell, pm = -1 on 15xx walls
void bc_res_level(const Level &L, double *ra) {
  for (int b = 0; b < L.nb; ++b) {
    B3 q(ra, L, b);
    const int *t = L.bct.data() + L.obct[b];
    for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
      Patch pa = patch_of(t + 10 * ibc, L.im[b], L.jm[b], L.km[b]);
      const double pm = pa.bctyp / 100 == 15 ? -1.0 : 1.0;
      const int ibcpt = pa.inrout == 1 ? 0 : pa.ijk[pa.idir];
      const int ibcn = pa.inrout == 1 ? 1 : pa.ijk[pa.idir] - 1;
      for (int n = 0; n < L.S; ++n)
        for (int v = 1; v <= L.npde; ++v)
          for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
            for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
              int a, bb, c, an, bn, cn;
              pidx(pa, ibcpt, i2, i3, a, bb, c);
              pidx(pa, ibcn, i2, i3, an, bn, cn);
              q(a, bb, c, v, n) = pm * q(an, bn, cn, v, n);
            }
    }
  }
}

// rest4_b (src/cosa.f90:3122-3160): volume-weighted restriction of a
// scalar P3 field (prd, delpls, divvel or mut)
void rest4_b(const Level &L1, const Level &L2, int b, const double *f1a, double *f2a, const double *v1a,
             const double *v2a) {
  B3s f1(const_cast<double *>(f1a), L1, b), f2(f2a, L2, b);
  B1 v1(const_cast<double *>(v1a), L1, b, 1), v2(const_cast<double *>(v2a), L2, b, 1);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  for (int n = 0; n < L1.S; ++n)
    for (int k1 = 1; k1 <= km1 - 2; k1 += 2)
      for (int j1 = 1; j1 <= jm1 - 2; j1 += 2)
        for (int i1 = 1; i1 <= im1 - 2; i1 += 2) {
          const int i2 = 1 + i1 / 2, j2 = 1 + j1 / 2, k2 = 1 + k1 / 2;
          f2(i2, j2, k2, n) =
              (v1(i1, j1, k1) * f1(i1, j1, k1, n) + v1(i1, j1 + 1, k1) * f1(i1, j1 + 1, k1, n) +
               v1(i1 + 1, j1, k1) * f1(i1 + 1, j1, k1, n) + v1(i1 + 1, j1 + 1, k1) * f1(i1 + 1, j1 + 1, k1, n) +
               v1(i1, j1, k1 + 1) * f1(i1, j1, k1 + 1, n) + v1(i1, j1 + 1, k1 + 1) * f1(i1, j1 + 1, k1 + 1, n) +
               v1(i1 + 1, j1, k1 + 1) * f1(i1 + 1, j1, k1 + 1, n) +
               v1(i1 + 1, j1 + 1, k1 + 1) * f1(i1 + 1, j1 + 1, k1 + 1, n)) /
              v2(i2, j2, k2);
        }
}

// lim_prod_mg_b (src/src.f90:708-745): the production limiter applied to
// prd before it is restricted; q is conservative here (the residual pass
// has converted it back), so tke and ome are rho k and rho omega
void lim_prod_mg_b(const Level &L, int b, const double *qa, double *prda, const double *muta,
                   const cosa_params &P) {
  B3 q(const_cast<double *>(qa), L, b);
  B3s prd(prda, L, b), mu(const_cast<double *>(muta), L, b);
  const double mor = P.machfs / P.reyno;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double rho = q(i, j, k, 1, n), tke = q(i, j, k, 6, n), ome = q(i, j, k, 7, n);
          const double mut = mu(i, j, k, n), prod = prd(i, j, k, n);
          const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
          if (mor * mut * prod > tstdis) prd(i, j, k, n) = tstdis / mor / mut;
        }
}

// lim_res_ome_b (src/update.f90:2585-2835), explicit branch without
// low-speed preconditioning: the omega residual is limited so that the
// point-implicit update cannot take rho omega below gkw cmu rho sqrt(prd);
// ttrm = (0, gkw, bkw) for the Wilcox model
void lim_res_ome_b(const Level &L, int b, double *ra, const double *qa, const double *va, const double *dtta,
                   const double *dpla, const double *prda, double ar, const cosa_params &P,
                   const double *ttrma = nullptr) {
  B3 res(ra, L, b), q(const_cast<double *>(qa), L, b);
  B1 vol(const_cast<double *>(va), L, b, 1), dtt(const_cast<double *>(dtta), L, b, L.S);
  B3s dpl(const_cast<double *>(dpla), L, b), prd(const_cast<double *>(prda), L, b);
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double gav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 2, n) : P.gkw;
          const double bav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 3, n) : P.bkw;
          const double dtau = dtt(i, j, k, n) * vol(i, j, k);
          const double rho = q(i, j, k, 1, n), ome = q(i, j, k, 7, n) / q(i, j, k, 1, n);
          if (P.rkimp && P.dualt) {
            // rkimp (src/update.f90:2785-2823): the physical-time term in the
            // denominator; the reference's den1 has no ar here
            const double fact = P.bdf1 ? 1.0 : 1.5;
            const double den1 = 1 + dtau * (gav * dpl(i, j, k, n) + 2 * bav * ome);
            const double den2 = ar * fact * dtau / P.dt;
            const double rhomega = q(i, j, k, 7, n) - ar * res(i, j, k, 7, n) * dtt(i, j, k, n) / (den1 + den2);
            const double rhomegamin = gav * P.cmu * rho * std::sqrt(prd(i, j, k, n));
            if (rhomega < rhomegamin)
              res(i, j, k, 7, n) = ((den1 + den2) * (q(i, j, k, 7, n) - rhomegamin)) / dtt(i, j, k, n) / ar;
            continue;
          }
          const double den1 = 1 + ar * dtau * (gav * dpl(i, j, k, n) + 2 * bav * ome);
          const double rhomega = q(i, j, k, 7, n) - ar * res(i, j, k, 7, n) * dtt(i, j, k, n) / den1;
          const double rhomegamin = gav * P.cmu * rho * std::sqrt(prd(i, j, k, n));
          if (rhomega < rhomegamin) res(i, j, k, 7, n) = den1 * (q(i, j, k, 7, n) - rhomegamin) / dtt(i, j, k, n) / ar;
        }
}

// q_bedges (src/flux.f90:3913-4263): the plane through three neighbours of
// each halo edge cell, evaluated at the edge cell.  Edge families: (i,j) at
// every interior k, (i,k) at every interior j, (j,k) at every interior i.
struct Edge2 { int x[4], y[4]; };
inline void edge_fit(double q1, double q2, double q3, const Edge2 &e, double &out) {
  const int x0 = e.x[0], y0 = e.y[0], x1 = e.x[1], y1 = e.y[1], x2 = e.x[2], y2 = e.y[2], x3 = e.x[3], y3 = e.y[3];
  const double b = ((q3 - q1) * (double)(x2 - x1) - (q2 - q1) * (double)(x3 - x1)) /
                   (double)((y3 - y1) * (x2 - x1) - (y2 - y1) * (x3 - x1));
  const double a = (q2 - q1 - b * (double)(y2 - y1)) / (double)(x2 - x1);
  const double c = q1 - a * (double)x1 - b * (double)y1;
  out = a * (double)x0 + b * (double)y0 + c;
}
// the 4 edges of one family: points 0 (target), 1, 2, 3 in the reference's order
inline void edge_table(int m1, int m2, Edge2 e[4]) {
  e[0] = {{0, 0, 1, 1}, {0, 1, 0, 1}};
  e[1] = {{m1, m1, m1 - 1, m1 - 1}, {0, 1, 0, 1}};
  e[2] = {{m1, m1, m1 - 1, m1 - 1}, {m2, m2 - 1, m2, m2 - 1}};
  e[3] = {{0, 0, 1, 1}, {m2, m2 - 1, m2, m2 - 1}};
}
void q_bedges(const Level &L, int b, double *qa, double *muta) {
  B3 q(qa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  Edge2 eij[4], eik[4], ejk[4];
  edge_table(im, jm, eij);
  edge_table(im, km, eik);
  edge_table(jm, km, ejk);
  auto fam = [&](auto &&at, int nv, int nsnap, const Edge2 *E, int lo, int hi) {
    for (int n = 0; n < nsnap; ++n)
      for (int v = 1; v <= nv; ++v)
        for (int t = lo; t <= hi; ++t)
          for (int ic = 0; ic < 4; ++ic) {
            const Edge2 &e = E[ic];
            double o;
            edge_fit(at(e.x[1], e.y[1], t, v, n), at(e.x[2], e.y[2], t, v, n), at(e.x[3], e.y[3], t, v, n), e, o);
            at(e.x[0], e.y[0], t, v, n) = o;
          }
  };
  auto qij = [&](int a, int c, int t, int v, int n) -> double & { return q(a, c, t, v, n); };
  auto qik = [&](int a, int c, int t, int v, int n) -> double & { return q(a, t, c, v, n); };
  auto qjk = [&](int a, int c, int t, int v, int n) -> double & { return q(t, a, c, v, n); };
  if (muta) {
    B3s mu(muta, L, b);
    auto mij = [&](int a, int c, int t, int, int n) -> double & { return mu(a, c, t, n); };
    auto mik = [&](int a, int c, int t, int, int n) -> double & { return mu(a, t, c, n); };
    auto mjk = [&](int a, int c, int t, int, int n) -> double & { return mu(t, a, c, n); };
    fam(qij, L.npde, L.S, eij, 1, km - 1); fam(mij, 1, L.S, eij, 1, km - 1);
    fam(qik, L.npde, L.S, eik, 1, jm - 1); fam(mik, 1, L.S, eik, 1, jm - 1);
    fam(qjk, L.npde, L.S, ejk, 1, im - 1); fam(mjk, 1, L.S, ejk, 1, im - 1);
  } else {
    fam(qij, L.npde, L.S, eij, 1, km - 1);
    fam(qik, L.npde, L.S, eik, 1, jm - 1);
    fam(qjk, L.npde, L.S, ejk, 1, im - 1);
  }
}

// q_bcorns (src/flux.f90:3156-3469): the plane a i + b j + c k + d through
// four neighbours of each of the 8 halo corner cells.  The coefficient
// expressions are integer arithmetic in the reference (every integer
// division is by +-1, so exact); they are kept as ints here.
struct Corner { int x[5], y[5], z[5]; };
inline void corner_table(int im, int jm, int km, Corner c[8]) {
  // points 0 (target), 1..4 in the reference's order (ijkc(:,0:4,ic))
  c[0] = {{0, 0, 1, 1, 1}, {0, 1, 1, 0, 1}, {0, 1, 0, 1, 1}};
  c[1] = {{im, im, im - 1, im - 1, im - 1}, {0, 1, 1, 0, 1}, {0, 1, 0, 1, 1}};
  c[2] = {{im, im, im - 1, im - 1, im - 1}, {jm, jm - 1, jm - 1, jm, jm - 1}, {0, 1, 0, 1, 1}};
  c[3] = {{0, 0, 1, 1, 1}, {jm, jm - 1, jm - 1, jm, jm - 1}, {0, 1, 0, 1, 1}};
  c[4] = {{0, 0, 1, 1, 1}, {0, 1, 1, 0, 1}, {km, km - 1, km, km - 1, km - 1}};
  c[5] = {{im, im, im - 1, im - 1, im - 1}, {0, 1, 1, 0, 1}, {km, km - 1, km, km - 1, km - 1}};
  c[6] = {{im, im, im - 1, im - 1, im - 1}, {jm, jm - 1, jm - 1, jm, jm - 1}, {km, km - 1, km, km - 1, km - 1}};
  c[7] = {{0, 0, 1, 1, 1}, {jm, jm - 1, jm - 1, jm, jm - 1}, {km, km - 1, km, km - 1, km - 1}};
}
inline double corner_fit(const Corner &C, double q1, double q2, double q3, double q4) {
  const int *x = C.x, *y = C.y, *z = C.z;
  const int dz = z[2] - z[1];
  const int t1 = ((z[3] - z[1]) * (y[4] - y[1]) - (z[4] - z[1]) * (y[3] - y[1])) / dz;
  const int t2 = ((z[2] - z[1]) * (y[1] - y[4]) + (z[4] - z[1]) * (y[2] - y[1])) / dz;
  const int t3 = ((z[2] - z[1]) * (y[3] - y[1]) + (z[3] - z[1]) * (y[1] - y[2])) / dz;
  const int den = ((x[4] - x[1]) * (y[3] - y[1]) + (x[1] - x[3]) * (y[4] - y[1])) +
                  ((x[4] - x[1]) * (y[1] - y[2]) + (x[2] - x[1]) * (y[4] - y[1])) * (z[3] - z[1]) / dz +
                  ((x[1] - x[2]) * (y[3] - y[1]) + (x[1] - x[3]) * (y[1] - y[2])) * (z[4] - z[1]) / dz;
  const double a = ((double)t1 * (q2 - q1) + (double)t2 * (q3 - q1) + (double)t3 * (q4 - q1)) / (double)den;
  const int e1 = (x[1] - x[3]) + (x[2] - x[1]) * (z[3] - z[1]) / dz;
  const int f1 = (z[3] - z[1]) / dz;
  const int g1 = (y[3] - y[1]) + (y[1] - y[2]) * (z[3] - z[1]) / dz;
  const double bb = ((double)e1 * a + (double)f1 * (q1 - q2) + (q3 - q1)) / (double)g1;
  const double c = ((double)(x[1] - x[2]) * a + (double)(y[1] - y[2]) * bb + (q2 - q1)) / (double)dz;
  const double d = q1 - a * (double)x[1] - bb * (double)y[1] - c * (double)z[1];
  return a * (double)x[0] + bb * (double)y[0] + c * (double)z[0] + d;
}
void q_bcorns(const Level &L, int b, double *qa, double *muta) {
  B3 q(qa, L, b);
  Corner C[8];
  corner_table(L.im[b], L.jm[b], L.km[b], C);
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int ic = 0; ic < 8; ++ic) {
        const Corner &c = C[ic];
        q(c.x[0], c.y[0], c.z[0], v, n) =
            corner_fit(c, q(c.x[1], c.y[1], c.z[1], v, n), q(c.x[2], c.y[2], c.z[2], v, n),
                       q(c.x[3], c.y[3], c.z[3], v, n), q(c.x[4], c.y[4], c.z[4], v, n));
      }
  if (muta) {
    B3s mu(muta, L, b);
    for (int n = 0; n < L.S; ++n)
      for (int ic = 0; ic < 8; ++ic) {
        const Corner &c = C[ic];
        mu(c.x[0], c.y[0], c.z[0], n) = corner_fit(c, mu(c.x[1], c.y[1], c.z[1], n), mu(c.x[2], c.y[2], c.z[2], n),
                                                   mu(c.x[3], c.y[3], c.z[3], n), mu(c.x[4], c.y[4], c.z[4], n));
      }
  }
}

// prol_bln_b (src/cosa.f90:3478-3888): trilinear (27/9/3/1)/64 prolongation
// of the coarse correction onto fine cells 0..imax1 (one halo layer
// included); turbulence variables only with one of the three positivity
// options (lim_corr 1..3).
inline double prol_w(double a, double b, double c, double d, double e, double f, double g, double h) {
  return (27 * a + 9 * b + 9 * c + 3 * d + 9 * e + 3 * f + 3 * g + h) / 64;
}
inline double lim2(double q, double c) {
  if ((q + c) <= 0) {
    if ((q + c / 2) > 0) return c / 2;
    if ((q + c / 4) > 0) return c / 4;
    return 0.0;
  }
  return c;
}
void prol_bln_b(const Level &L1, const Level &L2, int b, double *q1a, const double *q2a, int lim_corr) {
  B3 q1(q1a, L1, b), q2(const_cast<double *>(q2a), L2, b);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  const double beta = 100.0, epsl = 1.0e-12;
  for (int n = 0; n < L1.S; ++n)
    for (int v = 1; v <= L1.npde; ++v) {
      if (v >= 6 && lim_corr == 0) continue;
      for (int k1 = 0; k1 <= km1 - 1; k1 += 2)
        for (int j1 = 0; j1 <= jm1 - 1; j1 += 2)
          for (int i1 = 0; i1 <= im1 - 1; i1 += 2) {
            const int i2 = i1 / 2, j2 = j1 / 2, k2 = k1 / 2;
            const double nel = q2(i2 + 1, j2 + 1, k2, v, n), nwl = q2(i2, j2 + 1, k2, v, n);
            const double sel = q2(i2 + 1, j2, k2, v, n), swl = q2(i2, j2, k2, v, n);
            const double neu = q2(i2 + 1, j2 + 1, k2 + 1, v, n), nwu = q2(i2, j2 + 1, k2 + 1, v, n);
            const double seu = q2(i2 + 1, j2, k2 + 1, v, n), swu = q2(i2, j2, k2 + 1, v, n);
            double swf_l = prol_w(swl, sel, nwl, nel, swu, seu, nwu, neu);
            double sef_l = prol_w(sel, swl, nel, nwl, seu, swu, neu, nwu);
            double nef_l = prol_w(nel, nwl, sel, swl, neu, nwu, seu, swu);
            double nwf_l = prol_w(nwl, nel, swl, sel, nwu, neu, swu, seu);
            double swf_u = prol_w(swu, seu, nwu, neu, swl, sel, nwl, nel);
            double sef_u = prol_w(seu, swu, neu, nwu, sel, swl, nel, nwl);
            double nef_u = prol_w(neu, nwu, seu, swu, nel, nwl, sel, swl);
            double nwf_u = prol_w(nwu, neu, swu, seu, nwl, nel, swl, sel);
            double &a0 = q1(i1, j1, k1, v, n), &a1 = q1(i1 + 1, j1, k1, v, n);
            double &a2 = q1(i1 + 1, j1 + 1, k1, v, n), &a3 = q1(i1, j1 + 1, k1, v, n);
            double &a4 = q1(i1, j1, k1 + 1, v, n), &a5 = q1(i1 + 1, j1, k1 + 1, v, n);
            double &a6 = q1(i1 + 1, j1 + 1, k1 + 1, v, n), &a7 = q1(i1, j1 + 1, k1 + 1, v, n);
            if (v >= 6 && lim_corr == 2) {
              // the NE limits test the SE values in the reference (kept)
              const double qsw_l = a0, qse_l = a1, qne_l = a2, qnw_l = a3;
              const double qsw_u = a4, qse_u = a5, qne_u = a6, qnw_u = a7;
              swf_l = lim2(qsw_l, swf_l);
              sef_l = lim2(qse_l, sef_l);
              if ((qne_l + nef_l) <= 0) {
                if ((qne_l + nef_l / 2) > 0) nef_l = nef_l / 2;
                else if ((qse_l + sef_l / 4) > 0) nef_l = nef_l / 4;
                else nef_l = 0.0;
              }
              nwf_l = lim2(qnw_l, nwf_l);
              swf_u = lim2(qsw_u, swf_u);
              sef_u = lim2(qse_u, sef_u);
              if ((qne_u + nef_u) <= 0) {
                if ((qne_u + nef_u / 2) > 0) nef_u = nef_u / 2;
                else if ((qse_u + sef_u / 4) > 0) nef_u = nef_u / 4;
                else nef_u = 0.0;
              }
              nwf_u = lim2(qnw_u, nwf_u);
            }
            if (v >= 6 && lim_corr == 3) {
              auto el = [&](double &q, double c) { q = q + c / (1 - beta * std::min(c / (q + epsl), 0.0)); };
              el(a0, swf_l); el(a1, sef_l); el(a2, nef_l); el(a3, nwf_l);
              el(a4, swf_u); el(a5, sef_u); el(a6, nef_u); el(a7, nwf_u);
            } else {
              a0 = a0 + swf_l; a1 = a1 + sef_l; a2 = a2 + nef_l; a3 = a3 + nwf_l;
              a4 = a4 + swf_u; a5 = a5 + sef_u; a6 = a6 + nef_u; a7 = a7 + nwf_u;
            }
          }
    }
}

// prol_lin_b (src/cosa.f90:3315-3476): volume-weighted bilinear interpolation
// in each coarse k plane, then a volume-weighted blend between the planes
void prol_lin_b(const Level &L1, const Level &L2, int b, double *q1a, const double *q2a, const double *v1a) {
  B3 q1(q1a, L1, b), q2(const_cast<double *>(q2a), L2, b);
  B1 vol(const_cast<double *>(v1a), L1, b, 1);
  const int im1 = L1.im[b], jm1 = L1.jm[b], km1 = L1.km[b];
  for (int n = 0; n < L1.S; ++n)
    for (int v = 1; v <= L1.npde; ++v)
      for (int k1 = 0; k1 <= km1 - 1; k1 += 2)
        for (int j1 = 0; j1 <= jm1 - 1; j1 += 2)
          for (int i1 = 0; i1 <= im1 - 1; i1 += 2) {
            const int i2 = i1 / 2, j2 = j1 / 2, k2 = k1 / 2;
            double f[2][4];  // [plane][sw, se, nw, ne]
            for (int pl = 0; pl < 2; ++pl) {
              const int kc = k2 + pl, kf = k1 + pl;
              const double cne = q2(i2 + 1, j2 + 1, kc, v, n), cnw = q2(i2, j2 + 1, kc, v, n);
              const double cse = q2(i2 + 1, j2, kc, v, n), csw = q2(i2, j2, kc, v, n);
              const double dn = cne - cnw, ds = cse - csw, de = cne - cse, dw = cnw - csw;
              const double v00 = vol(i1, j1, kf), v10 = vol(i1 + 1, j1, kf), v01 = vol(i1, j1 + 1, kf),
                           v11 = vol(i1 + 1, j1 + 1, kf);
              f[pl][0] = csw + ds / 2 * v00 / (v00 + v10) + dw / 2 * v00 / (v00 + v01);
              f[pl][1] = cse - ds / 2 * v10 / (v00 + v10) + de / 2 * v10 / (v10 + v11);
              f[pl][2] = cnw + dn / 2 * v01 / (v01 + v11) - dw / 2 * v01 / (v00 + v01);
              f[pl][3] = cne - dn / 2 * v11 / (v11 + v01) - de / 2 * v11 / (v11 + v10);
            }
            const int di[4] = {0, 1, 0, 1}, dj[4] = {0, 0, 1, 1};
            // reference order of the corrections: sw, se, ne, nw
            const int ord[4] = {0, 1, 3, 2};
            for (int t = 0; t < 4; ++t) {
              const int c = ord[t], ii = i1 + di[c], jj = j1 + dj[c];
              const double fact = vol(ii, jj, k1) / 2 / (vol(ii, jj, k1) + vol(ii, jj, k1 + 1));
              q1(ii, jj, k1, v, n) = q1(ii, jj, k1, v, n) + f[0][c] + fact / 2 * (f[1][c] - f[0][c]);
              q1(ii, jj, k1 + 1, v, n) = q1(ii, jj, k1 + 1, v, n) + f[1][c] - (1 - fact) / 2 * (f[1][c] - f[0][c]);
            }
          }
}

// add_array over cells 0..imax (off_l = 1) or the interior (off_l = -1)
// (src/util.f90:137-222)
void add_level(const Level &L, double *v1a, const double *v2a, double fact, int off_l) {
  const int lo = off_l == 1 ? 0 : 1, hi_off = off_l == 1 ? 0 : -1;
  for (int b = 0; b < L.nb; ++b) {
    B3 a(v1a, L, b), c(const_cast<double *>(v2a), L, b);
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int k = lo; k <= L.km[b] + hi_off; ++k)
          for (int j = lo; j <= L.jm[b] + hi_off; ++j)
            for (int i = lo; i <= L.im[b] + hi_off; ++i) a(i, j, k, v, n) = a(i, j, k, v, n) + c(i, j, k, v, n) * fact;
  }
}

// fixq_b (src/update.f90:2216-2269): floors of k and omega
void fixq_level(const Level &L, double *qa, const cosa_params &P) {
  if (L.npde < 7) return;
  for (int b = 0; b < L.nb; ++b) {
    B3 q(qa, L, b);
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            const double rho = q(i, j, k, 1, n);
            double tke = q(i, j, k, 6, n) / rho, ome = q(i, j, k, 7, n) / rho;
            if (tke < P.qmin[5]) { tke = P.qmin[5]; q(i, j, k, 6, n) = rho * tke; }
            if (ome < P.qmin[6]) { ome = P.qmin[6]; q(i, j, k, 7, n) = rho * ome; }
          }
  }
}

// tur_vis_b (src/update.f90:2297-2337): mut over cells 0..imax
void tur_vis_level(const Level &L, const double *qa, double *muta, const cosa_params &P) {
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b);
    B3s mu(muta, L, b);
    for (int n = 0; n < L.S; ++n)
      for (int k = 0; k <= L.km[b]; ++k)
        for (int j = 0; j <= L.jm[b]; ++j)
          for (int i = 0; i <= L.im[b]; ++i) {
            const double rho = q(i, j, k, 1, n), tke = q(i, j, k, 6, n), ome = q(i, j, k, 7, n);
            mu(i, j, k, n) = P.cmu * rho * tke / (ome + P.epst) * P.reyno / P.machfs;
          }
  }
}

// ---- viscous set-up (src/grid.f90) -----------------------------------------
struct BGw {  // writable grid view (0:im+1, 0:jm+1, 0:km+1) of snapshot nh (moving grids: dim5h snapshots)
  double *p; int I, J;
  BGw(double *base, const Level &L, int b, int nh = 0) : I(L.im[b] + 2), J(L.jm[b] + 2) {
    p = base + L.op2[b] * L.dim5h + (int64_t)nh * I * J * (L.km[b] + 2);
  }
  inline double &operator()(int i, int j, int k) const { return p[i + (int64_t)I * (j + (int64_t)J * k)]; }
};
struct BV {  // face inverse metrics (3, imax, jmax, kmax), 1-based face index
  double *p; int I, J;
  BV(double *base, const Level &L, int b) : I(L.im[b]), J(L.jm[b]) { p = base + L.of0[b] * 3; }
  inline double &operator()(int c, int i, int j, int k) const {
    return p[((i - 1) + (int64_t)I * ((j - 1) + (int64_t)J * (k - 1))) * 3 + (c - 1)];
  }
};

// the face inverse metrics of grid snapshot nh (moving grids keep one set of
// 27 n0 values per snapshot, xideri(.., 0:2*nharms*hbmove))
inline const double *vm_snap(const Level &L, const double *vm, int nh) { return vm + (int64_t)nh * 27 * L.n0; }

// cordex_b (src/grid.f90:20-80): ghost nodes repeat the boundary nodes
void coordex_level(const Level &L, double *xa, double *ya, double *za, int nh = 0) {
  for (int b = 0; b < L.nb; ++b) {
    const int im = L.im[b], jm = L.jm[b], km = L.km[b];
    for (double *a : {xa, ya, za}) {
      BGw X(a, L, b, nh);
      for (int k = 1; k <= km; ++k) {
        for (int i = 1; i <= im; ++i) { X(i, 0, k) = X(i, 1, k); X(i, jm + 1, k) = X(i, jm, k); }
        for (int j = 1; j <= jm; ++j) { X(0, j, k) = X(1, j, k); X(im + 1, j, k) = X(im, j, k); }
      }
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) { X(i, j, 0) = X(i, j, 1); X(i, j, km + 1) = X(i, j, km); }
    }
  }
}

// cut_x, in-process branch (src/grid.f90:242-523): the ghost node plane of
// block 1 takes the nodes one plane inside block 2
void cutman_x_level(const Level &L, double *xa, double *ya, double *za, int nh = 0) {
  for (int icut = 0; icut < L.ncuts; ++icut) {
    const int *c = L.cut.data() + 21 * icut;
    const int b1 = c[0] - 1, b2 = c[9] - 1;
    int ijk1[4] = {0, L.im[b1], L.jm[b1], L.km[b1]}, ijk2[4] = {0, L.im[b2], L.jm[b2], L.km[b2]};
    const int idir1 = c[1], inout1 = c[2], idir2 = c[10], inout2 = c[11];
    int istr1[4] = {0, c[3], c[5], c[7]}, iend1[4] = {0, c[4], c[6], c[8]};
    int istr2[4] = {0, c[12], c[14], c[16]}, iend2[4] = {0, c[13], c[15], c[17]};
    const int iord[4] = {0, c[18], c[19], c[20]};
    const int ibcpt = inout1 == 1 ? 0 : ijk1[idir1] + 1;
    const int inr = inout2 == 1 ? 2 : ijk2[idir2] - 1;
    for (int l = 1; l <= 3; ++l)
      if (l != idir1) { if (iend1[l] > istr1[l]) iend1[l] += 1; else istr1[l] += 1; }
    for (int l = 1; l <= 3; ++l)
      if (l != idir2) { if (iend2[l] > istr2[l]) iend2[l] += 1; else istr2[l] += 1; }
    int len[4], isgn1[4], isgn2[4];
    for (int l = 1; l <= 3; ++l) {
      len[l] = std::abs(iend1[l] - istr1[l]);
      isgn1[l] = iend1[l] > istr1[l] ? 1 : -1;
      isgn2[l] = iend2[l] > istr2[l] ? 1 : -1;
    }
    const int ic1 = cyc(idir1, 1), ic2 = cyc(idir1, 2), ic3 = cyc(idir1, 3);
    const int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
    for (double *a : {xa, ya, za}) {
      BGw X1(a, L, b1, nh), X2(a, L, b2, nh);
      for (int i3 = 0; i3 <= len[ic3]; ++i3)
        for (int i2 = 0; i2 <= len[ic2]; ++i2) {
          const int a2_ = istr1[ic2] + isgn1[ic2] * i2, a3_ = istr1[ic3] + isgn1[ic3] * i3;
          const int ii1 = ibcpt * krd(ic1, 1) + a2_ * krd(ic2, 1) + a3_ * krd(ic3, 1);
          const int jj1 = ibcpt * krd(ic1, 2) + a2_ * krd(ic2, 2) + a3_ * krd(ic3, 2);
          const int kk1 = ibcpt * krd(ic1, 3) + a2_ * krd(ic2, 3) + a3_ * krd(ic3, 3);
          const int b2_ = istr2[jc2] + isgn2[jc2] * i2, b3_ = istr2[jc3] + isgn2[jc3] * i3;
          const int in1 = inr * krd(jc1, 1) + b2_ * krd(jc2, 1) + b3_ * krd(jc3, 1);
          const int jn1 = inr * krd(jc1, 2) + b2_ * krd(jc2, 2) + b3_ * krd(jc3, 2);
          const int kn1 = inr * krd(jc1, 3) + b2_ * krd(jc2, 3) + b3_ * krd(jc3, 3);
          X1(ii1, jj1, kk1) = X2(in1, jn1, kn1);
        }
    }
  }
}

// volex_b (src/grid.f90:110-136): face-halo volumes repeat the first cell
void volex_level(const Level &L, double *va) {
  for (int b = 0; b < L.nb; ++b) {
    B1 vol(va, L, b, 1);
    const int im = L.im[b], jm = L.jm[b], km = L.km[b];
    for (int k = 1; k <= km - 1; ++k) {
      for (int i = 1; i <= im - 1; ++i) { vol(i, 0, k) = vol(i, 1, k); vol(i, jm, k) = vol(i, jm - 1, k); }
      for (int j = 1; j <= jm - 1; ++j) { vol(0, j, k) = vol(1, j, k); vol(im, j, k) = vol(im - 1, j, k); }
    }
    for (int j = 1; j <= jm - 1; ++j)
      for (int i = 1; i <= im - 1; ++i) { vol(i, j, 0) = vol(i, j, 1); vol(i, j, km) = vol(i, j, km - 1); }
  }
}

// cut_v, in-process branch (src/grid.f90:612-700): one halo layer of volumes
void cutman_v_level(const Level &L, double *va) {
  for (int icut = 0; icut < L.ncuts; ++icut) {
    const int *c = L.cut.data() + 21 * icut;
    const int b1 = c[0] - 1, b2 = c[9] - 1;
    int ijk1[4] = {0, L.im[b1], L.jm[b1], L.km[b1]}, ijk2[4] = {0, L.im[b2], L.jm[b2], L.km[b2]};
    const int idir1 = c[1], inout1 = c[2], idir2 = c[10], inout2 = c[11];
    const int istr1[4] = {0, c[3], c[5], c[7]}, iend1[4] = {0, c[4], c[6], c[8]};
    const int istr2[4] = {0, c[12], c[14], c[16]}, iend2[4] = {0, c[13], c[15], c[17]};
    const int iord[4] = {0, c[18], c[19], c[20]};
    const int ibcpt = inout1 == 1 ? 0 : ijk1[idir1];
    const int inr = inout2 == 1 ? 1 : ijk2[idir2] - 1;
    int len[4], isgn1[4], isgn2[4];
    for (int l = 1; l <= 3; ++l) {
      len[l] = std::abs(iend1[l] - istr1[l]);
      isgn1[l] = iend1[l] > istr1[l] ? 1 : -1;
      isgn2[l] = iend2[l] > istr2[l] ? 1 : -1;
    }
    const int ic1 = cyc(idir1, 1), ic2 = cyc(idir1, 2), ic3 = cyc(idir1, 3);
    const int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
    B1 v1(va, L, b1, 1), v2(va, L, b2, 1);
    for (int i3 = 0; i3 <= len[ic3]; ++i3)
      for (int i2 = 0; i2 <= len[ic2]; ++i2) {
        const int a2_ = istr1[ic2] + isgn1[ic2] * i2, a3_ = istr1[ic3] + isgn1[ic3] * i3;
        const int ii1 = ibcpt * krd(ic1, 1) + a2_ * krd(ic2, 1) + a3_ * krd(ic3, 1);
        const int jj1 = ibcpt * krd(ic1, 2) + a2_ * krd(ic2, 2) + a3_ * krd(ic3, 2);
        const int kk1 = ibcpt * krd(ic1, 3) + a2_ * krd(ic2, 3) + a3_ * krd(ic3, 3);
        const int b2_ = istr2[jc2] + isgn2[jc2] * i2, b3_ = istr2[jc3] + isgn2[jc3] * i3;
        const int in1 = inr * krd(jc1, 1) + b2_ * krd(jc2, 1) + b3_ * krd(jc3, 1);
        const int jn1 = inr * krd(jc1, 2) + b2_ * krd(jc2, 2) + b3_ * krd(jc3, 2);
        const int kn1 = inr * krd(jc1, 3) + b2_ * krd(jc2, 3) + b3_ * krd(jc3, 3);
        v1(ii1, jj1, kk1) = v2(in1, jn1, kn1);
      }
  }
}

// vmetrix_b (src/grid.f90:3150-3582): the inverse metrics xi_x .. zeta_z on
// the faces of family d from node differences averaged over the face, with
// one-sided differences doubled where a ghost node coincides with its node
// (coordex), divided by the mean volume of the two cells of the face.
// vm[m] receives (xi, eta, zeta)_(x, y, z) for m = xi, eta, zeta.
void vmetrix_b(const Level &L, int b, int d, const double *xa, const double *ya, const double *za,
               const double *va, double *vm0, double *vm1, double *vm2, int nh = 0) {
  BGw X(const_cast<double *>(xa), L, b, nh), Y(const_cast<double *>(ya), L, b, nh), Z(const_cast<double *>(za), L, b, nh);
  B1 vol(const_cast<double *>(va), L, b, 1);
  BV o0(vm0, L, b), o1(vm1, L, b), o2(vm2, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const int ijkm[4] = {0, im, jm, km};
  // unit offsets and the corner lists of the reference
  auto e = [](int dir, int o[3]) { o[0] = dir == 1; o[1] = dir == 2; o[2] = dir == 3; };
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i) {
        const int p[3] = {i, j, k};
        double g[4][3][5];  // g[dir][xyz][0..4]
        for (int dir = 1; dir <= 3; ++dir) {
          int ed[3];
          e(dir, ed);
          if (dir == d) {
            // 4 corners of the face in the reference's order
            int cr[4][3];
            if (d == 1) { int t[4][3] = {{0,0,0},{0,1,0},{0,1,1},{0,0,1}}; std::memcpy(cr, t, sizeof t); }
            else if (d == 2) { int t[4][3] = {{0,0,0},{0,0,1},{1,0,1},{1,0,0}}; std::memcpy(cr, t, sizeof t); }
            else { int t[4][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0}}; std::memcpy(cr, t, sizeof t); }
            const int pos = p[d - 1];
            for (int m = 0; m < 4; ++m) {
              const int a0 = p[0] + cr[m][0], a1 = p[1] + cr[m][1], a2 = p[2] + cr[m][2];
              const int hp[3] = {a0 + ed[0], a1 + ed[1], a2 + ed[2]}, hm[3] = {a0 - ed[0], a1 - ed[1], a2 - ed[2]};
              double v3[3];
              int c = 0;
              for (BGw *A : {&X, &Y, &Z}) {
                v3[c] = ((*A)(hp[0], hp[1], hp[2]) - (*A)(hm[0], hm[1], hm[2])) / 2;
                ++c;
              }
              if (pos == 1 || pos == ijkm[d]) {
                const int *gh = pos == 1 ? hm : hp;
                const double dx = X(gh[0], gh[1], gh[2]) - X(a0, a1, a2);
                const double dy = Y(gh[0], gh[1], gh[2]) - Y(a0, a1, a2);
                const double dz = Z(gh[0], gh[1], gh[2]) - Z(a0, a1, a2);
                const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (dist < 1.0e-14) for (int c2 = 0; c2 < 3; ++c2) v3[c2] = 2 * v3[c2];
              }
              for (int c2 = 0; c2 < 3; ++c2) g[dir][c2][m + 1] = v3[c2];
            }
            for (int c2 = 0; c2 < 3; ++c2)
              g[dir][c2][0] = (g[dir][c2][1] + g[dir][c2][2] + g[dir][c2][3] + g[dir][c2][4]) / 4;
          } else {
            // two edge differences along dir, at the reference's positions
            int s[2][3];
            const int other = 6 - d - dir;  // the remaining direction
            int eo[3];
            e(other, eo);
            s[0][0] = 0; s[0][1] = 0; s[0][2] = 0;
            s[1][0] = eo[0]; s[1][1] = eo[1]; s[1][2] = eo[2];
            for (int m = 0; m < 2; ++m) {
              const int a0 = p[0] + s[m][0], a1 = p[1] + s[m][1], a2 = p[2] + s[m][2];
              int c = 0;
              for (BGw *A : {&X, &Y, &Z}) {
                g[dir][c][m + 1] = (*A)(a0 + ed[0], a1 + ed[1], a2 + ed[2]) - (*A)(a0, a1, a2);
                ++c;
              }
            }
            for (int c2 = 0; c2 < 3; ++c2) g[dir][c2][0] = (g[dir][c2][1] + g[dir][c2][2]) / 2;
          }
        }
        double volvisc;
        if (d == 1) volvisc = (vol(i - 1, j, k) + vol(i, j, k)) / 2;
        else if (d == 2) volvisc = (vol(i, j, k) + vol(i, j - 1, k)) / 2;
        else volvisc = (vol(i, j, k) + vol(i, j, k - 1)) / 2;
        const double x_xi = g[1][0][0], y_xi = g[1][1][0], z_xi = g[1][2][0];
        const double x_eta = g[2][0][0], y_eta = g[2][1][0], z_eta = g[2][2][0];
        const double x_zeta = g[3][0][0], y_zeta = g[3][1][0], z_zeta = g[3][2][0];
        o0(1, i, j, k) = (z_zeta * y_eta - z_eta * y_zeta) / volvisc;
        o0(2, i, j, k) = (x_zeta * z_eta - x_eta * z_zeta) / volvisc;
        o0(3, i, j, k) = (y_zeta * x_eta - y_eta * x_zeta) / volvisc;
        o1(1, i, j, k) = (z_xi * y_zeta - z_zeta * y_xi) / volvisc;
        o1(2, i, j, k) = (x_xi * z_zeta - x_zeta * z_xi) / volvisc;
        o1(3, i, j, k) = (y_xi * x_zeta - y_zeta * x_xi) / volvisc;
        o2(1, i, j, k) = (z_eta * y_xi - z_xi * y_eta) / volvisc;
        o2(2, i, j, k) = (x_eta * z_xi - x_xi * z_eta) / volvisc;
        o2(3, i, j, k) = (y_eta * x_xi - y_xi * x_eta) / volvisc;
      }
}

// ---- viscous residual (src/flux.f90) ----------------------------------------
// bq_face_* (src/flux.f90:2432-2801): face averages of the primitive state,
// the halo (wall) value on strong-boundary faces
void q_face_b(const Level &L, int b, int d, const double *qa, double *qfa) {
  B3 q(const_cast<double *>(qa), L, b), qf(qfa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const int di = d == 1, dj = d == 2, dk = d == 3;
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= ni; ++i)
            qf(i, j, k, v, n) = (q(i - di, j - dj, k - dk, v, n) + q(i, j, k, v, n)) / 2;
  const int *t = L.bct.data() + L.obct[b];
  for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
    Patch pa = patch_of(t + 10 * ibc, im, jm, km);
    if (pa.idir != d || !strong_bc(pa.bctyp)) continue;
    const int ibcpt = pa.inrout == 1 ? 0 : pa.ijk[d], iface = pa.inrout == 1 ? 1 : pa.ijk[d];
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
          for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
            int a, bb, c, e, f, g;
            pidx(pa, iface, i2, i3, a, bb, c);
            pidx(pa, ibcpt, i2, i3, e, f, g);
            qf(a, bb, c, v, n) = q(e, f, g, v, n);
          }
  }
}

// bq_der_* (src/flux.f90:1848-2390): face gradients in computational
// coordinates; one-sided three-point normal derivative and tangential
// derivatives along the halo (wall) line on strong-boundary faces
void q_der_b(const Level &L, int b, int d, const double *qa, double *dxa, double *dya, double *dza) {
  B3 q(const_cast<double *>(qa), L, b);
  B3 dqs[3] = {B3(dxa, L, b), B3(dya, L, b), B3(dza, L, b)};
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const int ed[3] = {d == 1, d == 2, d == 3};
  for (int n = 0; n < L.S; ++n)
    for (int v = 1; v <= L.npde; ++v)
      for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= ni; ++i) {
            const int mi = i - ed[0], mj = j - ed[1], mk = k - ed[2];
            for (int t = 1; t <= 3; ++t) {
              if (t == d) {
                dqs[t - 1](i, j, k, v, n) = q(i, j, k, v, n) - q(mi, mj, mk, v, n);
                continue;
              }
              const int ti = t == 1, tj = t == 2, tk = t == 3;
              const double q2 = (q(mi, mj, mk, v, n) + q(i, j, k, v, n) + q(i + ti, j + tj, k + tk, v, n) +
                                 q(mi + ti, mj + tj, mk + tk, v, n)) / 4;
              const double q1 = (q(mi - ti, mj - tj, mk - tk, v, n) + q(i - ti, j - tj, k - tk, v, n) +
                                 q(i, j, k, v, n) + q(mi, mj, mk, v, n)) / 4;
              dqs[t - 1](i, j, k, v, n) = q2 - q1;
            }
          }
  const int *tb = L.bct.data() + L.obct[b];
  for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
    Patch pa = patch_of(tb + 10 * ibc, im, jm, km);
    if (pa.idir != d || !strong_bc(pa.bctyp)) continue;
    const bool lo = pa.inrout == 1;
    const int iaux = lo ? 0 : pa.ijk[d], in1 = lo ? 1 : pa.ijk[d] - 1, in2 = lo ? 2 : pa.ijk[d] - 2;
    const int iface = lo ? 1 : pa.ijk[d];
    const double sgnm = lo ? 1.0 : -1.0;
    for (int n = 0; n < L.S; ++n)
      for (int v = 1; v <= L.npde; ++v)
        for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
          for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
            int fi, fj, fk, ai, aj, ak, n1i, n1j, n1k, n2i, n2j, n2k;
            pidx(pa, iface, i2, i3, fi, fj, fk);
            pidx(pa, iaux, i2, i3, ai, aj, ak);
            pidx(pa, in1, i2, i3, n1i, n1j, n1k);
            pidx(pa, in2, i2, i3, n2i, n2j, n2k);
            dqs[d - 1](fi, fj, fk, v, n) = sgnm / 3 *
                (-q(ai, aj, ak, v, n) * 8 + q(n1i, n1j, n1k, v, n) * 9 - q(n2i, n2j, n2k, v, n));
            for (int t = 1; t <= 3; ++t) {
              if (t == d) continue;
              const int ti = t == 1, tj = t == 2, tk = t == 3;
              const int pos = t == 1 ? ai : (t == 2 ? aj : ak);
              auto Q = [&](int s) { return q(ai + s * ti, aj + s * tj, ak + s * tk, v, n); };
              double q2, q1;
              if (pos == pa.istrt[t]) { q2 = (Q(0) + Q(1)) / 2; q1 = (Q(0) * 3 - Q(1)) / 2; }
              else if (pos == pa.iend[t]) { q2 = (Q(0) * 3 - Q(-1)) / 2; q1 = (Q(0) + Q(-1)) / 2; }
              else { q2 = (Q(0) + Q(1)) / 2; q1 = (Q(-1) + Q(0)) / 2; }
              dqs[t - 1](fi, fj, fk, v, n) = q2 - q1;
            }
          }
  }
}

// vflux_b, laminar branch (src/flux.f90:878-1180): viscous stresses and heat
// flux on the faces of family d; the energy row keeps the reference's terms
void vflux_b(const Level &L, int b, int d, const double *qfa, const double *dxa, const double *dya,
             const double *dza, const double *xd, const double *ed, const double *zd, const double *sijk,
             double *fa, const cosa_params &P, bool kom = false) {
  B3 qf(const_cast<double *>(qfa), L, b), dqx(const_cast<double *>(dxa), L, b);
  B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b);
  const int64_t vms = 27 * L.n0;  // per grid snapshot
  B2 s(sijk, L, b);
  B0 flux(fa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const double g = P.gamma, mr = P.machfs / P.reyno;
  if (!kom)  // laminar: the flux starts from zero (src/flux.f90:1073-1087)
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= nk; ++k)
        for (int j = 1; j <= nj; ++j)
          for (int i = 1; i <= ni; ++i)
            for (int v = 1; v <= 5; ++v) flux(i, j, k, v, n) = 0;
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          const double kx = s(1, i, j, k, nh), ky = s(2, i, j, k, nh), kz = s(3, i, j, k, nh), ds = s(4, i, j, k, nh);
          const double rho = qf(i, j, k, 1, n), u = qf(i, j, k, 2, n), v = qf(i, j, k, 3, n), w = qf(i, j, k, 4, n);
          const double p = qf(i, j, k, 5, n);
          const double t = g * p / rho;
          const double mu = (P.stemp + 1) / (t + P.stemp) * std::pow(t, 1.5);
          const double mut = flux(i, j, k, 1, n);
          const BV xv(const_cast<double *>(xd) + n * P.hbmove * vms, L, b), ev(const_cast<double *>(ed) + n * P.hbmove * vms, L, b),
              zv(const_cast<double *>(zd) + n * P.hbmove * vms, L, b);
          const double xix = xv(1, i, j, k), xiy = xv(2, i, j, k), xiz = xv(3, i, j, k);
          const double etax = ev(1, i, j, k), etay = ev(2, i, j, k), etaz = ev(3, i, j, k);
          const double zetax = zv(1, i, j, k), zetay = zv(2, i, j, k), zetaz = zv(3, i, j, k);
          const double uxi = dqx(i, j, k, 2, n), ueta = dqe(i, j, k, 2, n), uzeta = dqz(i, j, k, 2, n);
          const double vxi = dqx(i, j, k, 3, n), veta = dqe(i, j, k, 3, n), vzeta = dqz(i, j, k, 3, n);
          const double wxi = dqx(i, j, k, 4, n), weta = dqe(i, j, k, 4, n), wzeta = dqz(i, j, k, 4, n);
          const double txi = t * (dqx(i, j, k, 5, n) / p - dqx(i, j, k, 1, n) / rho);
          const double teta = t * (dqe(i, j, k, 5, n) / p - dqe(i, j, k, 1, n) / rho);
          const double tzeta = t * (dqz(i, j, k, 5, n) / p - dqz(i, j, k, 1, n) / rho);
          const double dudx = uxi * xix + ueta * etax + uzeta * zetax;
          const double dudy = uxi * xiy + ueta * etay + uzeta * zetay;
          const double dudz = uxi * xiz + ueta * etaz + uzeta * zetaz;
          const double dvdx = vxi * xix + veta * etax + vzeta * zetax;
          const double dvdy = vxi * xiy + veta * etay + vzeta * zetay;
          const double dvdz = vxi * xiz + veta * etaz + vzeta * zetaz;
          const double dwdx = wxi * xix + weta * etax + wzeta * zetax;
          const double dwdy = wxi * xiy + weta * etay + wzeta * zetay;
          const double dwdz = wxi * xiz + weta * etaz + wzeta * zetaz;
          const double dtdx = txi * xix + teta * etax + tzeta * zetax;
          const double dtdy = txi * xiy + teta * etay + tzeta * zetay;
          const double dtdz = txi * xiz + teta * etaz + tzeta * zetaz;
          const double divv = dudx + dvdy + dwdz;
          const double txx = mr * 2 * mu * (dudx - divv / 3);
          const double txy = mr * mu * (dudy + dvdx);
          const double txz = mr * mu * (dudz + dwdx);
          const double tyy = mr * 2 * mu * (dvdy - divv / 3);
          const double tyz = mr * mu * (dvdz + dwdy);
          const double tzz = mr * 2 * mu * (dwdz - divv / 3);
          const double cq = mr * (mu / P.pranl + mut / P.prant) / (g - 1);
          const double qx = -(cq * dtdx), qy = -(cq * dtdy), qz = -(cq * dtdz);
          flux(i, j, k, 1, n) = 0;
          flux(i, j, k, 2, n) = flux(i, j, k, 2, n) - (txx * kx + txy * ky + txz * kz) * ds;
          flux(i, j, k, 3, n) = flux(i, j, k, 3, n) - (txy * kx + tyy * ky + tyz * kz) * ds;
          flux(i, j, k, 4, n) = flux(i, j, k, 4, n) - (txz * kx + tyz * ky + tzz * kz) * ds;
          flux(i, j, k, 5, n) = flux(i, j, k, 5, n) -
                                ((u * txx + v * txy + w * txz) * kx + (u * txy + v * tyy + w * tyz) * ky +
                                 (u * txy + v * tyy + w * tyz) * kz) * ds +
                                (qx * kx + qy * ky + qz * kz) * ds;
        }
  }
}

// bc_walvis_15, laminar part (src/bc.f90:2144-2300): no-slip wall on a fixed
// grid; the wall pressure extrapolated, the density isentropic from cell 1
void bc_walvis_15(const Patch &pa, B3 &q, const Level &L, const cosa_params &P) {
  const int ibcpt = pa.inrout == 1 ? 0 : pa.ijk[pa.idir], ibcpt2 = pa.inrout == 1 ? -1 : pa.ijk[pa.idir] + 1;
  const int ibcn = pa.inrout == 1 ? 1 : pa.ijk[pa.idir] - 1, ibcn2 = pa.inrout == 1 ? 2 : pa.ijk[pa.idir] - 2;
  for (int n = 0; n < L.S; ++n)
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int hi, hj, hk, h2i, h2j, h2k, ni_, nj_, nk_, n2i, n2j, n2k;
        pidx(pa, ibcpt, i2, i3, hi, hj, hk);
        pidx(pa, ibcpt2, i2, i3, h2i, h2j, h2k);
        pidx(pa, ibcn, i2, i3, ni_, nj_, nk_);
        pidx(pa, ibcn2, i2, i3, n2i, n2j, n2k);
        const double p1 = q(ni_, nj_, nk_, 5, n), p2 = q(n2i, n2j, n2k, 5, n);
        const double pw = 0.5 * (3 * p1 - p2);
        const double rhow = std::pow(pw / p1, 1 / P.gamma) * q(ni_, nj_, nk_, 1, n);
        double uw = 0.0, vw = 0.0, ww = 0.0;
        if (P.moving && L.fv[pa.idir - 1]) {
          // the wall moves with its face (src/bc.f90:2256-2283)
          int mi, mj, mk;
          pidx(pa, pa.inrout == 1 ? 1 : pa.ijk[pa.idir], i2, i3, mi, mj, mk);
          BFv f(L.fv[pa.idir - 1], L, pa.blk);
          const int nh = n * P.hbmove;
          uw = f(1, mi, mj, mk, nh); vw = f(2, mi, mj, mk, nh); ww = f(3, mi, mj, mk, nh);
        }
        q(hi, hj, hk, 1, n) = rhow;
        q(hi, hj, hk, 2, n) = uw;
        q(hi, hj, hk, 3, n) = vw;
        q(hi, hj, hk, 4, n) = ww;
        q(hi, hj, hk, 5, n) = pw;
        for (int v = 1; v <= 5; ++v) q(h2i, h2j, h2k, v, n) = q(hi, hj, hk, v, n);
      }
}

// lambdab viscous branch + eig_ns (src/cosa.f90:1335-1423, 4236-4297): the
// convective lambdas and the viscous ones (kept in lamv(.,1:3)); the
// neighbour temperatures on the + side use rho of the - side, as the
// reference does
void lambda_ns_level(const Level &L, const double *qa, const double *si, const double *sj, const double *sk,
                     const double *va, const double *muta, double *lam, double *lamv, const cosa_params &P,
                     const double *cpga = nullptr, const double *cvsa = nullptr, int nl = 1) {
  const double g = P.gamma, st = P.stemp;
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b), lm(lam, L, b), lv(lamv, L, b);
    B2 vi(si, L, b), vj(sj, L, b), vk(sk, L, b);
    B1 vol(const_cast<double *>(va), L, b, 1);
    for (int n = 0; n < L.S; ++n) {
      const int nh = n * P.hbmove;
      auto MUT = [&](int i, int j, int k) -> double {
        if (!muta) return 0.0;
        B3s mu(const_cast<double *>(muta), L, b);
        return mu(i, j, k, n);
      };
      auto MU = [&](double t) { return (st + 1.0) / (t + st) * std::pow(t, 1.5); };
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            const double rho = q(i, j, k, 1, n), p = q(i, j, k, 5, n);
            const double t = g * p / rho, mu = MU(t), mutc = MUT(i, j, k);
            double mud[3], mutd[3];
            const int dd[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
            for (int d = 0; d < 3; ++d) {
              const int a = dd[d][0], bq = dd[d][1], c = dd[d][2];
              const double rhom = q(i - a, j - bq, k - c, 1, n), pm = q(i - a, j - bq, k - c, 5, n);
              const double tm = g * pm / rhom, mum = MU(tm), mutm = MUT(i - a, j - bq, k - c);
              const double pp = q(i + a, j + bq, k + c, 5, n);
              const double tp = g * pp / rhom, mup = MU(tp), mutp = MUT(i + a, j + bq, k + c);
              mud[d] = (mum + 2 * mu + mup) / 4;
              mutd[d] = (mutm + 2 * mutc + mutp) / 4;
            }
            double sim[5], sip[5], sjm[5], sjp[5], skm[5], skp[5];
            for (int c = 1; c <= 4; ++c) {
              sim[c] = vi(c, i, j, k, nh); sip[c] = vi(c, i + 1, j, k, nh);
              sjm[c] = vj(c, i, j, k, nh); sjp[c] = vj(c, i, j + 1, k, nh);
              skm[c] = vk(c, i, j, k, nh); skp[c] = vk(c, i, j, k + 1, nh);
            }
            double u = q(i, j, k, 2, n), v = q(i, j, k, 3, n), w = q(i, j, k, 4, n);
            if (P.moving && L.cv[0]) {
              // eig_ns: velocity relative to the cell's grid velocity (src/cosa.f90:4283-4287)
              u = u - BGs(L.cv[0], L, b, nh)(i, j, k);
              v = v - BGs(L.cv[1], L, b, nh)(i, j, k);
              w = w - BGs(L.cv[2], L, b, nh)(i, j, k);
            }
            const double a = std::sqrt(t);
            const double xix = 0.5 * (sim[1] * sim[4] + sip[1] * sip[4]);
            const double xiy = 0.5 * (sim[2] * sim[4] + sip[2] * sip[4]);
            const double xiz = 0.5 * (sim[3] * sim[4] + sip[3] * sip[4]);
            const double etax = 0.5 * (sjm[1] * sjm[4] + sjp[1] * sjp[4]);
            const double etay = 0.5 * (sjm[2] * sjm[4] + sjp[2] * sjp[4]);
            const double etaz = 0.5 * (sjm[3] * sjm[4] + sjp[3] * sjp[4]);
            const double zetax = 0.5 * (skm[1] * skm[4] + skp[1] * skp[4]);
            const double zetay = 0.5 * (skm[2] * skm[4] + skp[2] * skp[4]);
            const double zetaz = 0.5 * (skm[3] * skm[4] + skp[3] * skp[4]);
            const double axi = (sim[4] + sip[4]) / 2, aeta = (sjm[4] + sjp[4]) / 2, azeta = (skm[4] + skp[4]) / 2;
            if (P.lomach && cpga) {
              B1m cpg(const_cast<double *>(cpga), L, b), cvs(const_cast<double *>(cvsa), L, b);
              double l3[3];
              lsp_lambdas(P, nl, u, v, w, a, std::max(cpg(i, j, k, n), cvs(i, j, k, n)), xix, xiy, xiz, etax, etay,
                          etaz, zetax, zetay, zetaz, axi, aeta, azeta, l3);
              for (int c = 0; c < 3; ++c) lm(i, j, k, c + 1, n) = l3[c];
            } else {
              lm(i, j, k, 1, n) = std::fabs(u * xix + v * xiy + w * xiz) + a * axi;
              lm(i, j, k, 2, n) = std::fabs(u * etax + v * etay + w * etaz) + a * aeta;
              lm(i, j, k, 3, n) = std::fabs(u * zetax + v * zetay + w * zetaz) + a * azeta;
            }
            const double volc = vol(i, j, k), cm = P.cdff;
            lv(i, j, k, 1, n) = cm * axi * axi * g * P.machfs / P.reyno * (mud[0] / P.pranl + mutd[0] / P.prant) /
                                (rho * volc);
            lv(i, j, k, 2, n) = cm * aeta * aeta * g * P.machfs / P.reyno * (mud[1] / P.pranl + mutd[1] / P.prant) /
                                (rho * volc);
            lv(i, j, k, 3, n) = cm * azeta * azeta * g * P.machfs / P.reyno * (mud[2] / P.pranl + mutd[2] / P.prant) /
                                (rho * volc);
          }
    }
  }
}


// IRS coefficients of bdeltat (src/cosa.f90:4896-5200) for one cell with
// ratio `rat` (rat for the mean flow, ratt for k-omega); irsop 5 and 6 add
// the viscous floor c1/4 lamv / sum(lam)
void irs_coef(int irsop, double rat, double psirs, const double lam[3], const double lamv[3], double out[3]) {
  const double zeta = 0.4, c1 = 40.0;
  const double lami = lam[0], lamj = lam[1], lamk = lam[2];
  if (irsop == 2 || irsop == 5) {
    const double phixi = 1 + std::pow(lamj / lami, zeta) + std::pow(lamk / lami, zeta);
    const double phieta = 1 + std::pow(lami / lamj, zeta) + std::pow(lamk / lamj, zeta);
    const double phizeta = 1 + std::pow(lami / lamk, zeta) + std::pow(lamj / lamk, zeta);
    double t;
    t = (rat * lami * phixi / (lami + lamj + lamk));
    out[0] = std::max(0.0, (t * t - 1) / 4);
    t = (rat * lamj * phieta / (lami + lamj + lamk));
    out[1] = std::max(0.0, (t * t - 1) / 4);
    t = (rat * lamk * phizeta / (lami + lamj + lamk));
    out[2] = std::max(0.0, (t * t - 1) / 4);
    if (irsop == 5)
      for (int c = 0; c < 3; ++c) out[c] = std::max(out[c], c1 / 4 * lamv[c] / (lami + lamj + lamk));
  } else if (irsop == 3 || irsop == 6) {
    const double rji = lamj / lami, rki = lamk / lami, rij = lami / lamj;
    const double rkj = lamk / lamj, rik = lami / lamk, rjk = lamj / lamk;
    double t;
    t = rat / (1 + psirs * (rji + rki));
    out[0] = std::max(0.0, 0.25 * (t * t - 1));
    t = rat / (1 + psirs * (rij + rkj));
    out[1] = std::max(0.0, 0.25 * (t * t - 1));
    t = rat / (1 + psirs * (rik + rjk));
    out[2] = std::max(0.0, 0.25 * (t * t - 1));
    if (irsop == 6)
      for (int c = 0; c < 3; ++c) out[c] = std::max(out[c], 0.25 * c1 * lamv[c] / (lami + lamj + lamk));
  } else {
    out[0] = out[1] = out[2] = 0.0;
  }
}

// bdeltat, viscous branch (src/cosa.f90:4861-4876, 4895-5200): the viscous
// lambdas join the time step unless irsop is 5 or 6, where they raise the
// smoothing coefficients instead; k-omega: dtvolt = cflt/cfl dtvol and the
// turbulence coefficients with ratt
void deltat_ns_level(const Level &L, double *dtv, const double *lam, const double *lamv, double *bx_, double *by_,
                     double *bz_, const cosa_params &P, double *dtt_ = nullptr, double *tbx_ = nullptr,
                     double *tby_ = nullptr, double *tbz_ = nullptr) {
  const bool dt_visc = P.irsop != 5 && P.irsop != 6;
  for (int b = 0; b < L.nb; ++b) {
    B3 lm(const_cast<double *>(lam), L, b), lv(const_cast<double *>(lamv), L, b);
    B1 dt(dtv, L, b, L.S);
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            if (dt_visc)
              dt(i, j, k, n) = P.cfl / (lm(i, j, k, 1, n) + lm(i, j, k, 2, n) + lm(i, j, k, 3, n) +
                                        lv(i, j, k, 1, n) + lv(i, j, k, 2, n) + lv(i, j, k, 3, n));
            else
              dt(i, j, k, n) = P.cfl / (lm(i, j, k, 1, n) + lm(i, j, k, 2, n) + lm(i, j, k, 3, n));
            if (dtt_) {
              B1 dtt(dtt_, L, b, L.S);
              dtt(i, j, k, n) = P.cflt / P.cfl * dt(i, j, k, n);
            }
          }
    if (P.irsop < 2 || P.irsop == 4) continue;
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            const double l[3] = {lm(i, j, k, 1, n), lm(i, j, k, 2, n), lm(i, j, k, 3, n)};
            const double v[3] = {lv(i, j, k, 1, n), lv(i, j, k, 2, n), lv(i, j, k, 3, n)};
            double o[3];
            if (bx_) {
              irs_coef(P.irsop, P.rat, P.psirs, l, v, o);
              B1 bx(bx_, L, b, L.S), by(by_, L, b, L.S), bz(bz_, L, b, L.S);
              bx(i, j, k, n) = o[0]; by(i, j, k, n) = o[1]; bz(i, j, k, n) = o[2];
            }
            if (tbx_) {
              irs_coef(P.irsop, P.ratt, P.psirs, l, v, o);
              B1 bx(tbx_, L, b, L.S), by(tby_, L, b, L.S), bz(tbz_, L, b, L.S);
              bx(i, j, k, n) = o[0]; by(i, j, k, n) = o[1]; bz(i, j, k, n) = o[2];
            }
          }
  }
}

// ---- k-omega (Wilcox), src/flux.f90, src/src.f90, src/update.f90, src/bc.f90 --
// bc_walvis_15, k-omega part (src/bc.f90:2309-2470): k = 0 at the wall and
// omega from Wilcox's rough-wall law (wallwilc) or Menter's near-wall
// solution, both from the wall distance of the first cell
void bc_walvis_15_kom(const Patch &pa, B3 &q, const B2 &si, const B2 &sj, const B2 &sk, const double *dista,
                      const Level &L, int b, const cosa_params &P) {
  const double small = 1.0e-12, smasq = 1.0e-24, mor = P.machfs / P.reyno;
  const int ibcpt = pa.inrout == 1 ? 0 : pa.ijk[pa.idir], ibcpt2 = pa.inrout == 1 ? -1 : pa.ijk[pa.idir] + 1;
  const int ibcn = pa.inrout == 1 ? 1 : pa.ijk[pa.idir] - 1, ibcm = pa.inrout == 1 ? 1 : pa.ijk[pa.idir];
  B1 dist(const_cast<double *>(dista), L, b, 1);
  const B2 &sf = pa.idir == 1 ? si : (pa.idir == 2 ? sj : sk);
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
      for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
        int hi, hj, hk, h2i, h2j, h2k, ni_, nj_, nk_, mi, mj, mk;
        pidx(pa, ibcpt, i2, i3, hi, hj, hk);
        pidx(pa, ibcpt2, i2, i3, h2i, h2j, h2k);
        pidx(pa, ibcn, i2, i3, ni_, nj_, nk_);
        pidx(pa, ibcm, i2, i3, mi, mj, mk);
        const double rhow = q(hi, hj, hk, 1, n), pw = q(hi, hj, hk, 5, n);
        const double tw = pw * P.gamma / rhow;
        const double muw = (P.stemp + 1) / (tw + P.stemp) * std::pow(tw, 1.5);
        const double d = dist(ni_, nj_, nk_);
        double omew;
        if (P.wallwilc) {
          const double nx = sf(1, mi, mj, mk, nh), ny = sf(2, mi, mj, mk, nh), nz = sf(3, mi, mj, mk, nh);
          double uw = 0.0, vw = 0.0, ww = 0.0;
          if (P.moving && L.fv[pa.idir - 1]) {
            // velocity relative to the moving wall face (src/bc.f90:2346-2368, 2392-2394)
            BFv f(L.fv[pa.idir - 1], L, b);
            uw = f(1, mi, mj, mk, nh); vw = f(2, mi, mj, mk, nh); ww = f(3, mi, mj, mk, nh);
          }
          const double uc = q(ni_, nj_, nk_, 2, n) - uw, vc = q(ni_, nj_, nk_, 3, n) - vw;
          const double wc = q(ni_, nj_, nk_, 4, n) - ww;
          const double uorth = nx * uc + ny * vc + nz * wc;
          const double a = uc - uorth * nx, bb = vc - uorth * ny, c = wc - uorth * nz;
          const double upar = std::sqrt(a * a + bb * bb + c * c);
          const double dupardn = upar / (d + small);
          const double tauw = muw * std::fabs(dupardn);
          const double rkrpls = P.roughk > 0.0 ? std::max(1.0, std::sqrt(rhow * tauw / mor) * P.roughk / muw) : 1.0;
          const double sr = rkrpls >= 25.0 ? 100.0 / rkrpls : 2500.0 / (rkrpls * rkrpls);
          omew = std::fabs(dupardn) * sr;
        } else {
          omew = 60.0 * muw / (P.bkw * rhow * (d * d) + smasq) * P.machfs / P.reyno;
        }
        q(hi, hj, hk, 6, n) = 0.0;
        q(hi, hj, hk, 7, n) = omew;
        q(h2i, h2j, h2k, 6, n) = q(hi, hj, hk, 6, n);
        q(h2i, h2j, h2k, 7, n) = q(hi, hj, hk, 7, n);
      }
  }
}

// bq_face_* with calmut (src/flux.f90:2495-2540 and the j, k counterparts):
// face turbulent viscosity into flux(.,1), the halo value on strong faces
void q_face_mut_b(const Level &L, int b, int d, const double *muta, double *fa) {
  B3s mu(const_cast<double *>(muta), L, b);
  B0 f(fa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const int di = d == 1, dj = d == 2, dk = d == 3;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) f(i, j, k, 1, n) = (mu(i - di, j - dj, k - dk, n) + mu(i, j, k, n)) / 2;
  const int *t = L.bct.data() + L.obct[b];
  for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
    Patch pa = patch_of(t + 10 * ibc, im, jm, km);
    if (pa.idir != d || !strong_bc(pa.bctyp)) continue;
    const int ibcpt = pa.inrout == 1 ? 0 : pa.ijk[d], iface = pa.inrout == 1 ? 1 : pa.ijk[d];
    for (int n = 0; n < L.S; ++n)
      for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
        for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
          int a, bb, c, e, g, h;
          pidx(pa, iface, i2, i3, a, bb, c);
          pidx(pa, ibcpt, i2, i3, e, g, h);
          f(a, bb, c, 1, n) = mu(e, g, h, n);
        }
  }
}

// b_rtst (src/flux.f90:2846-2946): Reynolds stresses on the faces of family
// d, tau1(.,1..6) = txx, txy, txz, tyy, tyz, tzz, with -2/3 rho k on the
// diagonal
void rtst_b(const Level &L, int b, int d, const double *qfa, const double *dxa, const double *dya, const double *dza,
            const double *xd, const double *ed, const double *zd, double *taua, const double *fa,
            const cosa_params &P) {
  B3 qf(const_cast<double *>(qfa), L, b), dqx(const_cast<double *>(dxa), L, b);
  B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b), tau(taua, L, b);
  const int64_t vms = 27 * L.n0;  // per grid snapshot
  B0 f(const_cast<double *>(fa), L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  const double fact = 2.0 / 3.0;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          const double rho = qf(i, j, k, 1, n), tke = qf(i, j, k, 6, n), mut = f(i, j, k, 1, n);
          const BV xv(const_cast<double *>(xd) + n * P.hbmove * vms, L, b), ev(const_cast<double *>(ed) + n * P.hbmove * vms, L, b),
              zv(const_cast<double *>(zd) + n * P.hbmove * vms, L, b);
          const double xix = xv(1, i, j, k), xiy = xv(2, i, j, k), xiz = xv(3, i, j, k);
          const double etax = ev(1, i, j, k), etay = ev(2, i, j, k), etaz = ev(3, i, j, k);
          const double zetax = zv(1, i, j, k), zetay = zv(2, i, j, k), zetaz = zv(3, i, j, k);
          const double uxi = dqx(i, j, k, 2, n), ueta = dqe(i, j, k, 2, n), uzeta = dqz(i, j, k, 2, n);
          const double vxi = dqx(i, j, k, 3, n), veta = dqe(i, j, k, 3, n), vzeta = dqz(i, j, k, 3, n);
          const double wxi = dqx(i, j, k, 4, n), weta = dqe(i, j, k, 4, n), wzeta = dqz(i, j, k, 4, n);
          const double dudx = uxi * xix + ueta * etax + uzeta * zetax;
          const double dudy = uxi * xiy + ueta * etay + uzeta * zetay;
          const double dudz = uxi * xiz + ueta * etaz + uzeta * zetaz;
          const double dvdx = vxi * xix + veta * etax + vzeta * zetax;
          const double dvdy = vxi * xiy + veta * etay + vzeta * zetay;
          const double dvdz = vxi * xiz + veta * etaz + vzeta * zetaz;
          const double dwdx = wxi * xix + weta * etax + wzeta * zetax;
          const double dwdy = wxi * xiy + weta * etay + wzeta * zetay;
          const double dwdz = wxi * xiz + weta * etaz + wzeta * zetaz;
          const double divv = (dudx + dvdy + dwdz) * P.turcmp;
          const double txx = 2 * mut * (dudx - divv / 3), txy = mut * (dudy + dvdx), txz = mut * (dudz + dwdx);
          const double tyy = 2 * mut * (dvdy - divv / 3), tyz = mut * (dvdz + dwdy);
          const double tzz = 2 * mut * (dwdz - divv / 3);
          const double mr = P.machfs / P.reyno;
          tau(i, j, k, 1, n) = mr * txx - fact * rho * tke;
          tau(i, j, k, 2, n) = mr * txy;
          tau(i, j, k, 3, n) = mr * txz;
          tau(i, j, k, 4, n) = mr * tyy - fact * rho * tke;
          tau(i, j, k, 5, n) = mr * tyz;
          tau(i, j, k, 6, n) = mr * tzz - fact * rho * tke;
        }
}

// vflux_b, Wilcox k-omega branch (src/flux.f90:915-983): Reynolds-stress
// momentum flux and the k / omega diffusion, before the laminar terms; the
// omega row keeps the reference's dk/dz in place of domega/dz
void vflux_kom_b(const Level &L, int b, int d, const double *qfa, const double *dxa, const double *dya,
                 const double *dza, const double *taua, const double *xd, const double *ed, const double *zd,
                 const double *sijk, double *fa, const cosa_params &P, const double *fdista = nullptr) {
  B3 qf(const_cast<double *>(qfa), L, b), dqx(const_cast<double *>(dxa), L, b);
  B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b), tau(const_cast<double *>(taua), L, b);
  const int64_t vms = 27 * L.n0;  // per grid snapshot
  B2 s(sijk, L, b);
  B0 flux(fa, L, b);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  const int ni = d == 1 ? im : im - 1, nj = d == 2 ? jm : jm - 1, nk = d == 3 ? km : km - 1;
  for (int n = 0; n < L.S; ++n) {
    const int nh = n * P.hbmove;
    for (int k = 1; k <= nk; ++k)
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          const double kx = s(1, i, j, k, nh), ky = s(2, i, j, k, nh), kz = s(3, i, j, k, nh), ds = s(4, i, j, k, nh);
          const double rho = qf(i, j, k, 1, n), p = qf(i, j, k, 5, n);
          const double t = P.gamma * p / rho;
          const double mu = (P.stemp + 1) / (t + P.stemp) * std::pow(t, 1.5);
          const double mut = flux(i, j, k, 1, n);
          const BV xv(const_cast<double *>(xd) + n * P.hbmove * vms, L, b), ev(const_cast<double *>(ed) + n * P.hbmove * vms, L, b),
              zv(const_cast<double *>(zd) + n * P.hbmove * vms, L, b);
          const double xix = xv(1, i, j, k), xiy = xv(2, i, j, k), xiz = xv(3, i, j, k);
          const double etax = ev(1, i, j, k), etay = ev(2, i, j, k), etaz = ev(3, i, j, k);
          const double zetax = zv(1, i, j, k), zetay = zv(2, i, j, k), zetaz = zv(3, i, j, k);
          const double tkexi = dqx(i, j, k, 6, n), tkeeta = dqe(i, j, k, 6, n), tkezeta = dqz(i, j, k, 6, n);
          const double omexi = dqx(i, j, k, 7, n), omeeta = dqe(i, j, k, 7, n), omezeta = dqz(i, j, k, 7, n);
          const double dtkedx = tkexi * xix + tkeeta * etax + tkezeta * zetax;
          const double dtkedy = tkexi * xiy + tkeeta * etay + tkezeta * zetay;
          const double dtkedz = tkexi * xiz + tkeeta * etaz + tkezeta * zetaz;
          const double domedx = omexi * xix + omeeta * etax + omezeta * zetax;
          const double domedy = omexi * xiy + omeeta * etay + omezeta * zetay;
          const double txx = tau(i, j, k, 1, n), txy = tau(i, j, k, 2, n), txz = tau(i, j, k, 3, n);
          const double tyy = tau(i, j, k, 4, n), tyz = tau(i, j, k, 5, n), tzz = tau(i, j, k, 6, n);
          flux(i, j, k, 2, n) = -(txx * kx + txy * ky + txz * kz) * ds;
          flux(i, j, k, 3, n) = -(txy * kx + tyy * ky + tyz * kz) * ds;
          flux(i, j, k, 4, n) = -(txz * kx + tyz * ky + tzz * kz) * ds;
          double sigk = P.sigk, sigw = P.sigw;
          if (is_blend(P)) {
            // BSL/SST (src/flux.f90:987-1061): sigma_k and sigma_omega blended by
            // F1 of the face state and the face's wall distance
            const Blend c = blend_of(P);
            const double tke = qf(i, j, k, 6, n), ome = qf(i, j, k, 7, n);
            const double domedz = omexi * xiz + omeeta * etaz + omezeta * zetaz;
            const double fd = B0s(const_cast<double *>(fdista), L, b)(i, j, k) + P.epst;
            double arg1 = std::max(std::sqrt(tke) / 0.09 / ome / fd, 500 * mu / rho / ome / (fd * fd) * P.machfs / P.reyno);
            const double cdt = 2 * rho * c.sigw2 / ome * (dtkedx * domedx + dtkedy * domedy + dtkedz * domedz);
            const double acdt = std::max(cdt, 1.0e-20);
            arg1 = std::min(arg1, 4 * rho * c.sigw2 * tke / acdt / (fd * fd));
            arg1 = std::min(pow4(arg1), 1.0e2);
            const double f1 = tanh_ref(arg1);
            sigk = f1 * c.sigk1 + (1 - f1) * c.sigk2;
            sigw = f1 * c.sigw1 + (1 - f1) * c.sigw2;
          }
          const double ctke = (mu + sigk * mut) * P.machfs / P.reyno;
          const double come = (mu + sigw * mut) * P.machfs / P.reyno;
          flux(i, j, k, 5, n) = -ctke * (dtkedx * kx + dtkedy * ky + dtkedz * kz) * ds;
          flux(i, j, k, 6, n) = -ctke * (dtkedx * kx + dtkedy * ky + dtkedz * kz) * ds;
          flux(i, j, k, 7, n) = -come * (domedx * kx + domedy * ky + dtkedz * kz) * ds;
        }
  }
}

// bq_der_ci/cj/ck (src/flux.f90:2979-3130): cell-centred differences of the
// face values of family d for the velocity components, and for k and omega
// under BSL/SST
void q_der_c_b(const Level &L, int b, int d, const double *qfa, double *dca, bool blend = false) {
  B3 qf(const_cast<double *>(qfa), L, b), dc(dca, L, b);
  const int di = d == 1, dj = d == 2, dk = d == 3;
  for (int n = 0; n < L.S; ++n)
    for (int v = 2; v <= (blend ? 7 : 4); ++v) {
      if (v == 5) continue;
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i)
            dc(i, j, k, v, n) = qf(i + di, j + dj, k + dk, v, n) - qf(i, j, k, v, n);
    }
}

// turprod_b (src/src.f90:40-177): production P_d (alternative form), div u,
// delta+ = 2/3 max(div u, 0); the cell-centre metrics average the two faces
// of the family matching each Cartesian component, as the reference does
void turprod_b(const Level &L, int b, const double *qa, const double *dxa, const double *dya, const double *dza,
               const double *vm, double *prda, double *diva, double *dpla, const cosa_params &P) {
  B3 q(const_cast<double *>(qa), L, b), dqx(const_cast<double *>(dxa), L, b);
  B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b);
  B3s prd(prda, L, b), dvv(diva, L, b), dpl(dpla, L, b);
  // vm array (d, m): derivative m on faces of family d
  const double fact = 2.0 / 3.0;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double *vmn = vm_snap(L, vm, n * P.hbmove);
          auto V = [&](int d, int m) { return BV(const_cast<double *>(vmn) + (int64_t)((d - 1) * 3 + m) * 3 * L.n0, L, b); };
          const BV xi_i = V(1, 0), xi_j = V(2, 0), xi_k = V(3, 0);
          const BV et_i = V(1, 1), et_j = V(2, 1), et_k = V(3, 1);
          const BV ze_i = V(1, 2), ze_j = V(2, 2), ze_k = V(3, 2);
          const double xix = (xi_i(1, i + 1, j, k) + xi_i(1, i, j, k)) / 2;
          const double xiy = (xi_j(2, i, j + 1, k) + xi_j(2, i, j, k)) / 2;
          const double xiz = (xi_k(3, i, j, k + 1) + xi_k(3, i, j, k)) / 2;
          const double etax = (et_i(1, i + 1, j, k) + et_i(1, i, j, k)) / 2;
          const double etay = (et_j(2, i, j + 1, k) + et_j(2, i, j, k)) / 2;
          const double etaz = (et_k(3, i, j, k + 1) + et_k(3, i, j, k)) / 2;
          const double zetax = (ze_i(1, i + 1, j, k) + ze_i(1, i, j, k)) / 2;
          const double zetay = (ze_j(2, i, j + 1, k) + ze_j(2, i, j, k)) / 2;
          const double zetaz = (ze_k(3, i, j, k + 1) + ze_k(3, i, j, k)) / 2;
          const double uxi = dqx(i, j, k, 2, n), ueta = dqe(i, j, k, 2, n), uzeta = dqz(i, j, k, 2, n);
          const double vxi = dqx(i, j, k, 3, n), veta = dqe(i, j, k, 3, n), vzeta = dqz(i, j, k, 3, n);
          const double wxi = dqx(i, j, k, 4, n), weta = dqe(i, j, k, 4, n), wzeta = dqz(i, j, k, 4, n);
          const double dudx = uxi * xix + ueta * etax + uzeta * zetax;
          const double dudy = uxi * xiy + ueta * etay + uzeta * zetay;
          const double dudz = uxi * xiz + ueta * etaz + uzeta * zetaz;
          const double dvdx = vxi * xix + veta * etax + vzeta * zetax;
          const double dvdy = vxi * xiy + veta * etay + vzeta * zetay;
          const double dvdz = vxi * xiz + veta * etaz + vzeta * zetaz;
          const double dwdx = wxi * xix + weta * etax + wzeta * zetax;
          const double dwdy = wxi * xiy + weta * etay + wzeta * zetay;
          const double dwdz = wxi * xiz + weta * etaz + wzeta * zetaz;
          const double divv = (dudx + dvdy + dwdz) * P.turcmp;
          const double txx = dudx, txy = (dudy + dvdx) / 2, txz = (dudz + dwdx) / 2;
          const double tyy = dvdy, tyz = (dvdz + dwdy) / 2, tzz = dwdz;
          const double prod = 2 * (txx * txx + tyy * tyy + tzz * tzz + 2 * (txy * txy + txz * txz + tyz * tyz) -
                                   divv * divv / 3);
          (void)q;
          prd(i, j, k, n) = prod;
          dvv(i, j, k, n) = divv;
          dpl(i, j, k, n) = fact * std::max(divv, 0.0);
        }
}

// srckw_b (src/src.f90:196-272): k and omega sources into res(6:7)
void srckw_b(const Level &L, int b, int nl, const double *qa, const double *muta, const double *prda,
             const double *diva, double *ra, const double *va, const cosa_params &P) {
  B3 q(const_cast<double *>(qa), L, b), res(ra, L, b);
  B3s mu(const_cast<double *>(muta), L, b), prd(const_cast<double *>(prda), L, b), dvv(const_cast<double *>(diva), L, b);
  B1 vol(const_cast<double *>(va), L, b, 1);
  const double fact = 2.0 / 3.0, mor = P.machfs / P.reyno;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double rho = q(i, j, k, 1, n), tke = q(i, j, k, 6, n), ome = q(i, j, k, 7, n);
          const double mut = mu(i, j, k, n), divv = dvv(i, j, k, n);
          double prod = prd(i, j, k, n), prodw = prd(i, j, k, n);
          if (P.lim_prodtke && (nl == 1 || P.prd_all_lvls)) {
            const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
            if (mor * mut * prod > tstdis) {
              prod = tstdis / mor / mut;
              if (P.lim_prodomega) prodw = prod;
            }
          }
          res(i, j, k, 6, n) = res(i, j, k, 6, n) -
                               vol(i, j, k) * (mor * mut * prod - fact * divv * rho * tke - P.bstrkw * rho * tke * ome);
          res(i, j, k, 7, n) = res(i, j, k, 7, n) - vol(i, j, k) * (P.gkw * P.cmu * rho * prodw -
                                                                    P.gkw * fact * divv * rho * ome -
                                                                    P.bkw * rho * (ome * ome));
        }
}

// ---- BSL / SST (src/update.f90:2340-2460, 3000-3161; src/src.f90:275-378;
// src/grid.f90:2809-2870) ------------------------------------------------------
// facedist_b: wall distance of the faces of each family, the mean of the
// two cells' distances and the boundary cell's own on the block faces
void facedist_level(const Level &L, const double *dista, double *fi, double *fj, double *fk) {
  for (int b = 0; b < L.nb; ++b) {
    B1 dist(const_cast<double *>(dista), L, b, 1);
    B0s FI(fi, L, b), FJ(fj, L, b), FK(fk, L, b);
    const int im = L.im[b], jm = L.jm[b], km = L.km[b];
    for (int k = 1; k <= km - 1; ++k)
      for (int j = 1; j <= jm - 1; ++j) {
        FI(1, j, k) = dist(0, j, k);
        for (int i = 2; i <= im - 1; ++i) FI(i, j, k) = (dist(i - 1, j, k) + dist(i, j, k)) / 2;
        FI(im, j, k) = dist(im, j, k);
      }
    for (int k = 1; k <= km - 1; ++k)
      for (int i = 1; i <= im - 1; ++i) {
        FJ(i, 1, k) = dist(i, 0, k);
        for (int j = 2; j <= jm - 1; ++j) FJ(i, j, k) = (dist(i, j - 1, k) + dist(i, j, k)) / 2;
        FJ(i, jm, k) = dist(i, jm, k);
      }
    for (int j = 1; j <= jm - 1; ++j)
      for (int i = 1; i <= im - 1; ++i) {
        FK(i, j, 1) = dist(i, j, 0);
        for (int k = 2; k <= km - 1; ++k) FK(i, j, k) = (dist(i, j, k - 1) + dist(i, j, k)) / 2;
        FK(i, j, km) = dist(i, j, km);
      }
  }
}

// the cell-centre inverse metrics of turprod_b / update_ttrm_b: each
// Cartesian derivative of xi, eta, zeta averaged over the two faces of the
// family it is stored on
struct CellMet { double xix, xiy, xiz, etax, etay, etaz, zetax, zetay, zetaz; };
inline CellMet cell_met(const Level &L, int b, const double *vm, int i, int j, int k) {
  auto V = [&](int d, int m) { return BV(const_cast<double *>(vm) + (int64_t)((d - 1) * 3 + m) * 3 * L.n0, L, b); };
  const BV xi_i = V(1, 0), xi_j = V(2, 0), xi_k = V(3, 0);
  const BV et_i = V(1, 1), et_j = V(2, 1), et_k = V(3, 1);
  const BV ze_i = V(1, 2), ze_j = V(2, 2), ze_k = V(3, 2);
  CellMet m;
  m.xix = (xi_i(1, i + 1, j, k) + xi_i(1, i, j, k)) / 2;
  m.xiy = (xi_j(2, i, j + 1, k) + xi_j(2, i, j, k)) / 2;
  m.xiz = (xi_k(3, i, j, k + 1) + xi_k(3, i, j, k)) / 2;
  m.etax = (et_i(1, i + 1, j, k) + et_i(1, i, j, k)) / 2;
  m.etay = (et_j(2, i, j + 1, k) + et_j(2, i, j, k)) / 2;
  m.etaz = (et_k(3, i, j, k + 1) + et_k(3, i, j, k)) / 2;
  m.zetax = (ze_i(1, i + 1, j, k) + ze_i(1, i, j, k)) / 2;
  m.zetay = (ze_j(2, i, j + 1, k) + ze_j(2, i, j, k)) / 2;
  m.zetaz = (ze_k(3, i, j, k + 1) + ze_k(3, i, j, k)) / 2;
  return m;
}

// update_ttrm_b: ttrm = (cross diffusion (1 - F1) CD, gamma, beta) blended
// by F1 from the primitive state, the cell-centred k and omega differences
// and the cell wall distance; Wilcox: (0, gkw, bkw)
void update_ttrm_b(const Level &L, int b, const double *qa, const double *dxa, const double *dya, const double *dza,
                   const double *vm, double *ttrma, const double *dista, const cosa_params &P) {
  B3 q(const_cast<double *>(qa), L, b), dqx(const_cast<double *>(dxa), L, b);
  B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b);
  B3t ttrm(ttrma, L, b);
  B1 dist(const_cast<double *>(dista), L, b, 1);
  const int im = L.im[b], jm = L.jm[b], km = L.km[b];
  if (P.kom) {
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 1; i <= im - 1; ++i) {
            ttrm(i, j, k, 1, n) = 0.0;
            ttrm(i, j, k, 2, n) = P.gkw;
            ttrm(i, j, k, 3, n) = P.bkw;
          }
    return;
  }
  const Blend c = blend_of(P);
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= km - 1; ++k)
      for (int j = 1; j <= jm - 1; ++j)
        for (int i = 1; i <= im - 1; ++i) {
          const double rho = q(i, j, k, 1, n), tke = q(i, j, k, 6, n), ome = q(i, j, k, 7, n), p = q(i, j, k, 5, n);
          const double t = P.gamma * p / rho;
          const double mu = (P.stemp + 1) / (t + P.stemp) * std::pow(t, 1.5);
          const CellMet m = cell_met(L, b, vm_snap(L, vm, n * P.hbmove), i, j, k);
          const double tkexi = dqx(i, j, k, 6, n), tkeeta = dqe(i, j, k, 6, n), tkezeta = dqz(i, j, k, 6, n);
          const double omexi = dqx(i, j, k, 7, n), omeeta = dqe(i, j, k, 7, n), omezeta = dqz(i, j, k, 7, n);
          const double dtkedx = tkexi * m.xix + tkeeta * m.etax + tkezeta * m.zetax;
          const double dtkedy = tkexi * m.xiy + tkeeta * m.etay + tkezeta * m.zetay;
          const double dtkedz = tkexi * m.xiz + tkeeta * m.etaz + tkezeta * m.zetaz;
          const double domedx = omexi * m.xix + omeeta * m.etax + omezeta * m.zetax;
          const double domedy = omexi * m.xiy + omeeta * m.etay + omezeta * m.zetay;
          const double domedz = omexi * m.xiz + omeeta * m.etaz + omezeta * m.zetaz;
          const double dd = dist(i, j, k) + P.epst;
          double arg1 = std::max(std::sqrt(tke) / 0.09 / ome / dd, 500 * mu / rho / ome / (dd * dd) * P.machfs / P.reyno);
          const double cdt = 2 * rho * c.sigw2 / ome * (dtkedx * domedx + dtkedy * domedy + dtkedz * domedz);
          const double acdt = std::max(cdt, 1.0e-20);
          arg1 = std::min(arg1, 4 * rho * c.sigw2 * tke / acdt / (dd * dd));
          arg1 = pow4(arg1);
          arg1 = std::min(arg1, 1.0e2);
          const double f1 = tanh_ref(arg1);
          ttrm(i, j, k, 1, n) = cdt * (1 - f1);
          ttrm(i, j, k, 2, n) = f1 * c.g1 + (1 - f1) * c.g2;
          ttrm(i, j, k, 3, n) = f1 * c.b1 + (1 - f1) * c.b2;
        }
}

// srckw_sst_b: the k source of srckw_b and the omega source with the blended
// gamma, beta and the cross-diffusion term
void srckw_sst_b(const Level &L, int b, int nl, const double *qa, const double *muta, const double *prda,
                 const double *diva, double *ra, const double *ttrma, const double *va, const cosa_params &P) {
  B3 q(const_cast<double *>(qa), L, b), res(ra, L, b);
  B3s mu(const_cast<double *>(muta), L, b), prd(const_cast<double *>(prda), L, b), dvv(const_cast<double *>(diva), L, b);
  B3t ttrm(const_cast<double *>(ttrma), L, b);
  B1 vol(const_cast<double *>(va), L, b, 1);
  const double fact = 2.0 / 3.0, mor = P.machfs / P.reyno;
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          const double rho = q(i, j, k, 1, n), tke = q(i, j, k, 6, n), ome = q(i, j, k, 7, n);
          const double mut = mu(i, j, k, n), divv = dvv(i, j, k, n);
          double prod = prd(i, j, k, n), prodw = prd(i, j, k, n);
          const double cdif = ttrm(i, j, k, 1, n), gav = ttrm(i, j, k, 2, n), bav = ttrm(i, j, k, 3, n);
          if (P.lim_prodtke && (nl == 1 || P.prd_all_lvls)) {
            const double tstdis = P.prdlim * P.bstrkw * rho * tke * ome;
            if (mor * mut * prod > tstdis) {
              prod = tstdis / mor / mut;
              if (P.lim_prodomega) prodw = prod;
            }
          }
          res(i, j, k, 6, n) = res(i, j, k, 6, n) -
                               vol(i, j, k) * (mor * mut * prod - fact * divv * rho * tke - P.bstrkw * rho * tke * ome);
          res(i, j, k, 7, n) = res(i, j, k, 7, n) - vol(i, j, k) * (gav * P.cmu * rho * prodw - gav * fact * divv * rho * ome -
                                                                    bav * rho * (ome * ome) + cdif);
        }
}

// tur_vis_sst_b: mut = a1 rho k / max(a1 omega, sqrt(2 S) F2) of the
// conservative state with the stage's cell-centred velocity differences;
// the face halos copy the adjacent cell (edges and corners are left)
void tur_vis_sst_level(const Level &L, const double *qa, double *muta, const double *dxa, const double *dya,
                       const double *dza, const double *vm, const double *dista, const cosa_params &P) {
  const Blend c = blend_of(P);
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b), dqx(const_cast<double *>(dxa), L, b);
    B3 dqe(const_cast<double *>(dya), L, b), dqz(const_cast<double *>(dza), L, b);
    B3s mut(muta, L, b);
    B1 dist(const_cast<double *>(dista), L, b, 1);
    const int im = L.im[b], jm = L.jm[b], km = L.km[b];
    for (int n = 0; n < L.S; ++n) {
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 1; i <= im - 1; ++i) {
            const double q1 = q(i, j, k, 1, n), q2 = q(i, j, k, 2, n), q3 = q(i, j, k, 3, n), q4 = q(i, j, k, 4, n);
            const double p = (P.gamma - 1) * (q(i, j, k, 5, n) - (q2 * q2 + q3 * q3 + q4 * q4) / q1 / 2 - q(i, j, k, 6, n));
            const double rho = q1, tke = q(i, j, k, 6, n) / rho, ome = q(i, j, k, 7, n) / rho;
            const double t = P.gamma * p / rho;
            const double mu = (P.stemp + 1) / (t + P.stemp) * std::pow(t, 1.5);
            const CellMet m = cell_met(L, b, vm_snap(L, vm, n * P.hbmove), i, j, k);
            const double uxi = dqx(i, j, k, 2, n), ueta = dqe(i, j, k, 2, n), uzeta = dqz(i, j, k, 2, n);
            const double vxi = dqx(i, j, k, 3, n), veta = dqe(i, j, k, 3, n), vzeta = dqz(i, j, k, 3, n);
            const double wxi = dqx(i, j, k, 4, n), weta = dqe(i, j, k, 4, n), wzeta = dqz(i, j, k, 4, n);
            const double dudx = uxi * m.xix + ueta * m.etax + uzeta * m.zetax;
            const double dudy = uxi * m.xiy + ueta * m.etay + uzeta * m.zetay;
            const double dudz = uxi * m.xiz + ueta * m.etaz + uzeta * m.zetaz;
            const double dvdx = vxi * m.xix + veta * m.etax + vzeta * m.zetax;
            const double dvdy = vxi * m.xiy + veta * m.etay + vzeta * m.zetay;
            const double dvdz = vxi * m.xiz + veta * m.etaz + vzeta * m.zetaz;
            const double dwdx = wxi * m.xix + weta * m.etax + wzeta * m.zetax;
            const double dwdy = wxi * m.xiy + weta * m.etay + wzeta * m.zetay;
            const double dwdz = wxi * m.xiz + weta * m.etaz + wzeta * m.zetaz;
            const double sxx = dudx, sxy = (dudy + dvdx) / 2, sxz = (dudz + dwdx) / 2;
            const double syy = dvdy, syz = (dvdz + dwdy) / 2, szz = dwdz;
            const double sn = sxx * sxx + syy * syy + szz * szz + 2 * (sxy * sxy + sxz * sxz + syz * syz);
            const double dd = dist(i, j, k) + P.epst;
            double arg2 = std::max(2 * std::sqrt(tke) / 0.09 / ome / dd, 500 * mu / rho / ome / (dd * dd) * P.machfs / P.reyno);
            arg2 = arg2 * arg2;
            arg2 = std::min(arg2, 1.0e2);
            const double f2 = tanh_ref(arg2);
            const double fact = std::sqrt(2 * sn);
            mut(i, j, k, n) = c.a1 * rho * tke / std::max(c.a1 * ome, fact * f2) * P.reyno / P.machfs;
          }
      for (int k = 0; k <= km; k += km)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 1; i <= im - 1; ++i) mut(i, j, k, n) = mut(i, j, k == 0 ? 1 : km - 1, n);
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 0; j <= jm; j += jm)
          for (int i = 1; i <= im - 1; ++i) mut(i, j, k, n) = mut(i, j == 0 ? 1 : jm - 1, k, n);
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 0; i <= im; i += im) mut(i, j, k, n) = mut(i == 0 ? 1 : im - 1, j, k, n);
    }
  }
}

// update_b, explicit k-omega part (src/update.f90:601-640): point-implicit
// rho*omega then rho*k with the destruction terms, omega floored by the
// production; ttrm = (0, gkw, bkw) for the Wilcox model (update_ttrm_b)
void update_kom_b(const Level &L, int b, const double *ra, double *qa, const double *qoa, const double *va,
                  const double *dtta, const double *dpla, const double *prda, double ar, const cosa_params &P,
                  const double *ttrma = nullptr) {
  B3 res(const_cast<double *>(ra), L, b), q(qa, L, b), qold(const_cast<double *>(qoa), L, b);
  B1 vol(const_cast<double *>(va), L, b, 1), dtt(const_cast<double *>(dtta), L, b, L.S);
  B3s dpl(const_cast<double *>(dpla), L, b), prd(const_cast<double *>(prda), L, b);
  for (int n = 0; n < L.S; ++n)
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) {
          // ttrm(2:3) per cell under BSL/SST, (gkw, bkw) for Wilcox
          const double gav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 2, n) : P.gkw;
          const double bav = ttrma ? B3t(const_cast<double *>(ttrma), L, b)(i, j, k, 3, n) : P.bkw;
          const double rho = q(i, j, k, 1, n);
          const double ome = q(i, j, k, 7, n) / q(i, j, k, 1, n);
          const double tke = q(i, j, k, 6, n) / q(i, j, k, 1, n);
          const double dtau = dtt(i, j, k, n) * vol(i, j, k);
          double rhomega = (qold(i, j, k, 7, n) - ar * res(i, j, k, 7, n) * dtt(i, j, k, n) +
                            ar * dtau * rho * ome * (gav * dpl(i, j, k, n) + 2 * bav * ome)) /
                           (1 + ar * dtau * (gav * dpl(i, j, k, n) + 2 * bav * ome));
          const double rhomegamin = gav * P.cmu * rho * std::sqrt(prd(i, j, k, n));
          if (rhomega < rhomegamin) rhomega = rhomegamin;
          q(i, j, k, 7, n) = rhomega;
          const double drhomega = q(i, j, k, 7, n) - rho * ome;
          q(i, j, k, 6, n) = (qold(i, j, k, 6, n) - ar * res(i, j, k, 6, n) * dtt(i, j, k, n) +
                              ar * dtau * rho * tke * (dpl(i, j, k, n) + P.bstrkw * ome) -
                              ar * dtau * P.bstrkw * tke * drhomega) /
                             (1 + ar * dtau * (dpl(i, j, k, n) + P.bstrkw * ome));
        }
}

// cutman_mut (src/bc.f90:2713-2799): cut_q on the turbulent viscosity
void cutman_mut_level(const Level &L, double *muta) {
  for (int icut = 0; icut < L.ncuts; ++icut) {
    const int *c = L.cut.data() + 21 * icut;
    const int b1 = c[0] - 1, b2 = c[9] - 1;
    B3s m1(muta, L, b1), m2(muta, L, b2);
    const int ijk1[4] = {0, L.im[b1], L.jm[b1], L.km[b1]}, ijk2[4] = {0, L.im[b2], L.jm[b2], L.km[b2]};
    const int idir1 = c[1], inout1 = c[2], idir2 = c[10], inout2 = c[11];
    const int istr1[4] = {0, c[3], c[5], c[7]}, iend1[4] = {0, c[4], c[6], c[8]};
    const int istr2[4] = {0, c[12], c[14], c[16]}, iend2[4] = {0, c[13], c[15], c[17]};
    const int iord[4] = {0, c[18], c[19], c[20]};
    int ibcpt, ibcinc, inr, inrinc;
    if (inout1 == 1) { ibcpt = 0; ibcinc = -1; } else { ibcpt = ijk1[idir1]; ibcinc = 1; }
    if (inout2 == 1) { inr = 1; inrinc = 1; } else { inr = ijk2[idir2] - 1; inrinc = -1; }
    int len[4], isgn1[4], isgn2[4];
    for (int l = 1; l <= 3; ++l) {
      len[l] = std::abs(iend1[l] - istr1[l]);
      isgn1[l] = iend1[l] > istr1[l] ? 1 : -1;
      isgn2[l] = iend2[l] > istr2[l] ? 1 : -1;
    }
    const int ic1 = cyc(idir1, 1), ic2 = cyc(idir1, 2), ic3 = cyc(idir1, 3);
    const int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
    for (int i3 = 0; i3 <= len[ic3]; ++i3)
      for (int i2 = 0; i2 <= len[ic2]; ++i2) {
        int p1[4] = {0, 0, 0, 0}, p2[4] = {0, 0, 0, 0};
        p1[ic1] = ibcpt; p1[ic2] = istr1[ic2] + isgn1[ic2] * i2; p1[ic3] = istr1[ic3] + isgn1[ic3] * i3;
        p2[jc1] = inr; p2[jc2] = istr2[jc2] + isgn2[jc2] * i2; p2[jc3] = istr2[jc3] + isgn2[jc3] * i3;
        for (int n = 0; n < L.S; ++n) {
          m1(p1[1], p1[2], p1[3], n) = m2(p2[1], p2[2], p2[3], n);
          int a1[4] = {0, p1[1], p1[2], p1[3]}, a2[4] = {0, p2[1], p2[2], p2[3]};
          a1[ic1] += ibcinc; a2[jc1] += inrinc;
          m1(a1[1], a1[2], a1[3], n) = m2(a2[1], a2[2], a2[3], n);
        }
      }
  }
}

// viscous set-up of a level as the solver start does it (src/cosa.f90:
// 300-322): volume and node halos, then the face inverse metrics.
// vm holds the 9 arrays (xi, eta, zeta derivatives on i-, j-, k-faces),
// array (d, m) at vm + ((d-1)*3 + m) * 3 * n0.
// viscous set-up (src/cosa.f90:300-322); moving grids: the ghost nodes and
// cuts and one set of face inverse metrics per grid snapshot
void viscous_setup_level(const Level &L, double *x, double *y, double *z, double *vol, double *vm) {
  volex_level(L, vol);
  cutman_v_level(L, vol);
  for (int nh = 0; nh < L.dim5h; ++nh) {
    coordex_level(L, x, y, z, nh);
    cutman_x_level(L, x, y, z, nh);
    double *vn = vm + (int64_t)nh * 27 * L.n0;
    for (int d = 1; d <= 3; ++d) {
      double *a = vn + (int64_t)(d - 1) * 9 * L.n0;
      for (int b = 0; b < L.nb; ++b) vmetrix_b(L, b, d, x, y, z, vol, a, a + 3 * L.n0, a + 6 * L.n0, nh);
    }
  }
}

// force frame of force_b (src/output.f90:4448-4470): drag (ss), lift (aa)
// and side (bb) directions; the aircraft frame, else the turbine one
void force_frame(const cosa_params &P, double ss[3], double aa[3], double bb[3]) {
  if (P.aircraft) {
    const double ca = std::cos(P.alpha), sa = std::sin(P.alpha), cb = std::cos(P.beta), sb = std::sin(P.beta);
    ss[0] = ca * cb; ss[1] = sa * cb; ss[2] = sb;
    const double den = std::sqrt(sb * sb + ca * ca * cb * cb);
    aa[0] = -sa * ca * cb * cb / den; aa[1] = den; aa[2] = sa * sb * cb / den;
    bb[0] = -sb / den; bb[1] = 0.0; bb[2] = ca * cb / den;
  } else {
    ss[0] = 0; ss[1] = 1; ss[2] = 0;
    aa[0] = 1; aa[1] = 0; aa[2] = 0;
    bb[0] = 0; bb[1] = 0; bb[2] = 1;
  }
}

// force_b (src/output.f90:4388-4900) of every block, summed over blocks in
// block order as force() does (src/output.f90:4283-4320).  Surface isurf
// (1-based) is the patches with bctopo(1) == 1500 + isurf - 1.  The wall
// state is the halo cell's conservative q; the moment arm is the node at
// face index ibcw (0 on inrout = 1 patches: the ghost node written by
// coordex).  The viscous part (P.viscous) uses the wall-face inverse
// metric of the patch's own direction (xideri, etaderj, zetaderk: vm arrays
// (1,xi), (2,eta), (3,zeta)).  out[n*12 + c], c = cl_p, cd_p, cz_p, cmx_p,
// cmy_p, cm_p, cl_v, cd_v, cz_v, cmx_v, cmy_v, cm_v; a non-moving grid, so
// the moment centre is xmom itself.
// snapshot times and pitch angles of harmonic balance (src/input.f90:3182-3192,
// src/grid.f90:4536-4541): t_n = n 2 pi / (|omegas| S), theta_n = dtheta0 sin(omegas t_n)
void hb_motion(const cosa_params &P, int S, double *zeit, double *dth) {
  const double pi = 3.14159265358979323846;
  const double omega = std::fabs(P.omegas);
  const double dt = omega > 0 ? 2 * pi / omega / S : 0.0;
  for (int n = 0; n < S; ++n) {
    zeit[n] = n * dt;
    dth[n] = P.dtheta0 * std::sin(P.omegas * zeit[n]);
  }
}

void force_level(const Level &L, const double *qa, const double *xa, const double *ya, const double *za,
                 const double *si, const double *sj, const double *sk, const double *vm, const cosa_params &P,
                 int isurf, const double xmom0[3], const double lngth[3], double *out) {
  double zeit[COSA_MAX_SNAP], dth[COSA_MAX_SNAP];
  hb_motion(P, L.S, zeit, dth);
  const double mach = P.machfs > 1e-14 ? P.machfs : 1.0;
  double ss[3], aa[3], bb[3];
  force_frame(P, ss, aa, bb);
  const double cf = 2 / (lngth[0] * lngth[1] * mach * mach);
  const double cmf = 2 / (lngth[0] * lngth[1] * lngth[2] * mach * mach);
  const double mor = P.machfs / P.reyno;
  for (int n = 0; n < L.S * 12; ++n) out[n] = 0.0;
  for (int b = 0; b < L.nb; ++b) {
    B3 q(const_cast<double *>(qa), L, b);
    const B2 sd[3] = {B2(si, L, b), B2(sj, L, b), B2(sk, L, b)};
    const int ijk[4] = {0, L.im[b], L.jm[b], L.km[b]};
    for (int n = 0; n < L.S; ++n) {
      const int nh = n * P.hbmove;
      BGs X(xa, L, b, nh), Y(ya, L, b, nh), Z(za, L, b, nh);
      double xmom[3] = {xmom0[0], xmom0[1], xmom0[2]};
      if (P.moving) {
        // moment centre carried by the pitching motion (src/output.f90:4476-4485)
        const double dr1 = (xmom0[0] - P.xh) * (std::cos(dth[n]) - 1) - (xmom0[1] - P.yh) * std::sin(dth[n]);
        const double dr2 = (xmom0[0] - P.xh) * std::sin(dth[n]) + (xmom0[1] - P.yh) * (std::cos(dth[n]) - 1);
        xmom[0] = xmom0[0] + dr1;
        xmom[1] = xmom0[1] + dr2;
      }
      double fp[6] = {0, 0, 0, 0, 0, 0}, fv[6] = {0, 0, 0, 0, 0, 0};
      for (int ib = 0; ib < L.nbcs[b]; ++ib) {
        const int *t = &L.bct[L.obct[b] + 10 * ib];
        if (t[0] != 1500 + isurf - 1) continue;
        Patch pa = patch_of(t, L.im[b], L.jm[b], L.km[b]);
        const int d = pa.idir, in1 = pa.inrout == 1;
        const int ibcpt = in1 ? 0 : ijk[d], ibcm = in1 ? 1 : ijk[d], ibcw = in1 ? 0 : ijk[d];
        const int sgn = in1 ? 1 : -1;  // (-1)**(1+1/inrout)
        const B2 &s = sd[d - 1];
        BV vd(vm ? const_cast<double *>(vm_snap(L, vm, nh)) + (int64_t)((d - 1) * 3 + (d - 1)) * 3 * L.n0 : nullptr, L, b);
        auto pw_of = [&](int i, int j, int k) {
          const double r = q(i, j, k, 1, n);
          return (P.gamma - 1) * (q(i, j, k, 5, n) - q(i, j, k, 2, n) * q(i, j, k, 2, n) / r / 2 -
                                  q(i, j, k, 3, n) * q(i, j, k, 3, n) / r / 2 - q(i, j, k, 4, n) * q(i, j, k, 4, n) / r / 2);
        };
        // pressure force and moment (src/output.f90:4660-4700)
        for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
          for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
            int hi, hj, hk, mi, mj, mk, wi, wj, wk;
            pidx(pa, ibcpt, i2, i3, hi, hj, hk);
            pidx(pa, ibcm, i2, i3, mi, mj, mk);
            pidx(pa, ibcw, i2, i3, wi, wj, wk);
            const double kx = sgn * s(1, mi, mj, mk, nh), ky = sgn * s(2, mi, mj, mk, nh);
            const double kz = sgn * s(3, mi, mj, mk, nh), ds = s(4, mi, mj, mk, nh);
            const double pw = pw_of(hi, hj, hk);
            fp[0] = fp[0] - pw * kx * ds;
            fp[1] = fp[1] - pw * ky * ds;
            fp[2] = fp[2] - pw * kz * ds;
            const double xr = X(wi, wj, wk) - xmom[0], yr = Y(wi, wj, wk) - xmom[1], zr = Z(wi, wj, wk) - xmom[2];
            fp[3] = fp[3] + (ky * zr - kz * yr) * pw * ds;
            fp[4] = fp[4] + (kz * xr - kx * zr) * pw * ds;
            fp[5] = fp[5] + (kx * yr - ky * xr) * pw * ds;
          }
        if (!P.viscous) continue;
        // skin friction from the one-sided three-point wall derivative
        // (src/output.f90:4703-4860)
        for (int i3 = pa.istrt[pa.ic3]; i3 <= pa.iend[pa.ic3]; ++i3)
          for (int i2 = pa.istrt[pa.ic2]; i2 <= pa.iend[pa.ic2]; ++i2) {
            int hi, hj, hk, mi, mj, mk, wi, wj, wk;
            pidx(pa, ibcpt, i2, i3, hi, hj, hk);
            pidx(pa, ibcm, i2, i3, mi, mj, mk);
            pidx(pa, ibcw, i2, i3, wi, wj, wk);
            const int o1[3] = {sgn * krd(d, 1), sgn * krd(d, 2), sgn * krd(d, 3)};
            const double kx = sgn * s(1, mi, mj, mk, nh), ky = sgn * s(2, mi, mj, mk, nh);
            const double kz = sgn * s(3, mi, mj, mk, nh), ds = s(4, mi, mj, mk, nh);
            const double ex = vd(1, mi, mj, mk), ey = vd(2, mi, mj, mk), ez = vd(3, mi, mj, mk);
            const double rhow = q(hi, hj, hk, 1, n);
            const double pw = pw_of(hi, hj, hk);
            const double tw = pw * P.gamma / rhow;
            const double muw = (P.stemp + 1) / (tw + P.stemp) * std::pow(tw, 1.5);
            double eta[3];
            for (int m = 0; m < 3; ++m) {
              const double uw = q(hi, hj, hk, m + 2, n) / q(hi, hj, hk, 1, n);
              const double u1 = q(hi + o1[0], hj + o1[1], hk + o1[2], m + 2, n) / q(hi + o1[0], hj + o1[1], hk + o1[2], 1, n);
              const double u2 = q(hi + 2 * o1[0], hj + 2 * o1[1], hk + 2 * o1[2], m + 2, n) /
                                q(hi + 2 * o1[0], hj + 2 * o1[1], hk + 2 * o1[2], 1, n);
              double uwm = uw, u1m = u1, u2m = u2;
              if (P.moving && L.cv[m]) {
                // velocities relative to the grid (src/output.f90:4768-4806)
                const BGs G(L.cv[m], L, b, nh);
                uwm = uw - G(hi, hj, hk);
                u1m = u1 - G(hi + o1[0], hj + o1[1], hk + o1[2]);
                u2m = u2 - G(hi + 2 * o1[0], hj + 2 * o1[1], hk + 2 * o1[2]);
              }
              eta[m] = sgn * (-8 * uwm + 9 * u1m - u2m) / 3;
            }
            const double dudx = eta[0] * ex, dudy = eta[0] * ey, dudz = eta[0] * ez;
            const double dvdx = eta[1] * ex, dvdy = eta[1] * ey, dvdz = eta[1] * ez;
            const double dwdx = eta[2] * ex, dwdy = eta[2] * ey, dwdz = eta[2] * ez;
            const double divv = dudx + dvdy + dwdz;
            const double txx = 2 * muw * (dudx - divv / 3), txy = muw * (dudy + dvdx), txz = muw * (dudz + dwdx);
            const double tyy = 2 * muw * (dvdy - divv / 3), tyz = muw * (dvdz + dwdy), tzz = 2 * muw * (dwdz - divv / 3);
            const double tx = txx * kx + txy * ky + txz * kz;
            const double ty = txy * kx + tyy * ky + tyz * kz;
            const double tz = txz * kx + tyz * ky + tzz * kz;
            fv[0] = fv[0] + mor * ds * tx;
            fv[1] = fv[1] + mor * ds * ty;
            fv[2] = fv[2] + mor * ds * tz;
            const double xr = X(wi, wj, wk) - xmom[0], yr = Y(wi, wj, wk) - xmom[1], zr = Z(wi, wj, wk) - xmom[2];
            fv[3] = fv[3] + mor * ds * (-ty * zr + tz * yr);
            fv[4] = fv[4] + mor * ds * (-tz * xr + tx * zr);
            fv[5] = fv[5] + mor * ds * (-tx * yr + ty * xr);
          }
      }
      // block coefficients (src/output.f90:4870-4893), summed over blocks
      double *o = out + n * 12;
      const double *f[2] = {fp, fv};
      for (int pv = 0; pv < 2; ++pv) {
        const double *g = f[pv];
        double *c = o + 6 * pv;
        c[0] += (g[0] * aa[0] + g[1] * aa[1] + g[2] * aa[2]) * cf;
        c[1] += (g[0] * ss[0] + g[1] * ss[1] + g[2] * ss[2]) * cf;
        c[2] += (g[0] * bb[0] + g[1] * bb[1] + g[2] * bb[2]) * cf;
        c[3] += g[3] * cmf;
        c[4] += g[4] * cmf;
        c[5] += g[5] * cmf;
      }
    }
  }
}

}  // namespace

// ============================================================================
// extern "C" surface used by tests/ (ctypes)
// ============================================================================
// a level of the oracle: the block tables and the level's low-speed
// cut-offs (p_cutoff_pgr / p_cutoff_vis of the reference, interior layout x S)
struct orc_level {
  Level L;
  std::vector<double> cut_pgr, cut_vis;
  int nl = 1;  // the level's index in the multigrid drivers
};

// rest3 of the low-speed cut-offs in restrict (src/cosa.f90:2724-2731)
void lsp_restrict(orc_level *f, orc_level *c, const cosa_params *p, const double *vol1, const double *vol2) {
  if (!p->lomach) return;
  for (int b = 0; b < f->L.nb; ++b) {
    if (p->cutoff_type == 3) rest3_b(f->L, c->L, b, f->cut_pgr.data(), c->cut_pgr.data(), vol1, vol2);
    if (p->visprec) rest3_b(f->L, c->L, b, f->cut_vis.data(), c->cut_vis.data(), vol1, vol2);
  }
}

extern "C" {

orc_level *orc_level_new(const cosa_level_desc *d, int npde, int nharms) {
  auto *h = new orc_level;
  Level &L = h->L;
  L.nb = d->nblocks; L.npde = npde; L.S = 2 * nharms + 1; L.lmet = 4; L.dim5h = 1;
  int64_t a3 = 0, a2 = 0, a1 = 0, a0 = 0, am = 0, ab = 0;
  for (int b = 0; b < L.nb; ++b) {
    int im = d->dims[3 * b], jm = d->dims[3 * b + 1], km = d->dims[3 * b + 2];
    L.im.push_back(im); L.jm.push_back(jm); L.km.push_back(km);
    L.nbcs.push_back(d->nbcs[b]);
    L.op3.push_back(a3); L.op2.push_back(a2); L.op1.push_back(a1);
    L.of0.push_back(a0); L.om1.push_back(am); L.obct.push_back(ab);
    a3 += (int64_t)(im + 3) * (jm + 3) * (km + 3);
    a2 += (int64_t)(im + 2) * (jm + 2) * (km + 2);
    a1 += (int64_t)(im + 1) * (jm + 1) * (km + 1);
    a0 += (int64_t)im * jm * km;
    am += (int64_t)(im - 1) * (jm - 1) * (km - 1);
    ab += 10 * d->nbcs[b];
  }
  L.n3 = a3; L.n2 = a2; L.n1 = a1; L.n0 = a0; L.nm1 = am;
  h->cut_pgr.assign((size_t)am * L.S, 0.0);
  h->cut_vis.assign((size_t)am * L.S, 0.0);
  L.bct.assign(d->bctopo, d->bctopo + ab);
  L.ncuts = d->ncuts;
  L.cut.assign(d->cutopo, d->cutopo + 21 * d->ncuts);
  return h;
}
void orc_level_free(orc_level *h) { delete h; }
void orc_level_sizes(orc_level *h, int64_t *s) {
  s[0] = h->L.n3; s[1] = h->L.n2; s[2] = h->L.n1; s[3] = h->L.n0; s[4] = h->L.nm1;
}
int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// moving grid of harmonic balance: metrics, grid arrays and the face /
// cell velocities of every snapshot (dim5h = S); null pointers turn the
// face and cell velocities off again
void orc_set_moving(orc_level *h, int hbmove, const double *fvi, const double *fvj, const double *fvk,
                    const double *cvx, const double *cvy, const double *cvz) {
  Level &L = h->L;
  L.dim5h = hbmove ? L.S : 1;
  L.fv[0] = fvi; L.fv[1] = fvj; L.fv[2] = fvk;
  L.cv[0] = cvx; L.cv[1] = cvy; L.cv[2] = cvz;
}
void orc_pitch(orc_level *h, const cosa_params *p, const double *x0, const double *y0, const double *z0,
               const double *dx, const double *dy, const double *dz, double *x, double *y, double *z, double *xd,
               double *yd, double *zd) {
  double zeit[COSA_MAX_SNAP], dth[COSA_MAX_SNAP];
  hb_motion(*p, h->L.S, zeit, dth);
  for (int b = 0; b < h->L.nb; ++b) pitch_b(h->L, b, x0, y0, z0, dx, dy, dz, x, y, z, xd, yd, zd, *p, zeit, dth);
}
void orc_face_vel(orc_level *h, const double *xd, const double *yd, const double *zd, double *fvi, double *fvj,
                  double *fvk) {
  for (int b = 0; b < h->L.nb; ++b) face_vel_b(h->L, b, xd, yd, zd, fvi, fvj, fvk);
}
void orc_vert2cell(orc_level *h, double *w) {
  for (int b = 0; b < h->L.nb; ++b) vert2cell_b(h->L, b, w);
}
void orc_hb_motion(const cosa_params *p, int S, double *zeit, double *dth) { hb_motion(*p, S, zeit, dth); }

void orc_imetrix(orc_level *h, const double *x, const double *y, const double *z, double *si,
                 double *sj, double *sk) {
  for (int b = 0; b < h->L.nb; ++b) imetrix_b(h->L, b, x, y, z, si, sj, sk);
}
void orc_vols(orc_level *h, const double *x, const double *y, const double *z, double *vol) {
  for (int b = 0; b < h->L.nb; ++b) bvols(h->L, b, x, y, z, vol);
}
void orc_cons2prim(orc_level *h, const cosa_params *p, int xtnd, double *q) {
  for (int b = 0; b < h->L.nb; ++b) cons2prim_b(h->L, b, q, xtnd, *p);
}
void orc_prim2cons(orc_level *h, const cosa_params *p, double *q) {
  for (int b = 0; b < h->L.nb; ++b) prim2cons_b(h->L, b, q, *p);
}
int orc_bc(orc_level *h, const cosa_params *p, double *q, const double *si, const double *sj,
           const double *sk) {
  return bc_level(h->L, q, si, sj, sk, *p);
}
void orc_cutman_q(orc_level *h, double *q) { cutman_q_level(h->L, q); }
int orc_prtest(orc_level *h, const cosa_params *p, const double *q) { return prtest_level(h->L, q, *p); }
void orc_lambda(orc_level *h, const cosa_params *p, const double *q, const double *si,
                const double *sj, const double *sk, double *lam) {
  lambda_level(h->L, q, si, sj, sk, lam, *p);
}
void orc_deltat(orc_level *h, const cosa_params *p, double *dtvol, const double *lam, double *bx,
                double *by, double *bz) {
  deltat_level(h->L, dtvol, lam, bx, by, bz, *p);
}
void orc_muscl(orc_level *h, const cosa_params *p, int idir, int nl, double *q, double *qp,
               double *qm, double *dq, double *dqp, double *dqm) {
  for (int b = 0; b < h->L.nb; ++b) muscl_b(h->L, b, idir, nl, q, qp, qm, dq, dqp, dqm, *p);
}
void orc_roflux(orc_level *h, const cosa_params *p, int idir, double *qr, double *ql, double *flux,
                const double *sijk) {
  for (int b = 0; b < h->L.nb; ++b) roflux_b(h->L, b, idir, qr, ql, flux, sijk, *p);
}
void orc_resid(orc_level *h, int idir, double *flux, double *res) {
  for (int b = 0; b < h->L.nb; ++b) resid_b(h->L, b, idir, flux, res);
}
void orc_update(orc_level *h, double *res, double *q, double *qold, double *dtvol, double ar) {
  for (int b = 0; b < h->L.nb; ++b) update_b(h->L, b, res, q, qold, dtvol, ar);
}
void orc_resg_rms(orc_level *h, double *res, double *rhs, double *out) { resg_rms_level(h->L, res, rhs, out); }
void orc_zero_res(orc_level *h, double *res) { zero_res(h->L, res); }
void orc_copy_interior(orc_level *h, double *dst, const double *src) { copy_interior(h->L, dst, src); }
// Roe face flux on single states (for KATs): q = (rho,u,v,w,p) prim
// nrm = (kx, ky, kz, ds[, ubn]): with nrm5 != 0, nrm[4] is the face's normal
// grid speed
void orc_roe_face(const cosa_params *p, const double *nrm, const double *qr, const double *ql,
                  double *f, int nrm5) {
  double vr[6], vl[6], out[6];
  for (int m = 0; m < 5; ++m) { vr[m + 1] = qr[m]; vl[m + 1] = ql[m]; }
  roe_face(*p, nrm[0], nrm[1], nrm[2], nrm[3], nrm5 ? nrm[4] : 0.0, vr, vl, 0.0, 0.0, out);
  for (int m = 0; m < 5; ++m) f[m] = out[m + 1];
}

/*
 * One residual evaluation as smooth() performs it at stage 1 (src/cosa.f90:
 * 1721-1908), leaving res (conservative residual), q back in conservative
 * form, and lambdas/dtvol when want_dt.  Work arrays are caller-owned P3/F0.
 */
int residual_impl(orc_level *h, const cosa_params *p, int nl, double *q, const double *si,
                  const double *sj, const double *sk, double *res, double *qp, double *qm, double *dq,
                  double *dqp, double *dqm, double *flux, double *dtvol, int want_dt, double *bx, double *by,
                  double *bz, const double *vol = nullptr, const double *vm = nullptr, int to_coarse = 0);

// arrays of the viscous / k-omega residual beyond cosa_level_ptrs: the face
// inverse metrics, production, div u, delta+ and the turbulence IRS
// coefficients
struct VExtra {
  const double *vm;
  double *prd, *divvel, *delpls;
  double *tbx, *tby, *tbz;
  double *ttrm;         // BSL/SST: (cdif, gamma, beta) per cell, P3 x 3 x S
  const double *fdist;  // BSL/SST: face wall distances, families 1..3 at 0, n0, 2 n0
  int to_coarse;        // smooth()'s to_coarse (the fine-level cut-offs of low-speed preconditioning)
};
int residual_full(orc_level *h, const cosa_params *p, int nl, const cosa_level_ptrs &A, const VExtra &X,
                  int want_dt, bool mut_first = false);

int orc_residual(orc_level *h, const cosa_params *p, int nl, double *q, const double *si,
                 const double *sj, const double *sk, double *res, double *qp, double *qm, double *dq,
                 double *dqp, double *dqm, double *flux, double *dtvol, int want_dt) {
  return residual_impl(h, p, nl, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt, nullptr, nullptr,
                       nullptr);
}

int residual_impl(orc_level *h, const cosa_params *p, int nl, double *q, const double *si,
                  const double *sj, const double *sk, double *res, double *qp, double *qm, double *dq,
                  double *dqp, double *dqm, double *flux, double *dtvol, int want_dt, double *bx, double *by,
                  double *bz, const double *vol, const double *vm, int to_coarse) {
  cosa_level_ptrs A{};
  A.q = q; A.res = res; A.dtvol = dtvol;
  A.si = const_cast<double *>(si); A.sj = const_cast<double *>(sj); A.sk = const_cast<double *>(sk);
  A.vol = const_cast<double *>(vol);
  A.qp = qp; A.qm = qm; A.dq = dq; A.dqp = dqp; A.dqm = dqm; A.flux = flux;
  A.betaxi = bx; A.betaeta = by; A.betazeta = bz;
  VExtra X{};
  X.vm = vm;
  X.to_coarse = to_coarse;
  return residual_full(h, p, nl, A, X, want_dt);
}

/*
 * One residual evaluation of smooth() (src/cosa.f90:1721-1908) on the
 * arrays of A: Euler, laminar (viscous) or Wilcox k-omega (viscous + kom,
 * with A.mut, A.dist, A.dtvolt and the source arrays of X).  q is left in
 * conservative form, res holds the residual, and on want_dt the time steps
 * (and IRS coefficients when the beta arrays are set).
 */
int residual_full(orc_level *h, const cosa_params *p, int nl, const cosa_level_ptrs &A, const VExtra &X,
                  int want_dt, bool mut_first) {
  Level &L = h->L;
  const bool visc = p->viscous != 0, kom = is_kom(*p);
  const bool blend = is_blend(*p);
  if (visc && (!A.vol || !X.vm)) return COSA_ERR_ARG;
  if (kom && (!visc || !A.mut || !A.dist || !A.dtvolt || !X.prd || !X.divvel || !X.delpls)) return COSA_ERR_ARG;
  if (blend && (!X.ttrm || !X.fdist)) return COSA_ERR_ARG;
  // low-speed preconditioning of k-omega runs (ipkpi of update_lsp_b) is not restated
  if (p->lomach && (kom || p->rkimp)) return COSA_ERR_UNSUPPORTED;
  double *q = A.q;
  for (int b = 0; b < L.nb; ++b) cons2prim_b(L, b, q, 0, *p);
  int status = bc_level(L, q, A.si, A.sj, A.sk, *p, A.dist, nl);
  cutman_q_level(L, q);
  if (mut_first) {
    // coarse-level mut from the restricted (primitive) state at the first
    // stage of the first cycle's visit (src/cosa.f90:1727-1760); SST takes
    // the cell-centred differences of a copy of q, back in conservative form
    if (p->kom_sst) {
      std::vector<double> w(q, q + L.n3 * L.npde * L.S);
      double *dc[3] = {A.qp, A.qm, A.dqm};
      for (int d = 1; d <= 3; ++d)
        for (int b = 0; b < L.nb; ++b) {
          q_face_b(L, b, d, w.data(), A.dq);
          q_der_c_b(L, b, d, A.dq, dc[d - 1], true);
        }
      for (int b = 0; b < L.nb; ++b) prim2cons_b(L, b, w.data(), *p);
      tur_vis_sst_level(L, w.data(), A.mut, A.qp, A.qm, A.dqm, X.vm, A.dist, *p);
      // the reference works in res and zeroes all of it afterwards
      std::fill(A.res, A.res + L.n3 * L.npde * L.S, 0.0);
    } else {
      tur_vis_level(L, q, A.mut, *p);
    }
    cutman_mut_level(L, A.mut);
  }
  status |= prtest_level(L, q, *p);
  const double *cpg = p->lomach ? h->cut_pgr.data() : nullptr, *cvs = p->lomach ? h->cut_vis.data() : nullptr;
  if (p->lomach) {
    // Darmofal's pressure-gradient cut-off (every level, or the fine level
    // of a cycle that restricts) and the viscous cut-off (src/cosa.f90:1763-1778)
    const bool fine = (p->nlevel > 1 && nl == 1 && X.to_coarse) || p->nlevel == 1;
    if ((p->cutoff_type == 3 && fine) || p->cutoff_type == 2)
      for (int b = 0; b < L.nb; ++b) lm_bcutoff_pg(L, b, q, h->cut_pgr.data(), *p);
    if (p->visprec && fine)
      for (int b = 0; b < L.nb; ++b) lm_bviscoff(L, b, q, A.si, A.sj, A.sk, h->cut_vis.data(), *p);
  }
  if (want_dt) {
    if (visc) {
      lambda_ns_level(L, q, A.si, A.sj, A.sk, A.vol, kom ? A.mut : nullptr, A.qp, A.dq, *p, cpg, cvs, nl);
      deltat_ns_level(L, A.dtvol, A.qp, A.dq, A.betaxi, A.betaeta, A.betazeta, *p, kom ? A.dtvolt : nullptr,
                      kom ? X.tbx : nullptr, kom ? X.tby : nullptr, kom ? X.tbz : nullptr);
    } else {
      lambda_level(L, q, A.si, A.sj, A.sk, A.qp, *p, cpg, cvs, nl);
      deltat_level(L, A.dtvol, A.qp, A.betaxi, A.betaeta, A.betazeta, *p);
    }
  }
  zero_res(L, A.res);
  if (visc)
    for (int b = 0; b < L.nb; ++b) q_bedges(L, b, q, kom ? A.mut : nullptr);
  const double *sd[4] = {nullptr, A.si, A.sj, A.sk};
  for (int d = 1; d <= 3; ++d) {
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < L.nb; ++b) muscl_b(L, b, d, nl, q, A.qp, A.qm, A.dq, A.dqp, A.dqm, *p);
    if (p->lomach) {
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) proflux_b(L, b, d, nl, A.qp, A.qm, A.flux, sd[d], cpg, cvs, *p);
    } else {
      for (int b = 0; b < L.nb; ++b) roflux_b(L, b, d, A.qp, A.qm, A.flux, sd[d], *p);
    }
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < L.nb; ++b) resid_b(L, b, d, A.flux, A.res);
    if (visc) {
      // q_face / q_der / [rtst] / vflux / resid (src/cosa.f90:1809-1824)
      const double *a = X.vm + (int64_t)(d - 1) * 9 * L.n0;
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) {
        q_face_b(L, b, d, q, A.dq);
        if (kom) q_face_mut_b(L, b, d, A.mut, A.flux);
        q_der_b(L, b, d, q, A.qp, A.qm, A.dqm);
        if (kom) {
          rtst_b(L, b, d, A.dq, A.qp, A.qm, A.dqm, a, a + 3 * L.n0, a + 6 * L.n0, A.dqp, A.flux, *p);
          vflux_kom_b(L, b, d, A.dq, A.qp, A.qm, A.dqm, A.dqp, a, a + 3 * L.n0, a + 6 * L.n0, sd[d], A.flux, *p,
                      blend ? X.fdist + (int64_t)(d - 1) * L.n0 : nullptr);
        }
        vflux_b(L, b, d, A.dq, A.qp, A.qm, A.dqm, a, a + 3 * L.n0, a + 6 * L.n0, sd[d], A.flux, *p, kom);
        resid_b(L, b, d, A.flux, A.res);
      }
    }
  }
  if (kom) {
    // cell-centred velocity gradients, production and the k-omega sources
    // (src/cosa.f90:1878-1896)
    double *dc[3] = {A.qp, A.qm, A.dqm};
    for (int d = 1; d <= 3; ++d)
      for (int b = 0; b < L.nb; ++b) {
        q_face_b(L, b, d, q, A.dq);
        q_der_c_b(L, b, d, A.dq, dc[d - 1], blend);
      }
    if (nl == 1 || p->prd_all_lvls)
      for (int b = 0; b < L.nb; ++b)
        turprod_b(L, b, q, A.qp, A.qm, A.dqm, X.vm, X.prd, X.divvel, X.delpls, *p);
    if (blend) {
      for (int b = 0; b < L.nb; ++b) {
        update_ttrm_b(L, b, q, A.qp, A.qm, A.dqm, X.vm, X.ttrm, A.dist, *p);
        srckw_sst_b(L, b, nl, q, A.mut, X.prd, X.divvel, A.res, X.ttrm, A.vol, *p);
      }
    } else {
      for (int b = 0; b < L.nb; ++b) srckw_b(L, b, nl, q, A.mut, X.prd, X.divvel, A.res, A.vol, *p);
    }
  }
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < L.nb; ++b) prim2cons_b(L, b, q, *p);
  if (dual_src_in_res(*p)) {
    if (!A.vol) return COSA_ERR_ARG;
    src_uns_level(L, q, A.vol, A.res, *p);
  } else if (p->harbal && A.vol && (!kom || !p->rkimp || p->irsop > 0 || p->nlevel > 1)) {
    // src_hb unless rkimp without IRS on one level (src/cosa.f90:1918-1922);
    // the Euler callers pass no vol in that case
    src_hb_level(L, q, A.vol, A.res, *p);
  }
  return status;
}

/*
 * Single-level explicit RK driver: mg() with nlevel=1 calls smooth(1,...,
 * niter=1) once per cycle (src/cosa.f90:817-840); this runs `ncycles` such
 * cycles.  hist receives, for cycles with (mgit==1 || mgit%rms_every==0 ||
 * mgit==last), the stage-1 resrms(1..npde+1) at row (mgit-mgit0).
 */
int orc_smooth_irs(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every, double *q,
                   double *qold, const double *si, const double *sj, const double *sk, double *res,
                   double *rhs, double *qp, double *qm, double *dq, double *dqp, double *dqm, double *flux,
                   double *dtvol, double *bx, double *by, double *bz, double *hist);

int orc_smooth(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every, double *q,
               double *qold, const double *si, const double *sj, const double *sk, double *res,
               double *rhs, double *qp, double *qm, double *dq, double *dqp, double *dqm, double *flux,
               double *dtvol, double *hist) {
  if (p->dualt || p->rgkuns) return COSA_ERR_UNSUPPORTED;  // dual time: orc_mg / orc_mg_rans; rkuns: orc_rkuns
  if (p->irsop > 0) return -1;
  Level &L = h->L;
  int status = 0;
  const int last = mgit0 + ncycles - 1;
  for (int mgit = mgit0; mgit <= last; ++mgit) {
    const int iter = 1;
    copy_interior(L, qold, q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= orc_residual(h, p, 1, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt);
      if (irk == 1 && (mgit == 1 || mgit % rms_every == 0 || mgit == last) && hist) {
        resg_rms_level(L, res, rhs, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
      }
      if (p->lomach) lsp_precres_level(L, 1, q, res, h->cut_pgr.data(), h->cut_vis.data(), *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) update_b(L, b, res, q, qold, dtvol, p->alphas[irk - 1]);
    }
  }
  return status;
}

int orc_smooth_irs(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every, double *q,
                   double *qold, const double *si, const double *sj, const double *sk, double *res,
                   double *rhs, double *qp, double *qm, double *dq, double *dqp, double *dqm, double *flux,
                   double *dtvol, double *bx, double *by, double *bz, double *hist) {
  if (p->dualt || p->rgkuns) return COSA_ERR_UNSUPPORTED;  // dual time: orc_mg / orc_mg_rans; rkuns: orc_rkuns
  Level &L = h->L;
  int status = 0;
  const int last = mgit0 + ncycles - 1;
  for (int mgit = mgit0; mgit <= last; ++mgit) {
    const int iter = 1;
    copy_interior(L, qold, q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= residual_impl(h, p, 1, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt, bx, by, bz);
      if (irk == 1 && (mgit == 1 || mgit % rms_every == 0 || mgit == last) && hist)
        resg_rms_level(L, res, rhs, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
      if (p->lomach) lsp_precres_level(L, 1, q, res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (p->irsop > 0) irs_level(L, res, dtvol, nullptr, bx, by, bz, nullptr, nullptr, nullptr, *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) update_b(L, b, res, q, qold, dtvol, p->alphas[irk - 1]);
    }
  }
  return status;
}

int orc_smooth_hb(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every, double *q,
                  double *qold, const double *si, const double *sj, const double *sk, const double *vol,
                  double *res, double *qp, double *qm, double *dq, double *dqp, double *dqm, double *flux,
                  double *dtvol, double *hist) {
  if (p->dualt || p->rgkuns) return COSA_ERR_UNSUPPORTED;  // dual time: orc_mg / orc_mg_rans; rkuns: orc_rkuns
  Level &L = h->L;
  int status = 0;
  const int last = mgit0 + ncycles - 1;
  // rkimp without IRS on one level: the time-spectral term is not added to
  // the residual (src/cosa.f90:1918-1922) but solved in update_bhb; with IRS
  // src_hb adds it and update_bhb takes it out again
  const bool imp = p->rkimp != 0;
  const bool src_in_res = !imp || p->irsop > 0 || p->nlevel > 1;
  if (imp && L.npde != 5) return COSA_ERR_UNSUPPORTED;
  std::vector<double> beta;
  double *bx = nullptr, *by = nullptr, *bz = nullptr;
  if (p->irsop > 0) {
    beta.assign((size_t)3 * L.n1 * L.S, 0.0);
    bx = beta.data(); by = bx + L.n1 * L.S; bz = by + L.n1 * L.S;
  }
  for (int mgit = mgit0; mgit <= last; ++mgit) {
    const int iter = 1;
    copy_interior(L, qold, q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= residual_impl(h, p, 1, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt, bx, by, bz,
                              src_in_res ? vol : nullptr);
      if (irk == 1 && (mgit == 1 || mgit % rms_every == 0 || mgit == last) && hist) {
        if (!src_in_res) resg_rms_hbimp_level(L, res, q, vol, *p, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
        else resg_rms_hb_level(L, res, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
      }
      if (p->lomach) lsp_precres_level(L, 1, q, res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (p->irsop > 0) irs_level(L, res, dtvol, nullptr, bx, by, bz, nullptr, nullptr, nullptr, *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) {
        if (imp) update_bhb_b(L, b, res, q, qold, dtvol, vol, p->alphas[irk - 1], *p, src_in_res);
        else update_b(L, b, res, q, qold, dtvol, p->alphas[irk - 1]);
      }
    }
  }
  return status;
}

void orc_lu_solve(int n, double *a, double *b, int nrhs) { lu_solve(n, a, b, nrhs); }

// ---- low-speed preconditioning, per routine (src/losp.f90, src/flux.f90:390-830) ----
// cut-off arrays in the interior-cell layout (off_m1 x S); q primitive
void orc_lm_cutoff_pg(orc_level *h, const cosa_params *p, const double *q, double *cut) {
  for (int b = 0; b < h->L.nb; ++b) lm_bcutoff_pg(h->L, b, q, cut, *p);
}
void orc_lm_viscoff(orc_level *h, const cosa_params *p, const double *q, const double *si, const double *sj,
                    const double *sk, double *cut) {
  for (int b = 0; b < h->L.nb; ++b) lm_bviscoff(h->L, b, q, si, sj, sk, cut, *p);
}
void orc_proflux(orc_level *h, const cosa_params *p, int idir, int nl, double *qr, double *ql, double *flux,
                 const double *sijk, const double *cpg, const double *cvs) {
  for (int b = 0; b < h->L.nb; ++b) proflux_b(h->L, b, idir, nl, qr, ql, flux, sijk, cpg, cvs, *p);
}
// prec (imax-1, jmax-1, kmax-1, npde, npde, 0:S-1) per block at off_m1 npde^2 S,
// from the conservative state
void orc_lsp_prec(orc_level *h, const cosa_params *p, int nl, const double *q, const double *cpg, const double *cvs,
                  double *prec) {
  const Level &L = h->L;
  const int npde = L.npde;
  for (int b = 0; b < L.nb; ++b) {
    B3 qv(const_cast<double *>(q), L, b);
    B1m cp(const_cast<double *>(cpg), L, b), cv(const_cast<double *>(cvs), L, b);
    const int64_t nc = (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
    double *pb = prec + L.om1[b] * npde * npde * L.S;
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            double qc[8], pm[49];
            for (int v = 1; v <= npde; ++v) qc[v] = qv(i, j, k, v, n);
            lsp_prec_cell(*p, nl, npde, qc, cp(i, j, k, n), cv(i, j, k, n), pm);
            const int64_t c = (i - 1) + (int64_t)(L.im[b] - 1) * ((j - 1) + (int64_t)(L.jm[b] - 1) * (k - 1));
            for (int r = 1; r <= npde; ++r)
              for (int cc = 1; cc <= npde; ++cc)
                pb[(((int64_t)n * npde + (cc - 1)) * npde + (r - 1)) * nc + c] = pm[(r - 1) * npde + (cc - 1)];
          }
  }
}
// precres / prec_bres (src/cosa.f90:2446-2521): res <- prec res
void orc_precres(orc_level *h, double *res, const double *prec) {
  const Level &L = h->L;
  const int npde = L.npde;
  for (int b = 0; b < L.nb; ++b) {
    B3 r(res, L, b);
    const int64_t nc = (int64_t)(L.im[b] - 1) * (L.jm[b] - 1) * (L.km[b] - 1);
    const double *pb = prec + L.om1[b] * npde * npde * L.S;
    for (int n = 0; n < L.S; ++n)
      for (int k = 1; k <= L.km[b] - 1; ++k)
        for (int j = 1; j <= L.jm[b] - 1; ++j)
          for (int i = 1; i <= L.im[b] - 1; ++i) {
            const int64_t c = (i - 1) + (int64_t)(L.im[b] - 1) * ((j - 1) + (int64_t)(L.jm[b] - 1) * (k - 1));
            double w[8];
            for (int a = 1; a <= npde; ++a) {
              w[a] = 0.0;
              for (int cc = 1; cc <= npde; ++cc)
                w[a] = w[a] + pb[(((int64_t)n * npde + (cc - 1)) * npde + (a - 1)) * nc + c] * r(i, j, k, cc, n);
            }
            for (int a = 1; a <= npde; ++a) r(i, j, k, a, n) = w[a];
          }
  }
}
// lambda with lomach: eig_eul_p, or with viscous eig_ns_p (src/cosa.f90:1447-1590)
void orc_lambda_p(orc_level *h, const cosa_params *p, int nl, const double *q, const double *si, const double *sj,
                  const double *sk, const double *vol, double *lam, double *lamv, const double *cpg,
                  const double *cvs) {
  if (p->viscous) lambda_ns_level(h->L, q, si, sj, sk, vol, nullptr, lam, lamv, *p, cpg, cvs, nl);
  else lambda_level(h->L, q, si, sj, sk, lam, *p, cpg, cvs, nl);
}
void orc_rest3(orc_level *f, orc_level *c, const double *c1, double *c2, const double *vol1, const double *vol2) {
  for (int b = 0; b < f->L.nb; ++b) rest3_b(f->L, c->L, b, c1, c2, vol1, vol2);
}
// the level's own cut-off arrays (what smooth() computes and restricts)
void orc_get_cutoffs(orc_level *h, double *pgr, double *vis) {
  std::copy(h->cut_pgr.begin(), h->cut_pgr.end(), pgr);
  std::copy(h->cut_vis.begin(), h->cut_vis.end(), vis);
}
void orc_set_cutoffs(orc_level *h, const double *pgr, const double *vis) {
  std::copy(pgr, pgr + h->cut_pgr.size(), h->cut_pgr.begin());
  std::copy(vis, vis + h->cut_vis.size(), h->cut_vis.begin());
}

void orc_src_uns(orc_level *h, const cosa_params *p, const double *q, const double *vol, double *res) {
  src_uns_level(h->L, q, vol, res, *p);
}
void orc_rhs_uns(orc_level *h, const cosa_params *p, double *rhs, const double *q1, const double *q2,
                 const double *vol) {
  rhs_uns_level(h->L, rhs, q1, q2, vol, *p);
}

/*
 * rkuns (src/cosa.f90:3890-4180) on a fixed grid: ntime physical steps of
 * the nstage-stage RK scheme with the global time step dtvol = dt / V of
 * deltat_urk (src/cosa.f90:2525-2572); on printed steps (itime % iprint == 0
 * or the last) hist row itime - 1 receives the norm of the last stage's
 * residual, as the reference overwrites resrms at every stage.  Euler and
 * laminar: the k-omega variant of the reference advances k and omega with
 * dtvolt, which rkuns never sets.
 */
int orc_rkuns(orc_level *h, const cosa_params *p, const cosa_level_ptrs *Ap, const double *vm, int ntime, int iprint,
              double *hist) {
  Level &L = h->L;
  const cosa_level_ptrs &A = *Ap;
  if (!p->rgkuns || is_kom(*p) || p->harbal || p->dualt) return COSA_ERR_UNSUPPORTED;
  if (!A.vol || !A.dtvol || (p->viscous && !vm) || iprint < 1) return COSA_ERR_ARG;
  for (int b = 0; b < L.nb; ++b) {
    B1 dtv(A.dtvol, L, b, 1), vol(A.vol, L, b, 1);
    for (int k = 1; k <= L.km[b] - 1; ++k)
      for (int j = 1; j <= L.jm[b] - 1; ++j)
        for (int i = 1; i <= L.im[b] - 1; ++i) dtv(i, j, k) = p->dt / vol(i, j, k);
  }
  int status = 0;
  for (int itime = 1; itime <= ntime; ++itime) {
    copy_interior(L, A.qold, A.q);
    const bool printed = itime % iprint == 0 || itime == ntime;
    for (int irk = 1; irk <= p->nstage; ++irk) {
      status |= residual_impl(h, p, 1, A.q, A.si, A.sj, A.sk, A.res, A.qp, A.qm, A.dq, A.dqp, A.dqm, A.flux, A.dtvol,
                              0, nullptr, nullptr, nullptr, A.vol, vm);
      if (status & (COSA_ERR_ARG | COSA_ERR_UNSUPPORTED)) return status;
      if (printed && hist) resg_rms_level(L, A.res, nullptr, hist + (int64_t)(itime - 1) * (L.npde + 1));
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) update_b(L, b, A.res, A.q, A.qold, A.dtvol, p->alphas[irk - 1]);
    }
  }
  return status;
}

void orc_src_hb(orc_level *h, const cosa_params *p, const double *q, const double *vol, double *res) {
  src_hb_level(h->L, q, vol, res, *p);
}

void orc_irs(orc_level *h, const cosa_params *p, double *res, const double *dtvol, const double *bx,
             const double *by, const double *bz) {
  irs_level(h->L, res, dtvol, nullptr, bx, by, bz, nullptr, nullptr, nullptr, *p);
}
void orc_tridi(const double *a, const double *b, const double *c, double *x, int dim) { tridi(a, b, c, x, dim); }

// ---- multigrid -------------------------------------------------------------
void orc_q_edges(orc_level *h, double *q, double *mut) {
  for (int b = 0; b < h->L.nb; ++b) q_bedges(h->L, b, q, mut);
}
void orc_q_corns(orc_level *h, double *q, double *mut) {
  for (int b = 0; b < h->L.nb; ++b) q_bcorns(h->L, b, q, mut);
}
void orc_fixq(orc_level *h, const cosa_params *p, double *q) { fixq_level(h->L, q, *p); }
void orc_tur_vis(orc_level *h, const cosa_params *p, const double *q, double *mut) {
  tur_vis_level(h->L, q, mut, *p);
}
void orc_add_array(orc_level *h, double *v1, const double *v2, double fact, int off_l) {
  add_level(h->L, v1, v2, fact, off_l);
}
void orc_rest1(orc_level *f, orc_level *c, const double *q1, double *q2, const double *vol1, const double *vol2) {
  for (int b = 0; b < f->L.nb; ++b) rest1_b(f->L, c->L, b, q1, q2, vol1, vol2);
}
void orc_rest2(orc_level *f, orc_level *c, double *rhs2, const double *res1) {
  for (int b = 0; b < f->L.nb; ++b) rest2_lo_b(f->L, c->L, b, rhs2, res1);
}
void orc_rest2_ho(orc_level *f, orc_level *c, double *rhs2, const double *res1) {
  for (int b = 0; b < f->L.nb; ++b) rest2_ho_b(f->L, c->L, b, rhs2, res1);
}
void orc_bc_res(orc_level *h, double *res) { bc_res_level(h->L, res); }
void orc_prol_bln(orc_level *f, orc_level *c, double *q1, const double *q2, int lim_corr) {
  for (int b = 0; b < f->L.nb; ++b) prol_bln_b(f->L, c->L, b, q1, q2, lim_corr);
}
void orc_prol_lin(orc_level *f, orc_level *c, double *q1, const double *q2, const double *vol1) {
  for (int b = 0; b < f->L.nb; ++b) prol_lin_b(f->L, c->L, b, q1, q2, vol1);
}

// restrict (src/cosa.f90:2672-2755), Euler branch
int orc_restrict(orc_level *f, orc_level *c, const cosa_params *p, const cosa_level_ptrs *P1,
                 const cosa_level_ptrs *P2) {
  if (is_kom(*p)) return COSA_ERR_UNSUPPORTED;
  orc_rest1(f, c, P1->q, P2->q, P1->vol, P2->vol);
  lsp_restrict(f, c, p, P1->vol, P2->vol);
  // ho_rest reads res's first halo layer as smooth() left it (zeroed at
  // every stage, src/cosa.f90:1786-1792)
  if (p->ho_rest) orc_rest2_ho(f, c, P2->rhs, P1->res);
  else orc_rest2(f, c, P2->rhs, P1->res);
  return 0;
}

// prolong (src/cosa.f90:3167-3250)
int orc_prolong(orc_level *f, orc_level *c, const cosa_params *p, const cosa_level_ptrs *P1,
                const cosa_level_ptrs *P2) {
  const Level &L2 = c->L;
  int status = 0;
  orc_rest1(f, c, P1->q, P2->qold, P1->vol, P2->vol);
  for (double *a : {P2->qold, P2->q}) {
    for (int b = 0; b < L2.nb; ++b) cons2prim_b(L2, b, a, 0, *p);
    status |= bc_level(L2, a, P2->si, P2->sj, P2->sk, *p, P2->dist, c->nl);
    cutman_q_level(L2, a);
    for (int b = 0; b < L2.nb; ++b) prim2cons_b(L2, b, a, *p);
    for (int b = 0; b < L2.nb; ++b) q_bedges(L2, b, a, nullptr);
    for (int b = 0; b < L2.nb; ++b) q_bcorns(L2, b, a, nullptr);
  }
  add_level(L2, P2->q, P2->qold, -1.0, 1);
  if (p->bln_prol) orc_prol_bln(f, c, P1->q, P2->q, p->lim_corr);
  else orc_prol_lin(f, c, P1->q, P2->q, P1->vol);
  if (p->lim_corr == 1 || p->lim_corr == 3) fixq_level(f->L, P1->q, *p);
  return status;
}

// smooth(nl, from_fine, to_coarse, done, niter) (src/cosa.f90:1594-2032):
// explicit Euler branch with the multigrid forcing; `done` is not evaluated.
// hist_row receives the fine-level resrms of printed cycles (last iteration).
int orc_smooth_level(orc_level *h, const cosa_params *p, int nl, const cosa_level_ptrs *P, int niter,
                     int from_fine, int to_coarse, int mgit, int ncycle, int rms_every, double *hist_row) {
  Level &L = h->L;
  int status = 0;
  const int niterp = to_coarse ? niter + 1 : niter;
  std::vector<double> work;
  // harmonic balance: src_hb in the residual unless rkimp without IRS on one
  // level (src/cosa.f90:1918-1922)
  const bool imp = p->harbal && p->rkimp;
  const bool src_in_res = p->harbal && (!p->rkimp || p->irsop > 0 || p->nlevel > 1);
  if (imp && L.npde != 5) return COSA_ERR_UNSUPPORTED;
  // dual time: src_uns in the residual (unless rkimp without IRS on one
  // level), res -= rhs_uns on the fine level (src/cosa.f90:1910-1941)
  const bool dual_imp = p->dualt && p->rkimp;
  for (int iter = 1; iter <= niterp; ++iter) {
    if (iter <= niter) copy_interior(L, P->qold, P->q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= residual_impl(h, p, nl, P->q, P->si, P->sj, P->sk, P->res, P->qp, P->qm, P->dq, P->dqp, P->dqm,
                              P->flux, P->dtvol, want_dt, P->betaxi, P->betaeta, P->betazeta,
                              src_in_res || dual_src_in_res(*p) ? P->vol : nullptr, nullptr, to_coarse);
      if (nl == 1 && irk == 1 && iter != niter + 1 && hist_row &&
          (mgit == 1 || mgit % rms_every == 0 || mgit == ncycle)) {
        if (dual_imp && !dual_src_in_res(*p)) {
          resg_rms_dualimp_level(L, P->res, P->rhs, P->q, P->vol, *p, hist_row);
        } else if (imp && !src_in_res) {
          resg_rms_hbimp_level(L, P->res, P->q, P->vol, *p, hist_row);
        } else if (p->harbal) {
          work.assign(P->res, P->res + L.n3 * L.npde * L.S);
          resg_rms_hb_level(L, work.data(), hist_row);
        } else {
          resg_rms_level(L, P->res, P->rhs, hist_row);
        }
      }
      if (nl == 1 && p->dualt) add_level(L, P->res, P->rhs, -1.0, -1);
      // low-speed preconditioning of the residual (src/cosa.f90:1943-1947)
      if (p->lomach) lsp_precres_level(L, nl, P->q, P->res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (from_fine && iter == 1 && irk == 1) add_level(L, P->rhs, P->res, 1.0, -1);
      if (nl > 1) add_level(L, P->res, P->rhs, -1.0, -1);
      if (iter == niter + 1) return status;
      if (p->irsop > 0)
        irs_level(L, P->res, P->dtvol, nullptr, P->betaxi, P->betaeta, P->betazeta, nullptr, nullptr, nullptr, *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) {
        if (imp) update_bhb_b(L, b, P->res, P->q, P->qold, P->dtvol, P->vol, p->alphas[irk - 1], *p, src_in_res);
        else if (dual_imp) update_dual_b(L, b, P->res, P->q, P->qold, P->dtvol, P->vol, p->alphas[irk - 1], *p,
                                         dual_src_in_res(*p));
        else update_b(L, b, P->res, P->q, P->qold, P->dtvol, p->alphas[irk - 1]);
      }
    }
  }
  return status;
}

// mg() (src/cosa.f90:806-930) for cycles mgit0..mgit0+ncycles-1 of ncycle
int orc_mg(orc_level **lv, int nlevel, const cosa_params *p, const cosa_level_ptrs *P, int mgit0, int ncycles,
           int ncycle, int rms_every, double *hist) {
  int status = 0;
  const int npde = p->npde;
  int last = mgit0 - 1;
  for (int l = 0; l < nlevel; ++l) lv[l]->nl = l + 1;
  for (int mgit = mgit0; mgit < mgit0 + ncycles; ++mgit) {
    last = mgit;
    double *row = hist ? hist + (int64_t)(mgit - mgit0) * (npde + 1) : nullptr;
    int niter = nlevel == 1 ? 1 : (mgit == 1 ? p->nstart : p->npost);
    status |= orc_smooth_level(lv[0], p, 1, &P[0], niter, 0, nlevel > 1, mgit, ncycle, rms_every, row);
    if (nlevel > 1) {
      status |= orc_restrict(lv[0], lv[1], p, &P[0], &P[1]);
      niter = nlevel == 2 ? p->ncrs : p->npre;
      status |= orc_smooth_level(lv[1], p, 2, &P[1], niter, 1, nlevel > 2, mgit, ncycle, rms_every, nullptr);
      if (nlevel == 3) {
        status |= orc_restrict(lv[1], lv[2], p, &P[1], &P[2]);
        status |= orc_smooth_level(lv[2], p, 3, &P[2], p->ncrs, 1, 0, mgit, ncycle, rms_every, nullptr);
        status |= orc_prolong(lv[1], lv[2], p, &P[1], &P[2]);
        status |= orc_smooth_level(lv[1], p, 2, &P[1], p->npost, 0, 0, mgit, ncycle, rms_every, nullptr);
      }
      status |= orc_prolong(lv[0], lv[1], p, &P[0], &P[1]);
    }
  }
  if (nlevel > 1 && last == ncycle)
    status |= orc_smooth_level(lv[0], p, 1, &P[0], p->npost, 0, 0, ncycle + 1, ncycle, rms_every, nullptr);
  return status;
}


// ---- viscous path ----------------------------------------------------------
void orc_coordex(orc_level *h, double *x, double *y, double *z) { coordex_level(h->L, x, y, z); }
void orc_cutman_x(orc_level *h, double *x, double *y, double *z) { cutman_x_level(h->L, x, y, z); }
void orc_volex(orc_level *h, double *vol) { volex_level(h->L, vol); }
void orc_cutman_v(orc_level *h, double *vol) { cutman_v_level(h->L, vol); }
void orc_vmetrix(orc_level *h, const double *x, const double *y, const double *z, const double *vol, double *vm) {
  for (int d = 1; d <= 3; ++d) {
    double *a = vm + (int64_t)(d - 1) * 9 * h->L.n0;
    for (int b = 0; b < h->L.nb; ++b) vmetrix_b(h->L, b, d, x, y, z, vol, a, a + 3 * h->L.n0, a + 6 * h->L.n0);
  }
}
void orc_viscous_setup(orc_level *h, double *x, double *y, double *z, double *vol, double *vm) {
  viscous_setup_level(h->L, x, y, z, vol, vm);
}
void orc_q_face(orc_level *h, int idir, const double *q, double *qf) {
  for (int b = 0; b < h->L.nb; ++b) q_face_b(h->L, b, idir, q, qf);
}
void orc_q_der(orc_level *h, int idir, const double *q, double *dqxi, double *dqeta, double *dqzeta) {
  for (int b = 0; b < h->L.nb; ++b) q_der_b(h->L, b, idir, q, dqxi, dqeta, dqzeta);
}
void orc_vflux(orc_level *h, const cosa_params *p, int idir, const double *qf, const double *dqxi,
               const double *dqeta, const double *dqzeta, const double *vm, const double *sijk, double *flux) {
  const double *a = vm + (int64_t)(idir - 1) * 9 * h->L.n0;
  for (int b = 0; b < h->L.nb; ++b)
    vflux_b(h->L, b, idir, qf, dqxi, dqeta, dqzeta, a, a + 3 * h->L.n0, a + 6 * h->L.n0, sijk, flux, *p);
}
void orc_lambda_ns(orc_level *h, const cosa_params *p, const double *q, const double *si, const double *sj,
                   const double *sk, const double *vol, const double *mut, double *lam, double *lamv) {
  lambda_ns_level(h->L, q, si, sj, sk, vol, mut, lam, lamv, *p);
}
void orc_deltat_ns(orc_level *h, const cosa_params *p, double *dtvol, const double *lam, const double *lamv,
                   double *bx, double *by, double *bz) {
  deltat_ns_level(h->L, dtvol, lam, lamv, bx, by, bz, *p);
}
int orc_residual_ns(orc_level *h, const cosa_params *p, int nl, double *q, const double *si, const double *sj,
                    const double *sk, const double *vol, const double *vm, double *res, double *qp, double *qm,
                    double *dq, double *dqp, double *dqm, double *flux, double *dtvol, int want_dt, double *bx,
                    double *by, double *bz) {
  return residual_impl(h, p, nl, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt, bx, by, bz, vol,
                       vm);
}
/*
 * Viscous explicit RK driver (smooth() with viscous = .true., one level):
 * like orc_smooth_irs with the viscous residual; vol and vm come from
 * orc_viscous_setup.
 */
int orc_smooth_ns(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every, double *q,
                  double *qold, const double *si, const double *sj, const double *sk, const double *vol,
                  const double *vm, double *res, double *rhs, double *qp, double *qm, double *dq, double *dqp,
                  double *dqm, double *flux, double *dtvol, double *bx, double *by, double *bz, double *hist) {
  if (p->dualt || p->rgkuns) return COSA_ERR_UNSUPPORTED;  // dual time: orc_mg / orc_mg_rans; rkuns: orc_rkuns
  Level &L = h->L;
  int status = 0;
  const int last = mgit0 + ncycles - 1;
  for (int mgit = mgit0; mgit <= last; ++mgit) {
    const int iter = 1;
    copy_interior(L, qold, q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= residual_impl(h, p, 1, q, si, sj, sk, res, qp, qm, dq, dqp, dqm, flux, dtvol, want_dt, bx, by, bz,
                              vol, vm);
      if (status & COSA_ERR_ARG) return status;
      if (irk == 1 && (mgit == 1 || mgit % rms_every == 0 || mgit == last) && hist) {
        if (p->harbal) resg_rms_hb_level(L, res, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
        else resg_rms_level(L, res, rhs, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
      }
      if (p->lomach) lsp_precres_level(L, 1, q, res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (p->irsop > 0) irs_level(L, res, dtvol, nullptr, bx, by, bz, nullptr, nullptr, nullptr, *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) update_b(L, b, res, q, qold, dtvol, p->alphas[irk - 1]);
    }
  }
  return status;
}

// ---- k-omega ---------------------------------------------------------------
/*
 * Single-level RK cycles of smooth() for the viscous path with the Wilcox
 * k-omega model (or laminar, when kom is off): residual_full per stage,
 * implicit residual smoothing with the turbulence coefficients, the
 * point-implicit k/omega update (update_b), fixq, and tur_vis + cutman_mut
 * after the last stage (src/cosa.f90:1994-2016).  A.mut must hold the
 * turbulent viscosity of the initial state (tur_vis + cutman_mut).
 */
int orc_smooth_rans(orc_level *h, const cosa_params *p, int ncycles, int mgit0, int rms_every,
                    const cosa_level_ptrs *Ap, const double *vm, double *prd, double *divvel, double *delpls,
                    double *tbx, double *tby, double *tbz, double *ttrm, const double *fdist, double *hist) {
  if (p->dualt || p->rgkuns) return COSA_ERR_UNSUPPORTED;  // dual time: orc_mg / orc_mg_rans; rkuns: orc_rkuns
  Level &L = h->L;
  const cosa_level_ptrs &A = *Ap;
  VExtra X{vm, prd, divvel, delpls, tbx, tby, tbz, ttrm, fdist};
  const bool kom = is_kom(*p);
  int status = 0;
  const int last = mgit0 + ncycles - 1;
  for (int mgit = mgit0; mgit <= last; ++mgit) {
    const int iter = 1;
    copy_interior(L, A.qold, A.q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      status |= residual_full(h, p, 1, A, X, want_dt);
      if (status & (COSA_ERR_ARG | COSA_ERR_UNSUPPORTED)) return status;
      if (irk == 1 && (mgit == 1 || mgit % rms_every == 0 || mgit == last) && hist) {
        if (p->harbal) resg_rms_hb_level(L, A.res, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
        else resg_rms_level(L, A.res, A.rhs, hist + (int64_t)(mgit - mgit0) * (L.npde + 1));
      }
      if (p->lomach) lsp_precres_level(L, 1, A.q, A.res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (p->irsop > 0)
        irs_level(L, A.res, A.dtvol, kom ? A.dtvolt : nullptr, A.betaxi, A.betaeta, A.betazeta, X.tbx, X.tby, X.tbz,
                  *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) {
        if (kom)
          update_kom_b(L, b, A.res, A.q, A.qold, A.vol, A.dtvolt, X.delpls, X.prd, p->alphas[irk - 1], *p,
                       is_blend(*p) ? X.ttrm : nullptr);
        update_b(L, b, A.res, A.q, A.qold, A.dtvol, p->alphas[irk - 1]);
      }
      if (kom) {
        if (p->ifixq) fixq_level(L, A.q, *p);
        if (irk == p->nstage) {
          if (p->kom_sst) tur_vis_sst_level(L, A.q, A.mut, A.qp, A.qm, A.dqm, X.vm, A.dist, *p);
          else tur_vis_level(L, A.q, A.mut, *p);
          cutman_mut_level(L, A.mut);
        }
      }
    }
  }
  return status;
}
int orc_residual_rans(orc_level *h, const cosa_params *p, int nl, const cosa_level_ptrs *A, const double *vm,
                      double *prd, double *divvel, double *delpls, double *tbx, double *tby, double *tbz,
                      double *ttrm, const double *fdist, int want_dt) {
  VExtra X{vm, prd, divvel, delpls, tbx, tby, tbz, ttrm, fdist};
  return residual_full(h, p, nl, *A, X, want_dt);
}
void orc_cutman_mut(orc_level *h, double *mut) { cutman_mut_level(h->L, mut); }
int orc_bc_dist(orc_level *h, const cosa_params *p, double *q, const double *si, const double *sj, const double *sk,
                const double *dist) {
  return bc_level(h->L, q, si, sj, sk, *p, dist);
}
void orc_q_face_mut(orc_level *h, int idir, const double *mut, double *flux) {
  for (int b = 0; b < h->L.nb; ++b) q_face_mut_b(h->L, b, idir, mut, flux);
}
void orc_rtst(orc_level *h, const cosa_params *p, int idir, const double *qf, const double *dqxi, const double *dqeta,
              const double *dqzeta, const double *vm, double *tau1, const double *flux) {
  const double *a = vm + (int64_t)(idir - 1) * 9 * h->L.n0;
  for (int b = 0; b < h->L.nb; ++b)
    rtst_b(h->L, b, idir, qf, dqxi, dqeta, dqzeta, a, a + 3 * h->L.n0, a + 6 * h->L.n0, tau1, flux, *p);
}
void orc_vflux_kom(orc_level *h, const cosa_params *p, int idir, const double *qf, const double *dqxi,
                   const double *dqeta, const double *dqzeta, const double *tau1, const double *vm,
                   const double *sijk, double *flux, const double *fdist) {
  const double *a = vm + (int64_t)(idir - 1) * 9 * h->L.n0;
  for (int b = 0; b < h->L.nb; ++b) {
    vflux_kom_b(h->L, b, idir, qf, dqxi, dqeta, dqzeta, tau1, a, a + 3 * h->L.n0, a + 6 * h->L.n0, sijk, flux, *p,
                fdist);
    vflux_b(h->L, b, idir, qf, dqxi, dqeta, dqzeta, a, a + 3 * h->L.n0, a + 6 * h->L.n0, sijk, flux, *p, true);
  }
}
void orc_q_der_c(orc_level *h, const cosa_params *p, int idir, const double *qf, double *dqc) {
  for (int b = 0; b < h->L.nb; ++b) q_der_c_b(h->L, b, idir, qf, dqc, is_blend(*p));
}
void orc_facedist(orc_level *h, const double *dist, double *fdist) {
  const int64_t n0 = h->L.n0;
  facedist_level(h->L, dist, fdist, fdist + n0, fdist + 2 * n0);
}
void orc_update_ttrm(orc_level *h, const cosa_params *p, const double *q, const double *dqxi, const double *dqeta,
                     const double *dqzeta, const double *vm, double *ttrm, const double *dist) {
  for (int b = 0; b < h->L.nb; ++b) update_ttrm_b(h->L, b, q, dqxi, dqeta, dqzeta, vm, ttrm, dist, *p);
}
void orc_srckw_sst(orc_level *h, const cosa_params *p, int nl, const double *q, const double *mut, const double *prd,
                   const double *divvel, double *res, const double *ttrm, const double *vol) {
  for (int b = 0; b < h->L.nb; ++b) srckw_sst_b(h->L, b, nl, q, mut, prd, divvel, res, ttrm, vol, *p);
}
void orc_tur_vis_sst(orc_level *h, const cosa_params *p, const double *q, double *mut, const double *dqxi,
                     const double *dqeta, const double *dqzeta, const double *vm, const double *dist) {
  tur_vis_sst_level(h->L, q, mut, dqxi, dqeta, dqzeta, vm, dist, *p);
}
void orc_turprod(orc_level *h, const cosa_params *p, const double *q, const double *dqxi, const double *dqeta,
                 const double *dqzeta, const double *vm, double *prd, double *divvel, double *delpls) {
  for (int b = 0; b < h->L.nb; ++b) turprod_b(h->L, b, q, dqxi, dqeta, dqzeta, vm, prd, divvel, delpls, *p);
}
void orc_srckw(orc_level *h, const cosa_params *p, int nl, const double *q, const double *mut, const double *prd,
               const double *divvel, double *res, const double *vol) {
  for (int b = 0; b < h->L.nb; ++b) srckw_b(h->L, b, nl, q, mut, prd, divvel, res, vol, *p);
}
void orc_update_kom(orc_level *h, const cosa_params *p, const double *res, double *q, const double *qold,
                    const double *vol, const double *dtvolt, const double *delpls, const double *prd, double ar,
                    const double *ttrm) {
  for (int b = 0; b < h->L.nb; ++b) update_kom_b(h->L, b, res, q, qold, vol, dtvolt, delpls, prd, ar, *p, ttrm);
}
// ---- k-omega multigrid ------------------------------------------------------
// per-level arrays of the k-omega residual beyond cosa_level_ptrs
struct orc_vextra {
  const double *vm;
  double *prd, *divvel, *delpls, *tbx, *tby, *tbz, *ttrm;
  const double *fdist;
};
static VExtra vx(const orc_vextra &e) {
  return VExtra{e.vm, e.prd, e.divvel, e.delpls, e.tbx, e.tby, e.tbz, e.ttrm, e.fdist};
}

void orc_rest4(orc_level *f, orc_level *c, const double *f1, double *f2, const double *vol1, const double *vol2) {
  for (int b = 0; b < f->L.nb; ++b) rest4_b(f->L, c->L, b, f1, f2, vol1, vol2);
}
void orc_lim_prod_mg(orc_level *h, const cosa_params *p, const double *q, double *prd, const double *mut) {
  for (int b = 0; b < h->L.nb; ++b) lim_prod_mg_b(h->L, b, q, prd, mut, *p);
}
void orc_lim_res_ome(orc_level *h, const cosa_params *p, double *res, const double *q, const double *vol,
                     const double *dtvolt, const double *delpls, const double *prd, double ar) {
  for (int b = 0; b < h->L.nb; ++b) lim_res_ome_b(h->L, b, res, q, vol, dtvolt, delpls, prd, ar, *p);
}

// smooth(nl, from_fine, to_coarse, done, niter) with the k-omega terms
// (src/cosa.f90:1594-2032): mut of the coarse level from its restricted
// state at the first stage of the first cycle's visit, the forcing, and on
// the residual pass (to_coarse) lim_prod_mg and lim_res_ome
int orc_smooth_level_rans(orc_level *h, const cosa_params *p, int nl, int nlevel, const cosa_level_ptrs *Ap,
                          const orc_vextra *E, int niter, int from_fine, int to_coarse, int mgit, int ncycle,
                          int rms_every, double *hist_row) {
  Level &L = h->L;
  const cosa_level_ptrs &A = *Ap;
  VExtra X = vx(*E);
  X.to_coarse = to_coarse;
  int status = 0;
  const int niterp = to_coarse ? niter + 1 : niter;
  for (int iter = 1; iter <= niterp; ++iter) {
    if (iter <= niter) copy_interior(L, A.qold, A.q);
    for (int irk = 1; irk <= p->nstage; ++irk) {
      const bool want_dt = (iter / p->iupdt * p->iupdt == iter) && irk == 1;
      const bool mut_first = mgit == 1 && iter == 1 && irk == 1 && from_fine && !p->prd_all_lvls;
      status |= residual_full(h, p, nl, A, X, want_dt, mut_first);
      if (status & (COSA_ERR_ARG | COSA_ERR_UNSUPPORTED)) return status;
      if (nl == 1 && irk == 1 && iter != niter + 1 && hist_row &&
          (mgit == 1 || mgit % rms_every == 0 || mgit == ncycle)) {
        if (p->dualt && p->rkimp && !dual_src_in_res(*p)) {
          resg_rms_dualimp_level(L, A.res, A.rhs, A.q, A.vol, *p, hist_row);
        } else if (p->harbal && p->rkimp && p->irsop == 0 && p->nlevel == 1) {
          resg_rms_hbimp_level(L, A.res, A.q, A.vol, *p, hist_row);
        } else if (p->harbal) {
          std::vector<double> w(A.res, A.res + L.n3 * L.npde * L.S);
          resg_rms_hb_level(L, w.data(), hist_row);
        } else {
          resg_rms_level(L, A.res, A.rhs, hist_row);
        }
      }
      if (nl == 1 && p->dualt) add_level(L, A.res, A.rhs, -1.0, -1);
      if (p->lomach) lsp_precres_level(L, nl, A.q, A.res, h->cut_pgr.data(), h->cut_vis.data(), *p);
      if (from_fine && iter == 1 && irk == 1) add_level(L, A.rhs, A.res, 1.0, -1);
      if (nl > 1) add_level(L, A.res, A.rhs, -1.0, -1);
      if (iter == niter + 1) {
        if (nlevel > 1 && nl != nlevel && !p->prd_all_lvls && p->lim_prodtke)
          for (int b = 0; b < L.nb; ++b) lim_prod_mg_b(L, b, A.q, X.prd, A.mut, *p);
        for (int b = 0; b < L.nb; ++b) {
          if (p->harbal)
            lim_res_ome_bhb_b(L, b, A.res, A.q, A.qold, A.vol, A.dtvolt, X.delpls, X.prd, *p,
                              is_blend(*p) ? X.ttrm : nullptr);
          else
            lim_res_ome_b(L, b, A.res, A.q, A.vol, A.dtvolt, X.delpls, X.prd, p->alphas[irk - 1], *p,
                          is_blend(*p) ? X.ttrm : nullptr);
        }
        return status;
      }
      if (p->irsop > 0)
        irs_level(L, A.res, A.dtvol, A.dtvolt, A.betaxi, A.betaeta, A.betazeta, X.tbx, X.tby, X.tbz, *p);
#pragma omp parallel for schedule(dynamic)
      for (int b = 0; b < L.nb; ++b) {
        if (p->dualt && p->rkimp) {
          update_kom_dual_b(L, b, A.res, A.q, A.qold, A.vol, A.dtvolt, X.delpls, X.prd, p->alphas[irk - 1], *p,
                            is_blend(*p) ? X.ttrm : nullptr, dual_src_in_res(*p));
          update_dual_b(L, b, A.res, A.q, A.qold, A.dtvol, A.vol, p->alphas[irk - 1], *p, dual_src_in_res(*p));
        } else if (p->harbal && p->rkimp) {
          const bool sir = p->irsop > 0 || p->nlevel > 1;
          update_bhb_kom_b(L, b, A.res, A.q, A.qold, A.vol, A.dtvolt, X.delpls, X.prd, p->alphas[irk - 1], *p,
                           is_blend(*p) ? X.ttrm : nullptr, sir);
          update_bhb_b(L, b, A.res, A.q, A.qold, A.dtvol, A.vol, p->alphas[irk - 1], *p, sir);
        } else {
          update_kom_b(L, b, A.res, A.q, A.qold, A.vol, A.dtvolt, X.delpls, X.prd, p->alphas[irk - 1], *p,
                       is_blend(*p) ? X.ttrm : nullptr);
          update_b(L, b, A.res, A.q, A.qold, A.dtvol, p->alphas[irk - 1]);
        }
      }
      if (p->ifixq) fixq_level(L, A.q, *p);
      if (irk == p->nstage && (nl == 1 || !p->prd_all_lvls)) {
        if (p->kom_sst) tur_vis_sst_level(L, A.q, A.mut, A.qp, A.qm, A.dqm, X.vm, A.dist, *p);
        else tur_vis_level(L, A.q, A.mut, *p);
        cutman_mut_level(L, A.mut);
      }
    }
  }
  return status;
}

// restrict (src/cosa.f90:2672-2755), k-omega branch: q, the production terms
// (or mut with prd_all_lvls) and the residual sums (high order with ho_rest)
int orc_restrict_rans(orc_level *f, orc_level *c, const cosa_params *p, const cosa_level_ptrs *P1,
                      const cosa_level_ptrs *P2, const orc_vextra *E1, const orc_vextra *E2) {
  orc_rest1(f, c, P1->q, P2->q, P1->vol, P2->vol);
  lsp_restrict(f, c, p, P1->vol, P2->vol);
  if (!p->prd_all_lvls) {
    orc_rest4(f, c, E1->prd, E2->prd, P1->vol, P2->vol);
    orc_rest4(f, c, E1->delpls, E2->delpls, P1->vol, P2->vol);
    orc_rest4(f, c, E1->divvel, E2->divvel, P1->vol, P2->vol);
  } else {
    orc_rest4(f, c, P1->mut, P2->mut, P1->vol, P2->vol);
  }
  if (p->ho_rest) {
    // halo of the fine residual for the 4x4x4 stencil (src/cosa.f90:2742-2749)
    cutman_q_level(f->L, P1->res);
    bc_res_level(f->L, P1->res);
    orc_q_edges(f, P1->res, nullptr);
    orc_q_corns(f, P1->res, nullptr);
    orc_rest2_ho(f, c, P2->rhs, P1->res);
  } else {
    orc_rest2(f, c, P2->rhs, P1->res);
  }
  return 0;
}

// mg() (src/cosa.f90:806-930) with the k-omega smoothing and restriction
int orc_mg_rans(orc_level **lv, int nlevel, const cosa_params *p, const cosa_level_ptrs *P, const orc_vextra *E,
                int mgit0, int ncycles, int ncycle, int rms_every, double *hist) {
  int status = 0;
  const int npde = p->npde;
  int last = mgit0 - 1;
  for (int l = 0; l < nlevel; ++l) lv[l]->nl = l + 1;
  for (int mgit = mgit0; mgit < mgit0 + ncycles; ++mgit) {
    last = mgit;
    double *row = hist ? hist + (int64_t)(mgit - mgit0) * (npde + 1) : nullptr;
    int niter = nlevel == 1 ? 1 : (mgit == 1 ? p->nstart : p->npost);
    status |= orc_smooth_level_rans(lv[0], p, 1, nlevel, &P[0], &E[0], niter, 0, nlevel > 1, mgit, ncycle,
                                    rms_every, row);
    if (nlevel > 1) {
      status |= orc_restrict_rans(lv[0], lv[1], p, &P[0], &P[1], &E[0], &E[1]);
      niter = nlevel == 2 ? p->ncrs : p->npre;
      status |= orc_smooth_level_rans(lv[1], p, 2, nlevel, &P[1], &E[1], niter, 1, nlevel > 2, mgit, ncycle,
                                      rms_every, nullptr);
      if (nlevel == 3) {
        status |= orc_restrict_rans(lv[1], lv[2], p, &P[1], &P[2], &E[1], &E[2]);
        status |= orc_smooth_level_rans(lv[2], p, 3, nlevel, &P[2], &E[2], p->ncrs, 1, 0, mgit, ncycle, rms_every,
                                        nullptr);
        status |= orc_prolong(lv[1], lv[2], p, &P[1], &P[2]);
        status |= orc_smooth_level_rans(lv[1], p, 2, nlevel, &P[1], &E[1], p->npost, 0, 0, mgit, ncycle,
                                        rms_every, nullptr);
      }
      status |= orc_prolong(lv[0], lv[1], p, &P[0], &P[1]);
    }
    if (status & (COSA_ERR_ARG | COSA_ERR_UNSUPPORTED)) return status;
  }
  if (nlevel > 1 && last == ncycle)
    status |= orc_smooth_level_rans(lv[0], p, 1, nlevel, &P[0], &E[0], p->npost, 0, 0, ncycle + 1, ncycle,
                                    rms_every, nullptr);
  return status;
}

void orc_deltat_ns_full(orc_level *h, const cosa_params *p, double *dtvol, const double *lam, const double *lamv,
                        double *bx, double *by, double *bz, double *dtvolt, double *tbx, double *tby, double *tbz) {
  deltat_ns_level(h->L, dtvol, lam, lamv, bx, by, bz, *p, dtvolt, tbx, tby, tbz);
}
void orc_force(orc_level *h, const cosa_params *p, const double *q, const double *x, const double *y,
               const double *z, const double *si, const double *sj, const double *sk, const double *vm, int isurf,
               const double *xmom, const double *lngth, double *out) {
  force_level(h->L, q, x, y, z, si, sj, sk, vm, *p, isurf, xmom, lngth, out);
}
}  // extern "C"
