// Fused RK stage for sm_100a: halo fill + tiled residual/update kernel.
//
// One RK stage of smooth() (src/cosa.f90:1719-2016) for the explicit Euler
// path is cons2prim -> bc -> cutman_q -> prtest -> [lambda, deltat] ->
// muscl/roflux/resid x3 -> prim2cons -> [resg_rms] -> update: about 25
// full-array sweeps.  Here it is two kernels:
//
//  k_halo        one thread per boundary/cut face cell and snapshot: reads
//                the conservative interior next to the face, converts it to
//                primitive form, applies the BC (or the cut copy) and writes
//                the primitive halo values into the halo slots of the same
//                state array.  Halo cells written twice in the reference keep
//                the reference's last writer (mask computed on the host).
//  k_stage_tile  a CTA owns a TI x TJ column of cells of one block and
//                marches along k.  Planes of the state are staged in a 4-deep
//                shared-memory ring (interior cells converted cons->prim on
//                the way in, halo cells taken as written by k_halo); every
//                i-, j- and k-face of the tile is reconstructed (MUSCL +
//                limiter) and Roe-fluxed once per tile, the k-face flux is
//                carried in registers between planes, the flux divergence is
//                summed in the reference order, and the stage update
//                q = qold - alpha dt/V R is written directly.  On stage 1 it
//                also computes the local time step (lambda/deltat) and the
//                per-tile residual sums of squares for resg_rms.
#pragma once
#include <cuda_pipeline.h>

#include "physics.cuh"
#include "kernels_ref.cuh"

struct HaloItem {
  int dblk, sblk;   // destination / source block (0-based)
  int type;         // BC type, -1 = cut copy
  int idir;         // direction of the face (1..3)
  int mask;         // bit0: write first halo layer, bit1: second
  int sgn;          // sign applied to the face normal
  int64_t h1, h2;   // halo cells (p3 cell index in dblk)
  int64_t c1, c2;   // interior cells (p3 cell index in sblk)
  int64_t mface;    // metric cell index (i + I2*(j + J2*k)) of the face in dblk
  int ps;           // slot of the flow conditions (BC values) in the params array
  int nl;           // multigrid level of the item's block (the low-speed cut-off epsp(nl))
};

struct Tile {
  int blk, n, i0, j0, k0, k1;  // first cell (i0,j0), planes k0..k1 (inclusive)
};

// strong-boundary flags of one block: for each direction d and side s
// (0 = min, 1 = max) a byte per tangential cell (t2,t3), t2 fastest, with
// (t2,t3) = (j,k) for d=1, (i,k) for d=2, (i,j) for d=3 (1-based cells).
struct StrongMap {
  int64_t off[3][2];
  int n2[3];
};

__device__ __forceinline__ bool strong_at(const uint8_t *flags, const StrongMap &m, int d, int side, int t2, int t3) {
  const int64_t o = m.off[d][side];
  if (o < 0) return false;
  return flags[o + (t2 - 1) + (int64_t)m.n2[d] * (t3 - 1)] != 0;
}

// ---- k_halo ------------------------------------------------------------------------
// face velocities of a moving grid, the reference's sijk(5:7) of the three
// families: (3, 0:imax+1, 0:jmax+1, 0:kmax+1, 0:S2-1) per block at op2*3*S2
struct FaceVel {
  const double *f[3];
};

template <bool CONS>
__global__ void k_halo(const DevBlock *__restrict__ blocks, const HaloItem *__restrict__ items, int nitems,
                       const cosa_params *__restrict__ Pp, double *__restrict__ q,
                       const double *__restrict__ si, const double *__restrict__ sj,
                       const double *__restrict__ sk, int *status, const double *__restrict__ dist = nullptr,
                       FaceVel fvel = FaceVel{{nullptr, nullptr, nullptr}}) {
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int64_t total = (int64_t)nitems * S;
  int st = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const HaloItem it = items[t % nitems];
    const int n = (int)(t / nitems);
    const DevBlock sb = blocks[it.sblk], db = blocks[it.dblk];
    double c1[7], c2[7], h1[7], h2[7];
    for (int v = 0; v < npde; ++v) {
      const int64_t base = p3_var(sb, npde, S, v + 1, n);
      c1[v] = q[base + it.c1];
      c2[v] = q[base + it.c2];
    }
    if (CONS) {
      if (npde > 5) { c2p7(P.gamma, c1); c2p7(P.gamma, c2); }
      else { c2p5(P.gamma, c1); c2p5(P.gamma, c2); }
    }
    int mask = 0;
    if (it.type < 0) {
      for (int v = 0; v < npde; ++v) { h1[v] = c1[v]; h2[v] = c2[v]; }
      mask = 3;
    } else {
      double nx = 0, ny = 0, nz = 0;
      if (it.type == 14 || it.type == 21 || it.type == 30 || it.type == 31 || (it.type / 100 == 15 && npde > 5)) {
        const double *s = it.idir == 1 ? si : (it.idir == 2 ? sj : sk);
        const int nh = n * P.hbmove;
        const int64_t I2 = db.im + 2, J2 = db.jm + 2, K2 = db.km + 2;
        const int64_t e = ((db.op2 * S2) + (int64_t)nh * I2 * J2 * K2 + it.mface) * 4;
        nx = s[e] * it.sgn; ny = s[e + 1] * it.sgn; nz = s[e + 2] * it.sgn;
      }
      const BcPar B = make_bcpar(Pp[it.ps], it.nl);
      int err = 0;
      // moving walls: the velocity of the wall face (snapshot nh)
      double wv[3];
      const double *wvp = nullptr;
      if ((it.type == 14 || it.type / 100 == 15) && fvel.f[it.idir - 1]) {
        const int64_t I2 = db.im + 2, J2 = db.jm + 2, K2 = db.km + 2;
        const int64_t e = ((db.op2 * S2) + (int64_t)(n * P.hbmove) * I2 * J2 * K2 + it.mface) * 3;
        const double *f = fvel.f[it.idir - 1];
        wv[0] = f[e]; wv[1] = f[e + 1]; wv[2] = f[e + 2];
        wvp = wv;
      }
      switch (it.type) {
        case 80: mask = bc_sym(it.idir, npde, c1, c2, h1, h2); break;
        case 4: mask = bc_extrapol(npde, c1, h1, h2); break;
        case 14: mask = bc_walinv(npde, nx, ny, nz, c1, c2, h1, h2, wvp); break;
        case 21: mask = bc_insub(B, nx, ny, nz, c1, c2, h1, h2, &err); break;
        case 91: mask = bc_outsub(B, c1, c2, h1, h2); break;
        case 30: mask = bc_far0(B, nx, ny, nz, c1, h1, h2); break;
        case 31: mask = bc_far1(B, nx, ny, nz, c1, h1, h2); break;
        default:
          if (it.type / 100 == 15) {
            mask = bc_walvis(P.gamma, c1, c2, h1, h2, wvp);
            if (npde > 5) {
              // k-omega wall values from the wall distance of the first cell
              if (!dist) { st |= COSA_ERR_ARG; break; }
              const int64_t I3 = db.I3, J3 = db.J3;
              const int ci = (int)(it.c1 % I3) - 1, cj = (int)((it.c1 / I3) % J3) - 1;
              const int ck = (int)(it.c1 / (I3 * J3)) - 1;
              bc_walvis_kom(P, nx, ny, nz, dist[p1_idx(db, 1, ci, cj, ck, 0)], c1, h1, h2, wvp);
            }
          } else {
            st |= COSA_ERR_UNSUPPORTED;
          }
          break;
      }
      if (err) st |= COSA_ERR_INFLOW;
    }
    mask &= it.mask;
    for (int v = 0; v < npde; ++v) {
      const int64_t base = p3_var(db, npde, S, v + 1, n);
      if (mask & 1) q[base + it.h1] = h1[v];
      if (mask & 2) q[base + it.h2] = h2[v];
    }
    if (CONS && it.idir == 1) {  // bprtest also checks the i halos of the state (src/cosa.f90:1000)
      if (mask & 1) { if (h1[4] <= P.qmin[4]) st |= COSA_ERR_NEG_P; else if (h1[0] <= P.qmin[0]) st |= COSA_ERR_NEG_RHO; }
      if (mask & 2) { if (h2[4] <= P.qmin[4]) st |= COSA_ERR_NEG_P; else if (h2[0] <= P.qmin[0]) st |= COSA_ERR_NEG_RHO; }
    }
  }
  if (st) atomicOr(status, st);
}

// ---- k_stage_tile ------------------------------------------------------------------
struct StageArgs {
  const double *qin;     // stage input: interior conservative, halos primitive
  double *qout;          // stage output (interior written)
  const double *qold;    // RK base state q^n
  double *qold_copy;     // if set, q^n interior is copied here (stage 1)
  double *dtvol;         // Delta t / V, written when compute_dt, read otherwise
  const double *si, *sj, *sk;
  double *part;          // per-tile residual sums of squares (npde) or null
  double *rhs;           // multigrid forcing term of a coarse level, or null
  int rhs_mode;          // 1: r -= rhs; 2: rhs += r first (forcing), then r -= rhs
  double *res_out;       // if set, the residual is stored here (P3 layout)
  double *bx, *by, *bz;  // IRS coefficients written with the time step (irsop >= 2)
  const double *vol;     // cell volumes when the harmonic-balance source is on
  const double *vres;    // viscous flux balance of each cell (P3 layout), added to the residual, or null
  const uint8_t *strong; // strong-boundary flags
  const StrongMap *smap; // per block
  int *status;
  double ar;
  int compute_dt;
  int first_order;
  int update;            // 0: residual only (restriction pass)
  const double *cfl_blk; // per-block CFL number (serving: each solve's own), or null for P.cfl
};

// Thread layout: TJ main warps, warp w holds row j0+w of the tile (lane =
// i - i0) and computes that cell's left i-face, left j-face and upper k-face
// of every plane, then updates the cell; one extra warp computes the tile's
// boundary faces (the j-faces above the last row and the i-faces right of the
// last column), so every warp does a balanced share of the Roe fluxes.
template <int TI, int TJ, bool MIXED, bool RMS>
__global__ void __launch_bounds__(TI *TJ + 32, 2)
k_stage_tile(const DevBlock *__restrict__ blocks, const Tile *__restrict__ tiles, const cosa_params *__restrict__ Pp,
             StageArgs A) {
  static_assert(TI == 32, "a main warp is one row of the tile");
  constexpr int NM = TI * TJ;                             // main threads (one per cell)
  constexpr int NT = NM + 32;                             // + the boundary-face warp
  constexpr int PI = TI + 4, PJ = TJ + 4, PL = PI * PJ;  // padded plane
  constexpr int NSLOT = 5;                                // planes k-1..k+2 + the one in flight
  constexpr int CPT = (PL + NT - 1) / NT;                 // plane cells per thread
  extern __shared__ double smem[];
  double *ring = smem;                        // [NSLOT][5][PJ][PI]
  double *fi = ring + NSLOT * 5 * PL;         // [5][TJ][TI+1]
  double *fj = fi + 5 * TJ * (TI + 1);        // [5][TJ+1][TI]
  double *red = fj + 5 * (TJ + 1) * TI;       // [5][TJ]

  const cosa_params &P = *Pp;
  const Tile T = tiles[blockIdx.x];
  const DevBlock b = blocks[T.blk];
  const int npde = 5, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int n = T.n, nh = n * P.hbmove;
  const PhysPar ph = make_phys(P);
  const double g = P.gamma;
  const int tid = threadIdx.x;
  const bool main_warp = tid < NM;
  const int ti = tid % TI, tj = main_warp ? tid / TI : 0;
  const int ci = T.i0 + ti, cj = T.j0 + tj;          // this thread's cell column
  const bool cvalid = main_warp && ci <= b.im - 1 && cj <= b.jm - 1;
  const int64_t vstride = b.P3;
  const double *qin = A.qin + p3_var(b, npde, S, 1, n);
  const StrongMap sm = A.smap[T.blk];
  // metric plane strides (fixed grid per snapshot)
  const int64_t I2 = b.im + 2, J2 = b.jm + 2;
  const int64_t mbase = (b.op2 * S2 + (int64_t)nh * I2 * J2 * (b.km + 2)) * 4;
  int st = 0;

  auto slot = [](int k) { return ((k % NSLOT) + NSLOT) % NSLOT; };

  auto cell_kind = [&](int c, int k, int64_t &gcell) -> int {
    if (c >= PL) return 0;
    const int pi = c % PI, pj = c / PI;
    const int i = T.i0 - 2 + pi, j = T.j0 - 2 + pj;
    const bool iin = i >= 1 && i <= b.im - 1, jin = j >= 1 && j <= b.jm - 1, kin = k >= 1 && k <= b.km - 1;
    const int nout = (!iin) + (!jin) + (!kin);
    if (nout > 1 || i > b.im + 1 || j > b.jm + 1) return 0;  // corners, edges, outside
    gcell = p3_cell(b, i, j, k);
    return nout == 0 ? 1 : 2;
  };
  auto prefetch = [&](int k) {
    double *dst = ring + slot(k) * 5 * PL;
#pragma unroll
    for (int r = 0; r < CPT; ++r) {
      const int c = tid + r * NT;
      int64_t gc;
      if (!cell_kind(c, k, gc)) continue;
#pragma unroll
      for (int m = 0; m < 5; ++m) __pipeline_memcpy_async(dst + m * PL + c, qin + m * vstride + gc, sizeof(double));
    }
    __pipeline_commit();
  };
  auto convert = [&](int k) {
    double *dst = ring + slot(k) * 5 * PL;
#pragma unroll
    for (int r = 0; r < CPT; ++r) {
      const int c = tid + r * NT;
      int64_t gc;
      if (cell_kind(c, k, gc) != 1) continue;
      double v[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) v[m] = dst[m * PL + c];
      c2p5_nr(g, v);
      if (v[4] <= P.qmin[4]) st |= COSA_ERR_NEG_P;
      else if (v[0] <= P.qmin[0]) st |= COSA_ERR_NEG_RHO;
#pragma unroll
      for (int m = 0; m < 5; ++m) dst[m * PL + c] = v[m];
    }
  };

  // MUSCL + limiter + Roe flux of face f along a line: w0..w3 = cells f-2..f+1
  auto face = [&](const double *w0p, const double *w1p, const double *w2p, const double *w3p, int f, int mx,
                  bool slo, bool shi, const double *met, double *F) {
    double qr[5], ql[5];
    const bool ovr_lo = (f == 1 && slo), ovr_hi = (f == mx && shi);
    const bool d_lo = (f - 1 == 1 && slo) || (f - 1 == mx && shi);
    const bool d_mid = (f == 1 && slo) || (f == mx && shi);
    const bool d_hi = (f + 1 == 1 && slo) || (f + 1 == mx && shi);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const double a0 = w0p[m * PL], a1 = w1p[m * PL], a2 = w2p[m * PL], a3 = w3p[m * PL];
      if (A.first_order) {
        qr[m] = a2; ql[m] = a1;
      } else {
        double dlo = a1 - a0, dmid = a2 - a1, dhi = a3 - a2;
        if (d_lo) dlo = (a1 - a0) * 2;
        if (d_mid) dmid = (a2 - a1) * 2;
        if (d_hi) dhi = (a3 - a2) * 2;
        if (MIXED) {
          float dp, dm;
          limit_face_fast(ph.ilimf, (float)ph.epslimf, (float)ph.rkap, (float)dlo, (float)dmid, (float)dhi, dp, dm);
          qr[m] = a2 + (double)dp; ql[m] = a1 + (double)dm;
        } else {
          double dp, dm;
          limit_face_nr(ph.ilimf, ph.epslimf, ph.rkap, dlo, dmid, dhi, dp, dm);
          qr[m] = __dadd_rn(a2, dp); ql[m] = __dadd_rn(a1, dm);
        }
      }
      if (ovr_lo) { qr[m] = a1; ql[m] = a1; }
      if (ovr_hi) { qr[m] = a2; ql[m] = a2; }
    }
    if (MIXED) roe_flux_mixed(ph, met[0], met[1], met[2], met[3], qr, ql, F);
    else roe_flux_euler(ph, met[0], met[1], met[2], met[3], qr, ql, F);
  };

  auto load_metric = [&](const double *s, int i, int j, int k, double *m4) {
    const int64_t e = mbase + (i + I2 * (j + J2 * (int64_t)k)) * 4;
    const double2 a = __ldg(reinterpret_cast<const double2 *>(s + e));
    const double2 c = __ldg(reinterpret_cast<const double2 *>(s + e + 2));
    m4[0] = a.x; m4[1] = a.y; m4[2] = c.x; m4[3] = c.y;
  };

  // k-face flux at face kf (between planes kf-1 and kf) of this column
  auto kface = [&](int kf, double *F) {
    const int pc = (tj + 2) * PI + (ti + 2);
    double m4[4];
    load_metric(A.sk, ci, cj, kf, m4);
    const bool slo = (kf <= 2) && strong_at(A.strong, sm, 2, 0, ci, cj);
    const bool shi = (kf >= b.km - 1) && strong_at(A.strong, sm, 2, 1, ci, cj);
    face(ring + slot(kf - 2) * 5 * PL + pc, ring + slot(kf - 1) * 5 * PL + pc, ring + slot(kf) * 5 * PL + pc,
         ring + slot(kf + 1) * 5 * PL + pc, kf, b.km, slo, shi, m4, F);
  };

  // the (up to) two in-plane faces of this thread: task t = 0, 1
  //   main warps: t = 0 i-face (ci, cj), t = 1 j-face (ci, cj)
  //   extra warp: t = 0 j-face (i0+lane, j0+TJ), t = 1 i-face (i0+TI, j0+lane) for lane < TJ
  struct InTask { int dir, i, j; bool valid; };
  auto task = [&](int t) -> InTask {
    InTask r;
    if (main_warp) {
      r.dir = t; r.i = ci; r.j = cj;
      r.valid = t == 0 ? (ci <= b.im && cj <= b.jm - 1) : (ci <= b.im - 1 && cj <= b.jm);
    } else if (t == 0) {
      r.dir = 1; r.i = T.i0 + ti; r.j = T.j0 + TJ;
      r.valid = r.i <= b.im - 1 && r.j <= b.jm;
    } else {
      r.dir = 0; r.i = T.i0 + TI; r.j = T.j0 + ti;
      r.valid = ti < TJ && r.i <= b.im && r.j <= b.jm - 1;
    }
    return r;
  };

  double acc[5] = {0, 0, 0, 0, 0};
  for (int k = T.k0 - 2; k <= T.k0 + 2; ++k) prefetch(k);
  __pipeline_wait_prior(0);
  for (int k = T.k0 - 2; k <= T.k0 + 2; ++k) convert(k);
  __syncthreads();
  double fk_lo[5];
  if (cvalid) kface(T.k0, fk_lo);

  for (int k = T.k0; k <= T.k1; ++k) {
    if (k > T.k0) {
      __pipeline_wait_prior(0);  // plane k+2, issued during the previous face phase
      convert(k + 2);
    }
    __syncthreads();
    // the slot of plane k+3 held plane k-2, last read before the barrier above
    if (k + 3 <= T.k1 + 2) prefetch(k + 3);
    const double *pl = ring + slot(k) * 5 * PL;
    {
      InTask tk = task(0);
      double mcur[4], mnext[4];
      if (tk.valid) load_metric(tk.dir == 0 ? A.si : A.sj, tk.i, tk.j, k, mcur);
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const InTask tn = task(1);
        if (t == 0 && tn.valid) load_metric(tn.dir == 0 ? A.si : A.sj, tn.i, tn.j, k, mnext);
        if (tk.valid) {
          const int pc = (tk.j - T.j0 + 2) * PI + (tk.i - T.i0 + 2);
          const int stride = tk.dir == 0 ? 1 : PI;
          const int f = tk.dir == 0 ? tk.i : tk.j, mx = tk.dir == 0 ? b.im : b.jm;
          const int t2 = tk.dir == 0 ? tk.j : tk.i;
          const bool slo = (f <= 2) && strong_at(A.strong, sm, tk.dir, 0, t2, k);
          const bool shi = (f >= mx - 1) && strong_at(A.strong, sm, tk.dir, 1, t2, k);
          double F[5];
          face(pl + pc - 2 * stride, pl + pc - stride, pl + pc, pl + pc + stride, f, mx, slo, shi, mcur, F);
          if (tk.dir == 0) {
            const int a = tk.i - T.i0, r = tk.j - T.j0;
#pragma unroll
            for (int m = 0; m < 5; ++m) fi[(m * TJ + r) * (TI + 1) + a] = F[m];
          } else {
            const int a = tk.i - T.i0, r = tk.j - T.j0;
#pragma unroll
            for (int m = 0; m < 5; ++m) fj[(m * (TJ + 1) + r) * TI + a] = F[m];
          }
        }
        tk = tn;
#pragma unroll
        for (int m = 0; m < 4; ++m) mcur[m] = mnext[m];
      }
    }
    double fk_hi[5];
    if (cvalid) kface(k + 1, fk_hi);
    __syncthreads();
    if (cvalid) {
      const int64_t cell = p3_cell(b, ci, cj, k);
      const int64_t o1 = p1_idx(b, S, ci, cj, k, n);
      double dt;
      if (A.compute_dt) {
        // lambdab + bdeltat (src/cosa.f90:1293-1323, 4860-4870)
        double qc[5], sim[4], sip[4], sjm[4], sjp[4], skm[4], skp[4];
        const int pc = (tj + 2) * PI + (ti + 2);
#pragma unroll
        for (int m = 0; m < 5; ++m) qc[m] = pl[m * PL + pc];
        load_metric(A.si, ci, cj, k, sim); load_metric(A.si, ci + 1, cj, k, sip);
        load_metric(A.sj, ci, cj, k, sjm); load_metric(A.sj, ci, cj + 1, k, sjp);
        load_metric(A.sk, ci, cj, k, skm); load_metric(A.sk, ci, cj, k + 1, skp);
        double li, lj, lk;
        eig_eul(g, qc, sim, sip, sjm, sjp, skm, skp, li, lj, lk);
        dt = (A.cfl_blk ? A.cfl_blk[T.blk] : P.cfl) / (li + lj + lk);
        A.dtvol[o1] = dt;
        if (A.bx) {
          double ba, bb_, bc;
          irs_beta(P.irsop, P.rat, P.psirs, li, lj, lk, ba, bb_, bc);
          A.bx[o1] = ba; A.by[o1] = bb_; A.bz[o1] = bc;
        }
      } else {
        dt = A.dtvol[o1];
      }
      const double *qo = A.qold + p3_var(b, npde, S, 1, n);
      double *qw = A.qout + p3_var(b, npde, S, 1, n);
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        // bresid order: i, then j, then k (src/cosa.f90:1800-1876)
        double r = fi[(m * TJ + tj) * (TI + 1) + ti + 1] - fi[(m * TJ + tj) * (TI + 1) + ti];
        r = r + fj[(m * (TJ + 1) + tj + 1) * TI + ti] - fj[(m * (TJ + 1) + tj) * TI + ti];
        r = r + fk_hi[m] - fk_lo[m];
        // viscous terms (q_face/q_der/vflux/resid, src/cosa.f90:1809-1876)
        if (A.vres) r = r + A.vres[p3_var(b, npde, S, m + 1, n) + cell];
        if (A.vol) {
          // src_bhb (src/src.f90:556-613): harmonic-balance coupling of the snapshots
          const double ov = P.omega * A.vol[p1_idx(b, 1, ci, cj, k, 0)];
          double qhb = 0.0;
          for (int nj2 = 0; nj2 < S; ++nj2)
            qhb = qhb + ov * P.dhb[n * S + nj2] * A.qin[p3_var(b, npde, S, m + 1, nj2) + cell];
          r = r + qhb;
        }
        // resg_rms of the fine level, where rhs is zero (src/cosa.f90:1925-1936)
        if (RMS) acc[m] += r * r;
        if (A.rhs_mode) {
          // multigrid forcing on coarse levels (src/cosa.f90:1950-1960)
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
          const double q0 = qo[m * vstride + cell];
          if (A.qold_copy) A.qold_copy[p3_var(b, npde, S, m + 1, n) + cell] = q0;
          qw[m * vstride + cell] = q0 - A.ar * r * dt;
        }
      }
#pragma unroll
      for (int m = 0; m < 5; ++m) fk_lo[m] = fk_hi[m];
    }
  }
  if (RMS) {
    __syncthreads();
    // deterministic per-tile sums: warp shuffle then fixed-order warp sums
    if (main_warp) {
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        double x = acc[m];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((tid & 31) == 0) red[m * TJ + (tid >> 5)] = x;
      }
    }
    __syncthreads();
    if (tid < 5) {
      double x = 0;
      for (int w = 0; w < TJ; ++w) x += red[tid * TJ + w];
      A.part[(int64_t)blockIdx.x * 8 + tid] = x;
    }
  }
  if (st) atomicOr(A.status, st);
}

template <int TI, int TJ>
constexpr size_t stage_smem_bytes() {
  return sizeof(double) * (5 * 5 * (TI + 4) * (TJ + 4) + 5 * TJ * (TI + 1) + 5 * (TJ + 1) * TI + 5 * TJ);
}
template <int TI, int TJ>
constexpr int stage_threads() { return TI * TJ + 32; }

// ---- deterministic reduction of per-tile / per-CTA partials -> resrms ------------------
// resg_rms (src/cosa.f90:4458-4501): sqrt(sum/ncell), total sqrt(sum/ncell/npde)
__global__ void k_rms_final(const double *__restrict__ part, int nparts, int npde, double ncell,
                            double *__restrict__ out, int *row_counter, int nrows_max) {
  __shared__ double red[8][32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < nparts; p += blockDim.x)
    for (int v = 0; v < npde; ++v) acc[v] += part[(int64_t)p * 8 + v];
  for (int v = 0; v < npde; ++v) {
    double x = acc[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    double tot[8], all = 0;
    for (int v = 0; v < npde; ++v) {
      double x = 0;
      for (int w = 0; w < nw; ++w) x += red[v][w];
      tot[v] = x;
      all = all + x;
    }
    int row = 0;
    if (row_counter) { row = *row_counter; if (row < nrows_max) *row_counter = row + 1; else row = nrows_max - 1; }
    double *o = out + (int64_t)row * (npde + 1);
    for (int v = 0; v < npde; ++v) o[v] = sqrt(tot[v] / ncell);
    o[npde] = sqrt(all / ncell / npde);
  }
}

// per-segment version of k_rms_final: CTA s reduces tiles [seg[2s], +seg[2s+1])
// in the same fixed order into out[s * (npde + 1) ...]
__global__ void k_rms_seg(const double *__restrict__ part, const int *__restrict__ seg,
                          const double *__restrict__ seg_ncell, int npde, double *__restrict__ out) {
  __shared__ double red[8][32];
  const int s = blockIdx.x;
  const double *pp = part + (int64_t)seg[2 * s] * 8;
  const int nparts = seg[2 * s + 1];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < nparts; p += blockDim.x)
    for (int v = 0; v < npde; ++v) acc[v] += pp[(int64_t)p * 8 + v];
  for (int v = 0; v < npde; ++v) {
    double x = acc[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    const double ncell = seg_ncell[s];
    double tot[8], all = 0;
    for (int v = 0; v < npde; ++v) {
      double x = 0;
      for (int w = 0; w < nw; ++w) x += red[v][w];
      tot[v] = x;
      all = all + x;
    }
    double *o = out + (int64_t)s * (npde + 1);
    for (int v = 0; v < npde; ++v) o[v] = sqrt(tot[v] / ncell);
    o[npde] = sqrt(all / ncell / npde);
  }
}

// ---- interior copy (odd stage counts end in the second buffer) --------------------------
template <class BS>
__global__ void k_copy_interior(BS bs_, int nvar_snap, const double *__restrict__ src, double *__restrict__ dst) {
  const DevBlock b = bs_.get();
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t n = (int64_t)ni * nj * nk * nvar_snap;
  const int64_t base = b.op3 * nvar_snap;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1; r /= nk;
    const int64_t o = base + r * b.P3 + p3_cell(b, i, j, k);
    dst[o] = src[o];
  }
}

// ---- stage finalisation: face halos of q in conservative form ----------------------------
// After smooth(), the reference's q holds prim2cons of the last stage's
// halo values (src/cosa.f90:1908).  src holds those values in primitive form.
__global__ void k_halo_p2c(const DevBlock *__restrict__ blocks, const HaloItem *__restrict__ items, int nitems,
                           const cosa_params *__restrict__ Pp, const double *__restrict__ src, double *__restrict__ dst) {
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1;
  const int64_t total = (int64_t)nitems * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const HaloItem it = items[t % nitems];
    const int n = (int)(t / nitems);
    const DevBlock db = blocks[it.dblk];
    for (int layer = 0; layer < 2; ++layer) {
      if (!((it.mask >> layer) & 1)) continue;
      const int64_t c = layer ? it.h2 : it.h1;
      double v[7];
      for (int m = 0; m < npde; ++m) v[m] = src[p3_var(db, npde, S, m + 1, n) + c];
      p2c(P.gamma, v, npde);
      for (int m = 0; m < npde; ++m) dst[p3_var(db, npde, S, m + 1, n) + c] = v[m];
    }
  }
}
