// C-ABI of the B200 path (include/cosa_gpu.h): context, level tables,
// per-routine drop-in entry points and the fused smooth() loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>
#include <vector>

#include "kernels_ref.cuh"
#include "fused.cuh"
#include "mg.cuh"
#include "visc.cuh"
#include "kom.cuh"
#include "split.cuh"
#include "faces.cuh"
#include "moving.cuh"
#include "force.cuh"
#include "unsteady.cuh"
#include "lsp.cuh"

namespace {
// any k-omega variant: Wilcox (kom), BSL (kom_bsl), SST (kom_sst)
inline bool rans(const cosa_params &p) { return p.kom || p.kom_bsl || p.kom_sst; }
// the routine-by-routine stage (in place, one launch per pass): k-omega and
// low-speed preconditioning
inline bool routine_stage(const cosa_params &p) { return rans(p) || p.lomach; }
inline bool blend(const cosa_params &p) { return p.kom_bsl || p.kom_sst; }
// dual time: src_uns enters the residual unless rkimp without IRS on one
// level, where update_b takes the physical-time term alone (src/cosa.f90:1910-1915)
inline bool dual_src_in_res(const cosa_params &p) { return p.dualt && (!p.rkimp || p.irsop > 0 || p.nlevel > 1); }

constexpr int kTI = 32, kTJ = 7;  // tile of the fused stage kernel (7 rows + the boundary-face warp = 256 threads)

struct LevelState {
  int nb = 0;
  int nl = 1;  // the level's index (1 = finest)
  std::vector<DevBlock> hb;
  std::vector<int> nbcs, bct, cut;
  std::vector<int64_t> obct;
  int ncuts = 0;
  int64_t n3 = 0, n2 = 0, n1 = 0, n0 = 0, nm1 = 0;
  DevBlock *d_blocks = nullptr;
  int *d_bct = nullptr;
  // halo work list: BC items first (table order), then cut items
  std::vector<HaloItem> items;
  int n_bc_items = 0;
  HaloItem *d_items = nullptr;
  uint8_t *d_strong = nullptr;
  StrongMap *d_smap = nullptr;
  Tile *d_tiles = nullptr;
  int ntiles = 0, kchunk = 0;
  bool bound = false;
  cosa_level_ptrs ptrs{};
  double *d_T = nullptr;      // second state buffer of the fused stages
  double *d_part = nullptr;   // per-tile / per-CTA partial sums (8 doubles each)
  double *d_res = nullptr;    // residual of the IRS path (P3, zero halos)
  double *d_ores = nullptr;   // right-hand side copy of the cut-aware IRS
  double *d_irs_scr = nullptr;  // tridiagonal pivots, 2 doubles per P3 cell and snapshot
  double *d_beta[3] = {nullptr, nullptr, nullptr};  // IRS coefficients when not bound
  int npart_cap = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // iteration without / with rms
  long long graph_launches[2] = {0, 0};           // kernels per replay of each graph
  // viscous terms: strong-boundary faces, cut_x / cut_v copy lists, the
  // face inverse metrics (caller-owned, bound by cosa_gpu_viscous_setup) and
  // the per-stage work arrays
  std::vector<WallFace> walls;
  WallFace *d_walls = nullptr;
  CopyItem *d_cutx = nullptr, *d_cutv = nullptr;
  int ncutx = 0, ncutv = 0;
  const double *d_vm = nullptr;
  double *d_qprim = nullptr;  // primitive stage state (P3)
  double *d_vflux = nullptr;  // viscous face fluxes of the three families (3 x F0)
  double *d_vres = nullptr;   // viscous flux balance (P3)
  // k-omega: production, div u, delta+ (scalar P3) and the turbulence IRS
  // coefficients (P1 x S)
  double *d_prd = nullptr, *d_divvel = nullptr, *d_delpls = nullptr;
  double *d_ttrm = nullptr;   // BSL/SST: (cdif, gamma, beta) per cell (P3 x 3 x S)
  double *d_fdist = nullptr;  // BSL/SST: face wall distances, families 1..3 at 0, n0, 2 n0
  double *d_h0 = nullptr;     // k-omega: h0 of each family's last face (block x 3 x snapshot x 2)
  double *d_rflux = nullptr;  // k-omega: convective and viscous face fluxes of the three families (6 x F0 x npde x S)
  int rflux_S = 0;
  // low-speed preconditioning: the level's pressure-gradient and viscous
  // cut-offs (interior layout x S, the reference's p_cutoff_pgr / p_cutoff_vis)
  double *d_cut_pgr = nullptr, *d_cut_vis = nullptr;
  double *d_tbeta[3] = {nullptr, nullptr, nullptr};
  // stage schedule: 0 = fused tile kernel, 1 = face-split (k_faces + k_cells),
  // set by cosa_gpu_autotune
  int schedule = 0;
  double *d_cflux = nullptr;  // convective face fluxes of the split schedule (3 x F0)
  FaceTask *d_ftasks = nullptr;  // warp tasks of k_faces_line: i-face tasks first
  int nftasks = 0, nftasks1 = 0;
  // wall faces of each force surface (key: surface number), built on first use
  struct ForceList {
    ForceFace *d_faces = nullptr;
    int nfaces = 0;
    int *d_bstart = nullptr;
    double *d_buf = nullptr, *d_sums = nullptr, *d_xmom = nullptr;
  };
  std::map<int, ForceList> forces;
};

}  // namespace

struct ProfState {
  bool on = false;
  // kinds: 0 halo fill, 1 main kernel (k_stage_tile, or k_faces of the split
  // schedule), 2 the split schedule's k_cells
  cudaEvent_t ev[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};  // [kind][start/stop]
  double ms[3] = {0, 0, 0};
  long long n[3] = {0, 0, 0};
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;  // kernels per replay
};

struct cosa_ctx {
  ProfState prof;
  std::map<uint64_t, GraphEntry> graphs;  // captured launch sequences by key
  cosa_params p{};
  cosa_params *d_p = nullptr;
  int device = 0;
  cudaStream_t s = nullptr;
  int nlevels = 0;
  LevelState L[COSA_MAX_LEVELS];
  int *d_status = nullptr;
  int *d_row = nullptr;
  double *d_hist = nullptr;
  const cosa_params *d_halo_p = nullptr;  // flow-condition slots read by k_halo (default: d_p)
  // residual norms reduced per segment of tiles (one per served solve) when
  // set: segment s = tiles [d_seg[2s], +d_seg[2s+1]) with seg_ncell[s] cells
  int nseg = 0;
  double *d_cfl_blk = nullptr;  // serving: CFL number of each block's solve
  int *d_seg = nullptr;
  double *d_seg_ncell = nullptr;
  int hist_cap = 0;
  long long launches = 0;
  std::vector<void *> allocs;
};

namespace {

int cuda_ok(cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "cosa_gpu: CUDA error %s\n", cudaGetErrorString(e));
    return COSA_ERR_CUDA;
  }
  return COSA_OK;
}
#define CK(x) do { int _r = cuda_ok(x); if (_r) return _r; } while (0)

template <typename T>
int dalloc(cosa_ctx *c, T **p, size_t n) {
  void *v = nullptr;
  CK(cudaMalloc(&v, std::max<size_t>(n, 1) * sizeof(T)));
  c->allocs.push_back(v);
  *p = static_cast<T *>(v);
  return COSA_OK;
}

int grid_for(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// index of cell (i,j,k) on the normal/tangential decomposition of a face
inline void pcell(int idir, int nrm, int i2, int i3, int &i, int &j, int &k) {
  const int ic1 = cyc3(idir, 1), ic2 = cyc3(idir, 2), ic3 = cyc3(idir, 3);
  int v[4] = {0, 0, 0, 0};
  v[ic1] = nrm; v[ic2] = i2; v[ic3] = i3;
  i = v[1]; j = v[2]; k = v[3];
}

// offs (optional): per block the P3, P2 and P1 offsets in cells to use
// instead of the setoffs() concatenation (blocks placed in a shared pool);
// bps (optional): per block the slot of its flow conditions for k_halo
int build_level(cosa_ctx *c, LevelState &L, const cosa_level_desc &d, const int64_t *offs = nullptr,
                const int *bps = nullptr) {
  L.nb = d.nblocks;
  int64_t a3 = 0, a2 = 0, a1 = 0, a0 = 0, am = 0, ab = 0;
  for (int b = 0; b < L.nb; ++b) {
    DevBlock x{};
    x.im = d.dims[3 * b]; x.jm = d.dims[3 * b + 1]; x.km = d.dims[3 * b + 2];
    if (x.im < 3 || x.jm < 3 || x.km < 2) return COSA_ERR_ARG;
    x.I3 = x.im + 3; x.J3 = x.jm + 3;
    x.P3 = (int64_t)(x.im + 3) * (x.jm + 3) * (x.km + 3);
    x.op3 = a3; x.op2 = a2; x.op1 = a1; x.of0 = a0; x.om1 = am;
    if (offs) { x.op3 = offs[3 * b]; x.op2 = offs[3 * b + 1]; x.op1 = offs[3 * b + 2]; }
    x.obct = (int)ab; x.nbcs = d.nbcs[b];
    L.hb.push_back(x);
    L.nbcs.push_back(d.nbcs[b]);
    L.obct.push_back(ab);
    a3 += x.P3;
    a2 += (int64_t)(x.im + 2) * (x.jm + 2) * (x.km + 2);
    a1 += (int64_t)(x.im + 1) * (x.jm + 1) * (x.km + 1);
    a0 += (int64_t)x.im * x.jm * x.km;
    am += (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1);
    ab += 10 * d.nbcs[b];
  }
  L.n3 = a3; L.n2 = a2; L.n1 = a1; L.n0 = a0; L.nm1 = am;
  if (offs) {  // pool placement: array extents reach the furthest block end
    L.n3 = L.n2 = L.n1 = 0;
    for (const DevBlock &x : L.hb) {
      L.n3 = std::max(L.n3, x.op3 + x.P3);
      L.n2 = std::max(L.n2, x.op2 + (int64_t)(x.im + 2) * (x.jm + 2) * (x.km + 2));
      L.n1 = std::max(L.n1, x.op1 + (int64_t)(x.im + 1) * (x.jm + 1) * (x.km + 1));
    }
  }
  L.bct.assign(d.bctopo, d.bctopo + ab);
  L.ncuts = d.ncuts;
  L.cut.assign(d.cutopo, d.cutopo + 21 * (int64_t)d.ncuts);

  // ---- halo work list: bbc (src/bc.f90:35-121) then cut_q (src/bc.f90:1894-2141)
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    const int ijk[4] = {0, x.im, x.jm, x.km};
    const int64_t I2 = x.im + 2, J2 = x.jm + 2;
    for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
      const int *r = L.bct.data() + L.obct[b] + 10 * ibc;
      const int type = r[0], idir = r[1], inrout = r[2];
      if (idir < 1 || idir > 3) return COSA_ERR_ARG;
      // viscous walls: the laminar, fixed-grid branch of bc_walvis_15
      const bool wall15 = type / 100 == 15;
      const bool ok = type == 80 || type == 4 || type == 14 || type == 21 || type == 91 || type == 30 || type == 31 ||
                      wall15;
      if (!ok) return COSA_ERR_UNSUPPORTED;
      int istrt[4] = {0, r[3], r[5], r[7]}, iend[4] = {0, r[4], r[6], r[8]};
      const int ic2 = cyc3(idir, 2), ic3 = cyc3(idir, 3);
      int ibcpt, ibcpt2, ibcn, ibcn2, ibcm;
      if (inrout == 1) { ibcpt = 0; ibcpt2 = -1; ibcn = 1; ibcn2 = 2; ibcm = 1; }
      else { ibcpt = ijk[idir]; ibcpt2 = ibcpt + 1; ibcn = ibcpt - 1; ibcn2 = ibcpt - 2; ibcm = ibcpt; }
      int sgn = 1;
      if (type == 21) sgn = inrout == 1 ? 1 : -1;       // bc_insub sgnm
      else if (type == 30 || type == 31) sgn = inrout == 1 ? -1 : 1;  // bc_far0 / bc_far1 sgnm
      for (int i3 = istrt[ic3]; i3 <= iend[ic3]; ++i3)
        for (int i2 = istrt[ic2]; i2 <= iend[ic2]; ++i2) {
          HaloItem it{};
          it.dblk = it.sblk = b; it.type = type; it.idir = idir; it.mask = 3; it.sgn = sgn;
          int i, j, k;
          pcell(idir, ibcpt, i2, i3, i, j, k); it.h1 = p3_cell(x, i, j, k);
          pcell(idir, ibcpt2, i2, i3, i, j, k); it.h2 = p3_cell(x, i, j, k);
          pcell(idir, ibcn, i2, i3, i, j, k); it.c1 = p3_cell(x, i, j, k);
          pcell(idir, ibcn2, i2, i3, i, j, k); it.c2 = p3_cell(x, i, j, k);
          pcell(idir, ibcm, i2, i3, i, j, k); it.mface = i + I2 * (j + J2 * (int64_t)k);
          L.items.push_back(it);
        }
    }
  }
  L.n_bc_items = (int)L.items.size();
  for (int ic = 0; ic < L.ncuts; ++ic) {
    const int *cc = L.cut.data() + 21 * (int64_t)ic;
    const int b1 = cc[0] - 1, b2 = cc[9] - 1;
    if (b1 < 0 || b1 >= L.nb || b2 < 0 || b2 >= L.nb) return COSA_ERR_ARG;
    const DevBlock &x1 = L.hb[b1], &x2 = L.hb[b2];
    const int ijk1[4] = {0, x1.im, x1.jm, x1.km}, ijk2[4] = {0, x2.im, x2.jm, x2.km};
    const int idir1 = cc[1], inout1 = cc[2], idir2 = cc[10], inout2 = cc[11];
    const int istr1[4] = {0, cc[3], cc[5], cc[7]}, iend1[4] = {0, cc[4], cc[6], cc[8]};
    const int istr2[4] = {0, cc[12], cc[14], cc[16]}, iend2[4] = {0, cc[13], cc[15], cc[17]};
    const int iord[4] = {0, cc[18], cc[19], cc[20]};
    int ibcpt, ibcinc, inr, inrinc;
    if (inout1 == 1) { ibcpt = 0; ibcinc = -1; } else { ibcpt = ijk1[idir1]; ibcinc = 1; }
    if (inout2 == 1) { inr = 1; inrinc = 1; } else { inr = ijk2[idir2] - 1; inrinc = -1; }
    int len[4], isgn1[4], isgn2[4];
    for (int l = 1; l <= 3; ++l) {
      len[l] = std::abs(iend1[l] - istr1[l]);
      isgn1[l] = iend1[l] > istr1[l] ? 1 : -1;
      isgn2[l] = iend2[l] > istr2[l] ? 1 : -1;
    }
    const int ic1 = cyc3(idir1, 1), ic2 = cyc3(idir1, 2), ic3 = cyc3(idir1, 3);
    const int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
    for (int i3 = 0; i3 <= len[ic3]; ++i3)
      for (int i2 = 0; i2 <= len[ic2]; ++i2) {
        int p1[4] = {0, 0, 0, 0}, p2[4] = {0, 0, 0, 0};
        p1[ic1] = ibcpt; p1[ic2] = istr1[ic2] + isgn1[ic2] * i2; p1[ic3] = istr1[ic3] + isgn1[ic3] * i3;
        p2[jc1] = inr; p2[jc2] = istr2[jc2] + isgn2[jc2] * i2; p2[jc3] = istr2[jc3] + isgn2[jc3] * i3;
        HaloItem it{};
        it.dblk = b1; it.sblk = b2; it.type = -1; it.idir = idir1; it.mask = 3; it.sgn = 1;
        it.h1 = p3_cell(x1, p1[1], p1[2], p1[3]);
        p1[ic1] += ibcinc;
        it.h2 = p3_cell(x1, p1[1], p1[2], p1[3]);
        it.c1 = p3_cell(x2, p2[1], p2[2], p2[3]);
        p2[jc1] += inrinc;
        it.c2 = p3_cell(x2, p2[1], p2[2], p2[3]);
        it.mface = 0;
        L.items.push_back(it);
      }
  }
  if (bps)
    for (HaloItem &it : L.items) it.ps = bps[it.dblk];
  for (HaloItem &it : L.items) it.nl = L.nl;
  // last writer of every halo cell keeps its write (reference order)
  {
    std::unordered_map<int64_t, int64_t> owner;
    owner.reserve(L.items.size() * 2);
    for (size_t t = 0; t < L.items.size(); ++t) {
      const HaloItem &it = L.items[t];
      const int64_t base = L.hb[it.dblk].op3;
      owner[base + it.h1] = (int64_t)t * 2;
      owner[base + it.h2] = (int64_t)t * 2 + 1;
    }
    for (size_t t = 0; t < L.items.size(); ++t) {
      HaloItem &it = L.items[t];
      const int64_t base = L.hb[it.dblk].op3;
      int m = 0;
      if (owner[base + it.h1] == (int64_t)t * 2) m |= 1;
      if (owner[base + it.h2] == (int64_t)t * 2 + 1) m |= 2;
      it.mask = m;
    }
  }
  // ---- strong-boundary flags (muscl_b*, src/flux.f90:1318-1349, 1376-1406)
  std::vector<uint8_t> flags;
  std::vector<StrongMap> smap(L.nb);
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    const int nc[4] = {0, x.im - 1, x.jm - 1, x.km - 1};
    StrongMap &m = smap[b];
    for (int d = 1; d <= 3; ++d) {
      const int t2d = d == 1 ? 2 : 1, t3d = d == 3 ? 2 : 3;
      m.n2[d - 1] = nc[t2d];
      for (int side = 0; side < 2; ++side) {
        m.off[d - 1][side] = -1;
        for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
          const int *r = L.bct.data() + L.obct[b] + 10 * ibc;
          if (r[1] != d || !((r[0] == 13 || r[0] == 14 || r[0] / 100 == 15 || r[0] == 22 || r[0] == 23 ||
                               r[0] == 92 || r[0] == 93 || r[0] == 5)))
            continue;
          if ((r[2] == 1) != (side == 0)) continue;
          if (m.off[d - 1][side] < 0) {
            m.off[d - 1][side] = (int64_t)flags.size();
            flags.resize(flags.size() + (size_t)nc[t2d] * nc[t3d], 0);
          }
          const int lo[4] = {0, r[3], r[5], r[7]}, hi[4] = {0, r[4], r[6], r[8]};
          for (int t3 = std::max(1, lo[t3d]); t3 <= std::min(nc[t3d], hi[t3d]); ++t3)
            for (int t2 = std::max(1, lo[t2d]); t2 <= std::min(nc[t2d], hi[t2d]); ++t2)
              flags[(size_t)(m.off[d - 1][side] + (t2 - 1) + (int64_t)nc[t2d] * (t3 - 1))] = 1;
        }
      }
    }
  }
  // ---- strong-boundary faces of q_face / q_der (src/flux.f90:1884-1962, 2075-2143,
  // 2256-2324, 2466-2488): patches in table order, a later patch's values
  // replacing an earlier one's on a shared face
  L.walls.clear();
  {
    std::unordered_map<int64_t, size_t> wpos;
    for (int b = 0; b < L.nb; ++b) {
      const DevBlock &x = L.hb[b];
      const int ijk[4] = {0, x.im, x.jm, x.km};
      for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
        const int *r = L.bct.data() + L.obct[b] + 10 * ibc;
        if (!((r[0] == 13 || r[0] == 14 || r[0] / 100 == 15 || r[0] == 22 || r[0] == 23 || r[0] == 92 ||
               r[0] == 93 || r[0] == 5)))
          continue;
        const int d = r[1], inrout = r[2];
        const int lo[4] = {0, r[3], r[5], r[7]}, hi[4] = {0, r[4], r[6], r[8]};
        const int ic2 = cyc3(d, 2), ic3 = cyc3(d, 3);
        for (int l = 1; l <= 3; ++l)
          if (l != d && (lo[l] < 1 || hi[l] > ijk[l] - 1 || lo[l] > hi[l])) return COSA_ERR_ARG;
        if (ijk[d] < 3) return COSA_ERR_ARG;
        const int iface = inrout == 1 ? 1 : ijk[d];
        for (int i3 = lo[ic3]; i3 <= hi[ic3]; ++i3)
          for (int i2 = lo[ic2]; i2 <= hi[ic2]; ++i2) {
            WallFace w{};
            w.blk = b; w.d = d; w.inrout = inrout;
            int pp[4] = {0, 0, 0, 0};
            pp[d] = iface; pp[ic2] = i2; pp[ic3] = i3;
            w.fi = pp[1]; w.fj = pp[2]; w.fk = pp[3];
            for (int l = 1; l <= 3; ++l) { w.lo[l - 1] = lo[l]; w.hi[l - 1] = hi[l]; }
            const int64_t key = (((int64_t)b * 4 + d) << 40) +
                                (w.fi + (int64_t)(x.im + 1) * (w.fj + (int64_t)(x.jm + 1) * w.fk));
            auto f = wpos.find(key);
            if (f != wpos.end()) L.walls[f->second] = w;
            else { wpos[key] = L.walls.size(); L.walls.push_back(w); }
          }
      }
    }
  }
  // ---- cut_x / cut_v copy lists (src/grid.f90:242-523, 612-700), last writer kept
  std::vector<CopyItem> cutx, cutv;
  {
    std::unordered_map<int64_t, size_t> px, pv;
    auto put = [](std::vector<CopyItem> &v, std::unordered_map<int64_t, size_t> &pos, CopyItem it) {
      auto f = pos.find(it.dst);
      if (f != pos.end()) v[f->second] = it;
      else { pos[it.dst] = v.size(); v.push_back(it); }
    };
    for (int ic = 0; ic < L.ncuts; ++ic) {
      const int *cc = L.cut.data() + 21 * (int64_t)ic;
      const int b1 = cc[0] - 1, b2 = cc[9] - 1;
      const DevBlock &x1 = L.hb[b1], &x2 = L.hb[b2];
      const int ijk1[4] = {0, x1.im, x1.jm, x1.km}, ijk2[4] = {0, x2.im, x2.jm, x2.km};
      const int idir1 = cc[1], inout1 = cc[2], idir2 = cc[10], inout2 = cc[11];
      const int iord[4] = {0, cc[18], cc[19], cc[20]};
      const int ic1 = cyc3(idir1, 1), ic2 = cyc3(idir1, 2), ic3 = cyc3(idir1, 3);
      const int jc1 = iord[ic1], jc2 = iord[ic2], jc3 = iord[ic3];
      if (jc1 < 1 || jc1 > 3 || jc2 < 1 || jc2 > 3 || jc3 < 1 || jc3 > 3) return COSA_ERR_ARG;
      for (int pass = 0; pass < 2; ++pass) {  // 0: nodes (cut_x), 1: volumes (cut_v)
        int s1[4] = {0, cc[3], cc[5], cc[7]}, e1[4] = {0, cc[4], cc[6], cc[8]};
        int s2[4] = {0, cc[12], cc[14], cc[16]}, e2[4] = {0, cc[13], cc[15], cc[17]};
        int ibcpt, inr;
        if (pass == 0) {
          ibcpt = inout1 == 1 ? 0 : ijk1[idir1] + 1;
          inr = inout2 == 1 ? 2 : ijk2[idir2] - 1;
          for (int l = 1; l <= 3; ++l)
            if (l != idir1) { if (e1[l] > s1[l]) e1[l] += 1; else s1[l] += 1; }
          for (int l = 1; l <= 3; ++l)
            if (l != idir2) { if (e2[l] > s2[l]) e2[l] += 1; else s2[l] += 1; }
        } else {
          ibcpt = inout1 == 1 ? 0 : ijk1[idir1];
          inr = inout2 == 1 ? 1 : ijk2[idir2] - 1;
        }
        int len[4], g1[4], g2[4];
        for (int l = 1; l <= 3; ++l) {
          len[l] = std::abs(e1[l] - s1[l]);
          g1[l] = e1[l] > s1[l] ? 1 : -1;
          g2[l] = e2[l] > s2[l] ? 1 : -1;
        }
        const int top = pass == 0 ? 1 : 0;  // nodes 0..ijk+1, volumes 0..ijk
        for (int i3 = 0; i3 <= len[ic3]; ++i3)
          for (int i2 = 0; i2 <= len[ic2]; ++i2) {
            int p1[4] = {0, 0, 0, 0}, p2[4] = {0, 0, 0, 0};
            p1[ic1] = ibcpt; p1[ic2] = s1[ic2] + g1[ic2] * i2; p1[ic3] = s1[ic3] + g1[ic3] * i3;
            p2[jc1] = inr; p2[jc2] = s2[jc2] + g2[jc2] * i2; p2[jc3] = s2[jc3] + g2[jc3] * i3;
            for (int l = 1; l <= 3; ++l)
              if (p1[l] < 0 || p1[l] > ijk1[l] + top || p2[l] < 0 || p2[l] > ijk2[l] + top) return COSA_ERR_ARG;
            if (pass == 0)
              put(cutx, px, CopyItem{g2_idx(x1, p1[1], p1[2], p1[3]), g2_idx(x2, p2[1], p2[2], p2[3])});
            else
              put(cutv, pv, CopyItem{p1_idx(x1, 1, p1[1], p1[2], p1[3], 0), p1_idx(x2, 1, p2[1], p2[2], p2[3], 0)});
          }
      }
    }
  }
  L.ncutx = (int)cutx.size();
  L.ncutv = (int)cutv.size();
  // moving grids: the node copies of every snapshot (node arrays of S2
  // snapshots per block at op2 * S2, snapshot nh at nh * (im+2)(jm+2)(km+2))
  const int S2m = c->p.moving ? 2 * c->p.nharms * c->p.hbmove + 1 : 1;
  if (S2m > 1) {
    std::vector<std::pair<int64_t, int64_t>> base(L.nb);  // (op2, nodes per snapshot)
    for (int b = 0; b < L.nb; ++b)
      base[b] = {L.hb[b].op2, (int64_t)(L.hb[b].im + 2) * (L.hb[b].jm + 2) * (L.hb[b].km + 2)};
    auto shift = [&](int64_t g, int nh) {
      int b = L.nb - 1;
      while (b > 0 && base[b].first > g) --b;
      return g + base[b].first * (S2m - 1) + nh * base[b].second;
    };
    std::vector<CopyItem> all;
    all.reserve(cutx.size() * S2m);
    for (int nh = 0; nh < S2m; ++nh)
      for (const CopyItem &it : cutx) all.push_back(CopyItem{shift(it.dst, nh), shift(it.src, nh)});
    cutx.swap(all);
    L.ncutx = (int)cutx.size();
  }

  // ---- tiles of the fused stage kernel
  std::vector<Tile> tiles;
  const int S = 2 * c->p.nharms + 1;
  const int kc = 32;
  L.kchunk = kc;
  // snapshots innermost: the S tiles of one region run together, so the
  // harmonic-balance coupling re-reads the other snapshots from L2
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    for (int k0 = 1; k0 <= x.km - 1; k0 += kc)
      for (int j0 = 1; j0 <= x.jm - 1; j0 += kTJ)
        for (int i0 = 1; i0 <= x.im - 1; i0 += kTI)
          for (int n = 0; n < S; ++n)
            tiles.push_back(Tile{b, n, i0, j0, k0, std::min(k0 + kc - 1, x.km - 1)});
  }
  L.ntiles = (int)tiles.size();

  int r = 0;
  if ((r = dalloc(c, &L.d_blocks, L.hb.size()))) return r;
  if ((r = dalloc(c, &L.d_bct, std::max<size_t>(L.bct.size(), 1)))) return r;
  if ((r = dalloc(c, &L.d_items, std::max<size_t>(L.items.size(), 1)))) return r;
  if ((r = dalloc(c, &L.d_strong, std::max<size_t>(flags.size(), 1)))) return r;
  if ((r = dalloc(c, &L.d_smap, smap.size()))) return r;
  if ((r = dalloc(c, &L.d_tiles, std::max<size_t>(tiles.size(), 1)))) return r;
  CK(cudaMemcpy(L.d_blocks, L.hb.data(), L.hb.size() * sizeof(DevBlock), cudaMemcpyHostToDevice));
  if (!L.bct.empty()) CK(cudaMemcpy(L.d_bct, L.bct.data(), L.bct.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!L.items.empty())
    CK(cudaMemcpy(L.d_items, L.items.data(), L.items.size() * sizeof(HaloItem), cudaMemcpyHostToDevice));
  if (!flags.empty()) CK(cudaMemcpy(L.d_strong, flags.data(), flags.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(L.d_smap, smap.data(), smap.size() * sizeof(StrongMap), cudaMemcpyHostToDevice));
  if (!tiles.empty()) CK(cudaMemcpy(L.d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
  if ((r = dalloc(c, &L.d_walls, std::max<size_t>(L.walls.size(), 1)))) return r;
  if ((r = dalloc(c, &L.d_cutx, std::max<size_t>(cutx.size(), 1)))) return r;
  if ((r = dalloc(c, &L.d_cutv, std::max<size_t>(cutv.size(), 1)))) return r;
  if (!L.walls.empty())
    CK(cudaMemcpy(L.d_walls, L.walls.data(), L.walls.size() * sizeof(WallFace), cudaMemcpyHostToDevice));
  if (!cutx.empty()) CK(cudaMemcpy(L.d_cutx, cutx.data(), cutx.size() * sizeof(CopyItem), cudaMemcpyHostToDevice));
  if (!cutv.empty()) CK(cudaMemcpy(L.d_cutv, cutv.data(), cutv.size() * sizeof(CopyItem), cudaMemcpyHostToDevice));
  return COSA_OK;
}

LevelState *level(cosa_ctx *c, int nl) {
  if (!c || nl < 1 || nl > c->nlevels) return nullptr;
  return &c->L[nl - 1];
}

// face velocities of the bound level's moving grid (all null on fixed grids)
FaceVel face_vel_of(const cosa_ctx *c, const LevelState &L) {
  if (!c->p.moving) return FaceVel{{nullptr, nullptr, nullptr}};
  return FaceVel{{L.ptrs.fvi, L.ptrs.fvj, L.ptrs.fvk}};
}

int after_launch(cosa_ctx *c) {
  c->launches++;
  return cuda_ok(cudaGetLastError());
}

// CTAs along x for a multi-block launch over nb blocks of at most n items
int grid_x(int64_t n, int nb) {
  const int64_t g = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, std::max(148 * 16 / std::max(nb, 1), 148)));
}

// launch a per-block kernel once for all blocks of the level (grid y =
// block, x sized for the largest block); launch(BlockList, dim3 grid)
template <typename F>
int for_blocks(cosa_ctx *c, LevelState &L, int64_t (*count)(const DevBlock &, const cosa_params &), F launch) {
  int64_t m = 1;
  for (const DevBlock &b : L.hb) m = std::max<int64_t>(m, count(b, c->p));
  launch(BlockList{L.d_blocks}, dim3(grid_x(m, L.nb), L.nb));
  return after_launch(c);
}

// per snapshot: one item per node-indexed face (i,j,k <= imax,jmax,kmax) or per interior cell
int64_t cnt_faces(const DevBlock &b, const cosa_params &p) {
  return (int64_t)b.im * b.jm * b.km * (2 * p.nharms + 1);
}
int64_t cnt_cells(const DevBlock &b, const cosa_params &p) {
  return (int64_t)(b.im - 1) * (b.jm - 1) * (b.km - 1) * (2 * p.nharms + 1);
}
// halo edge cells of q_bedges, all variables
int64_t cnt_edges(const DevBlock &b, const cosa_params &p) {
  return 4 * ((int64_t)(b.im - 1) + (b.jm - 1) + (b.km - 1)) * (2 * p.nharms + 1) * p.npde;
}
int64_t cnt_interior(const DevBlock &b, const cosa_params &p) {
  return (int64_t)(b.im - 1) * (b.jm - 1) * (b.km - 1) * (2 * p.nharms + 1) * p.npde;
}
int64_t cnt_all(const DevBlock &b, const cosa_params &p) {
  return (int64_t)(b.im + 3) * (b.jm + 3) * (b.km + 3) * (2 * p.nharms + 1) * p.npde;
}

// once per process; contexts driven from several host threads (the serving
// engine's context lane) may reach it together
int set_smem_attrs() {
  static std::mutex mu;
  static bool done = false;
  std::lock_guard<std::mutex> lock(mu);
  if (done) return COSA_OK;
  const int smem = (int)stage_smem_bytes<kTI, kTJ>();
  CK(cudaFuncSetAttribute(k_stage_tile<kTI, kTJ, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(k_stage_tile<kTI, kTJ, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(k_stage_tile<kTI, kTJ, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(k_stage_tile<kTI, kTJ, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  done = true;
  return COSA_OK;
}

// the k-omega stage runs routine by routine (launch_rans_iteration); Wilcox,
// BSL and SST
int check_rans_supported(const cosa_params &p) {
  if (p.npde != 7 || !rans(p) || (p.kom + p.kom_bsl + p.kom_sst) != 1 || !p.viscous ||
      (p.rkimp && !p.dualt && !p.harbal) || (p.dualt && (p.dt <= 0 || p.harbal)) ||
      p.irsop < 0 || p.irsop > 6 || p.irsop == 4 || p.lmet != 4 || p.ilimf < 0 || p.ilimf > 4)
    return COSA_ERR_UNSUPPORTED;
  // moving grids: harmonic balance of a pitching body, explicit stages on one
  // level
  if (p.moving && (!p.harbal || !p.hbmove || p.rkimp || p.nlevel > 1)) return COSA_ERR_UNSUPPORTED;
  return COSA_OK;
}

// low-speed preconditioning: Euler or laminar flow, explicit stages, fixed
// grids (update_lsp_b's k-omega and implicit branches and the moving-frame
// preconditioner are not built); IRS 5 and 6 are refused by the reference
int check_lsp_supported(const cosa_params &p) {
  if (p.npde != 5 || rans(p) || p.rkimp || p.moving || p.rgkuns || p.cutoff_type < 1 || p.cutoff_type > 3 ||
      (p.visprec && !p.viscous) || p.irsop < 0 || p.irsop > 3 || p.lmet != 4 || p.ilimf < 0 || p.ilimf > 4 ||
      p.nlevel < 1 || p.nlevel > COSA_MAX_LEVELS || (p.dualt && (p.harbal || p.dt <= 0)))
    return COSA_ERR_UNSUPPORTED;
  return COSA_OK;
}

int check_fused_supported(const cosa_params &p) {
  if (p.lomach) return check_lsp_supported(p);
  if (rans(p)) return check_rans_supported(p);
  // rkimp: the implicit time-spectral update of harmonic balance (update_bhb,
  // src/update.f90:1564-1604 without IRS on one level, 1771-1836 with IRS or
  // multigrid)
  if (p.rkimp && !p.harbal && !p.dualt) return COSA_ERR_UNSUPPORTED;
  // dual time: one snapshot, fixed grid, a physical time step
  if (p.dualt && (p.harbal || p.moving || p.dt <= 0)) return COSA_ERR_UNSUPPORTED;
  if (p.npde != 5 || p.kom || p.kom_bsl || p.kom_sst ||
      p.irsop < 0 || p.irsop > 6 || p.irsop == 4 || p.lmet != 4 || p.ilimf < 0 || p.ilimf > 4)
    return COSA_ERR_UNSUPPORTED;
  // moving grids: harmonic balance of a pitching body (inviscid or laminar),
  // explicit (the face-split stage schedule carries the face speeds)
  if (p.moving && (!p.harbal || !p.hbmove || p.rkimp || p.nlevel > 1)) return COSA_ERR_UNSUPPORTED;
  return COSA_OK;
}

// A block with a single cell along a direction: the reference's BCs on the
// faces normal to it read "interior cell 2", which is the opposite face's
// halo, still holding the previous stage's value in conservative form
// (src/bc.f90 bc_* with ibcn2, after prim2cons of src/cosa.f90:1908).  The
// fused halo kernel fills all faces at once from primitive data, so it
// matches the reference there only where that second cell is never used:
// first-order reconstruction on the level (the second halo layer unread)
// and BCs whose first halo layer depends on the first interior cell alone
// (80 symmetry, 4 extrapolation, 30 far field).
int check_thin_blocks(const cosa_ctx *c, int nl) {
  const LevelState &L = c->L[nl - 1];
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    const int nc[4] = {0, x.im - 1, x.jm - 1, x.km - 1};
    for (int d = 1; d <= 3; ++d) {
      if (nc[d] > 1) continue;
      // the viscous face stencils and q_edges read across such a block too
      if (c->p.viscous) return COSA_ERR_UNSUPPORTED;
      if (nl < c->p.nl_crs) return COSA_ERR_UNSUPPORTED;
      for (int ibc = 0; ibc < L.nbcs[b]; ++ibc) {
        const int *r = L.bct.data() + L.obct[b] + 10 * ibc;
        if (r[1] == d && r[0] != 80 && r[0] != 4 && r[0] != 30 && r[0] != 31) return COSA_ERR_UNSUPPORTED;
      }
    }
  }
  return COSA_OK;
}

int ensure_irs_scratch(cosa_ctx *c, LevelState &L) {
  const int S = 2 * c->p.nharms + 1;
  const size_t n = (size_t)L.n3 * c->p.npde * S;
  int r = 0;
  if (!L.d_irs_scr && (r = dalloc(c, &L.d_irs_scr, (size_t)L.n3 * S * 2))) return r;
  if (!L.d_res) {
    if ((r = dalloc(c, &L.d_res, n))) return r;
    CK(cudaMemset(L.d_res, 0, n * sizeof(double)));
  }
  if (!L.d_ores && (r = dalloc(c, &L.d_ores, n))) return r;
  for (auto &bt : L.d_beta)
    if (!bt && (r = dalloc(c, &bt, (size_t)L.n1 * S))) return r;
  return COSA_OK;
}

// lines of kPcrMinLen..kPcrMaxLen cells are solved by cyclic reduction in
// shared memory (at most kPcrSmemBytes per CTA, within the 48 KB default);
// shorter lines (a warp per line would idle) and longer ones by the Thomas
// sweeps, one thread per line
constexpr int kPcrSmemBytes = 48 * 1024;
constexpr int kPcrMaxLen = kPcrSmemBytes / 64;
constexpr int kPcrMinLen = 16;

// the three line sweeps of cirs_b / ccirs_b on `res` for variables vs..ve
int irs_sweeps(cosa_ctx *c, LevelState &L, double *res, const double *ores, const double *const beta[3], double eps,
               int vs, int ve, int with_halo) {
  // blocks are independent here (each sweep writes its own block's interior,
  // halos were filled before), so a direction can run for all blocks at once
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde, nv = ve - vs + 1;
  for (int d = 1; d <= 3; ++d) {
    const double *bt = beta ? beta[d - 1] : nullptr;
    const double *src = d == 1 ? ores : nullptr;
    auto len_of = [&](const DevBlock &x) { return d == 1 ? x.im - 1 : (d == 2 ? x.jm - 1 : x.km - 1); };
    auto lines_of = [&](const DevBlock &x) {
      return d == 1 ? (int64_t)(x.jm - 1) * (x.km - 1)
                    : (d == 2 ? (int64_t)(x.im - 1) * (x.km - 1) : (int64_t)(x.im - 1) * (x.jm - 1));
    };
    bool all_pcr = true;
    int nmax = 1;
    int64_t wmax = 1;
    for (const DevBlock &x : L.hb) {
      const int len = len_of(x);
      all_pcr &= len >= kPcrMinLen && len <= kPcrMaxLen;
      nmax = std::max(nmax, len);
      wmax = std::max<int64_t>(wmax, lines_of(x) * S * nv);
    }
    if (all_pcr) {
      // parallel cyclic reduction, one warp per line and variable, all blocks
      const int wpc = std::max(1, std::min(4, kPcrSmemBytes / (64 * nmax)));
      const dim3 g((unsigned)grid_x(wmax * 32, L.nb) * 256 / (32 * wpc) + 1, L.nb);
      const size_t sm = (size_t)wpc * 8 * nmax * sizeof(double);
      const BlockList bl{L.d_blocks};
      if (d == 1) k_irs_pcr<1><<<g, 32 * wpc, sm, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, nmax);
      else if (d == 2) k_irs_pcr<2><<<g, 32 * wpc, sm, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, nmax);
      else k_irs_pcr<3><<<g, 32 * wpc, sm, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, nmax);
      const int r = after_launch(c);
      if (r) return r;
      continue;
    }
    bool all_thomas = true;
    for (const DevBlock &x : L.hb) all_thomas &= !(len_of(x) >= kPcrMinLen && len_of(x) <= kPcrMaxLen);
    if (all_thomas) {
      // Thomas sweeps, one thread per line, all blocks in one launch
      int64_t lmax = 1;
      for (const DevBlock &x : L.hb) lmax = std::max<int64_t>(lmax, lines_of(x) * S);
      const dim3 g(grid_x(lmax, L.nb) * 2, L.nb);  // 128-thread CTAs
      const BlockList bl{L.d_blocks};
      if (d == 1) k_irs_line<1><<<g, 128, 0, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
      else if (d == 2) k_irs_line<2><<<g, 128, 0, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
      else k_irs_line<3><<<g, 128, 0, c->s>>>(bl, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
      const int r = after_launch(c);
      if (r) return r;
      continue;
    }
    for (const DevBlock &x : L.hb) {
      const int len = len_of(x);
      const int64_t nl = lines_of(x);
      if (len >= kPcrMinLen && len <= kPcrMaxLen) {
        const int nm = std::max(len, 1);
        const int wpc = std::max(1, std::min(4, kPcrSmemBytes / (64 * nm)));
        const int g = grid_for(nl * S * nv * 32, 32 * wpc);  // one warp per line and variable
        const size_t sm = (size_t)wpc * 8 * nm * sizeof(double);
        if (d == 1) k_irs_pcr<1><<<g, 32 * wpc, sm, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, nm);
        else if (d == 2) k_irs_pcr<2><<<g, 32 * wpc, sm, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, nm);
        else k_irs_pcr<3><<<g, 32 * wpc, sm, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, nm);
      } else {
        const int g = grid_for(nl * S, 128);
        if (d == 1) k_irs_line<1><<<g, 128, 0, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
        else if (d == 2) k_irs_line<2><<<g, 128, 0, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
        else k_irs_line<3><<<g, 128, 0, c->s>>>(x, npde, S, res, src, bt, eps, vs, ve, with_halo, L.d_irs_scr);
      }
      const int r = after_launch(c);
      if (r) return r;
    }
  }
  return COSA_OK;
}

int irs_scale(cosa_ctx *c, LevelState &L, double *res, const double *dtv, const double *dtvt, int forward) {
  const int S = 2 * c->p.nharms + 1;
  return for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
    k_irs_scale<<<g, 256, 0, c->s>>>(b, c->p.npde, S, res, dtv, dtvt, forward);
  });
}

// cirs (cutcirs = 0) or scalef + 2 x (cutman_q + ccirs) + scaleb (cutcirs = 1)
// of smooth() (src/cosa.f90:1977-1998) for the mean-flow equations
// k-omega (npde 7): dtvt scales the turbulence equations and their sweeps
// use tbeta (irsop >= 2) or the constant coefficient (irsop 1)
int irs_apply(cosa_ctx *c, LevelState &L, double *res, double *ores, const double *dtv, const double *const beta[3],
              const double *dtvt = nullptr, const double *const tbeta[3] = nullptr) {
  const cosa_params &p = c->p;
  const double eps = 0.25 * (p.rat * p.rat - 1.0);
  const bool const_eps = p.irsop == 1;
  const bool kom = p.npde > 5;
  const int S = 2 * p.nharms + 1;
  auto sweeps = [&](const double *src, int with_halo) -> int {
    if (const_eps) return irs_sweeps(c, L, res, src, nullptr, eps, 1, p.npde, with_halo);
    int r2 = irs_sweeps(c, L, res, src, beta, eps, 1, 5, with_halo);
    if (!r2 && kom) r2 = irs_sweeps(c, L, res, src, tbeta, 0.0, 6, p.npde, with_halo);
    return r2;
  };
  int r = irs_scale(c, L, res, dtv, kom ? dtvt : nullptr, 1);
  if (r) return r;
  if (p.cutcirs == 0) {
    if ((r = sweeps(nullptr, 0))) return r;
  } else {
    CK(cudaMemcpyAsync(ores, res, (size_t)L.n3 * p.npde * S * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
    const int ncut = (int)L.items.size() - L.n_bc_items;
    for (int its = 0; its < 2; ++its) {
      if (ncut > 0) {
        k_halo<false><<<grid_for((int64_t)ncut * S), 256, 0, c->s>>>(L.d_blocks, L.d_items + L.n_bc_items, ncut, c->d_p,
                                                                    res, nullptr, nullptr, nullptr, c->d_status);
        if ((r = after_launch(c))) return r;
      }
      if ((r = sweeps(ores, 1))) return r;
    }
  }
  return irs_scale(c, L, res, dtv, kom ? dtvt : nullptr, 0);
}

// profiling: close the event pair of kernel class `k` and accumulate its time
void prof_stop(cosa_ctx *c, int k) {
  cudaEventRecord(c->prof.ev[k][1], c->s);
  cudaEventSynchronize(c->prof.ev[k][1]);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->prof.ev[k][0], c->prof.ev[k][1]);
  c->prof.ms[k] += ms;
  c->prof.n[k] += 1;
}

int launch_edges(cosa_ctx *c, LevelState &L, double *q, double *mut);

// x extent of a (x, nblocks[, 3]) grid covering `n` items per block
// viscous part of one stage on the halo-filled state qin: primitive copy,
// q_edges, [time step], face fluxes, wall faces, flux balance -> L.d_vres
int launch_visc(cosa_ctx *c, LevelState &L, const double *qin, bool dt, double *bx, double *by, double *bz,
                bool have_prim = false) {
  const cosa_params &p = c->p;
  const int S = 2 * p.nharms + 1;
  int64_t m3 = 0, mc = 0, mf = 0;
  for (const DevBlock &x : L.hb) {
    m3 = std::max<int64_t>(m3, x.P3 * S);
    mc = std::max<int64_t>(mc, (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1) * S);
    mf = std::max<int64_t>(mf, (int64_t)x.im * x.jm * x.km * S);
  }
  int r = 0;
  if (!have_prim) {
    k_prim<<<dim3(grid_x(m3, L.nb), L.nb), 256, 0, c->s>>>(L.d_blocks, c->d_p, qin, L.d_qprim);
    if ((r = after_launch(c))) return r;
  }
  if ((r = launch_edges(c, L, L.d_qprim, nullptr))) return r;
  const cosa_level_ptrs &P = L.ptrs;
  if (dt) {
    const bool mv = c->p.moving;
    k_dt_ns<<<dim3(grid_x(mc, L.nb), L.nb), 256, 0, c->s>>>(L.d_blocks, c->d_p, L.d_qprim, P.si, P.sj, P.sk, P.vol,
                                                            P.dtvol, bx, by, bz, mv ? P.xdot : nullptr,
                                                            mv ? P.ydot : nullptr, mv ? P.zdot : nullptr);
    if ((r = after_launch(c))) return r;
  }
  k_vface<<<dim3(grid_x(mf, L.nb), L.nb, 3), 256, 0, c->s>>>(L.d_blocks, c->d_p, L.d_qprim, P.si, P.sj, P.sk, L.d_vm,
                                                             L.n0, L.d_vflux);
  if ((r = after_launch(c))) return r;
  if (!L.walls.empty()) {
    const int nw = (int)L.walls.size();
    k_vwall<<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L.d_blocks, L.d_walls, nw, c->d_p, L.d_qprim, P.si, P.sj,
                                                         P.sk, L.d_vm, L.n0, L.d_vflux);
    if ((r = after_launch(c))) return r;
  }
  k_vdiv<<<dim3(grid_x(mc, L.nb), L.nb), 256, 0, c->s>>>(L.d_blocks, c->d_p, L.d_vflux, L.n0, L.d_vres);
  return after_launch(c);
}

constexpr int kCellsGX = 64;  // CTAs per block of k_cells (fixed: deterministic norm partials)

// split schedule after the halo fill (and, for viscous flows, the primitive
// copy): face fluxes, cell epilogue, norm reduction.  qsrc is the stage input
// (conv: interior cells converted on load) or the primitive copy.
int launch_split_tail(cosa_ctx *c, int nl, LevelState &L, StageArgs &A, bool want_rms, const double *qsrc,
                      bool conv) {
  const cosa_params &p = c->p;
  const int S = 2 * p.nharms + 1;
  const bool mixed = p.precision == COSA_PREC_MIXED;
  int r = 0;
  if (A.compute_dt) {
    int64_t mc = 0;
    for (const DevBlock &x : L.hb) mc = std::max<int64_t>(mc, (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1) * S);
    const dim3 g(grid_x(mc, L.nb), L.nb);
    const CellVel cv = p.moving ? CellVel{{L.ptrs.xdot, L.ptrs.ydot, L.ptrs.zdot}} : CellVel{{nullptr, nullptr, nullptr}};
    if (conv)
      k_dt_euler<true><<<g, 256, 0, c->s>>>(L.d_blocks, c->d_p, qsrc, A.si, A.sj, A.sk, A.dtvol, A.bx, A.by, A.bz,
                                            cv);
    else
      k_dt_euler<false><<<g, 256, 0, c->s>>>(L.d_blocks, c->d_p, qsrc, A.si, A.sj, A.sk, A.dtvol, A.bx, A.by, A.bz,
                                             cv);
    if ((r = after_launch(c))) return r;
  }
  A.part = want_rms ? L.d_part : nullptr;
  // i-face tasks, then the marching j- and k-face tasks
  auto faces = [&](int b0, int nb, cudaStream_t st) {
    (void)b0; (void)nb;
    const FaceTask *tk[2] = {L.d_ftasks, L.d_ftasks + L.nftasks1};
    const LinePar lp = make_line_par(p);
    const int nt[2] = {L.nftasks1, L.nftasks - L.nftasks1};
#define COSA_FACES_LINE(M, CV, IF)                                                                               \
  k_faces_line<M, CV, IF><<<(nt[IF ? 0 : 1] + 3) / 4, 128, 0, st>>>(                                           \
      L.d_blocks, tk[IF ? 0 : 1], nt[IF ? 0 : 1], lp, qsrc, A.si, A.sj, A.sk, L.d_strong, L.d_smap,              \
      A.first_order, L.n0, L.d_cflux, c->d_status)
#define COSA_FACES_MOVING(M, CV, IF)                                                                            \
  k_faces_line<M, CV, IF, true><<<(nt[IF ? 0 : 1] + 3) / 4, 128, 0, st>>>(                                     \
      L.d_blocks, tk[IF ? 0 : 1], nt[IF ? 0 : 1], lp, qsrc, A.si, A.sj, A.sk, L.d_strong, L.d_smap,              \
      A.first_order, L.n0, L.d_cflux, c->d_status, fvel)
    const FaceVel fvel = face_vel_of(c, L);
    // moving grids: the face speeds; viscous runs read the primitive copy (CV false)
    if (p.moving && conv && mixed) { COSA_FACES_MOVING(true, true, true); COSA_FACES_MOVING(true, true, false); }
    else if (p.moving && conv) { COSA_FACES_MOVING(false, true, true); COSA_FACES_MOVING(false, true, false); }
    else if (p.moving && mixed) { COSA_FACES_MOVING(true, false, true); COSA_FACES_MOVING(true, false, false); }
    else if (p.moving) { COSA_FACES_MOVING(false, false, true); COSA_FACES_MOVING(false, false, false); }
    else if (mixed && conv) { COSA_FACES_LINE(true, true, true); COSA_FACES_LINE(true, true, false); }
    else if (mixed) { COSA_FACES_LINE(true, false, true); COSA_FACES_LINE(true, false, false); }
    else if (conv) { COSA_FACES_LINE(false, true, true); COSA_FACES_LINE(false, true, false); }
    else { COSA_FACES_LINE(false, false, true); COSA_FACES_LINE(false, false, false); }
#undef COSA_FACES_LINE
#undef COSA_FACES_MOVING
  };
  auto cells = [&](int b0, int nb, cudaStream_t st) {
    const dim3 gc(kCellsGX, nb);
    if (want_rms) k_cells<true><<<gc, 256, 0, st>>>(L.d_blocks, c->d_p, A, L.d_cflux, L.n0, b0);
    else k_cells<false><<<gc, 256, 0, st>>>(L.d_blocks, c->d_p, A, L.d_cflux, L.n0, b0);
  };
  // one launch per kernel over all blocks: per-block launches on two streams
  // (cell pass of block b beside the faces of block b+1) measured slower, the
  // small blocks underfill the GPU
  if (c->prof.on) cudaEventRecord(c->prof.ev[1][0], c->s);
  faces(0, L.nb, c->s);
  if ((r = after_launch(c))) return r;
  if (c->prof.on) {
    prof_stop(c, 1);
    cudaEventRecord(c->prof.ev[2][0], c->s);
  }
  cells(0, L.nb, c->s);
  if ((r = after_launch(c))) return r;
  if (c->prof.on) prof_stop(c, 2);
  if (want_rms) {
    int64_t ncell = 0;
    for (auto &b : L.hb) ncell += (int64_t)(b.im - 1) * (b.jm - 1) * (b.km - 1);
    const double cnt = (double)ncell * (p.harbal ? S : 1);
    k_rms_final<<<1, 256, 0, c->s>>>(L.d_part, L.nb * kCellsGX, p.npde, cnt, c->d_hist, c->d_row, c->hist_cap);
    if ((r = after_launch(c))) return r;
  }
  (void)nl;
  return COSA_OK;
}

// one stage: halo fill + tile kernel (+ norm reduction)
int launch_stage(cosa_ctx *c, int nl, LevelState &L, double *qin, double *qout, const double *qold,
                 double *qold_copy, int irk, int compute_dt, bool want_rms, int update, double *res_out,
                 double *rhs = nullptr, int rhs_mode = 0) {
  const cosa_params &p = c->p;
  const int S = 2 * p.nharms + 1;
  const cosa_level_ptrs &P = L.ptrs;
  if (!L.items.empty()) {
    const int64_t n = (int64_t)L.items.size() * S;
    if (c->prof.on) cudaEventRecord(c->prof.ev[0][0], c->s);
    k_halo<true><<<grid_for(n), 256, 0, c->s>>>(L.d_blocks, L.d_items, (int)L.items.size(),
                                                c->d_halo_p ? c->d_halo_p : c->d_p, qin, P.si, P.sj, P.sk,
                                                c->d_status, nullptr, face_vel_of(c, L));
    int r = after_launch(c);
    if (r) return r;
    if (c->prof.on) prof_stop(c, 0);
  }
  StageArgs A{};
  A.qin = qin; A.qout = qout; A.qold = qold; A.qold_copy = qold_copy;
  A.dtvol = P.dtvol; A.si = P.si; A.sj = P.sj; A.sk = P.sk;
  A.part = want_rms ? L.d_part : nullptr;
  A.rhs = rhs;
  A.rhs_mode = rhs ? rhs_mode : 0;
  A.res_out = res_out;
  if (compute_dt && p.irsop >= 2) {
    A.bx = P.betaxi ? P.betaxi : L.d_beta[0];
    A.by = P.betaeta ? P.betaeta : L.d_beta[1];
    A.bz = P.betazeta ? P.betazeta : L.d_beta[2];
  }
  A.strong = L.d_strong; A.smap = L.d_smap; A.status = c->d_status;
  A.ar = p.alphas[irk - 1];
  // src_hb adds the time-spectral term to the residual except under rkimp
  // without IRS on one level, where update_bhb takes it alone
  // (src/cosa.f90:1918-1922)
  A.vol = p.harbal && (!p.rkimp || p.irsop > 0 || p.nlevel > 1) ? P.vol : nullptr;
  A.compute_dt = compute_dt;
  A.first_order = nl >= p.nl_crs;
  A.update = update;
  A.cfl_blk = c->d_cfl_blk;
  const bool split =
      L.schedule == 1 && c->nseg == 0 && L.d_cflux && (L.d_qprim || !p.viscous) && L.d_ftasks && !p.rkimp;
  if (split && p.viscous) {
    // primitive copy (with bprtest) shared by the viscous and convective faces
    int64_t m3 = 0;
    for (const DevBlock &x : L.hb) m3 = std::max<int64_t>(m3, x.P3 * S);
    k_prim<<<dim3(grid_x(m3, L.nb), L.nb), 256, 0, c->s>>>(L.d_blocks, c->d_p, qin, L.d_qprim, c->d_status);
    int r = after_launch(c);
    if (r) return r;
  }
  if (p.viscous) {
    // the viscous terms and, on stage 1, the viscous time step come first
    if (!L.d_vm || !L.d_vres || !P.vol) return COSA_ERR_ARG;
    int r = launch_visc(c, L, qin, compute_dt != 0, A.bx, A.by, A.bz, split);
    if (r) return r;
    A.vres = L.d_vres;
    A.compute_dt = 0;
    A.bx = A.by = A.bz = nullptr;
  }
  if (split) return launch_split_tail(c, nl, L, A, want_rms, p.viscous ? L.d_qprim : qin, !p.viscous);
  if (p.moving) return COSA_ERR_UNSUPPORTED;  // the tile kernel has no face speeds
  const size_t smem = stage_smem_bytes<kTI, kTJ>();
  if (c->prof.on) cudaEventRecord(c->prof.ev[1][0], c->s);
  // the residual-norm partials are a separate instantiation: their
  // accumulators would otherwise hold registers in every launch
  const int nthr = stage_threads<kTI, kTJ>();
  const bool mixed = p.precision == COSA_PREC_MIXED;
  if (mixed && want_rms)
    k_stage_tile<kTI, kTJ, true, true><<<L.ntiles, nthr, smem, c->s>>>(L.d_blocks, L.d_tiles, c->d_p, A);
  else if (mixed)
    k_stage_tile<kTI, kTJ, true, false><<<L.ntiles, nthr, smem, c->s>>>(L.d_blocks, L.d_tiles, c->d_p, A);
  else if (want_rms)
    k_stage_tile<kTI, kTJ, false, true><<<L.ntiles, nthr, smem, c->s>>>(L.d_blocks, L.d_tiles, c->d_p, A);
  else
    k_stage_tile<kTI, kTJ, false, false><<<L.ntiles, nthr, smem, c->s>>>(L.d_blocks, L.d_tiles, c->d_p, A);
  int r = after_launch(c);
  if (r) return r;
  if (c->prof.on) prof_stop(c, 1);
  if (want_rms && c->nseg > 0) {
    k_rms_seg<<<c->nseg, 256, 0, c->s>>>(L.d_part, c->d_seg, c->d_seg_ncell, p.npde, c->d_hist);
    r = after_launch(c);
    if (r) return r;
  } else if (want_rms) {
    int64_t ncell = 0;
    for (auto &b : L.hb) ncell += (int64_t)(b.im - 1) * (b.jm - 1) * (b.km - 1);
    // resg_rms_hb averages over the snapshots as well (src/cosa.f90:4620-4626)
    const double cnt = (double)ncell * (p.harbal ? (2 * p.nharms + 1) : 1);
    k_rms_final<<<1, 256, 0, c->s>>>(L.d_part, L.ntiles, p.npde, cnt, c->d_hist, c->d_row, c->hist_cap);
    r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

// what one RK iteration of smooth() does besides the stages themselves
struct IterOpts {
  bool want_rms = false;       // residual norm (fine level, printed cycle) at stage rms_stage
  int rms_stage = 1;           // 1 for smooth(); nstage for rkuns (the last stage's norm is kept)
  int compute_dt = 0;          // stage-1 local time step
  double *rhs = nullptr;       // coarse-level forcing: res -= rhs at every stage
  bool force = false;          // rhs += res at stage 1 (first iteration of a from_fine visit)
  bool copy_qold = true;       // qold = q at stage 1 (iter <= niter)
  double *res_only = nullptr;  // residual pass of to_coarse: stage-1 residual here, no update
  bool first_cycle = false;    // mgit == 1 (k-omega: coarse-level mut at the first visit)
  bool to_coarse = false;      // smooth()'s to_coarse (fine-level low-speed cut-offs)
};

int launch_rans_iteration(cosa_ctx *c, int nl, LevelState &L, const IterOpts &o);

// residual norm partials of every block (64 CTAs each) and the final sum;
// q_imp: the state whose implicit term is added back (dual time or harmonic
// balance with rkimp, no IRS, one level); harmonic balance averages over
// the snapshots
int launch_norm(cosa_ctx *c, LevelState &L, const double *res, const double *rhs, const double *q_imp) {
  int r = 0;
  int64_t ncell = 0;
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    double *part = L.d_part + (int64_t)b * 64 * 8;
    if (q_imp && c->p.harbal) k_rms_bhb_partial<<<64, 256, 0, c->s>>>(x, c->d_p, res, q_imp, L.ptrs.vol, part);
    else if (q_imp) k_rms_dualimp<<<64, 256, 0, c->s>>>(x, c->d_p, res, rhs, q_imp, L.ptrs.vol, part);
    else k_rms_partial<<<64, 256, 0, c->s>>>(x, c->d_p, res, rhs, part);
    if ((r = after_launch(c))) return r;
    ncell += (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1);
  }
  const double cnt = (double)ncell * (c->p.harbal ? 2 * c->p.nharms + 1 : 1);
  k_rms_final<<<1, 256, 0, c->s>>>(L.d_part, L.nb * 64, c->p.npde, cnt, c->d_hist, c->d_row, c->hist_cap);
  return after_launch(c);
}

// what follows the residual of a dual-time stage (src/cosa.f90:1908-1961):
// src_uns, the fine-level norm (printed cycles), res -= rhs_uns on the fine
// level, the multigrid forcing on coarse levels; q the stage state
int dual_tail(cosa_ctx *c, int nl, LevelState &L, const double *q, double *R, const IterOpts &o, int irk) {
  const cosa_params &p = c->p;
  const cosa_level_ptrs &P = L.ptrs;
  const int nvs = p.npde;
  int r = 0;
  if (dual_src_in_res(p) &&
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) { k_src_uns<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.vol, R); })))
    return r;
  if (nl == 1 && o.want_rms && irk == o.rms_stage &&
      (r = launch_norm(c, L, R, P.rhs, p.rkimp && !dual_src_in_res(p) ? q : nullptr)))
    return r;
  if (nl == 1 &&
      (r = for_blocks(c, L, cnt_interior, [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, R, P.rhs, -1.0); })))
    return r;
  if (o.rhs && o.force && irk == 1 &&
      (r = for_blocks(c, L, cnt_interior, [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, o.rhs, R, 1.0); })))
    return r;
  if (o.rhs &&
      (r = for_blocks(c, L, cnt_interior, [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, R, o.rhs, -1.0); })))
    return r;
  return COSA_OK;
}

// one RK iteration (nstage stages) of the fused path
int launch_iteration(cosa_ctx *c, int nl, LevelState &L, const IterOpts &o) {
  const cosa_params &p = c->p;
  if (routine_stage(p)) return launch_rans_iteration(c, nl, L, o);
  double *Q = L.ptrs.q, *T = L.d_T, *QO = L.ptrs.qold;
  const int S = 2 * p.nharms + 1;
  if (p.dualt) {
    // dual time: residual (no forcing, no update) -> dual_tail -> [IRS] ->
    // update_b, explicit or with the physical-time term implicit (rkimp)
    if (o.res_only) {
      int r = launch_stage(c, nl, L, Q, T, Q, nullptr, 1, o.compute_dt, false, 0, o.res_only);
      return r ? r : dual_tail(c, nl, L, Q, o.res_only, o, 1);
    }
    for (int irk = 1; irk <= p.nstage; ++irk) {
      double *qin = (irk % 2 == 1) ? Q : T;
      double *qout = (irk % 2 == 1) ? T : Q;
      const double *qold = irk == 1 ? Q : QO;
      double *qcopy = (irk == 1 && o.copy_qold) ? QO : nullptr;
      int r = launch_stage(c, nl, L, qin, qout, qold, nullptr, irk, o.compute_dt && irk == 1, false, 0, L.d_res);
      if (r || (r = dual_tail(c, nl, L, qin, L.d_res, o, irk))) return r;
      if (p.irsop > 0) {
        const double *beta[3] = {L.ptrs.betaxi ? L.ptrs.betaxi : L.d_beta[0],
                                 L.ptrs.betaeta ? L.ptrs.betaeta : L.d_beta[1],
                                 L.ptrs.betazeta ? L.ptrs.betazeta : L.d_beta[2]};
        if ((r = irs_apply(c, L, L.d_res, L.d_ores, L.ptrs.dtvol, beta))) return r;
      }
      const double ar = p.alphas[irk - 1];
      if (p.rkimp) {
        const int sir = dual_src_in_res(p) ? 1 : 0;
        r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
          k_update_dual<<<g, 256, 0, c->s>>>(b, c->d_p, L.d_res, qold, qin, qout, qcopy, L.ptrs.dtvol, L.ptrs.vol,
                                             ar, sir);
        });
      } else {
        for (int b = 0; b < L.nb && !r; ++b) {
          const DevBlock &x = L.hb[b];
          k_update_stage<<<grid_for((int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1)), 256, 0, c->s>>>(
              x, p.npde, 1, L.d_res, qold, qout, qcopy, L.ptrs.dtvol, ar);
          r = after_launch(c);
        }
      }
      if (r) return r;
    }
    if (p.nstage % 2 == 1)
      for (int b = 0; b < L.nb; ++b) {
        const DevBlock &x = L.hb[b];
        k_copy_interior<<<grid_for((int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1) * p.npde), 256, 0, c->s>>>(
            x, p.npde, T, Q);
        int r = after_launch(c);
        if (r) return r;
      }
    return COSA_OK;
  }
  if (o.res_only) {
    return launch_stage(c, nl, L, Q, T, Q, nullptr, 1, o.compute_dt, false, 0, o.res_only, o.rhs,
                        o.force ? 2 : 1);
  }
  for (int irk = 1; irk <= p.nstage; ++irk) {
    double *qin = (irk % 2 == 1) ? Q : T;
    double *qout = (irk % 2 == 1) ? T : Q;
    const double *qold = irk == 1 ? Q : QO;
    double *qcopy = (irk == 1 && o.copy_qold) ? QO : nullptr;
    const int rmode = (irk == 1 && o.force) ? 2 : 1;
    if (p.rkimp && (p.irsop > 0 || p.nlevel > 1)) {
      // residual with the time-spectral term -> [IRS] -> update_bhb, which
      // takes the unsmoothed term out again and solves for it implicitly
      int r = launch_stage(c, nl, L, qin, qout, qold, nullptr, irk, o.compute_dt && irk == 1, o.want_rms && irk == o.rms_stage,
                           0, L.d_res, o.rhs, rmode);
      if (r) return r;
      if (p.irsop > 0) {
        const double *beta[3] = {L.ptrs.betaxi ? L.ptrs.betaxi : L.d_beta[0],
                                 L.ptrs.betaeta ? L.ptrs.betaeta : L.d_beta[1],
                                 L.ptrs.betazeta ? L.ptrs.betazeta : L.d_beta[2]};
        if ((r = irs_apply(c, L, L.d_res, L.d_ores, L.ptrs.dtvol, beta))) return r;
      }
      const double *QOLD = qold, *QSRC = qin;
      r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
        k_update_bhb<<<g, 256, 0, c->s>>>(b, c->d_p, L.d_res, QOLD, qout, qcopy, L.ptrs.dtvol, L.ptrs.vol,
                                          p.alphas[irk - 1], QSRC);
      });
      if (r) return r;
      continue;
    }
    if (p.rkimp) {
      // residual without the time-spectral term -> [norm with it] -> the
      // per-cell snapshot solve of update_bhb
      int r = launch_stage(c, nl, L, qin, qout, qold, nullptr, irk, o.compute_dt && irk == 1, false, 0, L.d_res,
                           o.rhs, rmode);
      if (r) return r;
      if (o.want_rms && irk == o.rms_stage) {
        int64_t ncell = 0;
        for (int b = 0; b < L.nb; ++b) {
          const DevBlock &x = L.hb[b];
          k_rms_bhb_partial<<<64, 256, 0, c->s>>>(x, c->d_p, L.d_res, qin, L.ptrs.vol, L.d_part + (int64_t)b * 64 * 8);
          if ((r = after_launch(c))) return r;
          ncell += (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1);
        }
        k_rms_final<<<1, 256, 0, c->s>>>(L.d_part, L.nb * 64, p.npde, (double)ncell * S, c->d_hist, c->d_row,
                                         c->hist_cap);
        if ((r = after_launch(c))) return r;
      }
      const double *QOLD = qold;
      r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
        k_update_bhb<<<g, 256, 0, c->s>>>(b, c->d_p, L.d_res, QOLD, qout, qcopy, L.ptrs.dtvol, L.ptrs.vol,
                                          p.alphas[irk - 1], nullptr);
      });
      if (r) return r;
      continue;
    }
    if (p.irsop == 0) {
      int r = launch_stage(c, nl, L, qin, qout, qold, qcopy, irk, o.compute_dt && irk == 1, o.want_rms && irk == o.rms_stage, 1,
                           nullptr, o.rhs, rmode);
      if (r) return r;
    } else {
      // residual (no update) -> implicit smoothing -> update
      int r = launch_stage(c, nl, L, qin, qout, qold, nullptr, irk, o.compute_dt && irk == 1, o.want_rms && irk == o.rms_stage,
                           0, L.d_res, o.rhs, rmode);
      if (r) return r;
      const double *beta[3] = {L.ptrs.betaxi ? L.ptrs.betaxi : L.d_beta[0],
                               L.ptrs.betaeta ? L.ptrs.betaeta : L.d_beta[1],
                               L.ptrs.betazeta ? L.ptrs.betazeta : L.d_beta[2]};
      if ((r = irs_apply(c, L, L.d_res, L.d_ores, L.ptrs.dtvol, beta))) return r;
      for (int b = 0; b < L.nb; ++b) {
        const DevBlock &x = L.hb[b];
        k_update_stage<<<grid_for((int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1) * S), 256, 0, c->s>>>(
            x, p.npde, S, L.d_res, qold, qout, qcopy, L.ptrs.dtvol, p.alphas[irk - 1]);
        if ((r = after_launch(c))) return r;
      }
    }
  }
  if (p.nstage % 2 == 1) {
    // result landed in T: copy the interior back; Q keeps the last stage's
    // halo values for the finalisation of smooth()
    const int S = 2 * p.nharms + 1;
    for (int b = 0; b < L.nb; ++b) {
      const DevBlock &x = L.hb[b];
      k_copy_interior<<<grid_for((int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1) * p.npde * S), 256, 0, c->s>>>(
          x, p.npde * S, T, Q);
      int r = after_launch(c);
      if (r) return r;
    }
  }
  return COSA_OK;
}

void drop_graphs(cosa_ctx *c) {
  for (int l = 0; l < COSA_MAX_LEVELS; ++l)
    for (auto &g : c->L[l].graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto &kv : c->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  c->graphs.clear();
}

// replay the graph stored under `key`, capturing `issue` into it first if
// absent; the launch counter advances by the graph's kernel count
template <typename F>
int run_graph(cosa_ctx *c, uint64_t key, F &&issue) {
  GraphEntry &g = c->graphs[key];
  if (!g.exec) {
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
    const long long before = c->launches;
    const int r = issue();
    const long long n = c->launches - before;
    const cudaError_t e = cudaStreamEndCapture(c->s, &graph);
    c->launches = before;  // counted at replay
    if (r || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      c->graphs.erase(key);
      return r ? r : cuda_ok(e);
    }
    const cudaError_t e2 = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
      c->graphs.erase(key);
      return cuda_ok(e2);
    }
    g.launches = n;
  }
  const long long per = g.launches;
  CK(cudaGraphLaunch(g.exec, c->s));
  c->launches += per;
  return COSA_OK;
}

// the k-omega work arrays beyond the bound level pointers
int ensure_rans(cosa_ctx *c, LevelState &L) {
  const cosa_level_ptrs &P = L.ptrs;
  if (!P.res || !P.dtvolt || !P.qp || !P.qm || !P.dq || !P.dqp || !P.dqm || !P.flux || !P.mut || !P.dist ||
      !P.vol || !L.d_vm)
    return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1;
  int r = 0;
  for (double **a : {&L.d_prd, &L.d_divvel, &L.d_delpls})
    if (!*a) {
      if ((r = dalloc(c, a, (size_t)L.n3 * S))) return r;
      CK(cudaMemset(*a, 0, (size_t)L.n3 * S * sizeof(double)));
    }
  for (auto &t : L.d_tbeta)
    if (!t && (r = dalloc(c, &t, (size_t)L.n1 * S))) return r;
  if (!L.d_h0 && (r = dalloc(c, &L.d_h0, (size_t)L.nb * 3 * COSA_MAX_SNAP * 2))) return r;
  if (L.rflux_S < S) {
    drop_graphs(c);  // captured graphs hold the old buffer address
    if ((r = dalloc(c, &L.d_rflux, (size_t)6 * L.n0 * c->p.npde * S))) return r;
    L.rflux_S = S;
  }
  if (blend(c->p)) {
    if (!L.d_ttrm) {
      if ((r = dalloc(c, &L.d_ttrm, (size_t)L.n3 * 3 * S))) return r;
      CK(cudaMemset(L.d_ttrm, 0, (size_t)L.n3 * 3 * S * sizeof(double)));
    }
    if (!L.d_fdist && (r = dalloc(c, &L.d_fdist, (size_t)3 * L.n0))) return r;
    // the face distances of the bound wall distance (facedist, src/cosa.f90:209-211)
    for (const DevBlock &x : L.hb) {
      const int64_t nf = (int64_t)x.im * x.jm * x.km;
      k_facedist<1><<<grid_for(nf), 256, 0, c->s>>>(x, P.dist, L.d_fdist);
      k_facedist<2><<<grid_for(nf), 256, 0, c->s>>>(x, P.dist, L.d_fdist + L.n0);
      k_facedist<3><<<grid_for(nf), 256, 0, c->s>>>(x, P.dist, L.d_fdist + 2 * L.n0);
      if ((r = after_launch(c))) return r;
    }
  }
  if (c->p.irsop > 0 && (r = ensure_irs_scratch(c, L))) return r;
  if (L.npart_cap < L.nb * 64) {  // per-block norm partials of the routine-by-routine stage
    drop_graphs(c);
    if ((r = dalloc(c, &L.d_part, (size_t)L.nb * 64 * 8))) return r;
    L.npart_cap = L.nb * 64;
  }
  return COSA_OK;
}

// the preconditioned stage's arrays: the level's cut-offs (zero: cut-off
// type 1 and runs without the viscous cut-off keep them so), the face-flux
// planes, the norm partials and the IRS scratch
int ensure_lsp(cosa_ctx *c, LevelState &L) {
  const cosa_level_ptrs &P = L.ptrs;
  if (!P.res || !P.qp || !P.dq || !P.vol) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1;
  int r = 0;
  for (double **a : {&L.d_cut_pgr, &L.d_cut_vis})
    if (!*a) {
      drop_graphs(c);
      if ((r = dalloc(c, a, (size_t)L.nm1 * COSA_MAX_SNAP))) return r;
      CK(cudaMemset(*a, 0, (size_t)L.nm1 * COSA_MAX_SNAP * sizeof(double)));
    }
  if (L.rflux_S < S) {
    drop_graphs(c);
    if ((r = dalloc(c, &L.d_rflux, (size_t)6 * L.n0 * c->p.npde * S))) return r;
    L.rflux_S = S;
  }
  if (c->p.irsop > 0 && (r = ensure_irs_scratch(c, L))) return r;
  if (L.npart_cap < L.nb * 64) {
    drop_graphs(c);
    if ((r = dalloc(c, &L.d_part, (size_t)L.nb * 64 * 8))) return r;
    L.npart_cap = L.nb * 64;
  }
  return COSA_OK;
}

int ensure_hist(cosa_ctx *c, int rows) {
  if (rows <= c->hist_cap) return COSA_OK;
  drop_graphs(c);  // captured graphs hold the old buffer address
  int r = dalloc(c, &c->d_hist, (size_t)rows * 8);
  if (r) return r;
  c->hist_cap = rows;
  return COSA_OK;
}

}  // namespace

namespace {
int ensure_split(cosa_ctx *c, LevelState &L);
}

extern "C" {

int64_t cosa_gpu_params_size(void) { return (int64_t)sizeof(cosa_params); }

int cosa_gpu_init(const cosa_params *p, int32_t nlevels, const cosa_level_desc *levels, int32_t device,
                  cosa_ctx **out) {
  if (!p || !levels || !out || nlevels < 1 || nlevels > COSA_MAX_LEVELS) return COSA_ERR_ARG;
  if (p->npde != 5 && p->npde != 7) return COSA_ERR_ARG;
  if (2 * p->nharms + 1 > COSA_MAX_SNAP) return COSA_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return COSA_ERR_CUDA;
  CK(cudaSetDevice(device));
  cosa_ctx *c = new (std::nothrow) cosa_ctx;
  if (!c) return COSA_ERR_ARG;
  c->p = *p;
  c->device = device;
  c->nlevels = nlevels;
  int r = 0;
  if ((r = cuda_ok(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking))) ||
      (r = dalloc(c, &c->d_p, 1)) || (r = dalloc(c, &c->d_status, 1)) || (r = dalloc(c, &c->d_row, 1)) ||
      (r = set_smem_attrs())) {
    cosa_gpu_finalize(c);
    return r;
  }
  cudaMemcpy(c->d_p, p, sizeof(cosa_params), cudaMemcpyHostToDevice);
  cudaMemset(c->d_status, 0, sizeof(int));
  cudaMemset(c->d_row, 0, sizeof(int));
  for (int l = 0; l < nlevels; ++l) {
    c->L[l].nl = l + 1;
    if ((r = build_level(c, c->L[l], levels[l]))) {
      cosa_gpu_finalize(c);
      return r;
    }
  }
  *out = c;
  return COSA_OK;
}

int cosa_gpu_finalize(cosa_ctx *c) {
  if (!c) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->s) cudaStreamSynchronize(c->s);
  drop_graphs(c);
  for (auto &e2 : c->prof.ev)
    for (auto &e : e2)
      if (e) cudaEventDestroy(e);
  for (void *v : c->allocs) cudaFree(v);
  if (c->s) cudaStreamDestroy(c->s);
  delete c;
  return COSA_OK;
}

int cosa_gpu_set_params(cosa_ctx *c, const cosa_params *p) {
  if (!c || !p) return COSA_ERR_ARG;
  if (p->npde != c->p.npde || p->nharms != c->p.nharms) return COSA_ERR_ARG;
  c->p = *p;
  CK(cudaMemcpyAsync(c->d_p, p, sizeof(cosa_params), cudaMemcpyHostToDevice, c->s));
  CK(cudaStreamSynchronize(c->s));
  drop_graphs(c);
  return COSA_OK;
}

int cosa_gpu_level_sizes(cosa_ctx *c, int32_t nl, int64_t sizes[5]) {
  LevelState *L = level(c, nl);
  if (!L || !sizes) return COSA_ERR_ARG;
  sizes[0] = L->n3; sizes[1] = L->n2; sizes[2] = L->n1; sizes[3] = L->n0; sizes[4] = L->nm1;
  return COSA_OK;
}

int cosa_gpu_malloc(cosa_ctx *c, int64_t n, double **d) {
  if (!c || !d || n < 0) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  int r = dalloc(c, d, (size_t)n);
  if (r) return r;
  CK(cudaMemset(*d, 0, std::max<size_t>(n, 1) * sizeof(double)));  // cosa_all zeroes (src/input.f90:5125)
  return COSA_OK;
}

int cosa_gpu_memcpy_h2d(cosa_ctx *c, double *dst, const double *src, int64_t n) {
  if (!c || n < 0) return COSA_ERR_ARG;
  CK(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->s));
  return COSA_OK;
}

int cosa_gpu_memcpy_d2h(cosa_ctx *c, double *dst, const double *src, int64_t n) {
  if (!c || n < 0) return COSA_ERR_ARG;
  CK(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  return COSA_OK;
}

int cosa_gpu_synchronize(cosa_ctx *c) {
  if (!c) return COSA_ERR_ARG;
  CK(cudaStreamSynchronize(c->s));
  return COSA_OK;
}

int cosa_gpu_bind_level(cosa_ctx *c, int32_t nl, const cosa_level_ptrs *ptrs) {
  LevelState *L = level(c, nl);
  if (!L || !ptrs) return COSA_ERR_ARG;
  L->ptrs = *ptrs;
  const int S = 2 * c->p.nharms + 1;
  int r = 0;
  if (!L->d_T && (r = dalloc(c, &L->d_T, (size_t)L->n3 * c->p.npde * S))) return r;
  CK(cudaMemset(L->d_T, 0, (size_t)L->n3 * c->p.npde * S * sizeof(double)));
  const int need = std::max(L->ntiles, 148 * 16);
  if (L->npart_cap < need) {
    if ((r = dalloc(c, &L->d_part, (size_t)need * 8))) return r;
    L->npart_cap = need;
  }
  drop_graphs(c);  // graphs hold the previous pointers
  L->bound = true;
  if (c->p.moving) {
    // moving grids run the face-split schedule (the tile kernel has no face speeds)
    if (!ptrs->fvi || !ptrs->fvj || !ptrs->fvk || !ptrs->xdot || !ptrs->ydot || !ptrs->zdot) return COSA_ERR_ARG;
    if ((r = ensure_split(c, *L))) return r;
    L->schedule = 1;
  }
  return COSA_OK;
}

// ---- level drivers --------------------------------------------------------------------
int cosa_gpu_cons2prim(cosa_ctx *c, int32_t nl, int32_t xtnd, double *q) {
  LevelState *L = level(c, nl);
  if (!L || !q || xtnd < 0 || xtnd > 1) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_cons2prim<<<g, 256, 0, c->s>>>(b, c->d_p, q, xtnd);
  });
}

int cosa_gpu_prim2cons(cosa_ctx *c, int32_t nl, double *q) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
    k_prim2cons<<<g, 256, 0, c->s>>>(b, c->d_p, q);
  });
}

int cosa_gpu_bc(cosa_ctx *c, int32_t nl, double *q, const double *si, const double *sj, const double *sk,
                const double *dist) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  if (L->n_bc_items == 0) return COSA_OK;
  const int S = 2 * c->p.nharms + 1;
  k_halo<false><<<grid_for((int64_t)L->n_bc_items * S), 256, 0, c->s>>>(L->d_blocks, L->d_items, L->n_bc_items,
                                                                       c->d_p, q, si, sj, sk, c->d_status, dist,
                                                                       face_vel_of(c, *L));
  return after_launch(c);
}

int cosa_gpu_cutman_q(cosa_ctx *c, int32_t nl, double *q) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  const int ncut = (int)L->items.size() - L->n_bc_items;
  if (ncut == 0) return COSA_OK;
  const int S = 2 * c->p.nharms + 1;
  k_halo<false><<<grid_for((int64_t)ncut * S), 256, 0, c->s>>>(L->d_blocks, L->d_items + L->n_bc_items, ncut, c->d_p, q,
                                                              nullptr, nullptr, nullptr, c->d_status);
  return after_launch(c);
}

int cosa_gpu_prtest(cosa_ctx *c, int32_t nl, const double *q) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  int r = for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
    k_prtest<<<g, 256, 0, c->s>>>(b, c->d_p, q, c->d_status);
  });
  if (r) return r;
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_lambda(cosa_ctx *c, int32_t nl, const double *q, const double *si, const double *sj,
                    const double *sk, const double *, double *lam) {
  LevelState *L = level(c, nl);
  if (!L || !q || !lam) return COSA_ERR_ARG;
  if (c->p.viscous) return COSA_ERR_UNSUPPORTED;
  // moving grids: the cell grid velocities of the bound level
  const cosa_level_ptrs &P = L->ptrs;
  if (c->p.moving && (!P.xdot || !P.ydot || !P.zdot)) return COSA_ERR_ARG;
  const double *cx = c->p.moving ? P.xdot : nullptr, *cy = c->p.moving ? P.ydot : nullptr;
  const double *cz = c->p.moving ? P.zdot : nullptr;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_lambda<<<g, 256, 0, c->s>>>(b, c->d_p, q, si, sj, sk, lam, cx, cy, cz);
  });
}

int cosa_gpu_deltat(cosa_ctx *c, int32_t nl, double *dtvol, const double *lam, double *bx, double *by, double *bz) {
  LevelState *L = level(c, nl);
  if (!L || !dtvol || !lam) return COSA_ERR_ARG;
  if (c->p.viscous || rans(c->p) || c->p.irsop == 5 || c->p.irsop == 6) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_deltat<<<g, 256, 0, c->s>>>(b, c->d_p, dtvol, lam, bx, by, bz);
  });
}

}  // extern "C"

namespace {
// muscl / roflux of the routine-by-routine (k-omega) stage; mixed: limiter
// and Roe dissipation in FP32 on FP64 differences
int muscl_impl(cosa_ctx *c, int32_t idir, int32_t nl, const double *q, double *qp, double *qm, double *dq,
               double *dqp, double *dqm, int mixed);
int roflux_impl(cosa_ctx *c, int32_t idir, int32_t nl, const double *qr, const double *ql, double *flux,
                const double *sijk, int mixed);
}  // namespace

extern "C" {

int cosa_gpu_muscl(cosa_ctx *c, int32_t idir, int32_t nl, const double *q, double *qp, double *qm, double *dq,
                   double *dqp, double *dqm) {
  return muscl_impl(c, idir, nl, q, qp, qm, dq, dqp, dqm, 0);
}

int cosa_gpu_roflux(cosa_ctx *c, int32_t idir, int32_t nl, const double *qr, const double *ql, double *flux,
                    const double *sijk) {
  return roflux_impl(c, idir, nl, qr, ql, flux, sijk, 0);
}

}  // extern "C"

namespace {
int muscl_impl(cosa_ctx *c, int32_t idir, int32_t nl, const double *q, double *qp, double *qm, double *dq,
               double *dqp, double *dqm, int mixed) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !q || !qp || !qm || !dq || !dqp || !dqm) return COSA_ERR_ARG;
  const cosa_params &p = c->p;
  int so_beg = 1, so_end = p.npde;
  if (nl >= p.nl_crs) { so_beg = 0; so_end = -1; }
  else if (p.foturb) { so_beg = 1; so_end = 5; }
  const int *bct = L->d_bct;
  if (so_end >= so_beg) {
    const int r = for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
      k_muscl_dq<<<g, 256, 0, c->s>>>(b, c->d_p, idir, q, dq, bct, so_beg, so_end);
    });
    if (r) return r;
  }
  return for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
    k_muscl_face<<<g, 256, 0, c->s>>>(b, c->d_p, idir, nl, q, qp, qm, dq, dqp, dqm, bct, mixed);
  });
}

int roflux_impl(cosa_ctx *c, int32_t idir, int32_t nl, const double *qr, const double *ql, double *flux,
                const double *sijk, int mixed) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qr || !ql || !flux || !sijk) return COSA_ERR_ARG;
  // moving grids: the face velocities of the bound level (FP64 flux, inviscid)
  const double *fv = nullptr;
  if (c->p.moving) {
    if (mixed || c->p.npde != 5) return COSA_ERR_UNSUPPORTED;
    fv = idir == 1 ? L->ptrs.fvi : (idir == 2 ? L->ptrs.fvj : L->ptrs.fvk);
    if (!fv) return COSA_ERR_ARG;
  }
  return for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
    k_roflux<<<g, 256, 0, c->s>>>(b, c->d_p, idir, qr, ql, flux, sijk, mixed, fv);
  });
}
}  // namespace

extern "C" {

int cosa_gpu_resid(cosa_ctx *c, int32_t idir, int32_t nl, const double *flux, double *res) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !flux || !res) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_resid<<<g, 256, 0, c->s>>>(b, c->d_p, idir, flux, res);
  });
}

int cosa_gpu_update(cosa_ctx *c, int32_t nl, const double *res, double *q, const double *qold, const double *dtvol,
                    double ar) {
  LevelState *L = level(c, nl);
  if (!L || !res || !q || !qold || !dtvol) return COSA_ERR_ARG;
  if (c->p.harbal || c->p.rkimp) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_update<<<g, 256, 0, c->s>>>(b, c->d_p, res, q, qold, dtvol, ar);
  });
}

int cosa_gpu_src_uns(cosa_ctx *c, int32_t nl, const double *q, const double *vol, double *res) {
  LevelState *L = level(c, nl);
  if (!L || !q || !vol || !res) return COSA_ERR_ARG;
  if (c->p.harbal || c->p.dt <= 0) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) { k_src_uns<<<g, 256, 0, c->s>>>(b, c->d_p, q, vol, res); });
}

int cosa_gpu_copy_interior(cosa_ctx *c, int32_t nl, double *dst, const double *src) {
  LevelState *L = level(c, nl);
  if (!L || !dst || !src) return COSA_ERR_ARG;
  const int nvs = c->p.npde * (2 * c->p.nharms + 1);
  return for_blocks(c, *L, cnt_interior,
                    [&](auto b, dim3 g) { k_copy_interior<<<g, 256, 0, c->s>>>(b, nvs, src, dst); });
}

int cosa_gpu_rhs_uns(cosa_ctx *c, int32_t nl, double *rhs, const double *q1, const double *q2, const double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !rhs || !q1 || !q2 || !vol) return COSA_ERR_ARG;
  if (c->p.harbal || c->p.dt <= 0) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells,
                    [&](auto b, dim3 g) { k_rhs_uns<<<g, 256, 0, c->s>>>(b, c->d_p, rhs, q1, q2, vol); });
}

int cosa_gpu_zero(cosa_ctx *c, int32_t nl, double *a) {
  LevelState *L = level(c, nl);
  if (!L || !a) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) {
    k_zero_res<<<g, 256, 0, c->s>>>(b, c->d_p, a);
  });
}

int cosa_gpu_resg_rms(cosa_ctx *c, int32_t nl, const double *res, const double *rhs, double *resrms) {
  LevelState *L = level(c, nl);
  if (!L || !res || !resrms) return COSA_ERR_ARG;
  int r = 0;
  if (L->npart_cap < L->nb * 64) {
    drop_graphs(c);
    if ((r = dalloc(c, &L->d_part, (size_t)L->nb * 64 * 8))) return r;
    L->npart_cap = L->nb * 64;
  }
  for (int b = 0; b < L->nb; ++b) {
    k_rms_partial<<<64, 256, 0, c->s>>>(L->hb[b], c->d_p, res, rhs, L->d_part + (int64_t)b * 64 * 8);
    if ((r = after_launch(c))) return r;
  }
  if ((r = ensure_hist(c, 1))) return r;
  int64_t ncell = 0;
  for (auto &b : L->hb) ncell += (int64_t)(b.im - 1) * (b.jm - 1) * (b.km - 1);
  // resg_rms_hb: every snapshot, divided by ncell * dim5 (src/cosa.f90:4620-4626)
  const double cnt = (double)ncell * (c->p.harbal ? 2 * c->p.nharms + 1 : 1);
  k_rms_final<<<1, 256, 0, c->s>>>(L->d_part, L->nb * 64, c->p.npde, cnt, c->d_hist, nullptr, 1);
  if ((r = after_launch(c))) return r;
  CK(cudaMemcpyAsync(resrms, c->d_hist, (c->p.npde + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  return COSA_OK;
}

// ---- fused smooth ------------------------------------------------------------------------
int cosa_gpu_smooth(cosa_ctx *c, int32_t nl, int32_t niter, int32_t mgit0, int32_t rms_every, double *hist) {
  LevelState *L = level(c, nl);
  if (!L || !L->bound || niter < 0 || rms_every < 1) return COSA_ERR_ARG;
  int r = check_fused_supported(c->p);
  if (r || (r = check_thin_blocks(c, nl))) return r;
  const cosa_level_ptrs &P = L->ptrs;
  if (!P.q || !P.qold || !P.dtvol || !P.si || !P.sj || !P.sk) return COSA_ERR_ARG;
  if (c->p.harbal && !P.vol) return COSA_ERR_ARG;
  if (c->p.viscous && (!P.vol || !L->d_vm)) return COSA_ERR_ARG;
  if (c->p.dualt && (nl != 1 || !P.rhs || !P.vol)) return COSA_ERR_ARG;
  if (rans(c->p) && (r = ensure_rans(c, *L))) return r;
  if (c->p.lomach && (r = ensure_lsp(c, *L))) return r;
  cudaSetDevice(c->device);
  const int npde = c->p.npde;
  // schedule of printed iterations (src/cosa.f90:1925-1927)
  std::vector<int> rows;
  const int last = mgit0 + niter - 1;
  for (int it = 0; it < niter; ++it) {
    const int mgit = mgit0 + it;
    if (hist && (mgit == 1 || mgit % rms_every == 0 || mgit == last)) rows.push_back(it);
  }
  if ((r = ensure_hist(c, std::max<int>(1, (int)rows.size())))) return r;
  if ((c->p.irsop > 0 || c->p.rkimp || c->p.dualt) && (r = ensure_irs_scratch(c, *L))) return r;
  if ((c->p.rkimp || c->p.dualt) && L->npart_cap < L->nb * 64) {  // per-block norm partials (implicit HB, dual time)
    drop_graphs(c);
    if ((r = dalloc(c, &L->d_part, (size_t)L->nb * 64 * 8))) return r;
    L->npart_cap = L->nb * 64;
  }
  CK(cudaMemsetAsync(c->d_row, 0, sizeof(int), c->s));
  const int iter = 1;
  const int compute_dt = (iter / c->p.iupdt * c->p.iupdt == iter) ? 1 : 0;
  size_t ri = 0;
  for (int it = 0; it < niter; ++it) {
    const bool want = ri < rows.size() && rows[ri] == it;
    if (want) ++ri;
    cudaGraphExec_t &g = L->graph[want ? 1 : 0];
    if (!g) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
      const long long before = c->launches;
      IterOpts o;
      o.want_rms = want;
      o.compute_dt = compute_dt;
      r = launch_iteration(c, nl, *L, o);
      cudaError_t e = cudaStreamEndCapture(c->s, &graph);
      if (r) return r;
      CK(e);
      CK(cudaGraphInstantiate(&g, graph, 0));
      cudaGraphDestroy(graph);
      L->graph_launches[want ? 1 : 0] = c->launches - before;
      c->launches = before;  // counted at replay
    }
    CK(cudaGraphLaunch(g, c->s));
    c->launches += L->graph_launches[want ? 1 : 0];
  }
  // reference state after smooth(): face halos of q in conservative form
  // (the k-omega stage converts them itself, src/update.f90:1875-2084)
  if (niter > 0 && !L->items.empty() && !routine_stage(c->p)) {
    double *last_in = (c->p.nstage % 2 == 0) ? L->d_T : L->ptrs.q;
    const int S = 2 * c->p.nharms + 1;
    k_halo_p2c<<<grid_for((int64_t)L->items.size() * S), 256, 0, c->s>>>(L->d_blocks, L->d_items,
                                                                        (int)L->items.size(), c->d_p, last_in,
                                                                        L->ptrs.q);
    if ((r = after_launch(c))) return r;
  }
  if (hist) {
    std::vector<double> h(rows.size() * (npde + 1));
    if (!rows.empty())
      CK(cudaMemcpyAsync(h.data(), c->d_hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    for (int it = 0; it < niter; ++it)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)it * (npde + 1) + v] = NAN;
    for (size_t k = 0; k < rows.size(); ++k)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)rows[k] * (npde + 1) + v] = h[k * (npde + 1) + v];
  }
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_smooth_host(cosa_ctx *c, int32_t nl, double *q_host, int32_t niter, int32_t mgit0, int32_t rms_every,
                         double *hist) {
  LevelState *L = level(c, nl);
  if (!L || !L->bound || !q_host) return COSA_ERR_ARG;
  const int64_t n = L->n3 * c->p.npde * (2 * c->p.nharms + 1);
  int r = cosa_gpu_memcpy_h2d(c, L->ptrs.q, q_host, n);
  if (r) return r;
  r = cosa_gpu_smooth(c, nl, niter, mgit0, rms_every, hist);
  int r2 = cosa_gpu_memcpy_d2h(c, q_host, L->ptrs.q, n);
  return r ? r : r2;
}

int cosa_gpu_src_hb(cosa_ctx *c, int32_t nl, const double *q, const double *vol, double *res) {
  LevelState *L = level(c, nl);
  if (!L || !q || !vol || !res) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_src_hb<<<g, 256, 0, c->s>>>(b, c->d_p, q, vol, res);
  });
}

int cosa_gpu_scalef(cosa_ctx *c, int32_t nl, double *res, const double *dtvol, const double *dtvolt) {
  LevelState *L = level(c, nl);
  if (!L || !res || !dtvol) return COSA_ERR_ARG;
  return irs_scale(c, *L, res, dtvol, c->p.npde > 5 ? dtvolt : nullptr, 1);
}

int cosa_gpu_scaleb(cosa_ctx *c, int32_t nl, double *res, const double *dtvol, const double *dtvolt) {
  LevelState *L = level(c, nl);
  if (!L || !res || !dtvol) return COSA_ERR_ARG;
  return irs_scale(c, *L, res, dtvol, c->p.npde > 5 ? dtvolt : nullptr, 0);
}

int cosa_gpu_cirs(cosa_ctx *c, int32_t nl, double *res, const double *dtvol, const double *betaxi,
                  const double *betaeta, const double *betazeta) {
  LevelState *L = level(c, nl);
  if (!L || !res || !dtvol) return COSA_ERR_ARG;
  if (c->p.irsop < 1 || c->p.npde != 5) return COSA_ERR_UNSUPPORTED;
  int r = ensure_irs_scratch(c, *L);
  if (r) return r;
  const double *beta[3] = {betaxi, betaeta, betazeta};
  if (c->p.irsop >= 2 && (!betaxi || !betaeta || !betazeta)) return COSA_ERR_ARG;
  const double eps = 0.25 * (c->p.rat * c->p.rat - 1.0);
  if ((r = irs_scale(c, *L, res, dtvol, nullptr, 1))) return r;
  if ((r = irs_sweeps(c, *L, res, nullptr, c->p.irsop == 1 ? nullptr : beta, eps, 1, 5, 0))) return r;
  return irs_scale(c, *L, res, dtvol, nullptr, 0);
}

int cosa_gpu_ccirs(cosa_ctx *c, int32_t nl, double *res, const double *ores, const double *betaxi,
                   const double *betaeta, const double *betazeta) {
  LevelState *L = level(c, nl);
  if (!L || !res || !ores) return COSA_ERR_ARG;
  if (c->p.irsop < 1 || c->p.npde != 5) return COSA_ERR_UNSUPPORTED;
  int r = ensure_irs_scratch(c, *L);
  if (r) return r;
  const double *beta[3] = {betaxi, betaeta, betazeta};
  if (c->p.irsop >= 2 && (!betaxi || !betaeta || !betazeta)) return COSA_ERR_ARG;
  const double eps = 0.25 * (c->p.rat * c->p.rat - 1.0);
  return irs_sweeps(c, *L, res, ores, c->p.irsop == 1 ? nullptr : beta, eps, 1, 5, 1);
}

int cosa_gpu_imetrix(cosa_ctx *c, int32_t nl, const double *x, const double *y, const double *z, double *si,
                     double *sj, double *sk) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z || !si || !sj || !sk) return COSA_ERR_ARG;
  // one set of metrics per grid snapshot with hbmove (src/grid.f90:897-1062)
  const int S2 = 2 * c->p.nharms * c->p.hbmove + 1;
  double *s3[3] = {si, sj, sk};
  for (int nh = 0; nh < S2; ++nh)
    for (int b = 0; b < L->nb; ++b)
      for (int d = 1; d <= 3; ++d) {
        const DevBlock &x_ = L->hb[b];
        k_imetrix<<<grid_for((int64_t)(x_.im + 1) * (x_.jm + 1) * (x_.km + 1)), 256, 0, c->s>>>(x_, d, x, y, z,
                                                                                                 s3[d - 1], S2, nh);
        int r = after_launch(c);
        if (r) return r;
      }
  return COSA_OK;
}

int cosa_gpu_vols(cosa_ctx *c, int32_t nl, const double *x, const double *y, const double *z, double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z || !vol) return COSA_ERR_ARG;
  for (int b = 0; b < L->nb; ++b) {
    const DevBlock &x_ = L->hb[b];
    k_vols<<<grid_for((int64_t)x_.im * x_.jm * x_.km), 256, 0, c->s>>>(x_, x, y, z, vol,
                                                                       2 * c->p.nharms * c->p.hbmove + 1);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

// movegrid with pitch (src/grid.f90:1783-1966) for every snapshot
int cosa_gpu_movegrid(cosa_ctx *c, int32_t nl, const double *x0, const double *y0, const double *z0,
                      const double *dx, const double *dy, const double *dz, double *x, double *y, double *z,
                      double *xdot, double *ydot, double *zdot) {
  LevelState *L = level(c, nl);
  if (!L || !x0 || !y0 || !z0 || !dx || !dy || !x || !y || !z || !xdot || !ydot || !zdot) return COSA_ERR_ARG;
  (void)dz;
  const cosa_params &p = c->p;
  if (!p.moving || !p.harbal || !p.hbmove) return COSA_ERR_UNSUPPORTED;
  const int S2 = 2 * p.nharms * p.hbmove + 1;
  // snapshot times and angles (src/input.f90:3182-3192, src/grid.f90:4536-4541)
  std::vector<PitchSnap> snap(S2);
  const double pi = 3.14159265358979323846, omega = std::fabs(p.omegas);
  const double dt = omega > 0 ? 2 * pi / omega / (2 * p.nharms + 1) : 0.0;
  for (int n = 0; n < S2; ++n) {
    const double zeit = n * dt, dth = p.dtheta0 * std::sin(p.omegas * zeit);
    snap[n] = PitchSnap{std::cos(dth), std::sin(dth), std::cos(p.omegas * zeit)};
  }
  PitchSnap *d_snap = nullptr;
  int r = dalloc(c, &d_snap, snap.size());
  if (r) return r;
  CK(cudaMemcpyAsync(d_snap, snap.data(), snap.size() * sizeof(PitchSnap), cudaMemcpyHostToDevice, c->s));
  for (int b = 0; b < L->nb; ++b) {
    const DevBlock &x_ = L->hb[b];
    k_pitch<<<grid_for((int64_t)(x_.im + 2) * (x_.jm + 2) * (x_.km + 2) * S2), 256, 0, c->s>>>(
        x_, S2, d_snap, p.xh, p.yh, p.dtheta0, p.omegas, x0, y0, z0, dx, dy, x, y, z, xdot, ydot, zdot);
    if ((r = after_launch(c))) return r;
  }
  CK(cudaStreamSynchronize(c->s));
  return COSA_OK;
}

// face velocities from the node velocities (imetrix_b's moving part)
int cosa_gpu_face_vel(cosa_ctx *c, int32_t nl, const double *xdot, const double *ydot, const double *zdot,
                      double *fvi, double *fvj, double *fvk) {
  LevelState *L = level(c, nl);
  if (!L || !xdot || !ydot || !zdot || !fvi || !fvj || !fvk) return COSA_ERR_ARG;
  const int S2 = 2 * c->p.nharms * c->p.hbmove + 1;
  double *f3[3] = {fvi, fvj, fvk};
  for (int b = 0; b < L->nb; ++b)
    for (int d = 1; d <= 3; ++d) {
      const DevBlock &x_ = L->hb[b];
      k_face_vel<<<grid_for((int64_t)(x_.im + 1) * (x_.jm + 1) * (x_.km + 1) * S2), 256, 0, c->s>>>(
          x_, d, S2, xdot, ydot, zdot, f3[d - 1]);
      int r = after_launch(c);
      if (r) return r;
    }
  return COSA_OK;
}

// vert2cell_g (src/output.f90:3242-3480) of one node array, in place
int cosa_gpu_vert2cell(cosa_ctx *c, int32_t nl, double *w) {
  LevelState *L = level(c, nl);
  if (!L || !w) return COSA_ERR_ARG;
  const int S2 = 2 * c->p.nharms * c->p.hbmove + 1;
  const size_t n = (size_t)L->n2 * S2;
  double *tmp = nullptr;
  int r = dalloc(c, &tmp, n);
  if (r) return r;
  CK(cudaMemcpyAsync(tmp, w, n * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
  for (int b = 0; b < L->nb; ++b) {
    const DevBlock &x_ = L->hb[b];
    k_vert2cell<<<grid_for((int64_t)(x_.im + 1) * (x_.jm + 1) * (x_.km + 1) * S2), 256, 0, c->s>>>(x_, S2, tmp, w);
    if ((r = after_launch(c))) return r;
  }
  CK(cudaStreamSynchronize(c->s));
  return COSA_OK;
}

}  // extern "C"

// ---- multigrid ---------------------------------------------------------------------------
namespace {

// levels nl and nl+1 hold the same blocks with twice the cells per direction
int level_pair(cosa_ctx *c, int nl, LevelState *&L1, LevelState *&L2) {
  L1 = level(c, nl);
  L2 = level(c, nl + 1);
  if (!L1 || !L2 || L1->nb != L2->nb) return COSA_ERR_ARG;
  for (int b = 0; b < L1->nb; ++b) {
    const DevBlock &f = L1->hb[b], &g = L2->hb[b];
    if (f.im - 1 != 2 * (g.im - 1) || f.jm - 1 != 2 * (g.jm - 1) || f.km - 1 != 2 * (g.km - 1)) return COSA_ERR_ARG;
  }
  return COSA_OK;
}

int launch_edges(cosa_ctx *c, LevelState &L, double *q, double *mut) {
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  int r = for_blocks(c, L, cnt_edges, [&](auto b, dim3 g) { k_edges<<<g, 256, 0, c->s>>>(b, npde, S, q, -1); });
  if (r || !mut) return r;
  return for_blocks(c, L, cnt_edges, [&](auto b, dim3 g) { k_edges<<<g, 256, 0, c->s>>>(b, 1, S, mut, -1); });
}

int launch_corns(cosa_ctx *c, LevelState &L, double *q, double *mut) {
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    k_corns<<<1, 128, 0, c->s>>>(x, npde, S, q, x.op3 * npde * S);
    int r = after_launch(c);
    if (r) return r;
    if (mut) {
      k_corns<<<1, 128, 0, c->s>>>(x, 1, S, mut, x.op3 * S);
      if ((r = after_launch(c))) return r;
    }
  }
  return COSA_OK;
}

int launch_rest1(cosa_ctx *c, LevelState &L1, LevelState &L2, const double *q1, double *q2, const double *v1,
                 const double *v2) {
  const int S = 2 * c->p.nharms + 1;
  for (int b = 0; b < L1.nb; ++b) {
    const DevBlock &g = L2.hb[b];
    k_rest1<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * S), 256, 0, c->s>>>(L1.hb[b], g, c->p.npde, S,
                                                                                          q1, q2, v1, v2);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int launch_rest2(cosa_ctx *c, LevelState &L1, LevelState &L2, double *rhs2, const double *res1) {
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  for (int b = 0; b < L1.nb; ++b) {
    const DevBlock &g = L2.hb[b];
    k_rest2<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * npde * S), 256, 0, c->s>>>(L1.hb[b], g, npde,
                                                                                                 S, rhs2, res1);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int launch_prol(cosa_ctx *c, LevelState &L1, LevelState &L2, double *q1, const double *q2, const double *vol1,
                bool bilinear) {
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  for (int b = 0; b < L1.nb; ++b) {
    const DevBlock &g = L2.hb[b];
    const int64_t n = (int64_t)g.im * g.jm * g.km * npde * S;
    if (bilinear)
      k_prol_bln<<<grid_for(n), 256, 0, c->s>>>(L1.hb[b], g, npde, S, q1, q2, c->p.lim_corr);
    else
      k_prol_lin<<<grid_for(n), 256, 0, c->s>>>(L1.hb[b], g, npde, S, q1, q2, vol1);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int launch_rest2_ho(cosa_ctx *c, LevelState &L1, LevelState &L2, double *rhs2, const double *res1) {
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  for (int b = 0; b < L1.nb; ++b) {
    const DevBlock &g = L2.hb[b];
    k_rest2_ho<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * npde * S), 256, 0, c->s>>>(
        L1.hb[b], g, npde, S, rhs2, res1);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int launch_bc_res(cosa_ctx *c, LevelState &L, double *res) {
  if (L.n_bc_items == 0) return COSA_OK;
  const int S = 2 * c->p.nharms + 1;
  k_bc_res<<<grid_for((int64_t)L.n_bc_items * c->p.npde * S), 256, 0, c->s>>>(L.d_blocks, L.d_items, L.n_bc_items,
                                                                            c->p.npde, S, res);
  return after_launch(c);
}

// rest2 with ho_rest (src/cosa.f90:2742-2751): the fine residual's first halo
// layer as smooth() leaves it (zeroed every stage, src/cosa.f90:1786-1792) or,
// with k-omega, filled by cutman_q, bc_res, q_edges and q_corns
int issue_rest2_ho(cosa_ctx *c, LevelState &L1, LevelState &L2, int nl, double *rhs2, double *res1) {
  const int nvs = c->p.npde * (2 * c->p.nharms + 1);
  int r = 0;
  for (int b = 0; b < L1.nb; ++b) {
    const DevBlock &x = L1.hb[b];
    k_zero_shell1<<<grid_for((int64_t)(x.im + 1) * (x.jm + 1) * (x.km + 1) * nvs), 256, 0, c->s>>>(x, nvs, res1);
    if ((r = after_launch(c))) return r;
  }
  if (rans(c->p)) {
    if ((r = cosa_gpu_cutman_q(c, nl, res1)) || (r = launch_bc_res(c, L1, res1)) ||
        (r = launch_edges(c, L1, res1, nullptr)) || (r = launch_corns(c, L1, res1, nullptr)))
      return r;
  }
  return launch_rest2_ho(c, L1, L2, rhs2, res1);
}

// restrict(nl) (src/cosa.f90:2672-2755)
int issue_restrict(cosa_ctx *c, int nl) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  const cosa_level_ptrs &A = L1->ptrs, &B = L2->ptrs;
  if (!A.q || !A.vol || !A.res || !B.q || !B.vol || !B.rhs) return COSA_ERR_ARG;
  if ((r = launch_rest1(c, *L1, *L2, A.q, B.q, A.vol, B.vol))) return r;
  if (c->p.lomach) {
    // the low-speed cut-offs (src/cosa.f90:2724-2731)
    const int S = 2 * c->p.nharms + 1;
    std::vector<std::pair<const double *, double *>> cuts;
    if (c->p.cutoff_type == 3) cuts.push_back({L1->d_cut_pgr, L2->d_cut_pgr});
    if (c->p.visprec) cuts.push_back({L1->d_cut_vis, L2->d_cut_vis});
    for (auto &f : cuts) {
      if (!f.first || !f.second) return COSA_ERR_ARG;
      for (int b = 0; b < L2->nb; ++b) {
        const DevBlock &g = L2->hb[b];
        k_rest3<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * S), 256, 0, c->s>>>(
            L1->hb[b], g, S, f.first, f.second, A.vol, B.vol);
        if ((r = after_launch(c))) return r;
      }
    }
  }
  if (rans(c->p)) {
    // production terms (or mut with prd_all_lvls) restricted as well
    // (src/cosa.f90:2733-2741)
    const int S = 2 * c->p.nharms + 1;
    std::vector<std::pair<const double *, double *>> fields;
    if (!c->p.prd_all_lvls) {
      if (!L1->d_prd || !L2->d_prd) return COSA_ERR_ARG;
      fields = {{L1->d_prd, L2->d_prd}, {L1->d_delpls, L2->d_delpls}, {L1->d_divvel, L2->d_divvel}};
    } else {
      if (!A.mut || !B.mut) return COSA_ERR_ARG;
      fields = {{A.mut, B.mut}};
    }
    for (auto &f : fields)
      for (int b = 0; b < L2->nb; ++b) {
        const DevBlock &g = L2->hb[b];
        k_rest4<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * S), 256, 0, c->s>>>(
            L1->hb[b], g, S, f.first, f.second, A.vol, B.vol);
        if ((r = after_launch(c))) return r;
      }
  }
  if (c->p.ho_rest) return issue_rest2_ho(c, *L1, *L2, nl, B.rhs, A.res);
  return launch_rest2(c, *L1, *L2, B.rhs, A.res);
}

// prolong(nl) (src/cosa.f90:3167-3250)
int issue_prolong(cosa_ctx *c, int nl) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  const cosa_level_ptrs &A = L1->ptrs, &B = L2->ptrs;
  if (!A.q || !A.vol || !B.q || !B.qold || !B.vol || !B.si || !B.sj || !B.sk) return COSA_ERR_ARG;
  if ((r = launch_rest1(c, *L1, *L2, A.q, B.qold, A.vol, B.vol))) return r;
  for (double *a : {B.qold, B.q}) {
    if ((r = cosa_gpu_cons2prim(c, nl + 1, 0, a)) || (r = cosa_gpu_bc(c, nl + 1, a, B.si, B.sj, B.sk, B.dist)) ||
        (r = cosa_gpu_cutman_q(c, nl + 1, a)) || (r = cosa_gpu_prim2cons(c, nl + 1, a)) ||
        (r = launch_edges(c, *L2, a, nullptr)) || (r = launch_corns(c, *L2, a, nullptr)))
      return r;
  }
  const int nvs = c->p.npde * (2 * c->p.nharms + 1);
  for (int b = 0; b < L2->nb; ++b) {
    const DevBlock &g = L2->hb[b];
    k_add_ext1<<<grid_for((int64_t)(g.im + 1) * (g.jm + 1) * (g.km + 1) * nvs), 256, 0, c->s>>>(g, nvs, B.q, B.qold,
                                                                                               -1.0);
    if ((r = after_launch(c))) return r;
  }
  if ((r = launch_prol(c, *L1, *L2, A.q, B.q, A.vol, c->p.bln_prol != 0))) return r;
  if (c->p.lim_corr == 1 || c->p.lim_corr == 3) return cosa_gpu_fixq(c, nl, A.q);
  return COSA_OK;
}

// smooth(nl, from_fine, to_coarse, done, niter) of the fused path
int issue_smooth_level(cosa_ctx *c, int nl, int niter, bool from_fine, bool to_coarse, bool want_rms,
                       bool first_cycle = false) {
  LevelState &L = *level(c, nl);
  const cosa_params &p = c->p;
  const int niterp = to_coarse ? niter + 1 : niter;
  int r = 0;
  for (int iter = 1; iter <= niterp; ++iter) {
    IterOpts o;
    o.compute_dt = (iter / p.iupdt * p.iupdt == iter) ? 1 : 0;
    o.rhs = nl > 1 ? L.ptrs.rhs : nullptr;
    o.force = from_fine && iter == 1;
    o.copy_qold = iter <= niter;
    o.want_rms = want_rms && nl == 1 && iter == niter;
    o.res_only = iter == niter + 1 ? L.ptrs.res : nullptr;
    o.first_cycle = first_cycle;
    o.to_coarse = to_coarse;
    if ((r = launch_iteration(c, nl, L, o))) return r;
  }
  // reference state after smooth(): face halos of q in conservative form
  // (the k-omega stage converts them itself)
  if (niterp > 0 && !L.items.empty() && !routine_stage(p)) {
    double *last_in = (to_coarse || p.nstage % 2 == 1) ? L.ptrs.q : L.d_T;
    const int S = 2 * p.nharms + 1;
    k_halo_p2c<<<grid_for((int64_t)L.items.size() * S), 256, 0, c->s>>>(L.d_blocks, L.d_items, (int)L.items.size(),
                                                                       c->d_p, last_in, L.ptrs.q);
    if ((r = after_launch(c))) return r;
  }
  return COSA_OK;
}

// one cycle of mg() (src/cosa.f90:822-912)
int issue_mg_cycle(cosa_ctx *c, int mgit, bool want_rms) {
  const cosa_params &p = c->p;
  const int nlevel = p.nlevel;
  int r = 0;
  const bool first = mgit == 1;
  int niter = nlevel == 1 ? 1 : (mgit == 1 ? p.nstart : p.npost);
  if ((r = issue_smooth_level(c, 1, niter, false, nlevel > 1, want_rms, first))) return r;
  if (nlevel == 1) return COSA_OK;
  if ((r = issue_restrict(c, 1))) return r;
  niter = nlevel == 2 ? p.ncrs : p.npre;
  if ((r = issue_smooth_level(c, 2, niter, true, nlevel > 2, false, first))) return r;
  if (nlevel == 3) {
    if ((r = issue_restrict(c, 2)) || (r = issue_smooth_level(c, 3, p.ncrs, true, false, false, first)) ||
        (r = issue_prolong(c, 2)) || (r = issue_smooth_level(c, 2, p.npost, false, false, false, first)))
      return r;
  }
  return issue_prolong(c, 1);
}

// the bound levels' arrays that smoothing and the transfers of nlevel levels need
int check_mg_levels(cosa_ctx *c, int nlevel) {
  for (int nl = 1; nl <= nlevel; ++nl) {
    LevelState *L = level(c, nl);
    if (!L || !L->bound) return COSA_ERR_ARG;
    const cosa_level_ptrs &P = L->ptrs;
    if (!P.q || !P.qold || !P.dtvol || !P.si || !P.sj || !P.sk) return COSA_ERR_ARG;
    if ((c->p.harbal || nlevel > 1 || c->p.viscous) && !P.vol) return COSA_ERR_ARG;
    if (c->p.viscous && !L->d_vm) return COSA_ERR_ARG;  // cosa_gpu_viscous_setup on every level
    if (nl < nlevel && !P.res) return COSA_ERR_ARG;
    if (nl > 1 && !P.rhs) return COSA_ERR_ARG;
    if (nl < nlevel) {
      LevelState *L1, *L2;
      if (level_pair(c, nl, L1, L2)) return COSA_ERR_ARG;
    }
  }
  return COSA_OK;
}

uint64_t graph_key(int kind, int nl, int niter, int flags) {
  return ((uint64_t)kind << 56) | ((uint64_t)(nl & 0xff) << 48) | ((uint64_t)(uint32_t)niter << 16) |
         (uint64_t)(flags & 0xffff);
}

}  // namespace

extern "C" {

int cosa_gpu_q_edges(cosa_ctx *c, int32_t nl, double *q, double *mut) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  return launch_edges(c, *L, q, mut);
}

int cosa_gpu_q_corns(cosa_ctx *c, int32_t nl, double *q, double *mut) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  return launch_corns(c, *L, q, mut);
}

int cosa_gpu_fixq(cosa_ctx *c, int32_t nl, double *q) {
  LevelState *L = level(c, nl);
  if (!L || !q) return COSA_ERR_ARG;
  if (c->p.npde < 7) return COSA_OK;  // the reference calls it for k-omega only
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) { k_fixq<<<g, 256, 0, c->s>>>(b, c->d_p, q); });
}

int cosa_gpu_tur_vis(cosa_ctx *c, int32_t nl, const double *q, double *mut) {
  LevelState *L = level(c, nl);
  if (!L || !q || !mut || c->p.npde < 7) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_all, [&](auto b, dim3 g) { k_tur_vis<<<g, 256, 0, c->s>>>(b, c->d_p, q, mut); });
}

int cosa_gpu_rest1(cosa_ctx *c, int32_t nl, const double *q1, double *q2, const double *vol1, const double *vol2) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!q1 || !q2 || !vol1 || !vol2) return COSA_ERR_ARG;
  return launch_rest1(c, *L1, *L2, q1, q2, vol1, vol2);
}

int cosa_gpu_rest2(cosa_ctx *c, int32_t nl, double *rhs2, const double *res1) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!rhs2 || !res1) return COSA_ERR_ARG;
  return launch_rest2(c, *L1, *L2, rhs2, res1);
}

int cosa_gpu_rest2_ho(cosa_ctx *c, int32_t nl, double *rhs2, const double *res1) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!rhs2 || !res1) return COSA_ERR_ARG;
  return launch_rest2_ho(c, *L1, *L2, rhs2, res1);
}
int cosa_gpu_bc_res(cosa_ctx *c, int32_t nl, double *res) {
  LevelState *L = level(c, nl);
  if (!L || !res) return COSA_ERR_ARG;
  return launch_bc_res(c, *L, res);
}
int cosa_gpu_prol_bln(cosa_ctx *c, int32_t nl, double *q1, const double *q2) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!q1 || !q2) return COSA_ERR_ARG;
  return launch_prol(c, *L1, *L2, q1, q2, nullptr, true);
}

int cosa_gpu_prol_lin(cosa_ctx *c, int32_t nl, double *q1, const double *q2, const double *vol1) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!q1 || !q2 || !vol1) return COSA_ERR_ARG;
  return launch_prol(c, *L1, *L2, q1, q2, vol1, false);
}

int cosa_gpu_restrict(cosa_ctx *c, int32_t nl) {
  if (!c) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  return issue_restrict(c, nl);
}

int cosa_gpu_prolong(cosa_ctx *c, int32_t nl) {
  if (!c) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  int r = issue_prolong(c, nl);
  if (r) return r;
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_smooth_level(cosa_ctx *c, int32_t nl, int32_t niter, int32_t from_fine, int32_t to_coarse, int32_t mgit,
                          int32_t ncycle, int32_t rms_every, double *resrms) {
  LevelState *L = level(c, nl);
  if (!L || !L->bound || niter < 0 || rms_every < 1) return COSA_ERR_ARG;
  int r = check_fused_supported(c->p);
  if (r || (r = check_thin_blocks(c, nl))) return r;
  const cosa_level_ptrs &P = L->ptrs;
  if (!P.q || !P.qold || !P.dtvol || !P.si || !P.sj || !P.sk) return COSA_ERR_ARG;
  if ((c->p.harbal && !P.vol) || (to_coarse && !P.res) || (nl > 1 && !P.rhs)) return COSA_ERR_ARG;
  if (c->p.dualt && (!P.rhs || !P.vol)) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  const bool want = resrms && nl == 1 && niter > 0 && (mgit == 1 || mgit % rms_every == 0 || mgit == ncycle);
  if ((r = ensure_hist(c, 1))) return r;
  if ((c->p.irsop > 0 || c->p.rkimp || c->p.dualt) && (r = ensure_irs_scratch(c, *L))) return r;
  if ((c->p.rkimp || c->p.dualt) && L->npart_cap < L->nb * 64) {  // per-block norm partials (implicit HB, dual time)
    drop_graphs(c);
    if ((r = dalloc(c, &L->d_part, (size_t)L->nb * 64 * 8))) return r;
    L->npart_cap = L->nb * 64;
  }
  CK(cudaMemsetAsync(c->d_row, 0, sizeof(int), c->s));
  if (rans(c->p) && (r = ensure_rans(c, *L))) return r;
  if (c->p.lomach && (r = ensure_lsp(c, *L))) return r;
  const bool first = mgit == 1;
  const int flags = (from_fine ? 1 : 0) | (to_coarse ? 2 : 0) | (want ? 4 : 0) | (first ? 8 : 0);
  r = run_graph(c, graph_key(1, nl, niter, flags),
                [&] { return issue_smooth_level(c, nl, niter, from_fine != 0, to_coarse != 0, want, first); });
  if (r) return r;
  if (want) CK(cudaMemcpyAsync(resrms, c->d_hist, (c->p.npde + 1) * sizeof(double), cudaMemcpyDeviceToHost, c->s));
  CK(cudaStreamSynchronize(c->s));
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_rkuns(cosa_ctx *c, int32_t ntime, int32_t iprint, double *hist) {
  LevelState *L = level(c, 1);
  if (!L || !L->bound || ntime < 0 || iprint < 1) return COSA_ERR_ARG;
  const cosa_params &p = c->p;
  // fixed grids, Euler and laminar, no IRS (rkuns smooths nothing); the
  // reference's k-omega variant advances k and omega with a dtvolt that
  // rkuns never sets
  if (!p.rgkuns || rans(p) || p.harbal || p.dualt || p.moving || p.irsop != 0 || p.dt <= 0)
    return COSA_ERR_UNSUPPORTED;
  int r = check_fused_supported(p);
  if (r || (r = check_thin_blocks(c, 1))) return r;
  const cosa_level_ptrs &P = L->ptrs;
  if (!P.q || !P.qold || !P.dtvol || !P.si || !P.sj || !P.sk || !P.vol) return COSA_ERR_ARG;
  if (p.viscous && !L->d_vm) return COSA_ERR_ARG;
  cudaSetDevice(c->device);
  std::vector<int> rows;
  for (int it = 0; it < ntime; ++it)
    if (hist && ((it + 1) % iprint == 0 || it + 1 == ntime)) rows.push_back(it);
  if ((r = ensure_hist(c, std::max<int>(1, (int)rows.size())))) return r;
  // deltat_urk: the global time step, once (src/cosa.f90:4039-4041)
  if ((r = for_blocks(c, *L, cnt_cells,
                      [&](auto b, dim3 g) { k_deltat_urk<<<g, 256, 0, c->s>>>(b, c->d_p, P.vol, P.dtvol); })))
    return r;
  CK(cudaMemsetAsync(c->d_row, 0, sizeof(int), c->s));
  size_t ri = 0;
  for (int it = 0; it < ntime; ++it) {
    const bool want = ri < rows.size() && rows[ri] == it;
    if (want) ++ri;
    IterOpts o;
    o.want_rms = want;
    o.rms_stage = p.nstage;  // the norm of the last stage is the one kept
    o.compute_dt = 0;
    r = run_graph(c, graph_key(3, 1, 0, want ? 1 : 0), [&] { return launch_iteration(c, 1, *L, o); });
    if (r) return r;
  }
  if (ntime > 0 && !L->items.empty()) {
    double *last_in = (p.nstage % 2 == 0) ? L->d_T : L->ptrs.q;
    k_halo_p2c<<<grid_for((int64_t)L->items.size()), 256, 0, c->s>>>(L->d_blocks, L->d_items, (int)L->items.size(),
                                                                      c->d_p, last_in, L->ptrs.q);
    if ((r = after_launch(c))) return r;
  }
  if (hist) {
    const int npde = p.npde;
    std::vector<double> h(rows.size() * (npde + 1));
    if (!rows.empty())
      CK(cudaMemcpyAsync(h.data(), c->d_hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    for (int it = 0; it < ntime; ++it)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)it * (npde + 1) + v] = NAN;
    for (size_t k = 0; k < rows.size(); ++k)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)rows[k] * (npde + 1) + v] = h[k * (npde + 1) + v];
  }
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_mg(cosa_ctx *c, int32_t mgit0, int32_t ncycles, int32_t ncycle, int32_t rms_every, double *hist) {
  if (!c || ncycles < 0 || rms_every < 1 || mgit0 < 1) return COSA_ERR_ARG;
  const int nlevel = c->p.nlevel;
  if (nlevel < 1 || nlevel > c->nlevels) return COSA_ERR_ARG;
  int r = check_fused_supported(c->p);
  if (r) return r;
  if ((r = check_mg_levels(c, nlevel))) return r;
  // dual time: the fine level's rhs holds rhs_uns, the BDF term needs vol
  if (c->p.dualt && (!level(c, 1)->ptrs.rhs || !level(c, 1)->ptrs.vol)) return COSA_ERR_ARG;
  for (int nl = 1; nl <= nlevel; ++nl)
    if ((r = check_thin_blocks(c, nl))) return r;
  cudaSetDevice(c->device);
  const int npde = c->p.npde;
  std::vector<int> rows;
  for (int it = 0; it < ncycles; ++it) {
    const int mgit = mgit0 + it;
    if (hist && (mgit == 1 || mgit % rms_every == 0 || mgit == ncycle)) rows.push_back(it);
  }
  if ((r = ensure_hist(c, std::max<int>(1, (int)rows.size())))) return r;
  for (int nl = 1; nl <= nlevel; ++nl) {
    LevelState &Lv = *level(c, nl);
    if ((c->p.irsop > 0 || c->p.rkimp || c->p.dualt) && (r = ensure_irs_scratch(c, Lv))) return r;
    if ((c->p.rkimp || c->p.dualt) && Lv.npart_cap < Lv.nb * 64) {  // per-block norm partials (implicit HB, dual time)
      drop_graphs(c);
      if ((r = dalloc(c, &Lv.d_part, (size_t)Lv.nb * 64 * 8))) return r;
      Lv.npart_cap = Lv.nb * 64;
    }
    if (rans(c->p) && (r = ensure_rans(c, Lv))) return r;
    if (c->p.lomach && (r = ensure_lsp(c, Lv))) return r;
  }
  CK(cudaMemsetAsync(c->d_row, 0, sizeof(int), c->s));
  size_t ri = 0;
  int last = mgit0 - 1;
  for (int it = 0; it < ncycles; ++it) {
    const int mgit = mgit0 + it;
    const bool want = ri < rows.size() && rows[ri] == it;
    if (want) ++ri;
    const int flags = (mgit == 1 ? 1 : 0) | (want ? 2 : 0);
    r = run_graph(c, graph_key(2, nlevel, 0, flags), [&] { return issue_mg_cycle(c, mgit, want); });
    if (r) return r;
    last = mgit;
  }
  if (nlevel > 1 && last == ncycle) {
    r = run_graph(c, graph_key(1, 1, c->p.npost, 0),
                  [&] { return issue_smooth_level(c, 1, c->p.npost, false, false, false); });
    if (r) return r;
  }
  if (hist) {
    std::vector<double> h(rows.size() * (npde + 1));
    if (!rows.empty())
      CK(cudaMemcpyAsync(h.data(), c->d_hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    for (int it = 0; it < ncycles; ++it)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)it * (npde + 1) + v] = NAN;
    for (size_t k = 0; k < rows.size(); ++k)
      for (int v = 0; v <= npde; ++v) hist[(int64_t)rows[k] * (npde + 1) + v] = h[k * (npde + 1) + v];
  } else {
    CK(cudaStreamSynchronize(c->s));
  }
  return cosa_gpu_status(c, 0);
}

int cosa_gpu_profile(cosa_ctx *c, int32_t nl, int32_t niter, double ms[4], int64_t counts[4]) {
  LevelState *L = level(c, nl);
  if (!L || !L->bound || niter < 1 || !ms || !counts) return COSA_ERR_ARG;
  int r = check_fused_supported(c->p);
  if (r || (r = check_thin_blocks(c, nl))) return r;
  ProfState &pf = c->prof;
  for (auto &e2 : pf.ev)
    for (auto &e : e2)
      if (!e) CK(cudaEventCreate(&e));
  pf.ms[0] = pf.ms[1] = pf.ms[2] = 0;
  pf.n[0] = pf.n[1] = pf.n[2] = 0;
  pf.on = true;
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  const int compute_dt = (1 / c->p.iupdt * c->p.iupdt == 1) ? 1 : 0;
  if (c->p.irsop > 0 && (r = ensure_irs_scratch(c, *L))) return r;
  cudaEventRecord(t0, c->s);
  IterOpts o;
  o.compute_dt = compute_dt;
  for (int it = 0; it < niter && !r; ++it) r = launch_iteration(c, nl, *L, o);
  cudaEventRecord(t1, c->s);
  pf.on = false;
  CK(cudaEventSynchronize(t1));
  float tot = 0;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (r) return r;
  ms[0] = pf.n[0] ? pf.ms[0] / pf.n[0] : 0.0;
  ms[1] = pf.n[1] ? pf.ms[1] / pf.n[1] : 0.0;
  ms[2] = tot / niter;
  ms[3] = pf.n[2] ? pf.ms[2] / pf.n[2] : 0.0;
  counts[0] = pf.n[0];
  counts[1] = pf.n[1];
  counts[2] = niter;
  counts[3] = pf.n[2];
  return cosa_gpu_status(c, 0);
}

void *cosa_gpu_stream(cosa_ctx *c) { return c ? (void *)c->s : nullptr; }

}  // extern "C"

namespace {
__global__ void k_nr_selftest(int64_t n, const double *__restrict__ x, double *__restrict__ e) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[t];
    const double r = 1.0 / v, s = 1.0 / sqrt(v);
    e[2 * t] = fabs(rcp_nr(v) - r) / r;
    e[2 * t + 1] = fabs(rsqrt_nr(v) - s) / s;
  }
}
}  // namespace

extern "C" {

int cosa_gpu_nr_selftest(int64_t n, const double *x, double err[2]) {
  if (n < 1 || !x || !err) return COSA_ERR_ARG;
  double *dx = nullptr, *de = nullptr;
  CK(cudaMalloc(&dx, n * sizeof(double)));
  if (cudaMalloc(&de, 2 * n * sizeof(double)) != cudaSuccess) { cudaFree(dx); return COSA_ERR_CUDA; }
  std::vector<double> h(2 * n);
  int r = cuda_ok(cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice));
  if (!r) {
    k_nr_selftest<<<grid_for(n), 256>>>(n, dx, de);
    r = cuda_ok(cudaGetLastError());
  }
  if (!r) r = cuda_ok(cudaMemcpy(h.data(), de, 2 * n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(dx);
  cudaFree(de);
  if (r) return r;
  err[0] = err[1] = 0.0;
  for (int64_t t = 0; t < n; ++t) {
    err[0] = std::max(err[0], h[2 * t]);
    err[1] = std::max(err[1], h[2 * t + 1]);
  }
  return COSA_OK;
}

int64_t cosa_gpu_launch_count(cosa_ctx *c, int32_t reset) {
  if (!c) return -1;
  const long long v = c->launches;
  if (reset) c->launches = 0;
  return v;
}

int cosa_gpu_status(cosa_ctx *c, int32_t reset) {
  if (!c) return COSA_ERR_ARG;
  int st = 0;
  if (cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->s) != cudaSuccess) return COSA_ERR_CUDA;
  if (cudaStreamSynchronize(c->s) != cudaSuccess) return COSA_ERR_CUDA;
  if (reset) cudaMemsetAsync(c->d_status, 0, sizeof(int), c->s);
  return st;
}

}  // extern "C"

// ---- allocation-free residual norm ---------------------------------------------------
// Scratch of cosa_gpu_resg_rms_noalloc: per-CTA partial sums, 8 doubles each,
// COSA_NOALLOC_MAX_PARTS rows (256 KiB).  It lives in the library image, so
// every device that loads the library holds it until the process exits.  Host
// code must not pass the symbol itself to a kernel (on the host it is only a
// stand-in); the device address is looked up once per device below.
static __device__ __align__(256) double g_noalloc_rms_part[COSA_NOALLOC_MAX_PARTS * 8];

namespace {
constexpr int kMaxDevices = 64;
double *g_noalloc_part_dev[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;

int noalloc_scratch(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return COSA_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_part_dev[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_rms_part) != cudaSuccess || !p) return COSA_ERR_CUDA;
    g_noalloc_part_dev[dev] = static_cast<double *>(p);
  }
  *out = g_noalloc_part_dev[dev];
  return COSA_OK;
}
}  // namespace

extern "C" int cosa_gpu_resg_rms_noalloc(int32_t nblocks, const int32_t *dims, int32_t npde, int32_t nharms,
                                         const double *res, const double *rhs, double *resrms, void *stream) {
  if (nblocks < 1 || nblocks > COSA_NOALLOC_MAX_PARTS || !dims || !res || !resrms) return COSA_ERR_ARG;
  if ((npde != 5 && npde != 7) || nharms < 0 || 2 * nharms + 1 > COSA_MAX_SNAP) return COSA_ERR_ARG;
  for (int b = 0; b < nblocks; ++b)
    if (dims[3 * b] < 3 || dims[3 * b + 1] < 3 || dims[3 * b + 2] < 2) return COSA_ERR_ARG;
  double *part = nullptr;
  int r = noalloc_scratch(&part);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int per_block = std::max(1, std::min(64, COSA_NOALLOC_MAX_PARTS / nblocks));
  const int S = 2 * nharms + 1;
  int64_t op3 = 0, ncell = 0;
  for (int b = 0; b < nblocks; ++b) {
    DevBlock x{};
    x.im = dims[3 * b]; x.jm = dims[3 * b + 1]; x.km = dims[3 * b + 2];
    x.I3 = x.im + 3; x.J3 = x.jm + 3;
    x.P3 = (int64_t)(x.im + 3) * (x.jm + 3) * (x.km + 3);
    x.op3 = op3;
    k_rms_partial_noalloc<<<per_block, 256, 0, s>>>(x, npde, S, res, rhs, part + (int64_t)b * per_block * 8);
    if (cudaGetLastError() != cudaSuccess) return COSA_ERR_CUDA;
    op3 += x.P3;
    ncell += (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1);
  }
  // resg_rms_hb divides by ncell * dim5 (src/cosa.f90:4620-4626)
  k_rms_final<<<1, 256, 0, s>>>(part, nblocks * per_block, npde, (double)ncell * S, resrms, nullptr, 1);
  if (cudaGetLastError() != cudaSuccess) return COSA_ERR_CUDA;
  return COSA_OK;
}

// ---- laminar viscous path ---------------------------------------------------------------
extern "C" {

// a block's view of node snapshot nh of a moving level's node arrays
// (S2 snapshots per block at op2 * S2)
static DevBlock node_snapshot(const cosa_ctx *c, const DevBlock &b, int nh) {
  DevBlock x = b;
  if (c->p.moving) {
    const int S2 = 2 * c->p.nharms * c->p.hbmove + 1;
    x.op2 = b.op2 * S2 + (int64_t)nh * (b.im + 2) * (b.jm + 2) * (b.km + 2);
  }
  return x;
}

static int node_snapshots(const cosa_ctx *c) { return c->p.moving ? 2 * c->p.nharms * c->p.hbmove + 1 : 1; }

int cosa_gpu_coordex(cosa_ctx *c, int32_t nl, double *x, double *y, double *z) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z) return COSA_ERR_ARG;
  for (int nh = 0; nh < node_snapshots(c); ++nh)
    for (const DevBlock &b : L->hb) {
      const int64_t n = 2 * ((int64_t)b.im * b.km + (int64_t)b.jm * b.km + (int64_t)b.im * b.jm);
      k_coordex<<<grid_for(n), 256, 0, c->s>>>(node_snapshot(c, b, nh), x, y, z);
      int r = after_launch(c);
      if (r) return r;
    }
  return COSA_OK;
}

int cosa_gpu_cutman_x(cosa_ctx *c, int32_t nl, double *x, double *y, double *z) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z) return COSA_ERR_ARG;
  if (L->ncutx == 0) return COSA_OK;
  k_copy_list<<<grid_for(L->ncutx), 256, 0, c->s>>>(L->d_cutx, L->ncutx, x, y, z);
  return after_launch(c);
}

int cosa_gpu_volex(cosa_ctx *c, int32_t nl, double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !vol) return COSA_ERR_ARG;
  for (const DevBlock &b : L->hb) {
    const int64_t n = 2 * ((int64_t)(b.im - 1) * (b.km - 1) + (int64_t)(b.jm - 1) * (b.km - 1) +
                           (int64_t)(b.im - 1) * (b.jm - 1));
    k_volex<<<grid_for(n), 256, 0, c->s>>>(b, vol);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int cosa_gpu_cutman_v(cosa_ctx *c, int32_t nl, double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !vol) return COSA_ERR_ARG;
  if (L->ncutv == 0) return COSA_OK;
  k_copy_list<<<grid_for(L->ncutv), 256, 0, c->s>>>(L->d_cutv, L->ncutv, vol, nullptr, nullptr);
  return after_launch(c);
}

int cosa_gpu_vmetrix(cosa_ctx *c, int32_t nl, const double *x, const double *y, const double *z, const double *vol,
                     double *vm) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z || !vol || !vm) return COSA_ERR_ARG;
  // moving grids: the inverse metrics of every node snapshot, 27 * n0 each
  for (int nh = 0; nh < node_snapshots(c); ++nh)
    for (const DevBlock &b : L->hb)
      for (int d = 1; d <= 3; ++d) {
        k_vmetrix<<<grid_for((int64_t)b.im * b.jm * b.km), 256, 0, c->s>>>(node_snapshot(c, b, nh), d, x, y, z, vol,
                                                                           vm + (int64_t)nh * 27 * L->n0, L->n0);
        int r = after_launch(c);
        if (r) return r;
      }
  return COSA_OK;
}

int cosa_gpu_viscous_setup(cosa_ctx *c, int32_t nl, double *x, double *y, double *z, double *vol, double *vm) {
  LevelState *L = level(c, nl);
  if (!L || !x || !y || !z || !vol || !vm) return COSA_ERR_ARG;
  int r = 0;
  if ((r = cosa_gpu_volex(c, nl, vol)) || (r = cosa_gpu_cutman_v(c, nl, vol)) || (r = cosa_gpu_coordex(c, nl, x, y, z)) ||
      (r = cosa_gpu_cutman_x(c, nl, x, y, z)) || (r = cosa_gpu_vmetrix(c, nl, x, y, z, vol, vm)))
    return r;
  const int S = 2 * c->p.nharms + 1;
  const size_t n3 = (size_t)L->n3 * 5 * S;
  if (!L->d_qprim && (r = dalloc(c, &L->d_qprim, n3))) return r;
  if (!L->d_vres && (r = dalloc(c, &L->d_vres, n3))) return r;
  if (!L->d_vflux && (r = dalloc(c, &L->d_vflux, (size_t)3 * L->n0 * 5 * S))) return r;
  CK(cudaMemsetAsync(L->d_qprim, 0, n3 * sizeof(double), c->s));
  CK(cudaMemsetAsync(L->d_vres, 0, n3 * sizeof(double), c->s));
  CK(cudaMemsetAsync(L->d_vflux, 0, (size_t)3 * L->n0 * 5 * S * sizeof(double), c->s));
  L->d_vm = vm;
  drop_graphs(c);
  return COSA_OK;
}

int cosa_gpu_q_face(cosa_ctx *c, int32_t idir, int32_t nl, const double *q, double *qf) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !q || !qf) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1;
  for (const DevBlock &b : L->hb) {
    const int g = grid_for((int64_t)b.im * b.jm * b.km * S);
    const bool k7 = c->p.npde == 7;
    if (idir == 1) {
      if (k7) k_qface_qder<1, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
      else k_qface_qder<1, 5><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
    } else if (idir == 2) {
      if (k7) k_qface_qder<2, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
      else k_qface_qder<2, 5><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
    } else {
      if (k7) k_qface_qder<3, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
      else k_qface_qder<3, 5><<<g, 256, 0, c->s>>>(b, S, q, qf, nullptr, nullptr, nullptr);
    }
    int r = after_launch(c);
    if (r) return r;
  }
  if (L->walls.empty()) return COSA_OK;
  const int nw = (int)L->walls.size();
  if (c->p.npde == 7)
    k_qwall<7><<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L->d_blocks, L->d_walls, nw, idir, S, q, qf, nullptr,
                                                            nullptr, nullptr);
  else
    k_qwall<5><<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L->d_blocks, L->d_walls, nw, idir, S, q, qf, nullptr,
                                                            nullptr, nullptr);
  return after_launch(c);
}

int cosa_gpu_q_der(cosa_ctx *c, int32_t idir, int32_t nl, const double *q, double *dqxi, double *dqeta,
                   double *dqzeta) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !q || !dqxi || !dqeta || !dqzeta) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1;
  for (const DevBlock &b : L->hb) {
    const int g = grid_for((int64_t)b.im * b.jm * b.km * S);
    const bool k7 = c->p.npde == 7;
    if (idir == 1) {
      if (k7) k_qface_qder<1, 7><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
      else k_qface_qder<1, 5><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
    } else if (idir == 2) {
      if (k7) k_qface_qder<2, 7><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
      else k_qface_qder<2, 5><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
    } else {
      if (k7) k_qface_qder<3, 7><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
      else k_qface_qder<3, 5><<<g, 256, 0, c->s>>>(b, S, q, nullptr, dqxi, dqeta, dqzeta);
    }
    int r = after_launch(c);
    if (r) return r;
  }
  if (L->walls.empty()) return COSA_OK;
  const int nw = (int)L->walls.size();
  if (c->p.npde == 7)
    k_qwall<7><<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L->d_blocks, L->d_walls, nw, idir, S, q, nullptr, dqxi,
                                                            dqeta, dqzeta);
  else
    k_qwall<5><<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L->d_blocks, L->d_walls, nw, idir, S, q, nullptr, dqxi,
                                                            dqeta, dqzeta);
  return after_launch(c);
}

int cosa_gpu_vflux(cosa_ctx *c, int32_t idir, int32_t nl, const double *qf, const double *dqxi, const double *dqeta,
                   const double *dqzeta, const double *vm, const double *sijk, double *flux) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qf || !dqxi || !dqeta || !dqzeta || !vm || !sijk || !flux) return COSA_ERR_ARG;
  if (c->p.npde != 5 || c->p.moving) return COSA_ERR_UNSUPPORTED;
  const int S = 2 * c->p.nharms + 1;
  for (const DevBlock &b : L->hb) {
    k_vflux_ref<<<grid_for((int64_t)b.im * b.jm * b.km * S), 256, 0, c->s>>>(b, idir, c->d_p, qf, dqxi, dqeta, dqzeta,
                                                                            vm, L->n0, sijk, flux);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int cosa_gpu_lambda_ns(cosa_ctx *c, int32_t nl, const double *q, const double *si, const double *sj, const double *sk,
                       const double *vol, const double *mut, double *lam, double *lamv) {
  LevelState *L = level(c, nl);
  if (!L || !q || !si || !sj || !sk || !vol || !lam || !lamv) return COSA_ERR_ARG;
  if (c->p.moving) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_lambda_ns<<<g, 256, 0, c->s>>>(b, c->d_p, q, si, sj, sk, vol, rans(c->p) ? mut : nullptr, lam, lamv);
  });
}

int cosa_gpu_deltat_ns(cosa_ctx *c, int32_t nl, double *dtvol, const double *lam, const double *lamv, double *bx,
                       double *by, double *bz, double *dtvolt, double *tbx, double *tby, double *tbz) {
  LevelState *L = level(c, nl);
  if (!L || !dtvol || !lam || !lamv) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_interior, [&](auto b, dim3 g) {
    k_deltat_ns<<<g, 256, 0, c->s>>>(b, c->d_p, dtvol, lam, lamv, bx, by, bz, rans(c->p) ? dtvolt : nullptr,
                                     rans(c->p) ? tbx : nullptr, tby, tbz);
  });
}

}  // extern "C"

// ---- Wilcox k-omega path ------------------------------------------------------------------
extern "C" {

int cosa_gpu_q_face_mut(cosa_ctx *c, int32_t idir, int32_t nl, const double *mut, double *flux) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !mut || !flux) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  int r = for_blocks(c, *L, cnt_faces, [&](auto b, dim3 g) {
    if (idir == 1) k_qface_mut<1><<<g, 256, 0, c->s>>>(b, npde, S, mut, flux);
    else if (idir == 2) k_qface_mut<2><<<g, 256, 0, c->s>>>(b, npde, S, mut, flux);
    else k_qface_mut<3><<<g, 256, 0, c->s>>>(b, npde, S, mut, flux);
  });
  if (r) return r;
  if (L->walls.empty()) return COSA_OK;
  const int nw = (int)L->walls.size();
  k_qwall_mut<<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L->d_blocks, L->d_walls, nw, idir, npde, S, mut, flux);
  return after_launch(c);
}

int cosa_gpu_rtst(cosa_ctx *c, int32_t idir, int32_t nl, const double *qf, const double *dqxi, const double *dqeta,
                  const double *dqzeta, const double *vm, const double *flux, double *tau1) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qf || !dqxi || !dqeta || !dqzeta || !vm || !flux || !tau1) return COSA_ERR_ARG;
  if (c->p.npde != 7) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_faces, [&](auto b, dim3 g) {
    k_rtst<<<g, 256, 0, c->s>>>(b, idir, c->d_p, qf, dqxi, dqeta, dqzeta, vm, L->n0, flux, tau1);
  });
}

int cosa_gpu_vflux_kom(cosa_ctx *c, int32_t idir, int32_t nl, const double *qf, const double *dqxi,
                       const double *dqeta, const double *dqzeta, const double *tau1, const double *vm,
                       const double *sijk, double *flux, const double *fdist) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qf || !dqxi || !dqeta || !dqzeta || !tau1 || !vm || !sijk || !flux)
    return COSA_ERR_ARG;
  if (c->p.npde != 7 || !rans(c->p) || c->p.moving) return COSA_ERR_UNSUPPORTED;
  if (blend(c->p) != (fdist != nullptr)) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_faces, [&](auto b, dim3 g) {
    k_vflux_kom<<<g, 256, 0, c->s>>>(b, idir, c->d_p, qf, dqxi, dqeta, dqzeta, tau1, vm, L->n0, sijk, flux, fdist);
  });
}

int cosa_gpu_facedist(cosa_ctx *c, int32_t nl, const double *dist, double *fidist, double *fjdist, double *fkdist) {
  LevelState *L = level(c, nl);
  if (!L || !dist || !fidist || !fjdist || !fkdist) return COSA_ERR_ARG;
  for (const DevBlock &x : L->hb) {
    const int64_t nf = (int64_t)x.im * x.jm * x.km;
    k_facedist<1><<<grid_for(nf), 256, 0, c->s>>>(x, dist, fidist);
    k_facedist<2><<<grid_for(nf), 256, 0, c->s>>>(x, dist, fjdist);
    k_facedist<3><<<grid_for(nf), 256, 0, c->s>>>(x, dist, fkdist);
    int r = after_launch(c);
    if (r) return r;
  }
  return COSA_OK;
}

int cosa_gpu_update_ttrm(cosa_ctx *c, int32_t nl, const double *q, const double *dqxi, const double *dqeta,
                         const double *dqzeta, const double *vm, double *ttrm, const double *dist) {
  LevelState *L = level(c, nl);
  if (!L || !q || !dqxi || !dqeta || !dqzeta || !vm || !ttrm || !dist) return COSA_ERR_ARG;
  if (c->p.npde != 7 || !rans(c->p)) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_update_ttrm<<<g, 256, 0, c->s>>>(b, c->d_p, q, dqxi, dqeta, dqzeta, vm, L->n0, ttrm, dist);
  });
}

int cosa_gpu_srckw_sst(cosa_ctx *c, int32_t nl, const double *q, const double *prd, const double *divvel,
                       double *res, const double *mut, const double *ttrm, const double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !q || !prd || !divvel || !res || !mut || !ttrm || !vol) return COSA_ERR_ARG;
  if (c->p.npde != 7 || !blend(c->p)) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_srckw<<<g, 256, 0, c->s>>>(b, c->d_p, nl, q, mut, prd, divvel, res, vol, ttrm);
  });
}

int cosa_gpu_tur_vis_sst(cosa_ctx *c, int32_t nl, const double *q, double *mut, const double *dqxi,
                         const double *dqeta, const double *dqzeta, const double *vm, const double *dist) {
  LevelState *L = level(c, nl);
  if (!L || !q || !mut || !dqxi || !dqeta || !dqzeta || !vm || !dist) return COSA_ERR_ARG;
  if (c->p.npde != 7 || !c->p.kom_sst) return COSA_ERR_UNSUPPORTED;
  const int S = 2 * c->p.nharms + 1;
  int r = for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_tur_vis_sst<<<g, 256, 0, c->s>>>(b, c->d_p, q, mut, dqxi, dqeta, dqzeta, vm, L->n0, dist);
  });
  if (r) return r;
  for (const DevBlock &x : L->hb) {
    const int64_t nh = 2 * ((int64_t)(x.jm - 1) * (x.km - 1) + (int64_t)(x.im - 1) * (x.km - 1) +
                            (int64_t)(x.im - 1) * (x.jm - 1)) * S;
    k_tur_vis_sst_halo<<<grid_for(nh), 256, 0, c->s>>>(x, S, mut);
    if ((r = after_launch(c))) return r;
  }
  return COSA_OK;
}

int cosa_gpu_q_der_c(cosa_ctx *c, int32_t idir, int32_t nl, const double *qf, double *dqc) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qf || !dqc) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1, npde = c->p.npde;
  const int vhi = blend(c->p) ? 7 : 4;  // k and omega too under BSL/SST
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    if (idir == 1) k_qder_c<1><<<g, 256, 0, c->s>>>(b, npde, S, qf, dqc, vhi);
    else if (idir == 2) k_qder_c<2><<<g, 256, 0, c->s>>>(b, npde, S, qf, dqc, vhi);
    else k_qder_c<3><<<g, 256, 0, c->s>>>(b, npde, S, qf, dqc, vhi);
  });
}

int cosa_gpu_turprod(cosa_ctx *c, int32_t nl, const double *dqxi, const double *dqeta, const double *dqzeta,
                     const double *vm, double *prd, double *divvel, double *delpls) {
  LevelState *L = level(c, nl);
  if (!L || !dqxi || !dqeta || !dqzeta || !vm || !prd || !divvel || !delpls) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_turprod<<<g, 256, 0, c->s>>>(b, c->d_p, dqxi, dqeta, dqzeta, vm, L->n0, prd, divvel, delpls);
  });
}

int cosa_gpu_srckw(cosa_ctx *c, int32_t nl, const double *q, const double *mut, const double *prd,
                   const double *divvel, double *res, const double *vol) {
  LevelState *L = level(c, nl);
  if (!L || !q || !mut || !prd || !divvel || !res || !vol) return COSA_ERR_ARG;
  if (c->p.npde != 7) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_srckw<<<g, 256, 0, c->s>>>(b, c->d_p, nl, q, mut, prd, divvel, res, vol, nullptr);
  });
}

// ---- low-speed preconditioning, per routine ----------------------------------------
int cosa_gpu_lm_cutoff_pg(cosa_ctx *c, int32_t nl, const double *q, double *cutoff_pgr) {
  LevelState *L = level(c, nl);
  if (!L || !q || !cutoff_pgr) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_cells,
                    [&](auto b, dim3 g) { k_lm_cutoff_pg<<<g, 256, 0, c->s>>>(b, c->d_p, q, cutoff_pgr); });
}

int cosa_gpu_lm_viscoff(cosa_ctx *c, int32_t nl, const double *q, const double *si, const double *sj,
                        const double *sk, double *cutoff_vis) {
  LevelState *L = level(c, nl);
  if (!L || !q || !si || !sj || !sk || !cutoff_vis) return COSA_ERR_ARG;
  if (!c->p.viscous) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_lm_viscoff<<<g, 256, 0, c->s>>>(b, c->d_p, q, si, sj, sk, cutoff_vis);
  });
}

int cosa_gpu_rest3(cosa_ctx *c, int32_t nl, const double *cutoff1, double *cutoff2, const double *vol1,
                   const double *vol2) {
  LevelState *L1, *L2;
  int r = level_pair(c, nl, L1, L2);
  if (r) return r;
  if (!cutoff1 || !cutoff2 || !vol1 || !vol2) return COSA_ERR_ARG;
  const int S = 2 * c->p.nharms + 1;
  for (int b = 0; b < L2->nb; ++b) {
    const DevBlock &g = L2->hb[b];
    k_rest3<<<grid_for((int64_t)(g.im - 1) * (g.jm - 1) * (g.km - 1) * S), 256, 0, c->s>>>(L1->hb[b], g, S, cutoff1,
                                                                                          cutoff2, vol1, vol2);
    if ((r = after_launch(c))) return r;
  }
  return COSA_OK;
}

int cosa_gpu_proflux(cosa_ctx *c, int32_t idir, int32_t nl, const double *qr, const double *ql, double *flux,
                     const double *sijk, const double *cutoff_pgr, const double *cutoff_vis) {
  LevelState *L = level(c, nl);
  if (!L || idir < 1 || idir > 3 || !qr || !ql || !flux || !sijk || !cutoff_pgr || !cutoff_vis) return COSA_ERR_ARG;
  if (c->p.moving || nl > COSA_MAX_LEVELS) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_faces, [&](auto b, dim3 g) {
    k_proflux<<<g, 256, 0, c->s>>>(b, idir, c->d_p, nl, qr, ql, flux, sijk, cutoff_pgr, cutoff_vis);
  });
}

int cosa_gpu_lambda_p(cosa_ctx *c, int32_t nl, const double *q, const double *si, const double *sj,
                      const double *sk, const double *vol, double *lam, double *lamv, const double *cutoff_pgr,
                      const double *cutoff_vis) {
  LevelState *L = level(c, nl);
  if (!L || !q || !si || !sj || !sk || !lam || !cutoff_pgr || !cutoff_vis) return COSA_ERR_ARG;
  if (c->p.moving || rans(c->p) || nl > COSA_MAX_LEVELS) return COSA_ERR_UNSUPPORTED;
  if (c->p.viscous) {
    if (!vol || !lamv) return COSA_ERR_ARG;
    return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
      k_lambda_ns<<<g, 256, 0, c->s>>>(b, c->d_p, q, si, sj, sk, vol, nullptr, lam, lamv, cutoff_pgr, cutoff_vis, nl);
    });
  }
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_lambda<<<g, 256, 0, c->s>>>(b, c->d_p, q, si, sj, sk, lam, nullptr, nullptr, nullptr, cutoff_pgr, cutoff_vis, nl);
  });
}

int cosa_gpu_lsp(cosa_ctx *c, int32_t nl, const double *q, const double *cutoff_pgr, const double *cutoff_vis,
                 double *prec) {
  LevelState *L = level(c, nl);
  if (!L || !q || !cutoff_pgr || !cutoff_vis || !prec) return COSA_ERR_ARG;
  if (c->p.moving || nl > COSA_MAX_LEVELS) return COSA_ERR_UNSUPPORTED;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_lsp_prec<<<g, 256, 0, c->s>>>(b, c->d_p, nl, q, cutoff_pgr, cutoff_vis, prec);
  });
}

int cosa_gpu_precres(cosa_ctx *c, int32_t nl, double *res, const double *prec) {
  LevelState *L = level(c, nl);
  if (!L || !res || !prec) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) { k_precres<<<g, 256, 0, c->s>>>(b, c->d_p, res, prec); });
}

int cosa_gpu_lsp_cutoffs(cosa_ctx *c, int32_t nl, double *cutoff_pgr, double *cutoff_vis) {
  LevelState *L = level(c, nl);
  if (!L || !cutoff_pgr || !cutoff_vis) return COSA_ERR_ARG;
  if (!L->d_cut_pgr || !L->d_cut_vis) return COSA_ERR_ARG;
  const size_t n = (size_t)L->nm1 * (2 * c->p.nharms + 1) * sizeof(double);
  CK(cudaMemcpyAsync(cutoff_pgr, L->d_cut_pgr, n, cudaMemcpyDeviceToDevice, c->s));
  CK(cudaMemcpyAsync(cutoff_vis, L->d_cut_vis, n, cudaMemcpyDeviceToDevice, c->s));
  return COSA_OK;
}

int cosa_gpu_update_kom(cosa_ctx *c, int32_t nl, const double *res, double *q, const double *qold, const double *vol,
                        const double *dtvolt, const double *delpls, const double *prd, double ar,
                        const double *ttrm) {
  LevelState *L = level(c, nl);
  if (!L || !res || !q || !qold || !vol || !dtvolt || !delpls || !prd) return COSA_ERR_ARG;
  if (c->p.npde != 7 || c->p.rkimp) return COSA_ERR_UNSUPPORTED;
  if (blend(c->p) && !ttrm) return COSA_ERR_ARG;
  return for_blocks(c, *L, cnt_cells, [&](auto b, dim3 g) {
    k_update_kom<<<g, 256, 0, c->s>>>(b, c->d_p, res, q, qold, vol, dtvolt, delpls, prd, ar, ttrm);
  });
}

int cosa_gpu_force(cosa_ctx *c, int32_t nl, const double *q, const double *x, const double *y, const double *z,
                   const double *si, const double *sj, const double *sk, const double *vm, int32_t isurf,
                   const double *xmom, const double *lngth, double *coef) {
  LevelState *L = level(c, nl);
  if (!L || !q || !x || !y || !z || !si || !sj || !sk || !xmom || !lngth || !coef || isurf < 1) return COSA_ERR_ARG;
  const cosa_params &P = c->p;
  if (P.viscous && !vm) return COSA_ERR_ARG;
  // moving viscous grids: the wall derivative of the velocity relative to the
  // grid needs the bound level's cell grid velocities
  const bool mvisc = P.moving && P.viscous;
  if (mvisc && (!L->ptrs.xdot || !L->ptrs.ydot || !L->ptrs.zdot)) return COSA_ERR_ARG;
  if (lngth[0] == 0.0 || lngth[1] == 0.0 || lngth[2] == 0.0) return COSA_ERR_ARG;
  const int S = 2 * P.nharms + 1, nb = L->nb;
  // moment centre of every snapshot: on a pitching grid it moves with the
  // body (src/output.f90:4476-4485), theta_n as in cosa_gpu_movegrid
  std::vector<double> xms((size_t)3 * S);
  {
    const double pi = 3.14159265358979323846, omega = std::fabs(P.omegas);
    const double dt = omega > 0 ? 2 * pi / omega / S : 0.0;
    for (int n = 0; n < S; ++n) {
      double xr = xmom[0], yr = xmom[1];
      if (P.moving) {
        const double dth = P.dtheta0 * std::sin(P.omegas * (n * dt));
        const double dr1 = (xmom[0] - P.xh) * (std::cos(dth) - 1) - (xmom[1] - P.yh) * std::sin(dth);
        const double dr2 = (xmom[0] - P.xh) * std::sin(dth) + (xmom[1] - P.yh) * (std::cos(dth) - 1);
        xr = xmom[0] + dr1;
        yr = xmom[1] + dr2;
      }
      xms[3 * n] = xr; xms[3 * n + 1] = yr; xms[3 * n + 2] = xmom[2];
    }
  }
  auto it = L->forces.find(isurf);
  if (it == L->forces.end()) {
    // faces of the patches with bctopo(1) == 1500 + isurf - 1, block after
    // block, patches and faces in table order
    std::vector<ForceFace> faces;
    std::vector<int> bstart(nb + 1, 0);
    for (int b = 0; b < nb; ++b) {
      bstart[b] = (int)faces.size();
      const DevBlock &db = L->hb[b];
      const int ijk[4] = {0, db.im, db.jm, db.km};
      for (int ib = 0; ib < L->nbcs[b]; ++ib) {
        const int *t = &L->bct[L->obct[b] + 10 * ib];
        if (t[0] != 1500 + isurf - 1) continue;
        const int d = t[1], inrout = t[2];
        if (d < 1 || d > 3 || (inrout != 1 && inrout != 2)) return COSA_ERR_ARG;
        const int c2 = cyc3(d, 2), c3 = cyc3(d, 3);
        const int lo[4] = {0, t[3], t[5], t[7]}, hi[4] = {0, t[4], t[6], t[8]};
        for (int a : {c2, c3})
          if (lo[a] < 1 || hi[a] > ijk[a] - 1) return COSA_ERR_ARG;
        if (ijk[d] < 3) return COSA_ERR_ARG;  // the wall stencil reads two cells in
        const int h = inrout == 1 ? 0 : ijk[d];
        for (int i3 = lo[c3]; i3 <= hi[c3]; ++i3)
          for (int i2 = lo[c2]; i2 <= hi[c2]; ++i2) {
            int idx[4];
            idx[d] = h; idx[c2] = i2; idx[c3] = i3;
            faces.push_back(ForceFace{b, d, inrout == 1 ? 1 : -1, idx[1], idx[2], idx[3]});
          }
      }
    }
    bstart[nb] = (int)faces.size();
    LevelState::ForceList fl;
    fl.nfaces = (int)faces.size();
    int r;
    if ((r = dalloc(c, &fl.d_faces, faces.size())) || (r = dalloc(c, &fl.d_bstart, bstart.size())) ||
        (r = dalloc(c, &fl.d_buf, (size_t)fl.nfaces * 12 * S)) || (r = dalloc(c, &fl.d_sums, (size_t)nb * 12 * S)) ||
        (r = dalloc(c, &fl.d_xmom, (size_t)3 * S)))
      return r;
    if (!faces.empty())
      CK(cudaMemcpyAsync(fl.d_faces, faces.data(), faces.size() * sizeof(ForceFace), cudaMemcpyHostToDevice, c->s));
    CK(cudaMemcpyAsync(fl.d_bstart, bstart.data(), bstart.size() * sizeof(int), cudaMemcpyHostToDevice, c->s));
    CK(cudaStreamSynchronize(c->s));
    it = L->forces.emplace(isurf, fl).first;
  }
  const LevelState::ForceList &fl = it->second;
  std::vector<double> sums((size_t)nb * 12 * S, 0.0);
  if (fl.nfaces > 0) {
    CK(cudaMemcpyAsync(fl.d_xmom, xms.data(), xms.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
    k_force_faces<<<grid_for((int64_t)fl.nfaces * S), 256, 0, c->s>>>(L->d_blocks, c->d_p, fl.d_faces, fl.nfaces, q, x,
                                                                       y, z, si, sj, sk, vm, L->n0, fl.d_xmom,
                                                                       fl.d_buf, mvisc ? L->ptrs.xdot : nullptr,
                                                                       mvisc ? L->ptrs.ydot : nullptr,
                                                                       mvisc ? L->ptrs.zdot : nullptr);
    int r = after_launch(c);
    if (r) return r;
    k_force_sum<<<dim3(nb, S), 256, 0, c->s>>>(fl.d_bstart, fl.nfaces, fl.d_buf, fl.d_sums);
    if ((r = after_launch(c))) return r;
    CK(cudaMemcpyAsync(sums.data(), fl.d_sums, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
  }
  // coefficients of each block, summed in block order (src/output.f90:4870-4893, 4283-4320)
  const double mach = P.machfs > 1e-14 ? P.machfs : 1.0;
  double ss[3], aa[3], bb[3];
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
  const double cf = 2 / (lngth[0] * lngth[1] * mach * mach);
  const double cmf = 2 / (lngth[0] * lngth[1] * lngth[2] * mach * mach);
  for (int n = 0; n < S; ++n) {
    double *o = coef + (size_t)n * 12;
    for (int k = 0; k < 12; ++k) o[k] = 0.0;
    for (int b = 0; b < nb; ++b) {
      const double *g0 = &sums[((size_t)n * nb + b) * 12];
      for (int pv = 0; pv < 2; ++pv) {
        const double *g = g0 + 6 * pv;
        double *cc = o + 6 * pv;
        cc[0] += (g[0] * aa[0] + g[1] * aa[1] + g[2] * aa[2]) * cf;
        cc[1] += (g[0] * ss[0] + g[1] * ss[1] + g[2] * ss[2]) * cf;
        cc[2] += (g[0] * bb[0] + g[1] * bb[1] + g[2] * bb[2]) * cf;
        cc[3] += g[3] * cmf;
        cc[4] += g[4] * cmf;
        cc[5] += g[5] * cmf;
      }
    }
  }
  return COSA_OK;
}

int cosa_gpu_cutman_mut(cosa_ctx *c, int32_t nl, double *mut) {
  LevelState *L = level(c, nl);
  if (!L || !mut) return COSA_ERR_ARG;
  const int ncut = (int)L->items.size() - L->n_bc_items;
  if (ncut == 0) return COSA_OK;
  const int S = 2 * c->p.nharms + 1;
  k_cut_scalar<<<grid_for((int64_t)ncut * S), 256, 0, c->s>>>(L->d_blocks, L->d_items + L->n_bc_items, ncut, S, mut);
  return after_launch(c);
}

}  // extern "C"

namespace {

// q_face (calmut off) of family d into qf and, when g0 is set, q_der into
// g0..g2, bulk faces then strong-boundary faces, for npde = 7
int rans_face_state(cosa_ctx *c, LevelState &L, int d, const double *q, double *qf, double *g0, double *g1,
                    double *g2) {
  const int S = 2 * c->p.nharms + 1;
  int r = for_blocks(c, L, cnt_faces, [&](auto b, dim3 g) {
    if (d == 1) k_qface_qder<1, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, g0, g1, g2);
    else if (d == 2) k_qface_qder<2, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, g0, g1, g2);
    else k_qface_qder<3, 7><<<g, 256, 0, c->s>>>(b, S, q, qf, g0, g1, g2);
  });
  if (r) return r;
  if (L.walls.empty()) return COSA_OK;
  const int nw = (int)L.walls.size();
  k_qwall<7><<<grid_for((int64_t)nw * S), 256, 0, c->s>>>(L.d_blocks, L.d_walls, nw, d, S, q, qf, g0, g1, g2);
  return after_launch(c);
}

// one RK stage of the k-omega path, routine by routine as smooth() runs it
// (src/cosa.f90:1719-2016): every kernel is a full-array pass with the
// reference's arrays, captured with the rest of the iteration in a graph
int launch_rans_stage(cosa_ctx *c, int nl, LevelState &L, int irk, const IterOpts &o) {
  const bool compute_dt = o.compute_dt && irk == 1, want_rms = o.want_rms && irk == o.rms_stage, copy_qold = o.copy_qold;
  const cosa_params &p = c->p;
  const int S = 2 * p.nharms + 1, npde = p.npde;
  const cosa_level_ptrs &P = L.ptrs;
  double *q = P.q;
  int r = 0;
  if (irk == 1 && copy_qold &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_copy_interior<<<g, 256, 0, c->s>>>(b, npde * S, q, P.qold); })))
    return r;
  if ((r = cosa_gpu_cons2prim(c, nl, 0, q))) return r;
  if (!L.items.empty()) {
    // BC patches then cuts, last writers as in the reference
    k_halo<false><<<grid_for((int64_t)L.items.size() * S), 256, 0, c->s>>>(
        L.d_blocks, L.d_items, (int)L.items.size(), c->d_p, q, P.si, P.sj, P.sk, c->d_status, P.dist,
        face_vel_of(c, L));
    if ((r = after_launch(c))) return r;
  }
  if (o.first_cycle && o.force && irk == 1 && !p.prd_all_lvls) {
    // coarse-level mut from the restricted (primitive) state at the first
    // stage of the first cycle's visit (src/cosa.f90:1727-1760); SST takes
    // the cell-centred differences of a copy of q in res, back in
    // conservative form, and zeroes res after
    if (p.kom_sst) {
      const size_t bytes = (size_t)L.n3 * npde * S * sizeof(double);
      CK(cudaMemcpyAsync(P.res, q, bytes, cudaMemcpyDeviceToDevice, c->s));
      double *dc[3] = {P.qp, P.qm, P.dqm};
      for (int d = 1; d <= 3; ++d) {
        if ((r = rans_face_state(c, L, d, P.res, P.dq, nullptr, nullptr, nullptr))) return r;
        if ((r = cosa_gpu_q_der_c(c, d, nl, P.dq, dc[d - 1]))) return r;
      }
      if ((r = cosa_gpu_prim2cons(c, nl, P.res)) ||
          (r = cosa_gpu_tur_vis_sst(c, nl, P.res, P.mut, P.qp, P.qm, P.dqm, L.d_vm, P.dist)))
        return r;
      CK(cudaMemsetAsync(P.res, 0, bytes, c->s));
    } else if ((r = cosa_gpu_tur_vis(c, nl, q, P.mut))) {
      return r;
    }
    if ((r = cosa_gpu_cutman_mut(c, nl, P.mut))) return r;
  }
  if ((r = for_blocks(c, L, cnt_all, [&](auto b, dim3 g) { k_prtest<<<g, 256, 0, c->s>>>(b, c->d_p, q, c->d_status); })))
    return r;
  if (compute_dt) {
    if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           const bool mv = p.moving;
           k_lambda_ns<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.si, P.sj, P.sk, P.vol, P.mut, P.qp, P.dq, nullptr,
                                            nullptr, 1, mv ? P.xdot : nullptr, mv ? P.ydot : nullptr,
                                            mv ? P.zdot : nullptr);
         })))
      return r;
    const bool irs = p.irsop >= 2 && p.irsop != 4;
    if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_deltat_ns<<<g, 256, 0, c->s>>>(b, c->d_p, P.dtvol, P.qp, P.dq, irs ? P.betaxi : nullptr, P.betaeta,
                                            P.betazeta, P.dtvolt, irs ? L.d_tbeta[0] : nullptr, L.d_tbeta[1],
                                            L.d_tbeta[2]);
         })))
      return r;
  }
  if ((r = cosa_gpu_zero(c, nl, P.res))) return r;
  if ((r = launch_edges(c, L, q, P.mut))) return r;
  const bool mixed = p.precision == COSA_PREC_MIXED;
  const int *bct = L.d_bct;
  const BlockList bl{L.d_blocks};
  const int ntr = L.nb * 3 * S;
  if (mixed) k_rans_h0<true><<<grid_for(ntr, 64), 64, 0, c->s>>>(L.d_blocks, L.nb, c->d_p, bct, q, nl, L.d_h0);
  else k_rans_h0<false><<<grid_for(ntr, 64), 64, 0, c->s>>>(L.d_blocks, L.nb, c->d_p, bct, q, nl, L.d_h0);
  if ((r = after_launch(c))) return r;
  // muscl + roflux and q_face / q_der / rtst / vflux of the three families in
  // one launch, then resid of their sums (src/cosa.f90:1797-1824)
  if ((r = for_blocks(c, L, cnt_faces, [&](auto b, dim3 g) {
         (void)b;
         const dim3 g6(g.x * 2, g.y, 6);
         const double *fd = blend(p) ? L.d_fdist : nullptr;
         if (mixed)
           k_rans_faces<true><<<g6, 128, 0, c->s>>>(bl, c->d_p, bct, q, nl, P.si, P.sj, P.sk, L.d_h0, P.mut, L.d_vm,
                                                    L.n0, fd, L.d_rflux, face_vel_of(c, L));
         else
           k_rans_faces<false><<<g6, 128, 0, c->s>>>(bl, c->d_p, bct, q, nl, P.si, P.sj, P.sk, L.d_h0, P.mut, L.d_vm,
                                                     L.n0, fd, L.d_rflux, face_vel_of(c, L));
       })) ||
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
         (void)b;
         k_rans_resid<<<g, 256, 0, c->s>>>(bl, c->d_p, L.n0, L.d_rflux, P.res);
       })))
    return r;
  // cell-centred velocity gradients, production, BSL/SST blending and the
  // sources in one pass over the cells (src/cosa.f90:1878-1901)
  if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
         (void)b;
         if (blend(p))
           k_rans_cellsrc<true><<<g, 256, 0, c->s>>>(bl, c->d_p, nl, bct, q, P.qp, P.qm, P.dqm, L.d_vm, L.n0, P.mut,
                                                    P.dist, P.vol, L.d_prd, L.d_divvel, L.d_delpls, L.d_ttrm, P.res);
         else
           k_rans_cellsrc<false><<<g, 256, 0, c->s>>>(bl, c->d_p, nl, bct, q, P.qp, P.qm, P.dqm, L.d_vm, L.n0, P.mut,
                                                     P.dist, P.vol, L.d_prd, L.d_divvel, L.d_delpls, nullptr, P.res);
       })))
    return r;
  if ((r = cosa_gpu_prim2cons(c, nl, q))) return r;
  // dual time: src_uns, the norm with rhs_uns, res -= rhs_uns on the fine
  // level (src/cosa.f90:1908-1941)
  if (dual_src_in_res(p) &&
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) { k_src_uns<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.vol, P.res); })))
    return r;
  // harmonic balance: src_hb unless rkimp without IRS on one level
  // (src/cosa.f90:1918-1922)
  const bool hb_sir = p.harbal && (!p.rkimp || p.irsop > 0 || p.nlevel > 1);
  if (hb_sir &&
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) { k_src_hb<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.vol, P.res); })))
    return r;
  const bool imp_norm = p.rkimp && ((p.dualt && !dual_src_in_res(p)) || (p.harbal && !hb_sir));
  if (want_rms && (r = launch_norm(c, L, P.res, p.dualt ? P.rhs : nullptr, imp_norm ? q : nullptr))) return r;
  const int nvs = npde * S;
  if (p.dualt && nl == 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, P.res, P.rhs, -1.0); })))
    return r;
  // multigrid forcing: rhs += res at the first stage of a visit from the
  // finer level, then res -= rhs on coarse levels (src/cosa.f90:1950-1960)
  if (o.rhs && o.force && irk == 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, o.rhs, P.res, 1.0); })))
    return r;
  if (o.rhs && nl > 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, P.res, o.rhs, -1.0); })))
    return r;
  if (o.res_only) {
    // residual pass before the restriction (src/cosa.f90:1963-1975)
    if (p.nlevel > 1 && nl != p.nlevel && !p.prd_all_lvls && p.lim_prodtke &&
        (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_lim_prod_mg<<<g, 256, 0, c->s>>>(b, c->d_p, q, L.d_prd, P.mut);
         })))
      return r;
    return for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
      if (p.harbal)
        k_lim_res_ome_bhb<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.qold, P.vol, P.dtvolt, L.d_delpls, L.d_prd,
                                               blend(p) ? L.d_ttrm : nullptr);
      else
        k_lim_res_ome<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.vol, P.dtvolt, L.d_delpls, L.d_prd,
                                           p.alphas[irk - 1], blend(p) ? L.d_ttrm : nullptr);
    });
  }
  if (p.irsop > 0) {
    const double *beta[3] = {P.betaxi ? P.betaxi : L.d_beta[0], P.betaeta ? P.betaeta : L.d_beta[1],
                             P.betazeta ? P.betazeta : L.d_beta[2]};
    const double *tbeta[3] = {L.d_tbeta[0], L.d_tbeta[1], L.d_tbeta[2]};
    if ((r = irs_apply(c, L, P.res, L.d_ores, P.dtvol, beta, P.dtvolt, tbeta))) return r;
  }
  if (p.dualt && p.rkimp) {
    // update_b with the physical-time term implicit (src/update.f90:650-738)
    const int sir = dual_src_in_res(p) ? 1 : 0;
    const double ar = p.alphas[irk - 1];
    const double *tt = blend(p) ? L.d_ttrm : nullptr;
    if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_update_kom_dual<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.qold, P.vol, P.dtvolt, L.d_delpls, L.d_prd, ar,
                                                  tt, sir);
         })) ||
        (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_update_dual<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, P.qold, q, q, nullptr, P.dtvol, P.vol, ar, sir);
         })))
      return r;
  } else if (p.harbal && p.rkimp) {
    // update_bhb: k-omega snapshots coupled per cell, then the mean flow
    const int sir = hb_sir ? 1 : 0;
    const double ar = p.alphas[irk - 1];
    const double *tt = blend(p) ? L.d_ttrm : nullptr;
    if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_update_bhb_kom<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.qold, P.vol, P.dtvolt, L.d_delpls, L.d_prd, ar,
                                                 tt, sir);
         })) ||
        (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_update_bhb<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, P.qold, q, nullptr, P.dtvol, P.vol, ar,
                                             sir ? q : nullptr);
         })))
      return r;
  } else {
    // point-implicit k / omega, the mean-flow update and fixq in one pass
    const double ar = p.alphas[irk - 1];
    const double *tt = blend(p) ? L.d_ttrm : nullptr;
    if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
           k_update_rans<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.qold, P.vol, P.dtvolt, P.dtvol, L.d_delpls,
                                              L.d_prd, ar, tt);
         })))
      return r;
  }
  // k_update_rans applies fixq itself
  if (p.ifixq && p.rkimp && (p.dualt || p.harbal) && (r = cosa_gpu_fixq(c, nl, q))) return r;
  if (irk == p.nstage && (nl == 1 || !p.prd_all_lvls)) {
    // SST: the stage's cell-centred differences are still in qp, qm, dqm
    if (p.kom_sst) r = cosa_gpu_tur_vis_sst(c, nl, q, P.mut, P.qp, P.qm, P.dqm, L.d_vm, P.dist);
    else r = cosa_gpu_tur_vis(c, nl, q, P.mut);
    if (r || (r = cosa_gpu_cutman_mut(c, nl, P.mut))) return r;
  }
  return COSA_OK;
}

// one RK stage of the low-speed preconditioned path (npde = 5, Euler or
// laminar), smooth()'s routines with lomach (src/cosa.f90:1719-2016):
// cons2prim, BCs and cuts, bprtest, the cut-offs, the preconditioned time
// step, the preconditioned convective fluxes (MUSCL + proflux) and the laminar
// viscous ones in one launch, resid, prim2cons, the residual norm, lsp +
// precres, the multigrid forcing, IRS and update_b
int launch_lsp_stage(cosa_ctx *c, int nl, LevelState &L, int irk, const IterOpts &o) {
  const bool compute_dt = o.compute_dt && irk == 1, want_rms = o.want_rms && irk == o.rms_stage;
  const cosa_params &p = c->p;
  const int S = 2 * p.nharms + 1, npde = p.npde;
  const cosa_level_ptrs &P = L.ptrs;
  double *q = P.q;
  const BlockList bl{L.d_blocks};
  const int *bct = L.d_bct;
  double *beta[3] = {P.betaxi ? P.betaxi : L.d_beta[0], P.betaeta ? P.betaeta : L.d_beta[1],
                     P.betazeta ? P.betazeta : L.d_beta[2]};
  int r = 0;
  if (irk == 1 && o.copy_qold &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_copy_interior<<<g, 256, 0, c->s>>>(b, npde * S, q, P.qold); })))
    return r;
  if ((r = cosa_gpu_cons2prim(c, nl, 0, q))) return r;
  if (!L.items.empty()) {
    k_halo<false><<<grid_for((int64_t)L.items.size() * S), 256, 0, c->s>>>(
        L.d_blocks, L.d_items, (int)L.items.size(), c->d_p, q, P.si, P.sj, P.sk, c->d_status, P.dist,
        face_vel_of(c, L));
    if ((r = after_launch(c))) return r;
  }
  if ((r = for_blocks(c, L, cnt_all, [&](auto b, dim3 g) { k_prtest<<<g, 256, 0, c->s>>>(b, c->d_p, q, c->d_status); })))
    return r;
  // Darmofal's pressure-gradient cut-off (every level, or the fine level of a
  // cycle that restricts) and the viscous cut-off (src/cosa.f90:1763-1778)
  const bool fine = (p.nlevel > 1 && nl == 1 && o.to_coarse) || p.nlevel == 1;
  if (((p.cutoff_type == 3 && fine) || p.cutoff_type == 2) &&
      (r = for_blocks(c, L, cnt_cells,
                      [&](auto b, dim3 g) { k_lm_cutoff_pg<<<g, 256, 0, c->s>>>(b, c->d_p, q, L.d_cut_pgr); })))
    return r;
  if (p.visprec && fine && (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
                              k_lm_viscoff<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.si, P.sj, P.sk, L.d_cut_vis);
                            })))
    return r;
  if (compute_dt) {
    // eig_eul_p / eig_ns_p and bdeltat (src/cosa.f90:1447-1590)
    const bool irs = p.irsop >= 2;
    if (p.viscous) {
      if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
             k_lambda_ns<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.si, P.sj, P.sk, P.vol, nullptr, P.qp, P.dq, L.d_cut_pgr,
                                              L.d_cut_vis, nl);
           })) ||
          (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
             k_deltat_ns<<<g, 256, 0, c->s>>>(b, c->d_p, P.dtvol, P.qp, P.dq, irs ? beta[0] : nullptr, beta[1],
                                              beta[2], nullptr, nullptr, nullptr, nullptr);
           })))
        return r;
    } else {
      if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
             k_lambda<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.si, P.sj, P.sk, P.qp, nullptr, nullptr, nullptr, L.d_cut_pgr,
                                           L.d_cut_vis, nl);
           })) ||
          (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
             k_deltat<<<g, 256, 0, c->s>>>(b, c->d_p, P.dtvol, P.qp, irs ? beta[0] : nullptr, beta[1], beta[2]);
           })))
        return r;
    }
  }
  if ((r = cosa_gpu_zero(c, nl, P.res))) return r;
  if (p.viscous && (r = launch_edges(c, L, q, nullptr))) return r;
  // MUSCL + proflux (and the laminar viscous fluxes) of the three families,
  // then resid of their sums (src/cosa.f90:1797-1876)
  if ((r = for_blocks(c, L, cnt_faces, [&](auto b, dim3 g) {
         (void)b;
         const dim3 gz(g.x * 2, g.y, p.viscous ? 6 : 3);
         k_lsp_faces<<<gz, 128, 0, c->s>>>(bl, c->d_p, bct, q, nl, P.si, P.sj, P.sk, L.d_cut_pgr, L.d_cut_vis, L.d_vm,
                                           L.n0, L.d_rflux);
       })) ||
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
         (void)b;
         k_rans_resid<<<g, 256, 0, c->s>>>(bl, c->d_p, L.n0, L.d_rflux, P.res, p.viscous ? 1 : 0);
       })))
    return r;
  if ((r = cosa_gpu_prim2cons(c, nl, q))) return r;
  // unsteady source terms (src/cosa.f90:1908-1922)
  if (dual_src_in_res(p) &&
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) { k_src_uns<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.vol, P.res); })))
    return r;
  if (p.harbal &&
      (r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) { k_src_hb<<<g, 256, 0, c->s>>>(b, c->d_p, q, P.vol, P.res); })))
    return r;
  if (want_rms && (r = launch_norm(c, L, P.res, p.dualt ? P.rhs : nullptr, nullptr))) return r;
  const int nvs = npde * S;
  if (p.dualt && nl == 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, P.res, P.rhs, -1.0); })))
    return r;
  // lsp + precres (src/cosa.f90:1943-1947) on the conservative state
  if ((r = for_blocks(c, L, cnt_cells, [&](auto b, dim3 g) {
         k_lsp_precres<<<g, 256, 0, c->s>>>(b, c->d_p, nl, q, L.d_cut_pgr, L.d_cut_vis, P.res);
       })))
    return r;
  // multigrid forcing (src/cosa.f90:1950-1960)
  if (o.rhs && o.force && irk == 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, o.rhs, P.res, 1.0); })))
    return r;
  if (o.rhs && nl > 1 &&
      (r = for_blocks(c, L, cnt_interior,
                      [&](auto b, dim3 g) { k_add_interior<<<g, 256, 0, c->s>>>(b, nvs, P.res, o.rhs, -1.0); })))
    return r;
  if (o.res_only) return COSA_OK;
  if (p.irsop > 0 && (r = irs_apply(c, L, P.res, L.d_ores, P.dtvol, beta))) return r;
  // update_lsp_b / update_lsp_bhb without k-omega: q = q^n - ar R dt/V
  const double ar = p.alphas[irk - 1];
  return for_blocks(c, L, cnt_interior,
                    [&](auto b, dim3 g) { k_update<<<g, 256, 0, c->s>>>(b, c->d_p, P.res, q, P.qold, P.dtvol, ar); });
}

int launch_rans_iteration(cosa_ctx *c, int nl, LevelState &L, const IterOpts &o) {
  if (o.res_only && o.res_only != L.ptrs.res) return COSA_ERR_ARG;  // the residual pass leaves R in res
  auto stage = [&](int irk) {
    return rans(c->p) ? launch_rans_stage(c, nl, L, irk, o) : launch_lsp_stage(c, nl, L, irk, o);
  };
  if (o.res_only) return stage(1);
  for (int irk = 1; irk <= c->p.nstage; ++irk) {
    int r = stage(irk);
    if (r) return r;
  }
  return COSA_OK;
}

}  // namespace

// ---- stage schedule autotuner -----------------------------------------------------------
namespace {
// warp tasks of k_faces_line, block after block and snapshot after snapshot:
// first every d = 1 task (rows in groups of kLineRows, 31 faces per warp),
// then the d = 2, 3 tasks (lines of 32 lanes in segments of at most kLineSeg
// faces, the two families of a block back to back)
constexpr int kLineRows = 16, kLineSeg = 16;
int build_face_tasks(cosa_ctx *c, LevelState &L) {
  const int S = 2 * c->p.nharms + 1;
  std::vector<FaceTask> t;
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    const int nj = x.jm - 1, nk = x.km - 1;
    for (int n = 0; n < S; ++n)
      for (int k = 1; k <= nk; ++k)
        for (int j0 = 1; j0 <= nj; j0 += kLineRows)
          for (int i0 = 1; i0 <= x.im; i0 += 31)
            t.push_back(FaceTask{b, 1, n, i0, j0, k, 0, std::min(kLineRows, nj - j0 + 1)});
  }
  L.nftasks1 = (int)t.size();
  for (int b = 0; b < L.nb; ++b) {
    const DevBlock &x = L.hb[b];
    const int ni = x.im - 1, nj = x.jm - 1, nk = x.km - 1;
    for (int n = 0; n < S; ++n) {
      for (int d = 2; d <= 3; ++d) {
        const int mx = d == 2 ? x.jm : x.km, nt = d == 2 ? nk : nj;
        const int nseg = (mx + kLineSeg - 1) / kLineSeg, len = (mx + nseg - 1) / nseg;
        for (int tb = 1; tb <= nt; ++tb)
          for (int f0 = 1; f0 <= mx; f0 += len)
            for (int i0 = 1; i0 <= ni; i0 += 32)
              t.push_back(FaceTask{b, d, n, i0, 0, tb, f0, std::min(len, mx - f0 + 1)});
      }
    }
  }
  if (t.size() >= (size_t)1 << 30) return COSA_ERR_UNSUPPORTED;
  int r = dalloc(c, &L.d_ftasks, t.size());
  if (r) return r;
  CK(cudaMemcpy(L.d_ftasks, t.data(), t.size() * sizeof(FaceTask), cudaMemcpyHostToDevice));
  L.nftasks = (int)t.size();
  return COSA_OK;
}

int ensure_split(cosa_ctx *c, LevelState &L) {
  const int S = 2 * c->p.nharms + 1;
  int r = 0;
  if (!L.d_ftasks && (r = build_face_tasks(c, L))) return r;
  // the primitive copy only for viscous flows (the viscous set-up allocates it)
  if (c->p.viscous && !L.d_qprim && (r = dalloc(c, &L.d_qprim, (size_t)L.n3 * 5 * S))) return r;
  if (!L.d_cflux && (r = dalloc(c, &L.d_cflux, (size_t)3 * L.n0 * 5 * S))) return r;
  if (L.npart_cap < L.nb * kCellsGX) {
    drop_graphs(c);
    if ((r = dalloc(c, &L.d_part, (size_t)L.nb * kCellsGX * 8))) return r;
    L.npart_cap = L.nb * kCellsGX;
  }
  return COSA_OK;
}
}  // namespace

extern "C" int cosa_gpu_autotune(cosa_ctx *c, int32_t nl, int32_t niter, double ms[2], int32_t *choice) {
  LevelState *L = level(c, nl);
  if (!L || !L->bound || niter < 1 || !ms) return COSA_ERR_ARG;
  int r = check_fused_supported(c->p);
  if (r) return r;
  ms[0] = ms[1] = 0.0;
  if (routine_stage(c->p)) {  // the k-omega and preconditioned stages have one schedule
    L->schedule = 0;
    if (choice) *choice = 0;
    return COSA_OK;
  }
  cudaSetDevice(c->device);
  if ((r = ensure_split(c, *L))) return r;
  const int S = 2 * c->p.nharms + 1;
  const size_t nq = (size_t)L->n3 * c->p.npde * S;
  double *save = nullptr;
  CK(cudaMalloc(&save, nq * sizeof(double)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaMemcpyAsync(save, L->ptrs.q, nq * sizeof(double), cudaMemcpyDeviceToDevice, c->s);
  for (int sched = 0; sched < 2 && !r; ++sched) {
    L->schedule = sched;
    drop_graphs(c);
    if ((r = cosa_gpu_smooth(c, nl, 1, 1 << 30, 1 << 30, nullptr))) break;  // capture + warm-up
    cudaEventRecord(e0, c->s);
    if ((r = cosa_gpu_smooth(c, nl, niter, 1 << 30, 1 << 30, nullptr))) break;
    cudaEventRecord(e1, c->s);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    ms[sched] = t / niter;
    cudaMemcpyAsync(L->ptrs.q, save, nq * sizeof(double), cudaMemcpyDeviceToDevice, c->s);
  }
  const int best = (!r && ms[1] > 0.0 && ms[1] < ms[0]) ? 1 : 0;
  L->schedule = best;
  drop_graphs(c);
  cudaStreamSynchronize(c->s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(save);
  if (choice) *choice = best;
  return r ? r : cuda_ok(cudaGetLastError());
}

/* force a schedule (0 tile, 1 split) without timing */
extern "C" int cosa_gpu_set_schedule(cosa_ctx *c, int32_t nl, int32_t schedule) {
  LevelState *L = level(c, nl);
  if (!L || schedule < 0 || schedule > 1) return COSA_ERR_ARG;
  if (schedule == 1) {
    int r = ensure_split(c, *L);
    if (r) return r;
  }
  L->schedule = schedule;
  drop_graphs(c);
  return COSA_OK;
}

#include "serve.cuh"
