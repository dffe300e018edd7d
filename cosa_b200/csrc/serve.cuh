// Serving engine: several steady solves resident on one GPU, advanced
// together by the same stage launches.
//
// Included at the end of cosa_gpu.cu (it uses that file's level builder and
// launch helpers).  The engine owns one pool per state / metric array, in
// "slots" of one P3 cell: a solve of n3 P3 cells takes a contiguous range of
// n3 slots in every pool (its P2 and P1 arrays are smaller than its P3 one,
// so they fit the same range).  The active solves' blocks, placed at their
// pool offsets, form one merged level of the engine's context: one k_halo and
// one k_stage_tile launch per RK stage cover every tile of every solve.
// Flow conditions (free stream, inlet total state, outlet pressure) differ
// per solve and reach k_halo through a per-item parameter slot; the scheme
// (gamma, limiter, CFL, RK coefficients) is the engine's.
//
// Each solve's arithmetic touches only its own cells, its residual norm is
// reduced over its own tiles in a fixed order, and it is checked for
// convergence every check_every of its own iterations: a solve gives the
// same result alone and among others.  The convergence test is the
// residual drop rms / rms(first iteration) < tol on the total norm.
#pragma once
#include <chrono>
#include <deque>
#include <map>

namespace {

enum { SOLVE_QUEUED = 0, SOLVE_ACTIVE = 1, SOLVE_CONVERGED = 2, SOLVE_STOPPED = 3, SOLVE_FAILED = 4 };

struct ServeSolve {
  int state = SOLVE_QUEUED;
  int nb = 0, ncuts = 0;
  std::vector<int32_t> dims, nbcs, bct, cut;
  std::vector<double> x, y, z, q0;  // host inputs, released at admission
  cosa_params flow{};
  double tol = 0;
  int max_iter = 0;
  int64_t n3 = 0, n2 = 0, n1 = 0, off = -1, ncell = 0;
  std::vector<int64_t> lop;         // per block: local P3, P2, P1 offsets
  int64_t ntiles = 0;
  int iters = 0;
  double rms0 = 0, rms = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  std::vector<double> result;       // P3 state after retirement
};

constexpr int64_t kSlotBytes = (3 * 5 + 2 + 3 * 4) * 8;  // Q, T, QO (5 each), DT, VOL, SI, SJ, SK (4 each)

// per block of the merged level: 1 when an interior cell of the conservative
// state has rho <= qmin(1), p <= qmin(5) or a non-finite value (the
// positivity test of bprtest, src/cosa.f90:960-1120, used to find the solve
// that set the shared status word)
__global__ void k_block_bad(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                            const double *__restrict__ q, int *__restrict__ bad) {
  const DevBlock b = blocks[blockIdx.y];
  const cosa_params &P = *Pp;
  const int ni = b.im - 1, nj = b.jm - 1, nk = b.km - 1;
  const int64_t total = (int64_t)ni * nj * nk;
  int found = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1;
    const int k = (int)(r / nj) + 1;
    const int64_t c = p3_cell(b, i, j, k);
    double v[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) v[m] = q[p3_var(b, 5, 1, m + 1, 0) + c];
    const double pr = (P.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
    const bool ok = isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]) && isfinite(v[3]) && isfinite(v[4]) &&
                    v[0] > P.qmin[0] && pr > P.qmin[4];
    found |= ok ? 0 : 1;
  }
  if (__syncthreads_or(found) && threadIdx.x == 0) bad[blockIdx.y] = 1;
}

}  // namespace

struct cosa_serve {
  cosa_ctx *c = nullptr;
  int64_t cap = 0;
  double *Q = nullptr, *T = nullptr, *QO = nullptr, *DT = nullptr, *VOL = nullptr;
  double *SI = nullptr, *SJ = nullptr, *SK = nullptr;
  std::map<int64_t, int64_t> free_;  // offset -> length, in slots
  std::vector<ServeSolve> solves;    // index = request id
  std::deque<int64_t> queue;
  std::vector<int64_t> active;       // ids in the merged level's block order
  cosa_params *d_ps = nullptr;
  int ps_cap = 0;
  int *d_bad = nullptr;  // per-block positivity flags of the merged level
  int bad_cap = 0;
  int check_every = 10;
  bool dirty = true;
  uint64_t gen = 0;
  std::chrono::steady_clock::time_point t0;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

int64_t pool_alloc(cosa_serve *e, int64_t n) {
  for (auto it = e->free_.begin(); it != e->free_.end(); ++it) {
    if (it->second < n) continue;
    const int64_t off = it->first, len = it->second;
    e->free_.erase(it);
    if (len > n) e->free_[off + n] = len - n;
    return off;
  }
  return -1;
}

void pool_free(cosa_serve *e, int64_t off, int64_t n) {
  auto it = e->free_.emplace(off, n).first;
  auto nx = std::next(it);
  if (nx != e->free_.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    e->free_.erase(nx);
  }
  if (it != e->free_.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      e->free_.erase(it);
    }
  }
}

// the device tables of a level built by build_level, released before a rebuild
void free_level_tables(cosa_ctx *c, LevelState &L) {
  void *owned[] = {L.d_blocks, L.d_bct, L.d_items, L.d_strong, L.d_smap, L.d_tiles};
  for (void *v : owned) {
    if (!v) continue;
    cudaFree(v);
    c->allocs.erase(std::remove(c->allocs.begin(), c->allocs.end(), v), c->allocs.end());
  }
  double *part = L.d_part;
  const int cap = L.npart_cap;
  L = LevelState{};
  L.d_part = part;
  L.npart_cap = cap;
}

int64_t tiles_of(const int32_t *d) {
  const int64_t ni = d[0] - 1, nj = d[1] - 1, nk = d[2] - 1;
  return ((nk + 31) / 32) * ((nj + kTJ - 1) / kTJ) * ((ni + kTI - 1) / kTI);
}

// merged level of the active solves at their pool offsets
int serve_rebuild(cosa_serve *e) {
  cosa_ctx *c = e->c;
  LevelState &L = c->L[0];
  drop_graphs(c);
  free_level_tables(c, L);
  c->nseg = 0;
  const int na = (int)e->active.size();
  if (na == 0) { e->dirty = false; return COSA_OK; }
  std::vector<int32_t> dims, nbcs, bct, cut;
  std::vector<int64_t> offs;
  std::vector<int> bps;
  std::vector<int> seg;
  std::vector<double> segn, cflb;
  int nb = 0;
  int64_t tile0 = 0;
  for (int a = 0; a < na; ++a) {
    const ServeSolve &s = e->solves[(size_t)e->active[a]];
    dims.insert(dims.end(), s.dims.begin(), s.dims.end());
    nbcs.insert(nbcs.end(), s.nbcs.begin(), s.nbcs.end());
    bct.insert(bct.end(), s.bct.begin(), s.bct.end());
    for (int ic = 0; ic < s.ncuts; ++ic) {
      int32_t rec[21];
      std::copy(s.cut.begin() + 21 * ic, s.cut.begin() + 21 * (ic + 1), rec);
      rec[0] += nb;  // block numbers of the merged level
      rec[9] += nb;
      cut.insert(cut.end(), rec, rec + 21);
    }
    for (int b = 0; b < s.nb; ++b) {
      offs.push_back(s.off + s.lop[3 * b]);
      offs.push_back(s.off + s.lop[3 * b + 1]);
      offs.push_back(s.off + s.lop[3 * b + 2]);
      bps.push_back(a);
      cflb.push_back(s.flow.cfl > 0 ? s.flow.cfl : c->p.cfl);
    }
    seg.push_back((int)tile0);
    seg.push_back((int)s.ntiles);
    segn.push_back((double)s.ncell);
    tile0 += s.ntiles;
    nb += s.nb;
  }
  cosa_level_desc d{nb, dims.data(), nbcs.data(), bct.data(), (int32_t)(cut.size() / 21), cut.data()};
  int r = build_level(c, L, d, offs.data(), bps.data());
  if (r) return r;
  if (L.ntiles != tile0) return COSA_ERR_ARG;
  // per-solve flow conditions on the scheme's parameters
  if (e->ps_cap < na) {
    if (e->d_ps) { cudaFree(e->d_ps); e->d_ps = nullptr; }
    CK(cudaMalloc(&e->d_ps, (size_t)na * sizeof(cosa_params)));
    e->ps_cap = na;
  }
  std::vector<cosa_params> ps((size_t)na);
  for (int a = 0; a < na; ++a) ps[(size_t)a] = e->solves[(size_t)e->active[a]].flow;
  CK(cudaMemcpyAsync(e->d_ps, ps.data(), ps.size() * sizeof(cosa_params), cudaMemcpyHostToDevice, c->s));
  c->d_halo_p = e->d_ps;
  // residual-norm segments and their output rows
  if ((r = ensure_hist(c, na))) return r;
  // each solve's CFL number on its blocks (the flow conditions' cfl, else the scheme's)
  if (c->d_cfl_blk) { cudaFree(c->d_cfl_blk); c->d_cfl_blk = nullptr; }
  CK(cudaMalloc(&c->d_cfl_blk, cflb.size() * sizeof(double)));
  CK(cudaMemcpyAsync(c->d_cfl_blk, cflb.data(), cflb.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
  if (c->d_seg) { cudaFree(c->d_seg); c->d_seg = nullptr; }
  if (c->d_seg_ncell) { cudaFree(c->d_seg_ncell); c->d_seg_ncell = nullptr; }
  CK(cudaMalloc(&c->d_seg, seg.size() * sizeof(int)));
  CK(cudaMalloc(&c->d_seg_ncell, segn.size() * sizeof(double)));
  CK(cudaMemcpyAsync(c->d_seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice, c->s));
  CK(cudaMemcpyAsync(c->d_seg_ncell, segn.data(), segn.size() * sizeof(double), cudaMemcpyHostToDevice, c->s));
  c->nseg = na;
  if (L.npart_cap < L.ntiles) {
    if (L.d_part) cudaFree(L.d_part);
    L.d_part = nullptr;
    CK(cudaMalloc(&L.d_part, (size_t)L.ntiles * 8 * sizeof(double)));
    L.npart_cap = L.ntiles;
  }
  L.ptrs = cosa_level_ptrs{};
  L.ptrs.q = e->Q; L.ptrs.qold = e->QO; L.ptrs.dtvol = e->DT;
  L.ptrs.si = e->SI; L.ptrs.sj = e->SJ; L.ptrs.sk = e->SK; L.ptrs.vol = e->VOL;
  L.d_T = e->T;
  L.bound = true;
  CK(cudaStreamSynchronize(c->s));
  e->dirty = false;
  ++e->gen;
  return COSA_OK;
}

// place queued solves (first come, first served) while the pool has room
int serve_admit(cosa_serve *e) {
  cosa_ctx *c = e->c;
  while (!e->queue.empty()) {
    ServeSolve &s = e->solves[(size_t)e->queue.front()];
    const int64_t off = pool_alloc(e, s.n3);
    if (off < 0) break;
    s.off = off;
    // grid into scratch, metrics and volumes into the pools
    double *g = nullptr;
    CK(cudaMalloc(&g, (size_t)s.n2 * 3 * sizeof(double)));
    int r = cuda_ok(cudaMemcpyAsync(g, s.x.data(), s.n2 * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (!r) r = cuda_ok(cudaMemcpyAsync(g + s.n2, s.y.data(), s.n2 * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (!r) r = cuda_ok(cudaMemcpyAsync(g + 2 * s.n2, s.z.data(), s.n2 * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (!r) r = cuda_ok(cudaMemcpyAsync(e->Q + off * 5, s.q0.data(), s.n3 * 5 * sizeof(double),
                                        cudaMemcpyHostToDevice, c->s));
    double *sd[3] = {e->SI + off * 4, e->SJ + off * 4, e->SK + off * 4};
    for (int b = 0; b < s.nb && !r; ++b) {
      DevBlock x{};
      x.im = s.dims[3 * b]; x.jm = s.dims[3 * b + 1]; x.km = s.dims[3 * b + 2];
      x.I3 = x.im + 3; x.J3 = x.jm + 3;
      x.P3 = (int64_t)(x.im + 3) * (x.jm + 3) * (x.km + 3);
      x.op3 = s.lop[3 * b]; x.op2 = s.lop[3 * b + 1]; x.op1 = s.lop[3 * b + 2];
      for (int dd = 1; dd <= 3 && !r; ++dd) {
        k_imetrix<<<grid_for((int64_t)(x.im + 1) * (x.jm + 1) * (x.km + 1)), 256, 0, c->s>>>(x, dd, g, g + s.n2,
                                                                                           g + 2 * s.n2, sd[dd - 1]);
        r = after_launch(c);
      }
      if (!r) {
        k_vols<<<grid_for((int64_t)x.im * x.jm * x.km), 256, 0, c->s>>>(x, g, g + s.n2, g + 2 * s.n2, e->VOL + off);
        r = after_launch(c);
      }
    }
    if (!r) r = cuda_ok(cudaStreamSynchronize(c->s));
    cudaFree(g);
    if (r) { pool_free(e, off, s.n3); return r; }
    std::vector<double>().swap(s.x);
    std::vector<double>().swap(s.y);
    std::vector<double>().swap(s.z);
    std::vector<double>().swap(s.q0);
    s.state = SOLVE_ACTIVE;
    s.t_admit = e->now();
    e->active.push_back(e->queue.front());
    e->queue.pop_front();
    e->dirty = true;
  }
  return COSA_OK;
}

// one RK iteration of every active solve (graph per active set and norm flag)
int serve_iteration(cosa_serve *e, bool want_rms) {
  cosa_ctx *c = e->c;
  const uint64_t key = (3ull << 56) | ((e->gen & 0xffffffffull) << 8) | (want_rms ? 1u : 0u);
  return run_graph(c, key, [&] {
    IterOpts o;
    o.want_rms = want_rms;
    o.compute_dt = 1;
    int r = launch_iteration(c, 1, c->L[0], o);
    if (r || !want_rms) return r;
    return COSA_OK;
  });
}

// the retiring solves' states back to the host; their slots back to the pool
int serve_retire(cosa_serve *e, const std::vector<int64_t> &done) {
  cosa_ctx *c = e->c;
  LevelState &L = c->L[0];
  // face halos of the state in conservative form, as after smooth()
  if (!L.items.empty()) {
    const double *last_in = (c->p.nstage % 2 == 1) ? e->Q : e->T;
    k_halo_p2c<<<grid_for((int64_t)L.items.size()), 256, 0, c->s>>>(L.d_blocks, L.d_items, (int)L.items.size(),
                                                                   c->d_p, last_in, e->Q);
    int r = after_launch(c);
    if (r) return r;
  }
  for (int64_t id : done) {
    ServeSolve &s = e->solves[(size_t)id];
    s.result.resize((size_t)(s.n3 * 5));
    CK(cudaMemcpyAsync(s.result.data(), e->Q + s.off * 5, s.n3 * 5 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
  }
  CK(cudaStreamSynchronize(c->s));
  const double t = e->now();
  for (int64_t id : done) {
    ServeSolve &s = e->solves[(size_t)id];
    pool_free(e, s.off, s.n3);
    s.t_done = t;
    e->active.erase(std::find(e->active.begin(), e->active.end(), id));
  }
  e->dirty = true;
  return COSA_OK;
}

}  // namespace

extern "C" {

int cosa_serve_create(const cosa_params *scheme, int64_t budget_bytes, int32_t device, int32_t check_every,
                      cosa_serve **out) {
  if (!scheme || !out || budget_bytes < kSlotBytes || check_every < 1) return COSA_ERR_ARG;
  if (scheme->npde != 5 || scheme->nharms != 0 || scheme->irsop != 0 || scheme->iupdt != 1 || scheme->viscous)
    return COSA_ERR_UNSUPPORTED;
  int r = check_fused_supported(*scheme);
  if (r) return r;
  // a one-level context over a placeholder block; its level is rebuilt from the active set
  const int32_t dims[3] = {3, 3, 2}, nbcs[1] = {0};
  cosa_level_desc d{1, dims, nbcs, nullptr, 0, nullptr};
  cosa_ctx *c = nullptr;
  if ((r = cosa_gpu_init(scheme, 1, &d, device, &c))) return r;
  cosa_serve *e = new (std::nothrow) cosa_serve;
  if (!e) { cosa_gpu_finalize(c); return COSA_ERR_ARG; }
  e->c = c;
  e->check_every = check_every;
  e->cap = budget_bytes / kSlotBytes;
  double **pools[8] = {&e->Q, &e->T, &e->QO, &e->DT, &e->VOL, &e->SI, &e->SJ, &e->SK};
  const int width[8] = {5, 5, 5, 1, 1, 4, 4, 4};
  for (int i = 0; i < 8 && !r; ++i) r = dalloc(c, pools[i], (size_t)(e->cap * width[i]));
  if (!r) r = cuda_ok(cudaMemset(e->T, 0, (size_t)e->cap * 5 * sizeof(double)));
  if (r) { cosa_gpu_finalize(c); delete e; return r; }
  e->free_[0] = e->cap;
  e->t0 = std::chrono::steady_clock::now();
  *out = e;
  return COSA_OK;
}

int cosa_serve_destroy(cosa_serve *e) {
  if (!e) return COSA_ERR_ARG;
  cosa_ctx *c = e->c;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->s);
  if (e->d_ps) cudaFree(e->d_ps);
  if (e->d_bad) cudaFree(e->d_bad);
  if (c->d_seg) cudaFree(c->d_seg);
  if (c->d_seg_ncell) cudaFree(c->d_seg_ncell);
  if (c->d_cfl_blk) cudaFree(c->d_cfl_blk);
  if (c->L[0].d_part) cudaFree(c->L[0].d_part);
  c->L[0].d_part = nullptr;
  cosa_gpu_finalize(c);
  delete e;
  return COSA_OK;
}

int cosa_serve_submit(cosa_serve *e, const cosa_level_desc *grid, const double *x, const double *y, const double *z,
                      const double *q0, const cosa_params *flow, double tol, int32_t max_iter, int64_t *id) {
  if (!e || !grid || !x || !y || !z || !q0 || !flow || !id || grid->nblocks < 1 || max_iter < 1) return COSA_ERR_ARG;
  const cosa_params &sc = e->c->p;
  if (flow->npde != sc.npde || flow->nharms != 0 || flow->gamma != sc.gamma) return COSA_ERR_ARG;
  ServeSolve s;
  s.nb = grid->nblocks;
  s.ncuts = grid->ncuts;
  s.dims.assign(grid->dims, grid->dims + 3 * s.nb);
  s.nbcs.assign(grid->nbcs, grid->nbcs + s.nb);
  int64_t nbct = 0;
  for (int b = 0; b < s.nb; ++b) nbct += 10 * (int64_t)s.nbcs[(size_t)b];
  if (nbct) s.bct.assign(grid->bctopo, grid->bctopo + nbct);
  if (s.ncuts) s.cut.assign(grid->cutopo, grid->cutopo + 21 * (int64_t)s.ncuts);
  for (int b = 0; b < s.nb; ++b) {
    const int64_t im = s.dims[3 * b], jm = s.dims[3 * b + 1], km = s.dims[3 * b + 2];
    if (im < 3 || jm < 3 || km < 3) return COSA_ERR_ARG;  // no one-cell-thick blocks here
    s.lop.push_back(s.n3); s.lop.push_back(s.n2); s.lop.push_back(s.n1);
    s.n3 += (im + 3) * (jm + 3) * (km + 3);
    s.n2 += (im + 2) * (jm + 2) * (km + 2);
    s.n1 += (im + 1) * (jm + 1) * (km + 1);
    s.ncell += (im - 1) * (jm - 1) * (km - 1);
    s.ntiles += tiles_of(s.dims.data() + 3 * b);
  }
  if (s.n3 > e->cap) return COSA_ERR_ARG;  // can never be admitted
  s.x.assign(x, x + s.n2);
  s.y.assign(y, y + s.n2);
  s.z.assign(z, z + s.n2);
  s.q0.assign(q0, q0 + s.n3 * 5);
  s.flow = sc;  // the engine's scheme with this request's flow conditions
  s.flow.machfs = flow->machfs; s.flow.alpha = flow->alpha; s.flow.beta = flow->beta;
  s.flow.rhoinf = flow->rhoinf; s.flow.pinf = flow->pinf; s.flow.ainf = flow->ainf; s.flow.tinf = flow->tinf;
  s.flow.inlet_t0 = flow->inlet_t0; s.flow.inlet_p0 = flow->inlet_p0;
  for (int i = 0; i < 3; ++i) { s.flow.inlet_dir[i] = flow->inlet_dir[i]; s.flow.outlet_p[i] = flow->outlet_p[i]; }
  if (flow->cfl > 0) s.flow.cfl = flow->cfl;  // the request's own CFL number (local time step)
  s.tol = tol;
  s.max_iter = max_iter;
  s.t_submit = e->now();
  *id = (int64_t)e->solves.size();
  e->solves.push_back(std::move(s));
  e->queue.push_back(*id);
  return COSA_OK;
}

int cosa_serve_step(cosa_serve *e, int32_t niter, int32_t *nactive, int32_t *nqueued) {
  if (!e || niter < 0) return COSA_ERR_ARG;
  cosa_ctx *c = e->c;
  cudaSetDevice(c->device);
  const int npde = c->p.npde;
  int r = 0;
  for (int it = 0; it < niter; ++it) {
    if ((r = serve_admit(e))) return r;
    if (e->dirty && (r = serve_rebuild(e))) return r;
    if (e->active.empty()) break;
    // a solve's norm is taken on its iterations 1, check_every+1, 2 check_every+1, ...
    bool want = false;
    for (int64_t id : e->active) want |= e->solves[(size_t)id].iters % e->check_every == 0;
    if ((r = serve_iteration(e, want))) return r;
    std::vector<double> h;
    if (want) {
      h.resize(e->active.size() * (npde + 1));
      CK(cudaMemcpyAsync(h.data(), c->d_hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->s));
      CK(cudaStreamSynchronize(c->s));
    }
    std::vector<int64_t> done;
    for (size_t a = 0; a < e->active.size(); ++a) {
      ServeSolve &s = e->solves[(size_t)e->active[a]];
      const bool due = s.iters % e->check_every == 0;
      s.iters += 1;
      if (due) {
        const double rms = h[a * (npde + 1) + npde];
        if (s.iters == 1) s.rms0 = rms;
        s.rms = rms;
        if (!std::isfinite(rms)) { s.state = SOLVE_FAILED; done.push_back(e->active[a]); continue; }
        if (s.rms0 > 0 && rms < s.tol * s.rms0) { s.state = SOLVE_CONVERGED; done.push_back(e->active[a]); continue; }
      }
      if (s.iters >= s.max_iter) { s.state = SOLVE_STOPPED; done.push_back(e->active[a]); }
    }
    if (!done.empty() && (r = serve_retire(e, done))) return r;
  }
  const int st = cosa_gpu_status(c, 1);
  const int soft = COSA_ERR_NEG_P | COSA_ERR_NEG_RHO | COSA_ERR_NAN;
  if (st & ~soft) return st;
  if (st && !e->active.empty() && !e->dirty) {
    // a solve lost positivity: the status word is shared, so find the
    // solves whose blocks hold a bad cell and retire them as failed; the
    // other solves never read their cells and go on
    LevelState &L = c->L[0];
    if (e->bad_cap < L.nb) {
      if (e->d_bad) { cudaFree(e->d_bad); e->d_bad = nullptr; }
      CK(cudaMalloc(&e->d_bad, (size_t)L.nb * sizeof(int)));
      e->bad_cap = L.nb;
    }
    CK(cudaMemsetAsync(e->d_bad, 0, (size_t)L.nb * sizeof(int), c->s));
    int64_t mc = 1;
    for (const DevBlock &x : L.hb) mc = std::max<int64_t>(mc, (int64_t)(x.im - 1) * (x.jm - 1) * (x.km - 1));
    k_block_bad<<<dim3(grid_x(mc, L.nb), L.nb), 256, 0, c->s>>>(L.d_blocks, c->d_p, e->Q, e->d_bad);
    if ((r = after_launch(c))) return r;
    std::vector<int> bad((size_t)L.nb);
    CK(cudaMemcpyAsync(bad.data(), e->d_bad, bad.size() * sizeof(int), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    std::vector<int64_t> failed;
    int b0 = 0;
    for (int64_t id : e->active) {
      ServeSolve &s = e->solves[(size_t)id];
      bool any = false;
      for (int b = 0; b < s.nb; ++b) any |= bad[(size_t)(b0 + b)] != 0;
      b0 += s.nb;
      if (any) { s.state = SOLVE_FAILED; failed.push_back(id); }
    }
    if (!failed.empty() && (r = serve_retire(e, failed))) return r;
  }
  if (nactive) *nactive = (int32_t)e->active.size();
  if (nqueued) *nqueued = (int32_t)e->queue.size();
  return COSA_OK;
}

int cosa_serve_result(cosa_serve *e, int64_t id, int32_t *state, int32_t *iters, double *rms_drop, double times[3],
                      double *q_out) {
  if (!e || id < 0 || id >= (int64_t)e->solves.size()) return COSA_ERR_ARG;
  const ServeSolve &s = e->solves[(size_t)id];
  if (state) *state = s.state;
  if (iters) *iters = s.iters;
  if (rms_drop) *rms_drop = s.rms0 > 0 ? s.rms / s.rms0 : 0.0;
  if (times) { times[0] = s.t_submit; times[1] = s.t_admit; times[2] = s.t_done; }
  if (q_out && !s.result.empty()) std::copy(s.result.begin(), s.result.end(), q_out);
  return COSA_OK;
}

int64_t cosa_serve_free_slots(cosa_serve *e) {
  if (!e) return -1;
  int64_t n = 0;
  for (auto &kv : e->free_) n += kv.second;
  return n;
}

}  // extern "C"
