/*
 * cosa_gpu.h -- C-ABI of the B200 (sm_100a) explicit residual-and-update
 * path of COSA (LANCASTER-CFD/COSA, Fortran 90).
 *
 * COSA's hot routines are external Fortran procedures with implicit
 * interfaces that receive flat real(8) arrays (Cray pointers p_q(nl), ...,
 * src/cosa_variables.f90:184-211) and read every scalar from module
 * globals (src/common_variables.f90:11-129).  This header replaces them
 * one-for-one:
 *
 *   - the module globals become the POD struct cosa_params (uploaded once
 *     per solve) plus per-level block/BC/cut tables (cosa_level_desc);
 *   - every array argument is a DEVICE pointer to an array with exactly the
 *     reference's shape and block concatenation (offsets as in setoffs,
 *     src/input.f90:5502-5585), so the Fortran driver's arrays map 1:1;
 *   - every entry point returns an int status (0 = ok, COSA_ERR_* bits)
 *     instead of calling `stop` (src/cosa.f90:985-1000, src/bc.f90:1100-1105).
 *
 * Array shapes per block (node counts imax,jmax,kmax of the level; S =
 * 2*nharms+1 snapshots), all column-major with i fastest:
 *   P3 arrays (q, qold, res, rhs, qp, qm, dq, dqp, dqm, lambdas):
 *       (-1:imax+1,-1:jmax+1,-1:kmax+1, npde, 0:S-1)
 *   P2 metric arrays (si, sj, sk):   (lmet=4, 0:imax+1,0:jmax+1,0:kmax+1, 0:S*hbmove-1... )
 *   P1 arrays (vol):                 (0:imax,0:jmax,0:kmax)
 *   P1 x S arrays (dtvol, dtvolt, beta*):  (0:imax,0:jmax,0:kmax, 0:S-1)
 *   F0 arrays (flux):                (imax,jmax,kmax, npde, 0:S-1)
 *   Grid (x, y, z):                  (0:imax+1,0:jmax+1,0:kmax+1)
 */
#ifndef COSA_GPU_H
#define COSA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COSA_MAX_SNAP 15   /* 2*NH+1 for NH <= 7 */
#define COSA_MAX_LEVELS 3  /* nlevel <= 3 in mg(), src/cosa.f90:806-930 */

/* status bits (replace the reference's fatal stops) */
#define COSA_OK              0
#define COSA_ERR_NEG_P       0x001 /* p <= qmin(5): bprtest, src/cosa.f90:1000-1040 */
#define COSA_ERR_NEG_RHO     0x002 /* rho <= qmin(1): bprtest */
#define COSA_ERR_INFLOW      0x004 /* inlet Newton > 10 iterations, src/bc.f90:1100-1105 */
#define COSA_ERR_NAN         0x008 /* non-finite residual norm */
#define COSA_ERR_ARG         0x010 /* bad argument / size / level */
#define COSA_ERR_CUDA        0x020 /* CUDA runtime error */
#define COSA_ERR_TIMEOUT     0x040 /* a bounded device wait ran out */
#define COSA_ERR_UNSUPPORTED 0x080 /* option outside the implemented path */

/* precision of the reconstruction / Roe flux (state always FP64) */
#define COSA_PREC_FP64  0
#define COSA_PREC_MIXED 1

/*
 * Physics and scheme parameters: the common_variables module globals the
 * hot path reads (src/common_variables.f90:19-50), with the defaults of
 * input() (src/input.f90:2400-2540).  Boolean flags are int32 0/1.
 */
typedef struct cosa_params {
  /* flow */
  double gamma, machfs, alpha, beta, reyno, pranl, prant, stemp;
  double pinf, rhoinf, ainf, tinf;
  /* MUSCL + limiters (src/flux.f90:1221-1810, 3472-3888) */
  double rkap, epslimf, epslimt;
  int32_t ilimf, ilimt;
  int32_t nl_crs;       /* first-order on levels nl >= nl_crs */
  int32_t foturb;       /* first-order turbulence equations */
  /* Roe entropy fix / eigenvalue cut-off (src/flux.f90:162-200) */
  int32_t efx_setup_f, efx_all_f, eig_limit_f, eig_lim_all_f;
  int32_t efx_setup_t, efx_all_t, eig_limit_t, eig_lim_all_t;
  int32_t entfx_f_w[3], entfx_t_w[3];
  double cntrpy_f, entfxctf_f, eig_cutoff_f;
  double cntrpy_t, entfxctf_t, eig_cutoff_t;
  /* local time step, IRS (src/cosa.f90:4733-5203, 2035-2443) */
  double cfl, cflt, cdff, rat, ratt, psirs;
  int32_t irsop, cutcirs, iupdt, nstage;
  double alphas[5];     /* RK coefficients: ar4 = (0.25,0.333333,0.5,1.0) */
  /* equation set / flags */
  int32_t npde, nharms, hbmove, lmet;
  int32_t viscous, kom, kom_bsl, kom_sst, harbal, rkimp, moving;
  int32_t aircraft, rgkuns, dualt, nlevel;
  double qmin[7];
  /* k-omega (src/input.f90:2513-2540) */
  double tkefar, omefar, mutfar, cmu, bstrkw, gkw, bkw, sigk, sigw, epst, kappa;
  /* boundary values hard-wired in the reference, parameterised here;
     defaults are the reference literals:
       inlet  T0=1.008, p0=0.734486515085076, dir=(1,0,0)  (src/bc.f90:996-1000)
       outlet p=0.714285714285714 in both halo layers and on the face
                                                          (src/bc.f90:1310-1312) */
  double inlet_t0, inlet_p0, inlet_dir[3];
  double outlet_p[3];
  /* harmonic balance: omega and D (src/input.f90:5206-5284) */
  double omega;
  double dhb[COSA_MAX_SNAP * COSA_MAX_SNAP]; /* dhb[n*S + m] = D(n,m) */
  /* GPU-only knobs */
  int32_t precision;    /* COSA_PREC_FP64 | COSA_PREC_MIXED */
  /* multigrid controls (src/input.f90:3509-3570, common/mgpars):
     iterations per visit nstart (fine, first cycle), npre, npost, ncrs
     (coarsest); bln_prol 1 = bilinear prol_bln, 0 = linear prol_lin;
     lim_corr 0..3 = none / lim_corr1..3 of prol_bln (turbulence only) */
  int32_t nstart, npre, npost, ncrs, bln_prol, lim_corr;
  /* k-omega options (src/input.f90:2722-2765, 3565-3575): production
     limiter on k (lim_prodtke) and omega (lim_prodomega) with factor prdlim;
     production on every MG level (prd_all_lvls); k/omega floors after each
     update (ifixq); compressibility term switch turcmp (0 or 1); omega wall
     value (wallwilc 1: Wilcox rough wall with roughness roughk, 0: Menter);
     ho_rest 1: high-order residual restriction rest2_ho_b in restrict()
     (src/cosa.f90:2742-2751, 2871-2954), 0: rest2_lo_b */
  int32_t lim_prodtke, lim_prodomega, prd_all_lvls, ifixq, wallwilc, ho_rest;
  double turcmp, prdlim, roughk;
  /* rigid pitching of the grid (moving = 1, harmonic balance, hbmove = 1):
     theta(t) = dtheta0 sin(omegas t) about the hinge (xh, yh); dtheta0 in
     radians, omegas = 2 pi x the input frequency (src/input.f90:2960-2980,
     src/grid.f90:4540) */
  double dtheta0, omegas, xh, yh;
  /* time-accurate runs: the physical time step dt of dual time stepping
     (dualt, BDF2 with src_uns / rhs_uns, src/src.f90:381-527) and of the
     explicit RK integration (rgkuns, src/cosa.f90:3890-4180); bdf1 = 1 on
     the first physical step of a run not started from a dual-time restart
     (itime = 1 and not dual_prop_start: first-order backward difference) */
  double dt;
  int32_t bdf1, reserved_t;
  /* low-speed preconditioning, lomach = 1 (src/losp.f90, src/flux.f90:390-830,
     src/input.f90:3585-3700): cutoff_type 1 no pressure-gradient cut-off,
     2 lm_cutoff_pg on every level, 3 on the fine level and restricted
     (rest3) to the coarse ones; visprec 1 adds the viscous cut-off
     lm_viscoff (viscous runs); mixpi 0 standard, 1 mixed preconditioner;
     uprv the unsteady reference velocity (0 in steady runs); epsp[nl-1] the
     constant cut-off of level nl */
  int32_t lomach, cutoff_type, visprec, mixpi;
  double uprv;
  double epsp[COSA_MAX_LEVELS];
} cosa_params;

/*
 * One multigrid level of the block table.  dims/nbcs/bctopo/cutopo are the
 * reference's per-level tables: i_imax/j_jmax/k_kmax (src/input.f90:4426),
 * bctopo(10,nbcs) (src/input.f90:3839-3872) and cutopo(21,ncuts) with the
 * cut pairs already doubled (src/input.f90:3903-4000).
 */
typedef struct cosa_level_desc {
  int32_t nblocks;
  const int32_t *dims;    /* 3*nblocks: imax, jmax, kmax (node counts) */
  const int32_t *nbcs;    /* nblocks */
  const int32_t *bctopo;  /* 10 * sum(nbcs), block after block */
  int32_t ncuts;          /* number of cutopo records (2 per input cut) */
  const int32_t *cutopo;  /* 21 * ncuts */
} cosa_level_desc;

/*
 * Device pointer table of one level: the Cray-pointer bases p_*(nl) that
 * smooth() binds at its top (src/cosa.f90:1650-1703).
 */
typedef struct cosa_level_ptrs {
  double *q, *qold, *res, *rhs, *dtvol, *dtvolt;
  double *si, *sj, *sk, *vol;
  double *qp, *qm, *dq, *dqp, *dqm, *flux;           /* unfused scratch */
  double *betaxi, *betaeta, *betazeta;               /* IRS coefficients */
  double *mut, *dist;                                /* RANS */
  /* moving grids: xdot, ydot, zdot the cell grid velocities (the node
     arrays after vert2cell_g, P2 layout x S snapshots); fvi, fvj, fvk the
     face velocities of the three families, the reference's sijk(5:7) kept
     beside the lmet = 4 metric records: (3, 0:imax+1, 0:jmax+1, 0:kmax+1,
     0:S-1) per block at offset op2*3*S */
  double *xdot, *ydot, *zdot;
  double *fvi, *fvj, *fvk;
} cosa_level_ptrs;

typedef struct cosa_ctx cosa_ctx;

/* sizeof(cosa_params) as compiled into the library (ABI check) */
int64_t cosa_gpu_params_size(void);

/* ---- context: replaces the module state set up by input()/alloc() ---- */
int cosa_gpu_init(const cosa_params *p, int32_t nlevels,
                  const cosa_level_desc *levels, int32_t device,
                  cosa_ctx **out);
int cosa_gpu_finalize(cosa_ctx *ctx);
int cosa_gpu_set_params(cosa_ctx *ctx, const cosa_params *p);
/* sizes in doubles of the level's arrays: [P3 cells, P2 cells, P1 cells,
   F0 cells, interior cells]; a P3 array holds P3*npde*S doubles */
int cosa_gpu_level_sizes(cosa_ctx *ctx, int32_t nl, int64_t sizes[5]);
/* cosa_all replacement (src/input.f90:5072-5133): device allocation owned
   by the context, freed by cosa_gpu_finalize */
int cosa_gpu_malloc(cosa_ctx *ctx, int64_t ndoubles, double **dptr);
int cosa_gpu_memcpy_h2d(cosa_ctx *ctx, double *dst, const double *src, int64_t n);
int cosa_gpu_memcpy_d2h(cosa_ctx *ctx, double *dst, const double *src, int64_t n);
int cosa_gpu_synchronize(cosa_ctx *ctx);
int cosa_gpu_bind_level(cosa_ctx *ctx, int32_t nl, const cosa_level_ptrs *ptrs);

/* ---- level drivers: one per reference routine, device arrays ---- */
/* cons2prim (src/update.f90:2112-2188), xtnd as in the reference */
int cosa_gpu_cons2prim(cosa_ctx *ctx, int32_t nl, int32_t xtnd, double *q);
/* prim2cons (src/update.f90:1851-2084) */
int cosa_gpu_prim2cons(cosa_ctx *ctx, int32_t nl, double *q);
/* bc (src/bc.f90:2-121): every patch of every block, in table order */
int cosa_gpu_bc(cosa_ctx *ctx, int32_t nl, double *q, const double *si,
                const double *sj, const double *sk, const double *dist);
/* cutman_q (src/bc.f90:1801-1891), in-process branch of cut_q */
int cosa_gpu_cutman_q(cosa_ctx *ctx, int32_t nl, double *q);
/* prtest (src/cosa.f90:933-1120): status bits instead of stop */
int cosa_gpu_prtest(cosa_ctx *ctx, int32_t nl, const double *q);
/* lambda (src/cosa.f90:1214-1591): lambdas(.,1:3,n) */
int cosa_gpu_lambda(cosa_ctx *ctx, int32_t nl, const double *q,
                    const double *si, const double *sj, const double *sk,
                    const double *vol, double *lambdas);
/* deltat (src/cosa.f90:4701-5203): dtvol and IRS beta */
int cosa_gpu_deltat(cosa_ctx *ctx, int32_t nl, double *dtvol,
                    const double *lambdas, double *betaxi, double *betaeta,
                    double *betazeta);
/* muscl (src/flux.f90:1183-1810) */
int cosa_gpu_muscl(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *q,
                   double *qp, double *qm, double *dq, double *dqp, double *dqm);
/* roflux (src/flux.f90:2-387); flux is an F0 array */
int cosa_gpu_roflux(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qr,
                    const double *ql, double *flux, const double *sijk);
/* resid (src/cosa.f90:1123-1211) */
int cosa_gpu_resid(cosa_ctx *ctx, int32_t idir, int32_t nl,
                   const double *flux, double *res);
/* update (src/update.f90:2-100, 568-762), explicit branch: variables 1..5
   (with k-omega, cosa_gpu_update_kom first) */
int cosa_gpu_update(cosa_ctx *ctx, int32_t nl, const double *res, double *q,
                    const double *qold, const double *dtvol, double ar);
/* resg_rms (src/cosa.f90:4458-4582): resrms[0..npde]; with harbal the
   resg_rms_hb norm (src/cosa.f90:4585-4697): every snapshot of res - rhs,
   divided by ncell * (2 nharms + 1) */
int cosa_gpu_resg_rms(cosa_ctx *ctx, int32_t nl, const double *res,
                      const double *rhs, double *resrms);
/* zero (src/util.f90) of a P3 array including halo layer `ext` */
int cosa_gpu_zero(cosa_ctx *ctx, int32_t nl, double *a);

/* src_hb (src/src.f90:530-613): harmonic-balance source
   res(n) += omega * vol * sum_m D(n,m) q(m), q conservative, D from params */
int cosa_gpu_src_hb(cosa_ctx *ctx, int32_t nl, const double *q, const double *vol, double *res);
/* scalef / scaleb (src/cosa.f90:5626-5773): res *= / res /= dt/V (dtvolt
   for the turbulence equations when npde = 7) */
int cosa_gpu_scalef(cosa_ctx *ctx, int32_t nl, double *res, const double *dtvol,
                    const double *dtvolt);
int cosa_gpu_scaleb(cosa_ctx *ctx, int32_t nl, double *res, const double *dtvol,
                    const double *dtvolt);
/* cirs (src/cosa.f90:5206-5623): central implicit residual smoothing with
   constant (irsop 1) or per-cell (irsop 2,3,5,6) coefficients, including
   the scaling by dt/V; Thomas sweeps in i, j, k */
int cosa_gpu_cirs(cosa_ctx *ctx, int32_t nl, double *res, const double *dtvol,
                  const double *betaxi, const double *betaeta, const double *betazeta);
/* ccirs (src/cosa.f90:2035-2443): the cut-aware sweeps (right-hand side of
   the i sweep from ores, halo values of res on the boundary rows); called by
   smooth() twice after cutman_q on res, between scalef and scaleb */
int cosa_gpu_ccirs(cosa_ctx *ctx, int32_t nl, double *res, const double *ores,
                   const double *betaxi, const double *betaeta, const double *betazeta);
/* imetrix (src/grid.f90:820-1255): face unit normals and areas into si/sj/sk
   (lmet = 4) from the grid x,y,z; fixed grids */
int cosa_gpu_imetrix(cosa_ctx *ctx, int32_t nl, const double *x, const double *y,
                     const double *z, double *si, double *sj, double *sk);
/* ---- moving grids: harmonic balance of a rigidly pitching body (moving = 1,
   hbmove = 1, lmet stays 4: the face velocities live in their own arrays).
   Node arrays hold every snapshot: (0:imax+1,0:jmax+1,0:kmax+1,0:S-1) per
   block at offset op2*S; imetrix then writes one set of metrics per
   snapshot.  The set-up order is the reference's (src/cosa.f90:281-330):
   movegrid, vols, imetrix, face_vel, vert2cell of xdot, ydot, zdot. ---- */
/* movegrid + pitch (src/grid.f90:1783-1966): node positions x, y, z and
   velocities xdot, ydot, zdot of every snapshot t_n = n 2 pi / (|omegas| S),
   theta_n = dtheta0 sin(omegas t_n), from the reference grid x0, y0, z0 (P2
   node arrays) and the displacement scales dx, dy (P1 arrays, nodes
   1..imax; the mesh file's displacement record, src/input.f90:4562-4566).
   Ghost nodes (index 0, imax+1) rotate rigidly (unit scales). */
int cosa_gpu_movegrid(cosa_ctx *ctx, int32_t nl, const double *x0, const double *y0, const double *z0,
                      const double *dx, const double *dy, const double *dz, double *x, double *y, double *z,
                      double *xdot, double *ydot, double *zdot);
/* face velocities (imetrix_b, src/grid.f90:1024-1062): the mean of each
   face's four node velocities into fvi, fvj, fvk (layout as in
   cosa_level_ptrs) */
int cosa_gpu_face_vel(cosa_ctx *ctx, int32_t nl, const double *xdot, const double *ydot, const double *zdot,
                      double *fvi, double *fvj, double *fvk);
/* vert2cell_g (src/output.f90:3242-3480): node values of every snapshot to
   cell values (cells 0..imax), in place; the cell grid velocities that
   eig_eul reads */
int cosa_gpu_vert2cell(cosa_ctx *ctx, int32_t nl, double *w);
/* vols (src/grid.f90:2133-2230): cell volumes */
int cosa_gpu_vols(cosa_ctx *ctx, int32_t nl, const double *x, const double *y,
                  const double *z, double *vol);

/* q_edges / q_corns (src/flux.f90:3889-4263, 3132-3469): linear
   extrapolation of q (and of mut when mut != NULL, calmut) into the halo
   edge cells (plane through three neighbours) and the 8 halo corner cells
   (plane through four neighbours) of every block */
int cosa_gpu_q_edges(cosa_ctx *ctx, int32_t nl, double *q, double *mut);
int cosa_gpu_q_corns(cosa_ctx *ctx, int32_t nl, double *q, double *mut);
/* fixq (src/update.f90:2191-2269): k and omega floors qmin(6:7), npde = 7 */
int cosa_gpu_fixq(cosa_ctx *ctx, int32_t nl, double *q);
/* tur_vis (src/update.f90:2271-2337): mut = cmu rho k/(omega+epst) Re/M
   over cells 0..imax of every block (q conservative) */
int cosa_gpu_tur_vis(cosa_ctx *ctx, int32_t nl, const double *q, double *mut);

/* ---- multigrid transfers between level nl (fine) and nl+1 (coarse) ---- */
/* rest1 (src/cosa.f90:2757-2833): q2 = volume-weighted mean of the 8 fine
   cells of each coarse interior cell */
int cosa_gpu_rest1(cosa_ctx *ctx, int32_t nl, const double *q1, double *q2,
                   const double *vol1, const double *vol2);
/* rest2 with lo_rest (src/cosa.f90:2835-2869, 2955-3012):
   rhs2 = -(sum of the 8 fine residuals) */
int cosa_gpu_rest2(cosa_ctx *ctx, int32_t nl, double *rhs2, const double *res1);
/* rest2 with ho_rest (src/cosa.f90:2871-2954): rhs2 = -(27/9/3/1-weighted
   sum of the 4x4x4 fine residuals around each coarse cell) / 64; reads the
   first halo layer of res1, edges and corners included */
int cosa_gpu_rest2_ho(cosa_ctx *ctx, int32_t nl, double *rhs2, const double *res1);
/* bc_res (src/bc.f90:2802-2995): first halo layer of a residual array at
   every boundary patch = pm * first interior cell, pm = -1 on 15xx walls
   and +1 elsewhere (all npde equations) */
int cosa_gpu_bc_res(cosa_ctx *ctx, int32_t nl, double *res);
/* prol_bln (src/cosa.f90:3282-3313, 3478-3888): q1 += trilinear
   27/9/3/1 interpolation of the coarse correction q2 on fine cells
   0..imax (one halo layer), lim_corr from params for npde = 7 */
int cosa_gpu_prol_bln(cosa_ctx *ctx, int32_t nl, double *q1, const double *q2);
/* prol_lin (src/cosa.f90:3252-3280, 3315-3476): volume-weighted variant;
   vol1 must hold the halo volumes (volex/cutman_v/vol_edges) */
int cosa_gpu_prol_lin(cosa_ctx *ctx, int32_t nl, double *q1, const double *q2,
                      const double *vol1);
/* restrict (src/cosa.f90:2672-2755) on bound levels nl and nl+1: rest1 of
   q into q(nl+1), rest2 of res(nl) into rhs(nl+1); with ho_rest the
   high-order rest2 on res(nl) whose first halo layer is zero (smooth()
   zeroes it every stage) or, with k-omega, filled by cutman_q, bc_res,
   q_edges and q_corns as restrict() does */
int cosa_gpu_restrict(cosa_ctx *ctx, int32_t nl);
/* prolong (src/cosa.f90:3167-3250) on bound levels nl and nl+1:
   qold(nl+1) = rest1(q(nl)); both coarse states through cons2prim, bc,
   cutman_q, prim2cons, q_edges, q_corns; q(nl+1) -= qold(nl+1) over cells
   0..imax; then prol_bln (bln_prol) or prol_lin into q(nl); fixq for
   lim_corr 1 and 3 */
int cosa_gpu_prolong(cosa_ctx *ctx, int32_t nl);

/* ---- laminar viscous terms (viscous = .true., no turbulence model, fixed
   grid); q in primitive form where the reference has it so ---- */
/* coordex (src/grid.f90:2-80): ghost nodes 0 and imax+1 (j, k alike)
   repeat the boundary nodes; x, y, z are node arrays of cosa_level_desc's
   P2 extent (no lmet factor).  On a moving grid (moving, hbmove) the node
   arrays hold every snapshot (P2 x S2, as cosa_gpu_movegrid writes them)
   and coordex, cutman_x and vmetrix run on every snapshot */
int cosa_gpu_coordex(cosa_ctx *ctx, int32_t nl, double *x, double *y, double *z);
/* cutman_x / cut_x (src/grid.f90:242-523): ghost nodes of cut faces from
   the neighbour block's nodes one plane inside */
int cosa_gpu_cutman_x(cosa_ctx *ctx, int32_t nl, double *x, double *y, double *z);
/* volex (src/grid.f90:83-136): face-halo volumes repeat the first cell */
int cosa_gpu_volex(cosa_ctx *ctx, int32_t nl, double *vol);
/* cutman_v / cut_v (src/grid.f90:612-700): cut-face halo volumes from the
   neighbour block */
int cosa_gpu_cutman_v(cosa_ctx *ctx, int32_t nl, double *vol);
/* vmetrix (src/grid.f90:3118-3582): face inverse metrics.  vm holds the
   reference's nine arrays xideri, etaderi, zetaderi, xiderj, ... zetaderk,
   each (3, imax, jmax, kmax) per block at offset off_0*3 of a 3*n0 slab:
   array (d, m) (d = face family 1..3, m = 0 xi, 1 eta, 2 zeta) starts at
   ((d-1)*3 + m)*3*n0, n0 = sizes[3] of cosa_gpu_level_sizes; on a moving
   grid one such set per node snapshot, snapshot nh at nh*27*n0 */
int cosa_gpu_vmetrix(cosa_ctx *ctx, int32_t nl, const double *x, const double *y,
                     const double *z, const double *vol, double *vm);
/* the viscous start-up of the solver (src/cosa.f90:300-322): volex,
   cutman_v, coordex, cutman_x, vmetrix; binds vm (27*n0 doubles, times S2
   on a moving grid, kept by the caller) to level nl for cosa_gpu_smooth /
   smooth_level / mg */
int cosa_gpu_viscous_setup(cosa_ctx *ctx, int32_t nl, double *x, double *y, double *z,
                           double *vol, double *vm);
/* q_face (src/flux.f90:2391-2801), calmut = .false.: face averages of the
   primitive state, the halo (wall) value on strong-boundary faces; qf P3 */
int cosa_gpu_q_face(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *q, double *qf);
/* q_der (src/flux.f90:1813-2390): face gradients along xi, eta, zeta (P3
   each), one-sided three-point normal derivative and tangential
   derivatives along the halo line on strong-boundary faces */
int cosa_gpu_q_der(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *q, double *dqxi,
                   double *dqeta, double *dqzeta);
/* vflux (src/flux.f90:831-1180), laminar: flux = viscous face flux (F0) of
   face family idir with the family's metrics sijk and vm as above */
int cosa_gpu_vflux(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qf, const double *dqxi,
                   const double *dqeta, const double *dqzeta, const double *vm,
                   const double *sijk, double *flux);
/* lambda with viscous = .true. (src/cosa.f90:1349-1423, eig_ns
   4239-4297): lam(.,1:3) convective and lamv(.,1:3) viscous spectral radii
   (P3 layout, q primitive with halos) */
int cosa_gpu_lambda_ns(cosa_ctx *ctx, int32_t nl, const double *q, const double *si,
                       const double *sj, const double *sk, const double *vol, const double *mut,
                       double *lam, double *lamv);
/* deltat with viscous = .true. (src/cosa.f90:4831-5180): dtvol with the
   viscous radii (irsop other than 5, 6), IRS coefficients with the viscous
   floor for irsop 5 and 6; with k-omega also dtvolt = cflt/cfl dtvol and
   the turbulence coefficients tb* (ratt).  NULL pointers are skipped. */
int cosa_gpu_deltat_ns(cosa_ctx *ctx, int32_t nl, double *dtvol, const double *lam,
                       const double *lamv, double *bx, double *by, double *bz,
                       double *dtvolt, double *tbx, double *tby, double *tbz);

/* ---- time-accurate runs (one snapshot; params.dt, params.bdf1) ---- */
/* src_uns (src/src.f90:381-451): res += 3/2 q V / dt, or q V / dt with bdf1;
   the dual-time stages of cosa_gpu_smooth / cosa_gpu_mg add it themselves
   (and subtract the fine level's rhs, rhs_uns, src/cosa.f90:1908-1941) */
int cosa_gpu_src_uns(cosa_ctx *ctx, int32_t nl, const double *q, const double *vol, double *res);
/* rhs_uns (src/src.f90:453-527): rhs = (2 q1 - q2 / 2) V / dt, or q1 V / dt
   with bdf1; q1 = q^n, q2 = q^(n-1).  One physical step of dual time is
   q1 <- q, cosa_gpu_rhs_uns into the fine level's rhs, cosa_gpu_mg for the
   pseudo-time cycles, q2 <- q1 (src/cosa.f90:548-667). */
int cosa_gpu_rhs_uns(cosa_ctx *ctx, int32_t nl, double *rhs, const double *q1, const double *q2, const double *vol);
/* copy_array over the interior cells of every variable and snapshot
   (offset -1, src/util.f90:2-135): dst = src, e.g. q1 <- q */
int cosa_gpu_copy_interior(cosa_ctx *ctx, int32_t nl, double *dst, const double *src);
/* rkuns (src/cosa.f90:3890-4180) on level 1 of a fixed grid: ntime physical
   steps of the nstage-stage RK scheme with dtvol = dt / V (deltat_urk);
   hist receives (npde+1) values per step, the norm of the last stage's
   residual on steps with itime % iprint == 0 and the last (NaN elsewhere).
   Euler and laminar without IRS (COSA_ERR_UNSUPPORTED otherwise). */
int cosa_gpu_rkuns(cosa_ctx *ctx, int32_t ntime, int32_t iprint, double *hist);

/* ---- k-omega: Wilcox (kom), BSL (kom_bsl), SST (kom_sst); npde = 7; mut,
   prd, divvel, delpls are scalar P3 arrays (-1:imax+1,...,0:S-1); ttrm
   (BSL/SST) is (-1:imax+1,...,3,0:S-1) per block at off_p3 * 3 * S; the face
   wall distances are one F0 scalar array (imax,jmax,kmax) per face family ---- */
/* q_face with calmut (src/flux.f90:2495-2540): face mut into flux(.,1) */
int cosa_gpu_q_face_mut(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *mut, double *flux);
/* rtst (src/flux.f90:2803-2946): Reynolds stresses tau1(.,1..6) on the faces
   from q_face/q_der output, vm and the face mut in flux(.,1) */
int cosa_gpu_rtst(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qf, const double *dqxi,
                  const double *dqeta, const double *dqzeta, const double *vm,
                  const double *flux, double *tau1);
/* vflux with k-omega (src/flux.f90:915-1180): Reynolds-stress and k/omega
   diffusion fluxes plus the laminar terms; flux(.,1) holds the face mut on
   entry; fdist, the face wall distances of family idir, for BSL/SST (sigma
   blended by F1, src/flux.f90:987-1061) and null for Wilcox */
int cosa_gpu_vflux_kom(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qf, const double *dqxi,
                       const double *dqeta, const double *dqzeta, const double *tau1,
                       const double *vm, const double *sijk, double *flux, const double *fdist);
/* q_der_c (src/flux.f90:2949-3130): cell-centred velocity differences of
   the face values of family idir (and of k, omega under BSL/SST) */
int cosa_gpu_q_der_c(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qf, double *dqc);
/* turprod (src/src.f90:2-177): production, div u and delta+ */
int cosa_gpu_turprod(cosa_ctx *ctx, int32_t nl, const double *dqxi, const double *dqeta,
                     const double *dqzeta, const double *vm, double *prd, double *divvel,
                     double *delpls);
/* srckw (src/src.f90:179-272): k and omega sources into res(6:7) */
int cosa_gpu_srckw(cosa_ctx *ctx, int32_t nl, const double *q, const double *mut, const double *prd,
                   const double *divvel, double *res, const double *vol);
/* update_b, k-omega part (src/update.f90:601-640): point-implicit rho omega
   and rho k; call before cosa_gpu_update (which updates variables 1..5);
   ttrm: gamma and beta per cell (BSL/SST), null for Wilcox's constants */
int cosa_gpu_update_kom(cosa_ctx *ctx, int32_t nl, const double *res, double *q, const double *qold,
                        const double *vol, const double *dtvolt, const double *delpls,
                        const double *prd, double ar, const double *ttrm);
/* ---- low-speed preconditioning (lomach; src/losp.f90, src/flux.f90:390-830).
   Cut-off arrays are in the reference's interior-cell layout
   (imax-1, jmax-1, kmax-1, 0:S-1) per block, off_m1 * S (p_cutoff_pgr /
   p_cutoff_vis); prec is (imax-1, jmax-1, kmax-1, npde, npde, 0:S-1) per
   block at off_m1 * npde^2 * S (p_prec).  q primitive unless stated. */
/* lm_cutoff_pg (src/losp.f90:1085-1165): pressure-gradient cut-off */
int cosa_gpu_lm_cutoff_pg(cosa_ctx *ctx, int32_t nl, const double *q, double *cutoff_pgr);
/* lm_viscoff (src/losp.f90:1290-1414): viscous cut-off (viscous runs) */
int cosa_gpu_lm_viscoff(cosa_ctx *ctx, int32_t nl, const double *q, const double *si, const double *sj,
                        const double *sk, double *cutoff_vis);
/* rest3 (src/cosa.f90:3014-3088): cut-offs of level nl restricted to nl+1 */
int cosa_gpu_rest3(cosa_ctx *ctx, int32_t nl, const double *cutoff1, double *cutoff2, const double *vol1,
                   const double *vol2);
/* lm_cutoff + proflux (src/losp.f90:1416-1447, src/flux.f90:390-830): the
   preconditioned Roe flux of family idir from the MUSCL states qr (qp) and
   ql (qm) */
int cosa_gpu_proflux(cosa_ctx *ctx, int32_t idir, int32_t nl, const double *qr, const double *ql, double *flux,
                     const double *sijk, const double *cutoff_pgr, const double *cutoff_vis);
/* lambda with lomach (src/cosa.f90:1447-1590): eig_eul_p, or with viscous
   eig_ns_p (vol and lamv then required) */
int cosa_gpu_lambda_p(cosa_ctx *ctx, int32_t nl, const double *q, const double *si, const double *sj,
                      const double *sk, const double *vol, double *lam, double *lamv, const double *cutoff_pgr,
                      const double *cutoff_vis);
/* lsp (src/losp.f90:2-195): the preconditioner of every interior cell from
   the conservative q */
int cosa_gpu_lsp(cosa_ctx *ctx, int32_t nl, const double *q, const double *cutoff_pgr, const double *cutoff_vis,
                 double *prec);
/* precres (src/cosa.f90:2446-2521): res <- prec res over the interior cells */
int cosa_gpu_precres(cosa_ctx *ctx, int32_t nl, double *res, const double *prec);
/* the level's own cut-offs as the smooth/multigrid drivers left them
   (device to device copies into the two arrays given) */
int cosa_gpu_lsp_cutoffs(cosa_ctx *ctx, int32_t nl, double *cutoff_pgr, double *cutoff_vis);
/* facedist (src/grid.f90:2809-2870): face wall distances of the three
   families from the cell distances dist (P1) */
int cosa_gpu_facedist(cosa_ctx *ctx, int32_t nl, const double *dist, double *fidist, double *fjdist,
                      double *fkdist);
/* update_ttrm (src/update.f90:3000-3161): ttrm = ((1 - F1) CD, gamma, beta)
   blended by F1 from the primitive state, the cell-centred k and omega
   differences of q_der_c and dist; Wilcox: (0, gkw, bkw) */
int cosa_gpu_update_ttrm(cosa_ctx *ctx, int32_t nl, const double *q, const double *dqxi, const double *dqeta,
                         const double *dqzeta, const double *vm, double *ttrm, const double *dist);
/* srckw_sst (src/src.f90:275-378): BSL/SST k and omega sources into res(6:7) */
int cosa_gpu_srckw_sst(cosa_ctx *ctx, int32_t nl, const double *q, const double *prd, const double *divvel,
                       double *res, const double *mut, const double *ttrm, const double *vol);
/* tur_vis_sst (src/update.f90:2340-2460): SST eddy viscosity of the
   conservative state with the cell-centred velocity differences; the face
   halos copy the adjacent cell */
int cosa_gpu_tur_vis_sst(cosa_ctx *ctx, int32_t nl, const double *q, double *mut, const double *dqxi,
                         const double *dqeta, const double *dqzeta, const double *vm, const double *dist);
/* cutman_mut (src/bc.f90:2713-2799) */
int cosa_gpu_cutman_mut(cosa_ctx *ctx, int32_t nl, double *mut);

/* ---- wall forces ---- */
/* force (src/output.f90:4027-4387) over force_b (src/output.f90:4388-4900):
   pressure and skin-friction force and moment coefficients of surface isurf
   (the patches with bctopo(1) == 1500 + isurf - 1) of level nl, per block
   in the reference's order and summed over blocks.  q conservative with the
   halos of the last bc (as smooth() leaves them); x, y, z the P2 node arrays
   with the ghost nodes of coordex (the moment arm of an inrout = 1 patch is
   the ghost node); vm the face inverse metrics (viscous flows; may be NULL
   otherwise); xmom the moment centre, lngth = lref1..3 of the input file.
   coef (host, 12 * S doubles): snapshot n at coef[12n ..] = cl_p, cd_p,
   cz_p, cmx_p, cmy_p, cm_p, cl_v, cd_v, cz_v, cmx_v, cmy_v, cm_v.  On a
   pitching grid (moving) each snapshot uses its own metrics and nodes and
   the moment centre carried with the body (src/output.f90:4476-4485);
   inviscid only there. */
int cosa_gpu_force(cosa_ctx *ctx, int32_t nl, const double *q, const double *x, const double *y,
                   const double *z, const double *si, const double *sj, const double *sk,
                   const double *vm, int32_t isurf, const double *xmom, const double *lngth,
                   double *coef);

/* ---- fused: what smooth() calls when the GPU path is on ---- */
/*
 * One RK iteration sequence of smooth() (src/cosa.f90:1711-2029) on the
 * level bound with cosa_gpu_bind_level, niter iterations of nstage stages.
 * For every iteration whose number is listed in want_rms (mgit values;
 * iteration numbering starts at mgit0), the stage-1 residual RMS is written
 * to hist[(it-mgit0)*(npde+1) + 0..npde].  The state stays on the device.
 */
int cosa_gpu_smooth(cosa_ctx *ctx, int32_t nl, int32_t niter, int32_t mgit0,
                    int32_t rms_every, double *hist);
/* same, with the state q passed in HOST memory (copied in and out) */
int cosa_gpu_smooth_host(cosa_ctx *ctx, int32_t nl, double *q_host,
                         int32_t niter, int32_t mgit0, int32_t rms_every,
                         double *hist);
/*
 * smooth(nl, from_fine, to_coarse, done, niter) (src/cosa.f90:1594-2032) on
 * the bound level nl: niter RK iterations; with to_coarse one more stage-1
 * residual pass whose result (res - rhs on coarse levels) is left in the
 * level's res array for restrict; on coarse levels the forcing rhs += res at
 * the first stage of a from_fine visit and res -= rhs at every stage.  mgit
 * and ncycle select the printed cycle (mgit == 1, mgit % rms_every == 0 or
 * mgit == ncycle) whose fine-level resrms[0..npde] goes to resrms (NULL:
 * none).  The convergence test `done` is left to the caller.
 */
int cosa_gpu_smooth_level(cosa_ctx *ctx, int32_t nl, int32_t niter, int32_t from_fine,
                          int32_t to_coarse, int32_t mgit, int32_t ncycle,
                          int32_t rms_every, double *resrms);
/*
 * mg() (src/cosa.f90:806-930): cycles mgit0 .. mgit0+ncycles-1 of a run of
 * ncycle multigrid V-cycles on the nlevel (params) bound levels; smoothing
 * counts nstart/npre/npost/ncrs from params.  When the last cycle run is
 * ncycle, the final npost fine-level smoothing follows.  hist as in
 * cosa_gpu_smooth, one row per cycle.
 */
int cosa_gpu_mg(cosa_ctx *ctx, int32_t mgit0, int32_t ncycles, int32_t ncycle,
                int32_t rms_every, double *hist);
/* stage-schedule autotuner (no reference counterpart): times niter
   iterations of level nl with the fused tile kernel (schedule 0) and with
   the face-split schedule (1: face fluxes through HBM, then a cell pass),
   keeps the faster for the level and returns the ms per iteration of each;
   the level's state is restored afterwards.  set_schedule forces one. */
int cosa_gpu_autotune(cosa_ctx *ctx, int32_t nl, int32_t niter, double ms[2], int32_t *choice);
int cosa_gpu_set_schedule(cosa_ctx *ctx, int32_t nl, int32_t schedule);
/* niter fused iterations without graphs, with CUDA events around every
   kernel: ms[0] = mean halo-kernel time, ms[1] = mean time of the main
   kernel (k_stage_tile, or k_faces under the split schedule), ms[2] = mean
   iteration time, ms[3] = mean k_cells time (split schedule);
   counts = launches timed */
int cosa_gpu_profile(cosa_ctx *ctx, int32_t nl, int32_t niter, double ms[4],
                     int64_t counts[4]);
/* diagnostics: evaluates the fused kernel's Newton-Raphson reciprocal and
   reciprocal square root on n host values x (positive normal numbers) on
   the current device and returns in err[0], err[1] the largest relative
   differences from IEEE 1/x and 1/sqrt(x) computed there */
int cosa_gpu_nr_selftest(int64_t n, const double *x, double err[2]);
/* the context's CUDA stream (cudaStream_t), for callers that time with
   their own events */
void *cosa_gpu_stream(cosa_ctx *ctx);
/* number of this library's kernels launched since the last call */
int64_t cosa_gpu_launch_count(cosa_ctx *ctx, int32_t reset);
/* latched device status bits (COSA_ERR_*), cleared when reset != 0 */
int cosa_gpu_status(cosa_ctx *ctx, int32_t reset);

/*
 * Residual RMS that allocates nothing.  No counterpart in the reference: it
 * is the resg_rms computation for callers that cannot call cudaMalloc, such
 * as a Fortran driver whose device memory is owned and pooled by another
 * runtime, or code running where a new allocation would fail or is not
 * permitted.  It needs no context: the caller passes the block table (host
 * array dims[3*nblocks], node counts as in cosa_level_desc), npde, nharms,
 * the device arrays res and rhs (rhs may be NULL) in the P3 layout, a device
 * output resrms[npde+1] (per-equation RMS, then the total as in resg_rms),
 * and a CUDA stream (NULL = default stream).  With nharms > 0 the norm is
 * resg_rms_hb's (src/cosa.f90:4585-4697): the squares of every snapshot are
 * summed and divided by ncell * (2 nharms + 1); res must then already hold
 * any time-spectral term.  The per-CTA partial sums go to
 * a static device array of COSA_NOALLOC_MAX_PARTS rows of 8 doubles
 * (256 KiB) that every GPU loading the library holds until exit.  The first
 * call on a device looks up that array's device address; make that first
 * call before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race.  nblocks above COSA_NOALLOC_MAX_PARTS returns
 * COSA_ERR_ARG.
 */
#define COSA_NOALLOC_MAX_PARTS 4096
int cosa_gpu_resg_rms_noalloc(int32_t nblocks, const int32_t *dims, int32_t npde,
                              int32_t nharms, const double *res, const double *rhs,
                              double *resrms, void *stream);

/*
 * ---- serving: several steady solves resident on one GPU ----
 * No counterpart in the reference, which runs one solve per process.  An
 * engine holds device pools sized by budget_bytes; submitted solves (grid
 * tables, node coordinates in the P2 layout, initial P3 state, flow
 * conditions) wait in a first-come queue, are admitted when their arrays fit
 * in the pools, are advanced together (every RK stage of every active solve
 * in the same halo and tile launches) and retire when their total residual
 * norm falls below tol times its first-iteration value (checked every
 * check_every of their own iterations) or after max_iter iterations.  The
 * scheme (gamma, limiter, RK coefficients, and the CFL number unless the
 * request sets cfl > 0) is the engine's; machfs, alpha, beta, the free
 * stream, the inlet total state, the outlet pressure and the CFL number
 * come from each request.  Explicit Euler, single grid, S = 1,
 * blocks of at least two cells per direction.
 */
#define COSA_SOLVE_QUEUED    0
#define COSA_SOLVE_ACTIVE    1
#define COSA_SOLVE_CONVERGED 2
#define COSA_SOLVE_STOPPED   3  /* max_iter reached */
#define COSA_SOLVE_FAILED    4  /* non-finite residual norm */
typedef struct cosa_serve cosa_serve;
int cosa_serve_create(const cosa_params *scheme, int64_t budget_bytes, int32_t device,
                      int32_t check_every, cosa_serve **out);
int cosa_serve_destroy(cosa_serve *e);
int cosa_serve_submit(cosa_serve *e, const cosa_level_desc *grid, const double *x,
                      const double *y, const double *z, const double *q0,
                      const cosa_params *flow, double tol, int32_t max_iter, int64_t *id);
/* admit what fits, then advance the active solves by up to niter iterations
   (fewer when none is left); retired solves free their pool slots */
int cosa_serve_step(cosa_serve *e, int32_t niter, int32_t *nactive, int32_t *nqueued);
/* state, own iteration count, last residual drop, times (submitted,
   admitted, done; seconds since the engine was created) and, once retired,
   the P3 state (q_out may be NULL) */
int cosa_serve_result(cosa_serve *e, int64_t id, int32_t *state, int32_t *iters, double *rms_drop,
                      double times[3], double *q_out);
/* free pool slots (one slot holds one P3 cell of every pool) */
int64_t cosa_serve_free_slots(cosa_serve *e);

#ifdef __cplusplus
}
#endif
#endif /* COSA_GPU_H */
