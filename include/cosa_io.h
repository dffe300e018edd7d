/*
 * cosa_io.h -- the reference's case files, read and written on the host:
 * input.dat (input(), src/input.f90:2271-4392), mesh.dat (readgrid,
 * src/input.f90:4482-4570) and restart (readrest, src/input.f90:4620-4716;
 * writerest, src/output.f90:3484-3566).
 *
 * mesh.dat and restart are gfortran unformatted sequential files: every
 * record is framed by 4-byte little-endian length markers; a record longer
 * than 2147483639 bytes is split into subrecords whose leading markers are
 * negative (all but the last).  Arrays use this library's layouts (the
 * reference's): node arrays P2 (0:imax+1,0:jmax+1,0:kmax+1) per block at the
 * setoffs offsets, displacement scales P1 (0:imax,0:jmax,0:kmax), states P3
 * (-1:imax+1,...,npde,0:2*nharms).  Every function returns 0 or COSA_ERR_*
 * bits (COSA_ERR_ARG for a missing, short or malformed file).
 */
#ifndef COSA_IO_H
#define COSA_IO_H

#include <stdint.h>
#include "cosa_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* input()'s defaults (src/input.f90:2400-2540) */
int cosa_io_default_params(cosa_params *p);

/* the run controls of input.dat that are not cosa_params fields */
typedef struct cosa_run_opts {
  int32_t debug, exter, irest, srest, lmax, nl_fmg, dgn_cell, wri_res, wri_tec, calfor, nsurface;
  int32_t ntime, nsave, wrifl[3];
  double toler, tref, dt, xmom[3], lngth[3];
  char flow_kind[16];   /* aircraft, saircraft, vawt, rhawt, shawt */
  char out_format[16];  /* cgns, plt, szplt, bin or empty */
  int32_t n_surblo[8];  /* blocks of each force surface (nsurface <= 8) */
  int32_t i_surbl[8][64];
} cosa_run_opts;

typedef struct cosa_input cosa_input;
/* input.dat: params (the module globals with input()'s derived values:
   alpha and beta in radians, pinf, tkefar and omefar scaled, cfl/cflt and
   rat/ratt from the CFL entries, the harmonic-balance D matrix), the run
   controls and the fine level's block, BC and cut tables as input() builds
   them (bcdata, cutdata with the cut pairs doubled).  Options outside this
   library (CGNS grids, rotors, plunging, low-speed preconditioning,
   periodic sectors) return COSA_ERR_UNSUPPORTED. */
int cosa_io_read_input(const char *path, cosa_params *p, cosa_run_opts *run, cosa_input **out);
/* the tables of a parsed input: pointers into the handle */
int cosa_io_input_level(const cosa_input *in, cosa_level_desc *d);
int cosa_io_free_input(cosa_input *in);
/* input.dat from params, run controls and a level table, in the grammar
   cosa_io_read_input reads (so a Fortran run and this library can share a
   case) */
int cosa_io_write_input(const char *path, const cosa_params *p, const cosa_run_opts *run,
                        const cosa_level_desc *d);

/* mesh.dat: per block one record of x, y, z at nodes 1..imax, 1..jmax,
   1..kmax (i fastest), and with_disp (moving pitching grids) a second
   record of the displacement scales dx, dy, dz */
int cosa_io_read_mesh(const char *path, int32_t nblocks, const int32_t *dims, int32_t with_disp, double *x,
                      double *y, double *z, double *dx, double *dy, double *dz);
int cosa_io_write_mesh(const char *path, int32_t nblocks, const int32_t *dims, int32_t with_disp,
                       const double *x, const double *y, const double *z, const double *dx, const double *dy,
                       const double *dz);

/* restart: per block one record of q (every cell, halos included, all
   snapshots), with_q1 a record of the previous time level q1 (npde
   variables; dual time, so nharms = 0), with_mut a record of mut (all
   snapshots; k-omega).  The writer takes every array at its own block
   offset; the reference's writerest passes q1 and mut with each other's
   offsets (src/output.f90:3519), which only the first block survives. */
int cosa_io_read_restart(const char *path, int32_t nblocks, const int32_t *dims, int32_t npde, int32_t nharms,
                         int32_t with_q1, int32_t with_mut, double *q, double *q1, double *mut);
int cosa_io_write_restart(const char *path, int32_t nblocks, const int32_t *dims, int32_t npde, int32_t nharms,
                          int32_t with_q1, int32_t with_mut, const double *q, const double *q1,
                          const double *mut);

/* History and force files, one WRITE each, as text in buf (records end in
   '\n'; COSA_ERR_ARG when cap is too small).  cosa_io_hist_record: a line of
   hist.dat (resrms 1..5), histur.dat (6..npde) or histg.dat, format
   (i7,2x,i7,5(1x,e13.5)) of output() (src/output.f90:4941-4965, 5005).
   cosa_io_force_header: the title and variable list force() writes when it
   creates forces_tec.dat or forces_hb_<nnn>.dat of snapshot n
   (src/output.f90:4100-4240).  cosa_io_force_record: one record of that
   file (formats 212-220, src/output.f90:4310-4380); coef holds per surface
   cl_p, cl_v, cd_p, cd_v, cz_p, cz_v, cmx_p, cmx_v, cmy_p, cmy_v, cm_p, cm_v. */
int cosa_io_hist_record(int32_t itime, int32_t it, const double *res, int32_t n, char *buf, int64_t cap);
int cosa_io_force_header(const cosa_params *p, int32_t nsurface, int32_t n, char *buf, int64_t cap);
int cosa_io_force_record(const cosa_params *p, int32_t nsurface, int32_t itime, int32_t it, double time,
                         double zeit, const double *coef, double alpha_deg, char *buf, int64_t cap);

#ifdef __cplusplus
}
#endif
#endif /* COSA_IO_H */
