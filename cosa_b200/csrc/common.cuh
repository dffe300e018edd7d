// Layout helpers shared by every kernel of the B200 path.
//
// All state arrays use COSA's own layout (src/input.f90:5502-5585): per
// block, column-major with i fastest, dimensions
//   P3: (-1:imax+1, -1:jmax+1, -1:kmax+1, npde, 0:S-1)
//   P2: (lmet=4, 0:imax+1, 0:jmax+1, 0:kmax+1, 0:S*hbmove)   (face metrics)
//   P1: (0:imax, 0:jmax, 0:kmax [, 0:S-1])
//   F0: (imax, jmax, kmax, npde, 0:S-1)
// with the per-block arrays concatenated at setoffs() offsets.  Every
// variable plane of a block is contiguous along i, so a warp reading 32
// consecutive i of one variable issues fully coalesced 256-byte loads.
#pragma once
#include <cstdint>
#include "../../include/cosa_gpu.h"

struct DevBlock {
  int im, jm, km;          // node counts imax, jmax, kmax
  int I3, J3;              // im+3, jm+3
  int64_t P3;              // (im+3)(jm+3)(km+3)
  int64_t op3, op2, op1, of0;  // setoffs offsets in cells
  int64_t om1;                 // offset in the interior-cell layout (off_m1)
  int obct, nbcs;          // the block's rows of the level's BC table (offset in ints, count)
  // a per-block kernel launched for this block alone
  __host__ __device__ DevBlock get() const { return *this; }
};

// a per-block kernel launched once for all blocks of a level: block
// blockIdx.y of the level's device table (grid-stride loops use x only)
struct BlockList {
  const DevBlock *p;
  __device__ DevBlock get() const { return p[blockIdx.y]; }
};

// element (i,j,k) [Fortran indices] of the cell plane of a P3 block
__host__ __device__ __forceinline__ int64_t p3_cell(const DevBlock &b, int i, int j, int k) {
  return (int64_t)(i + 1) + (int64_t)b.I3 * ((j + 1) + (int64_t)b.J3 * (k + 1));
}
// base of variable v (1-based) of snapshot n of block b inside a P3 array
__host__ __device__ __forceinline__ int64_t p3_var(const DevBlock &b, int npde, int S, int v, int n) {
  return b.op3 * npde * S + ((int64_t)n * npde + (v - 1)) * b.P3;
}
// metric component c (1..4) of face (i,j,k) snapshot nh
__host__ __device__ __forceinline__ int64_t p2_idx(const DevBlock &b, int S2, int c, int i, int j, int k, int nh) {
  const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
  return ((b.op2 * S2) + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k)) * 4 + (c - 1);
}
__host__ __device__ __forceinline__ int64_t p1_idx(const DevBlock &b, int nsnap, int i, int j, int k, int n) {
  const int64_t I1 = b.im + 1, J1 = b.jm + 1, K1 = b.km + 1;
  return b.op1 * nsnap + (int64_t)n * I1 * J1 * K1 + i + I1 * (j + J1 * (int64_t)k);
}
__host__ __device__ __forceinline__ int64_t f0_idx(const DevBlock &b, int npde, int S, int i, int j, int k, int v, int n) {
  const int64_t I = b.im, J = b.jm, K = b.km;
  return b.of0 * npde * S + ((int64_t)n * npde + (v - 1)) * I * J * K + (i - 1) + I * ((j - 1) + J * (int64_t)(k - 1));
}

// cyc(idir,m) of input() (src/input.f90:2409), 1-based
__host__ __device__ __forceinline__ int cyc3(int idir, int m) {
  int r = idir + m - 1;
  return r > 3 ? r - 3 : r;
}

#define COSA_CUDA_MAX_NPDE 7
