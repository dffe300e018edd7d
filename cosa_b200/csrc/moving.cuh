// Moving grids of harmonic balance: a rigidly pitching body.
//
//   k_pitch       movegrid_b + pitch (src/grid.f90:1814-1966): the node
//                 positions and velocities of every snapshot from the
//                 reference grid x0 and the per-node displacement scales
//   k_face_vel    imetrix_b's moving part (src/grid.f90:1024-1062): face
//                 midpoint velocities, the reference's sijk(5:7), kept in
//                 their own arrays (3 doubles per face) beside the 32-byte
//                 lmet = 4 metric records the stage kernels load as pairs
//   k_vert2cell   vert2cell_bg (src/output.f90:3276-3480): node values to
//                 cell values, the cell grid velocities that eig_eul reads
//
// Node arrays of a moving grid hold every snapshot: (0:imax+1, 0:jmax+1,
// 0:kmax+1, 0:S2-1) per block at op2*S2 (S2 = 2 nharms hbmove + 1).
#pragma once
#include "common.cuh"

__host__ __device__ __forceinline__ int64_t gs_idx(const DevBlock &b, int S2, int i, int j, int k, int nh) {
  const int64_t I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
  return b.op2 * S2 + (int64_t)nh * I2 * J2 * K2 + i + I2 * (j + J2 * (int64_t)k);
}

// snapshot motion: sin/cos of theta_n and cos(omegas t_n), computed on the
// host in FP64 (the reference's dcos/dsin of the same arguments)
struct PitchSnap {
  double c, s, cw;
};

// one thread per node (all nodes 0..imax+1 of every snapshot).  Nodes
// 1..imax follow pitch() with their displacement scales dx, dy (P1 arrays);
// the ghost nodes rotate rigidly (unit scales), since the forces read them
// as moment arms.  The branch for |dx| or |dy| <= 1e-4 keeps the reference's
// y0 (not y0 - yh) in its rotation terms.
__global__ void k_pitch(DevBlock b, int S2, const PitchSnap *__restrict__ snap, double xh, double yh,
                        double dtheta0, double omegas, const double *__restrict__ x0, const double *__restrict__ y0,
                        const double *__restrict__ z0, const double *__restrict__ dx, const double *__restrict__ dy,
                        double *__restrict__ x, double *__restrict__ y, double *__restrict__ z,
                        double *__restrict__ xd, double *__restrict__ yd, double *__restrict__ zd) {
  const int I2 = b.im + 2, J2 = b.jm + 2, K2 = b.km + 2;
  const int64_t nn = (int64_t)I2 * J2 * K2, total = nn * S2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c0 = t % nn;
    const int n = (int)(t / nn);
    const int i = (int)(c0 % I2), j = (int)((c0 / I2) % J2), k = (int)(c0 / ((int64_t)I2 * J2));
    const int64_t g0 = b.op2 + c0, gn = gs_idx(b, S2, i, j, k, n);
    const PitchSnap m = snap[n];
    const bool ghost = i == 0 || j == 0 || k == 0 || i > b.im || j > b.jm || k > b.km;
    const double X0 = x0[g0], Y0 = y0[g0];
    const int64_t p1 = b.op1 + i + (int64_t)(b.im + 1) * (j + (int64_t)(b.jm + 1) * k);
    const double DX = ghost ? 1.0 : dx[p1], DY = ghost ? 1.0 : dy[p1];
    z[gn] = z0[g0];
    zd[gn] = 0.0;
    if (fabs(DX) > 1e-4 && fabs(DY) > 1e-4) {
      const double d1 = ((X0 - xh) * (m.c - 1) - (Y0 - yh) * m.s) / DX;
      const double d2 = ((X0 - xh) * m.s + (Y0 - yh) * (m.c - 1)) / DY;
      x[gn] = X0 + d1 * DX;
      y[gn] = Y0 + d2 * DY;
      const double v1 = (-(X0 - xh) * m.s - (Y0 - yh) * m.c) * dtheta0 * m.cw / DX;
      const double v2 = ((X0 - xh) * m.c - (Y0 - yh) * m.s) * dtheta0 * m.cw / DY;
      xd[gn] = omegas * v1 * DX;
      yd[gn] = omegas * v2 * DY;
    } else {
      const double d1 = ((X0 - xh) * (m.c - 1.0) - Y0 * m.s);
      const double d2 = ((X0 - xh) * m.s + Y0 * (m.c - 1.0));
      x[gn] = X0 + d1;
      y[gn] = Y0 + d2;
      const double v1 = dtheta0 * m.cw * (-(X0 - xh) * m.s - Y0 * m.c);
      const double v2 = dtheta0 * m.cw * ((X0 - xh) * m.c - Y0 * m.s);
      xd[gn] = omegas * v1;
      yd[gn] = omegas * v2;
    }
  }
}

// one thread per (face of family d, snapshot): the mean of the face's four
// node velocities, component by component
__global__ void k_face_vel(DevBlock b, int d, int S2, const double *__restrict__ xd, const double *__restrict__ yd,
                           const double *__restrict__ zd, double *__restrict__ fv) {
  const int ni = d == 1 ? b.im : b.im - 1, nj = d == 2 ? b.jm : b.jm - 1, nk = d == 3 ? b.km : b.km - 1;
  const int64_t nf = (int64_t)ni * nj * nk, total = nf * S2;
  const int64_t I2 = b.im + 2, J2 = b.jm + 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % ni) + 1; r /= ni;
    const int j = (int)(r % nj) + 1; r /= nj;
    const int k = (int)(r % nk) + 1;
    const int n = (int)(r / nk);
    const int64_t g = gs_idx(b, S2, i, j, k, n);
    // the four nodes in the reference's order
    int64_t o[4];
    if (d == 1) { o[0] = I2 + I2 * J2; o[1] = I2; o[2] = I2 * J2; o[3] = 0; }
    else if (d == 2) { o[0] = 1 + I2 * J2; o[1] = 1; o[2] = I2 * J2; o[3] = 0; }
    else { o[0] = 1 + I2; o[1] = 1; o[2] = I2; o[3] = 0; }
    const double *v[3] = {xd, yd, zd};
    double *out = fv + g * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = (v[c][g + o[0]] + v[c][g + o[1]] + v[c][g + o[2]] + v[c][g + o[3]]) / 4;
  }
}

// one thread per (cell 0..imax, 0..jmax, 0..kmax, snapshot): w from the node
// copy src (same layout)
__global__ void k_vert2cell(DevBlock b, int S2, const double *__restrict__ src, double *__restrict__ w) {
  const int im = b.im, jm = b.jm, km = b.km;
  const int64_t nc = (int64_t)(im + 1) * (jm + 1) * (km + 1), total = nc * S2;
  const int64_t I2 = im + 2, J2 = jm + 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = t;
    const int i = (int)(r % (im + 1)); r /= (im + 1);
    const int j = (int)(r % (jm + 1)); r /= (jm + 1);
    const int k = (int)(r % (km + 1));
    const int n = (int)(r / (km + 1));
    const int64_t base = gs_idx(b, S2, 0, 0, 0, n);
    auto W = [&](int a, int c, int e) { return src[base + a + I2 * (c + J2 * (int64_t)e)]; };
    const bool bi = i == 0 || i == im, bj = j == 0 || j == jm, bk = k == 0 || k == km;
    const int i1 = i == 0 ? 1 : im, j1 = j == 0 ? 1 : jm, k1 = k == 0 ? 1 : km;
    double v;
    if (bi && bj && bk) v = W(i1, j1, k1);
    else if (bj && bk) v = (W(i, j1, k1) + W(i + 1, j1, k1)) / 2;
    else if (bi && bk) v = (W(i1, j, k1) + W(i1, j + 1, k1)) / 2;
    else if (bi && bj) v = (W(i1, j1, k) + W(i1, j1, k + 1)) / 2;
    else if (bk) v = (W(i, j, k1) + W(i + 1, j, k1) + W(i, j + 1, k1) + W(i + 1, j + 1, k1)) / 4;
    else if (bj) v = (W(i, j1, k) + W(i + 1, j1, k) + W(i, j1, k + 1) + W(i + 1, j1, k + 1)) / 4;
    else if (bi) v = (W(i1, j, k) + W(i1, j, k + 1) + W(i1, j + 1, k) + W(i1, j + 1, k + 1)) / 4;
    else
      v = (W(i, j, k) + W(i + 1, j, k) + W(i, j + 1, k) + W(i + 1, j + 1, k) + W(i, j, k + 1) + W(i + 1, j, k + 1) +
           W(i, j + 1, k + 1) + W(i + 1, j + 1, k + 1)) / 8;
    w[base + i + I2 * (j + J2 * (int64_t)k)] = v;
  }
}
