// Wall force and moment integration of one surface: force_b
// (src/output.f90:4388-4900).
//
//  k_force_faces  one thread per wall face and snapshot: the pressure force
//                 and moment of the face (src/output.f90:4660-4700) and, for
//                 viscous flows, the skin-friction force and moment from the
//                 one-sided three-point wall derivative (4703-4860); the 12
//                 raw sums are written per face as buf[(n*12 + c)*nfaces + f].
//  k_force_sum    one CTA per (block, snapshot): fixed-order tree sum of the
//                 faces of the block, so the result does not depend on the
//                 launch; the host turns the block sums into coefficients in
//                 block order as force() does (src/output.f90:4283-4320).
#pragma once
#include "common.cuh"

// one face of a 15xx patch: halo cell (i,j,k) of the wall side, patch
// direction d (1..3) and sgn = (-1)**(1+1/inrout)
struct ForceFace {
  int32_t blk, d, sgn, i, j, k;
};

__global__ void k_force_faces(const DevBlock *__restrict__ blocks, const cosa_params *__restrict__ Pp,
                              const ForceFace *__restrict__ faces, int nfaces, const double *__restrict__ q,
                              const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ si,
                              const double *__restrict__ sj, const double *__restrict__ sk,
                              const double *__restrict__ vm, int64_t n0, const double *__restrict__ xmoms,
                              double *__restrict__ buf, const double *__restrict__ cvx = nullptr,
                              const double *__restrict__ cvy = nullptr, const double *__restrict__ cvz = nullptr) {
  // xmoms: the moment centre of every snapshot (3 doubles each; on moving
  // grids carried with the body, src/output.f90:4476-4485); metrics and
  // nodes of snapshot n hbmove; on moving grids the inverse metrics of
  // snapshot nh at vm + nh * 27 n0 and the cell grid velocities cv* (node
  // layout) make the wall derivative one of the velocity relative to the grid
  const cosa_params &P = *Pp;
  const int npde = P.npde, S = 2 * P.nharms + 1, S2 = 2 * P.nharms * P.hbmove + 1;
  const int64_t total = (int64_t)nfaces * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int f = (int)(t % nfaces), n = (int)(t / nfaces);
    const ForceFace F = faces[f];
    const DevBlock b = blocks[F.blk];
    const int d = F.d, sgn = F.sgn;
    const int di = d == 1, dj = d == 2, dk = d == 3;
    // face index ibcm: one past the halo on inrout = 1 patches, the halo index on inrout = 2
    const int up = sgn > 0 ? 1 : 0;
    const int mi = F.i + up * di, mj = F.j + up * dj, mk = F.k + up * dk;
    const double *s = d == 1 ? si : (d == 2 ? sj : sk);
    const int nh = n * P.hbmove;
    const double xm0 = xmoms[3 * n], xm1 = xmoms[3 * n + 1], xm2 = xmoms[3 * n + 2];
    const int64_t e = p2_idx(b, S2, 1, mi, mj, mk, nh);
    const double kx = sgn * s[e], ky = sgn * s[e + 1], kz = sgn * s[e + 2], ds = s[e + 3];
    const int64_t hc = p3_cell(b, F.i, F.j, F.k);
    auto Q = [&](int v, int64_t cell) { return q[p3_var(b, npde, S, v, n) + cell]; };
    const double r = Q(1, hc);
    const double u2 = Q(2, hc), v2 = Q(3, hc), w2 = Q(4, hc);
    const double pw = (P.gamma - 1) * (Q(5, hc) - u2 * u2 / r / 2 - v2 * v2 / r / 2 - w2 * w2 / r / 2);
    // moment arm: node (ibcw) with the halo cell's index
    const int64_t I2 = b.im + 2, J2 = b.jm + 2;
    const int64_t gw = b.op2 * S2 + (int64_t)nh * I2 * J2 * (b.km + 2) + F.i + I2 * (F.j + J2 * (int64_t)F.k);
    const double xr = x[gw] - xm0, yr = y[gw] - xm1, zr = z[gw] - xm2;
    double o[12];
    o[0] = -pw * kx * ds;
    o[1] = -pw * ky * ds;
    o[2] = -pw * kz * ds;
    o[3] = (ky * zr - kz * yr) * pw * ds;
    o[4] = (kz * xr - kx * zr) * pw * ds;
    o[5] = (kx * yr - ky * xr) * pw * ds;
    if (P.viscous) {
      const int64_t vb = (int64_t)nh * 27 * n0 + ((int64_t)((d - 1) * 3 + (d - 1)) * 3) * n0 + b.of0 * 3 +
                         ((mi - 1) + (int64_t)b.im * ((mj - 1) + (int64_t)b.jm * (mk - 1))) * 3;
      const double ex = vm[vb], ey = vm[vb + 1], ez = vm[vb + 2];
      const double tw = pw * P.gamma / r;
      const double muw = (P.stemp + 1) / (tw + P.stemp) * (tw * sqrt(tw));
      const int64_t c1 = p3_cell(b, F.i + sgn * di, F.j + sgn * dj, F.k + sgn * dk);
      const int64_t c2 = p3_cell(b, F.i + 2 * sgn * di, F.j + 2 * sgn * dj, F.k + 2 * sgn * dk);
      const double r1 = Q(1, c1), r2 = Q(1, c2);
      // node-layout offsets of the three cells (src/output.f90:4768-4806)
      const int64_t g0 = b.op2 * S2 + (int64_t)nh * I2 * J2 * (b.km + 2);
      const int64_t gh = g0 + F.i + I2 * (F.j + J2 * (int64_t)F.k);
      const int64_t g1 = gh + sgn * (di + I2 * (dj + J2 * (int64_t)dk));
      const int64_t g2 = gh + 2 * sgn * (di + I2 * (dj + J2 * (int64_t)dk));
      double eta[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double uw = Q(m + 2, hc) / r, ua = Q(m + 2, c1) / r1, ub = Q(m + 2, c2) / r2;
        if (cvx) {
          const double *cv = m == 0 ? cvx : (m == 1 ? cvy : cvz);
          uw = uw - cv[gh]; ua = ua - cv[g1]; ub = ub - cv[g2];
        }
        eta[m] = sgn * (-8 * uw + 9 * ua - ub) / 3;
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
      const double mor = P.machfs / P.reyno;
      o[6] = mor * ds * tx;
      o[7] = mor * ds * ty;
      o[8] = mor * ds * tz;
      o[9] = mor * ds * (-ty * zr + tz * yr);
      o[10] = mor * ds * (-tz * xr + tx * zr);
      o[11] = mor * ds * (-tx * yr + ty * xr);
    } else {
#pragma unroll
      for (int c = 6; c < 12; ++c) o[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < 12; ++c) buf[((int64_t)n * 12 + c) * nfaces + f] = o[c];
  }
}

// blockIdx.x = block of the table, blockIdx.y = snapshot; faces of block b
// are [bstart[b], bstart[b+1]); 256 threads
__global__ void __launch_bounds__(256) k_force_sum(const int *__restrict__ bstart, int nfaces,
                                                   const double *__restrict__ buf, double *__restrict__ sums) {
  __shared__ double red[12][256];
  const int b = blockIdx.x, n = blockIdx.y, nb = gridDim.x;
  const int f0 = bstart[b], f1 = bstart[b + 1];
  double acc[12];
#pragma unroll
  for (int c = 0; c < 12; ++c) acc[c] = 0.0;
  for (int f = f0 + threadIdx.x; f < f1; f += blockDim.x)
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] += buf[((int64_t)n * 12 + c) * nfaces + f];
#pragma unroll
  for (int c = 0; c < 12; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 12; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 12) sums[((int64_t)n * nb + b) * 12 + threadIdx.x] = red[threadIdx.x][0];
}
