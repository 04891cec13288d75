// Surface passes.
//
// surfTrack (periodic; periodicFFT/surfTrack.cpp:592-626, 744-806):
//
// surface_prep (elementwise, state n): from psi, grad psi, L psi, u and the
// second derivatives psi_xx, psi_yy, psi_xy (all real fields) it forms
//   |grad psi|, d_t psi = eps psi - L psi + N(psi) - u.grad psi   (= C2R of
//   scale (aLin psihat + Nhat), since aLin = eps - opSH), H-numerator
//   psi_xx + psi_yy and K-numerator psi_xx psi_yy - psi_xy^2.
// surface_scan (one thread per (x, y) column, state n+1): the first psi < 0
// after psi > 0.1 scanning +z, stepping back one voxel when that one is closer
// to zero; outputs the unadjusted z index (the reference writes k), v_n, H, K.
//
// Neumann curvature pass (cosFFT/comet/cosNoAdvMorphCurv.cpp:742-965):
// curv_scan, one thread per (x, y) column at state n, scanning -z from the top
// for the first psi < 0 after psi > 0.7 and moving up one voxel when that one
// is closer to zero; at that voxel the gradient is taken by centred
// differences (one-sided at the walls), the mixed derivatives as differences
// of the gradient, psi_xx, psi_yy, psi_zz and L psi come from the spectral
// fields, d_t psi = eps psi - L psi + N(psi), and Megrabov's H and K follow.
#pragma once
#include "sh_common.cuh"

namespace shb {

// Gradient of psi on the Neumann box by centred differences, one-sided at the
// walls: (psi[i+1] - psi[i-1]) / 2dx inside, 2 (psi[1] - psi[0]) / 2dx and
// 2 (psi[N-1] - psi[N-2]) / 2dx at the walls, in x, y and z
// (cosFFT/comet/morphSurfK.cpp:700-766).  One thread per point, replicas in y.
template <typename T>
__global__ void grad_wall_kernel(const T* __restrict__ psi, T* __restrict__ gx, T* __restrict__ gy,
                                 T* __restrict__ gz, int n, T inv2dx) {
  const long long n3 = (long long)n * n * n, nn = (long long)n * n;
  const size_t off = size_t(blockIdx.y) * n3;
  const T* p = psi + off;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x) {
    const int z = int(i % n), y = int((i / n) % n), x = int(i / nn);
    auto diff = [&](int c, long long s) {
      if (c == 0) return T(2) * (p[i + s] - p[i]) * inv2dx;
      if (c == n - 1) return T(2) * (p[i] - p[i - s]) * inv2dx;
      return (p[i + s] - p[i - s]) * inv2dx;
    };
    gx[off + i] = diff(x, nn);
    gy[off + i] = diff(y, n);
    gz[off + i] = diff(z, 1);
  }
}

template <typename T>
struct SurfArgs {
  const T* psi;      // state n
  const T* gx;
  const T* gy;
  const T* gz;
  const T* lpsi;
  const T* ux;
  const T* uy;
  const T* uz;
  T* dxx;            // in: psi_xx  out: |grad psi|
  T* dyy;            // in: psi_yy  out: d_t psi
  T* dxy;            // in: psi_xy  out: psi_xx psi_yy - psi_xy^2
  T* hnum;           // out: psi_xx + psi_yy
  PointParams pp;
  long long n3;
  int n;
};

template <typename T>
__global__ void surface_prep_kernel(SurfArgs<T> a) {
  const int rep = blockIdx.y;
  const T eps = T(a.pp.eps[rep]);
  const T beta = T(a.pp.beta), gamma = T(a.pp.gamma);
  const T cpen = T(2.0 * a.pp.w_mid * a.pp.inv_dz2);
  const int n = a.n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n3; i += (long long)gridDim.x * blockDim.x) {
    const size_t j = size_t(rep) * a.n3 + i;
    const T p = a.psi[j];
    const T gx = a.gx[j], gy = a.gy[j], gz = a.gz[j];
    T nl = nonlin_eval<T>(p, beta, gamma, a.pp.nonlin) - (a.ux[j] * gx + a.uy[j] * gy + a.uz[j] * gz);
    if (a.pp.w_mid != 0.0 && int(i % n) == n / 2) nl += cpen * (a.psi[j - 1] - T(2) * p + a.psi[j + 1]);
    const T xx = a.dxx[j], yy = a.dyy[j], xy = a.dxy[j];
    a.hnum[j] = xx + yy;
    a.dxy[j] = xx * yy - xy * xy;
    a.dyy[j] = eps * p - a.lpsi[j] + nl;
    a.dxx[j] = sqrt(gx * gx + gy * gy + gz * gz);
  }
}

template <typename T>
__global__ void surface_scan_kernel(const T* __restrict__ psi_new, const T* __restrict__ gradmag,
                                    const T* __restrict__ dtpsi, const T* __restrict__ hnum, const T* __restrict__ knum,
                                    int n, int* __restrict__ zout, double* __restrict__ vn, double* __restrict__ hh,
                                    double* __restrict__ kk) {
  const int rep = blockIdx.y;
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)n * n) return;
  const size_t base = (size_t(rep) * n * n + col) * n;
  const size_t o = size_t(rep) * n * n + col;
  int track = 0;
  int zf = -1;
  size_t idx = 0;
  for (int k = 0; k < n; ++k) {
    const T v = psi_new[base + k];
    if (v > T(0.1) && track == 0) track = 1;
    if (v < T(0) && track == 1) {
      idx = base + k;
      if (fabs(v) > fabs(psi_new[base + k - 1])) idx = base + k - 1;
      zf = k;
      break;
    }
  }
  zout[o] = zf;
  if (zf < 0) {
    vn[o] = hh[o] = kk[o] = nan("");
    return;
  }
  const double g = double(gradmag[idx]);
  vn[o] = double(dtpsi[idx]) / g;
  hh[o] = double(hnum[idx]) / g;
  kk[o] = double(knum[idx]) / (g * g);
}

template <typename T>
struct CurvArgs {
  const T* psi;    // state n, [rep][x][y][z]
  const T* dxx;    // psi_xx, psi_yy, psi_zz (spectral)
  const T* dyy;
  const T* dzz;
  const T* lpsi;   // L psi = opSH psi
  const T* wall;   // substrate term of N, planes z < kwall (optional)
  const T* lperp;
  int kwall;
  PointParams pp;
  int n;
  double dx;
  int* zout;
  double* vn;
  double* hh;
  double* kk;
  // optional exact derivatives of the cosine series: psi_x, psi_y, psi_z,
  // psi_xy, psi_xz, psi_yz (in place of the differences; all or none)
  const T* spec[6];
};

// centred difference along one axis (stride s, index i of n), one-sided at the walls
template <typename T>
__device__ __forceinline__ double curv_grad(const T* f, size_t at, size_t s, int i, int n, double td) {
  if (i > 0 && i < n - 1) return (double(f[at + s]) - double(f[at - s])) / td;
  if (i == 0) return 2.0 * (double(f[at + s]) - double(f[at])) / td;
  return 2.0 * (double(f[at]) - double(f[at - s])) / td;
}

template <typename T>
__global__ void curv_scan_kernel(CurvArgs<T> a) {
  const int rep = blockIdx.y;
  const int n = a.n;
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)n * n) return;
  const int i = int(col / n), j = int(col % n);
  const size_t sx = size_t(n) * n, sy = size_t(n);
  const size_t base = size_t(rep) * n * sx + size_t(col) * n;  // (rep, i, j, 0)
  const size_t o = size_t(rep) * n * n + col;
  const T* psi = a.psi;
  int k2 = -1, kf = -1;
  int track = 0;
  for (int k = n - 1; k >= 0; --k) {
    const T v = psi[base + k];
    if (v > T(0.7) && track == 0) track = 1;
    if (v < T(0) && track == 1) {
      kf = k;
      k2 = fabs(double(v)) > fabs(double(psi[base + k + 1])) ? k + 1 : k;
      break;
    }
  }
  a.zout[o] = k2;
  if (k2 < 0) {
    a.vn[o] = a.hh[o] = a.kk[o] = nan("");
    return;
  }
  const double td = 2.0 * a.dx;
  const size_t at = base + k2;
  const bool spec = a.spec[0] != nullptr;
  const double gx = spec ? double(a.spec[0][at]) : curv_grad(psi, at, sx, i, n, td);
  const double gy = spec ? double(a.spec[1][at]) : curv_grad(psi, at, sy, j, n, td);
  const double gz = spec ? double(a.spec[2][at]) : curv_grad(psi, at, 1, k2, n, td);
  const double g = sqrt(gx * gx + gy * gy + gz * gz);
  // psi_xy: y difference of the x gradient at k2
  double dxy;
  {
    const int jp = j < n - 1 ? j + 1 : j, jm = j > 0 ? j - 1 : j;
    const double gp = curv_grad(psi, at + (size_t(jp) - j) * sy, sx, i, n, td);
    const double gm = curv_grad(psi, at - (size_t(j) - jm) * sy, sx, i, n, td);
    dxy = (j > 0 && j < n - 1) ? (gp - gm) / td : 2.0 * (gp - gm) / td;
  }
  // psi_xz, psi_yz: z differences of the x and y gradients; the formula follows
  // the scan index k, as the reference does, and the top of the column is one-sided
  double dxz, dyz;
  {
    int zp, zm;
    if (kf > 0 && kf < n - 1 && k2 + 1 < n) {
      zp = k2 + 1;
      zm = k2 - 1;
    } else if (kf == 0) {
      zp = k2 + 1;
      zm = k2;
    } else {
      zp = k2;
      zm = k2 - 1;
    }
    const double c = (zp - zm == 2) ? 1.0 : 2.0;
    dxz = c * (curv_grad(psi, base + zp, sx, i, n, td) - curv_grad(psi, base + zm, sx, i, n, td)) / td;
    dyz = c * (curv_grad(psi, base + zp, sy, j, n, td) - curv_grad(psi, base + zm, sy, j, n, td)) / td;
  }
  if (spec) {
    dxy = a.spec[3][at];
    dxz = a.spec[4][at];
    dyz = a.spec[5][at];
  }
  const double xx = a.dxx[at], yy = a.dyy[at], zz = a.dzz[at];
  const double p = psi[at];
  double nl = double(nonlin_eval<double>(p, a.pp.beta, a.pp.gamma, a.pp.nonlin));
  if (a.pp.w_mid != 0.0 && k2 == n / 2)
    nl += 2.0 * a.pp.w_mid * a.pp.inv_dz2 * (double(psi[at - 1]) - 2.0 * p + double(psi[at + 1]));
  if (k2 < a.kwall) nl += double(a.wall[k2]) * double(a.lperp[(size_t(rep) * sx + col) * a.kwall + k2]);
  const double dt_psi = a.pp.eps[rep] * p - double(a.lpsi[at]) + nl;
  a.vn[o] = dt_psi / g;
  a.hh[o] = ((gy * gy + gz * gz) * xx + (gx * gx + gz * gz) * yy + (gx * gx + gy * gy) * zz -
             2.0 * (gx * gy * dxy + gx * gz * dxz + gy * gz * dyz)) /
            (g * g * g);
  a.kk[o] = (gz * gz * (xx * yy - dxy * dxy) + gx * gx * (yy * zz - dyz * dyz) + gy * gy * (xx * zz - dxz * dxz) +
             2.0 * (gy * dxy * (gz * dxz - gx * zz) + gx * dxz * (gy * dyz - gz * yy) + gz * dyz * (gx * dxy - gy * xx))) /
            (g * g * g * g);
}

}  // namespace shb
