// surfTrack surface pass (periodicFFT/surfTrack.cpp:592-626, 744-806).
//
// surface_prep (elementwise, state n): from psi, grad psi, L psi, u and the
// second derivatives psi_xx, psi_yy, psi_xy (all real fields) it forms
//   |grad psi|, d_t psi = eps psi - L psi + N(psi) - u.grad psi   (= C2R of
//   scale (aLin psihat + Nhat), since aLin = eps - opSH), H-numerator
//   psi_xx + psi_yy and K-numerator psi_xx psi_yy - psi_xy^2.
// surface_scan (one thread per (x, y) column, state n+1): the first psi < 0
// after psi > 0.1 scanning +z, stepping back one voxel when that one is closer
// to zero; outputs the unadjusted z index (the reference writes k), v_n, H, K.
#pragma once
#include "sh_common.cuh"

namespace shb {

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

}  // namespace shb
