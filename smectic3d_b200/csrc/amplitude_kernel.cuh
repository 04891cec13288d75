// Local-amplitude map of cosFFT/comet/morphSurfAmp.cpp:1005-1125.
//
// psiAvg(i,j,k) = T3[psi^2 over the box [i +- nl] x [j +- nl] x [k +- nl],
// clipped to the grid] / (psiRef * l1 l2 l3 / lambda^3), with T3 the nested
// trapezoid rule of the reference (trapz, morphSurfAmp.cpp:76-86), nl = Nw/2,
// l_a the clipped box edge lengths, lambda = 2 pi / q0 and psiRef the same
// integral over the fixed box [nl, 3 nl]^3.  The box is a product domain, so
// T3 is three 1-D clipped-window trapezoids, one axis after the other: each
// pass is a sliding-window sum along its lines (O(N^3) in all, where the
// reference's loops cost O(N^3 Nw^3)).
#pragma once
#include <cuda_runtime.h>

namespace shb {

// One line per thread: out[p] = h (sum f[a..b] - (f[a] + f[b]) / 2), a = max(0, p - nl),
// b = min(n - 1, p + nl), along axis 0 (x), 1 (y) or 2 (z) of [rep][x][y][z].
// ``square`` squares the input on the fly (first pass).
__global__ void amp_window_kernel(const double* __restrict__ in, double* __restrict__ out, int n, int axis, int nl,
                                  double h, int square) {
  const long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (line >= (long long)n * n) return;
  const size_t n3 = size_t(n) * n * n;
  const size_t rep = blockIdx.y;
  const int u = int(line / n), w = int(line % n);
  size_t base, stride;
  if (axis == 0) {  // lines (y=u, z=w) along x: neighbouring threads read neighbouring z
    base = (size_t(u) * n + w);
    stride = size_t(n) * n;
  } else if (axis == 1) {  // lines (x=u, z=w) along y
    base = size_t(u) * n * n + w;
    stride = size_t(n);
  } else {  // lines (x=u, y=w) along z
    base = (size_t(u) * n + w) * n;
    stride = 1;
  }
  const double* src = in + rep * n3 + base;
  double* dst = out + rep * n3 + base;
  auto f = [&](int m) {
    const double v = src[size_t(m) * stride];
    return square ? v * v : v;
  };
  double run = 0.0;
  for (int m = 0; m <= nl && m < n; ++m) run += f(m);
  for (int p = 0; p < n; ++p) {
    const int a = p - nl > 0 ? p - nl : 0, b = p + nl < n - 1 ? p + nl : n - 1;
    dst[size_t(p) * stride] = h * (run - 0.5 * (f(a) + f(b)));
    if (p + 1 + nl < n) run += f(p + 1 + nl);
    if (p - nl >= 0) run -= f(p - nl);
  }
}

// psiAvg = T3 / (psiRef l1 l2 l3 / lambda^3), psiRef = T3 at (2 nl, 2 nl, 2 nl)
__global__ void amp_normalise_kernel(const double* __restrict__ t3, double* __restrict__ out, int n, int nl, double dx,
                                     double lambda3) {
  const size_t n3 = size_t(n) * n * n;
  const size_t rep = blockIdx.y;
  const double ref = t3[rep * n3 + (size_t(2 * nl) * n + 2 * nl) * n + 2 * nl];
  for (size_t idx = blockIdx.x * size_t(blockDim.x) + threadIdx.x; idx < n3; idx += size_t(gridDim.x) * blockDim.x) {
    const int i = int(idx / (size_t(n) * n)), j = int((idx / n) % n), k = int(idx % n);
    auto len = [&](int c) {
      const int a = c - nl > 0 ? c - nl : 0, b = c + nl < n - 1 ? c + nl : n - 1;
      return (b - a) * dx;
    };
    out[rep * n3 + idx] = t3[rep * n3 + idx] / (ref * len(i) * len(j) * len(k) / lambda3);
  }
}

}  // namespace shb
