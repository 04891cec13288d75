// Shared definitions of the smectic3d_b200 kernels.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "fft_engine.cuh"

namespace shb {
namespace cg = cooperative_groups;

__host__ __device__ constexpr size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Wait for phase ``parity`` of an mbarrier, for about a second at most: on
// expiry set *timeout and return, so that a lost transfer cannot hang the SM.
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* mbar, uint32_t parity, int* timeout) {
  const uint32_t a = smem_u32(mbar);
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return;
    if (clock64() - t0 > (1ll << 31)) {
      atomicExch(timeout, 1);
      return;
    }
  }
}

// Programmatic dependent launch: the step kernels are launched so that they
// may start while the previous kernel of the stream drains; everything before
// this wait touches only data no kernel of the step writes (twiddles,
// wavenumbers, shared memory set-up).
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

enum NonlinKind : int { kQuintic = 0, kQuadCubic = 1 };
enum SchemeKind : int { kCNAB2 = 0, kIMEXEuler = 1 };
enum PassFlags : int {
  kFlPsiOut = 1,    // plane: write psi (double)
  kFlL1 = 2,        // plane: L1 monitor partial sums
  kFlEnergy = 4,    // plane / pencil: energy partial sums
  kFlRealOut = 8,   // plane step: write psi (T) to real_out
  kFlSpecOut = 16,  // pencil step: write psihat^{n+1} (pencil-major) to spec_out
  kFlShell = 32,    // pencil energy pass: spectral power per |k| shell into PencilArgs::shell
};

// Per-launch scalar parameters of the pointwise stages.
struct PointParams {
  double dt;
  double beta, gamma, alpha, q0;
  double eta_rho;       // rho * eta (Stokes)
  double w_mid;         // pinning penalty weight
  double inv_dz2;       // 1 / dz^2
  double scale;         // 1/N^3 (periodic) or 1/(8 N^3) (Neumann)
  int nonlin;           // NonlinKind
  int scheme;           // SchemeKind
  const double* eps;    // per-replica epsilon
};

template <typename T>
__device__ __forceinline__ T nonlin_eval(T p, T beta, T gamma, int kind) {
  const T p2 = p * p;
  // beta psi^3 - gamma psi^5  (periodicFFT/pf3d.cpp:368-369)
  if (kind == kQuintic) return p * p2 * (beta - gamma * p2);
  // beta psi^2 - gamma psi^3
  return p2 * (beta - gamma * p);
}

// dN/dpsi
template <typename T>
__device__ __forceinline__ T nonlin_deriv(T p, T beta, T gamma, int kind) {
  const T p2 = p * p;
  if (kind == kQuintic) return p2 * (T(3) * beta - T(5) * gamma * p2);
  return p * (T(2) * beta - T(3) * gamma * p);
}

// Local part of the Lyapunov density (energyPsi.m:225-228 without the gradient
// term, which is accumulated spectrally).
__device__ __forceinline__ double local_density(double p, double eps, double beta, double gamma, int kind) {
  const double p2 = p * p;
  if (kind == kQuintic) return -0.5 * eps * p2 + p2 * p2 * (-0.25 * beta + gamma / 6.0 * p2);
  return -0.5 * eps * p2 + p2 * p * (-beta / 3.0 + 0.25 * gamma * p);
}

// Kahan-compensated FP64 accumulator
struct KahanSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    double y = x - c;
    double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// Block-wide FP64 sum; every thread returns the total.  ``scratch`` holds one
// double per warp.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) scratch[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  double t = 0.0;
  for (int i = 0; i < nw; ++i) t += scratch[i];
  return t;
}

}  // namespace shb
