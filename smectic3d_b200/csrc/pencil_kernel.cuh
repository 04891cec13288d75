// Pencil pass: the x transform, fused with the spectral time update.
//
// A CTA owns TK consecutive in-plane positions f (128 bytes of every x-plane
// row, so each x step is one coalesced segment) and all N values of x.  The
// forward x transform completes the 3-D spectrum of the nonlinear term; the
// CNAB2 update runs in registers; the inverse x transform of the new psi
// spectrum starts from the same registers (the inverse radix plan is the
// forward plan reversed).
//
// The spectral state is W^n = C1 psihat^n - dt/2 Nhat^{n-1}, stored
// pencil-major ([f][kx], kx contiguous) so that each thread's register slots
// map to coalesced addresses.  The reference update
//   psihat^{n+1} = (C1 psihat^n + dt/2 (3 Nhat^n - Nhat^{n-1})) / C2
// (periodicFFT/pf3d.cpp:476-478, cosFFT/mesabi/cosNoAdvMorph.cpp:524-525)
// becomes psihat^{n+1} = (W^n + 3 dt/2 Nhat^n) / C2 and
// W^{n+1} = C1 psihat^{n+1} - dt/2 Nhat^n: one state read and one write.
#pragma once
#include "sh_common.cuh"

namespace shb {

enum PencilMode : int { kPencilStep = 0, kPencilInit = 1, kPencilEnergy = 2 };

template <typename T, int N, bool DCT>
struct PencilCfg {
  static constexpr int E = Plan<N>::E;
  static constexpr int G = N / E;
  static constexpr int TK = sizeof(T) == 4 ? 16 : 8;
  static constexpr int THREADS = TK * G;
  static constexpr int LS = line_stride(N);
  static constexpr int FP = DCT ? N * (N / 2) : N * (N / 2 + 1);
  static constexpr int TILES = FP / TK;
  static constexpr int RL = radix_of<N, -1, Plan<N>::P - 1>();
  static constexpr size_t TW_OFF = size_t(TK) * LS * sizeof(cplx<T>);
  static constexpr size_t RED_OFF = TW_OFF + size_t(tw_total<N>()) * sizeof(cplx<T>);
  static constexpr size_t SMEM = RED_OFF + 64 * sizeof(double);
  static_assert(FP % TK == 0, "tile must divide the plane");
  static_assert(THREADS % 32 == 0, "pencil CTA must be whole warps");
};

template <typename T>
struct PencilArgs {
  const cplx<T>* src;   // step: partial of N ; init: partial of psi   [rep][x][FP]
  const cplx<T>* src2;  // init: partial of N(psi)
  cplx<T>* w;           // state W [rep][FP][N]
  cplx<T>* dst;         // partial of scale * psihat^{n+1}, x-inverse applied [rep][x][FP]
  double* red;          // per-CTA spectral energy partial [rep][grid.x]
  int* nonfinite;       // set to 1 when a new coefficient is NaN/Inf
  const T* q;           // wavenumber table (N entries)
  const cplx<T>* tw;    // twiddle table [forward | inverse | quarter-wave]
  PointParams pp;
  int flags;
};

template <typename T, int N, bool DCT>
struct PencilOps {
  using Cfg = PencilCfg<T, N, DCT>;
  static constexpr int E = Cfg::E, G = Cfg::G, TK = Cfg::TK, LS = Cfg::LS, FP = Cfg::FP, RL = Cfg::RL;

  // TK * N == THREADS * E: all E loads of a thread are issued before its stores
  static __device__ __forceinline__ void load_tile(cplx<T>* buf, const cplx<T>* __restrict__ src, int f0) {
    cplx<T> tmp[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + Cfg::THREADS * e;
      tmp[e] = src[size_t(idx / TK) * FP + f0 + idx % TK];
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + Cfg::THREADS * e;
      buf[(idx % TK) * LS + pad(idx / TK)] = tmp[e];
    }
  }
  static __device__ __forceinline__ void store_tile(const cplx<T>* buf, cplx<T>* __restrict__ dst, int f0) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + Cfg::THREADS * e;
      dst[size_t(idx / TK) * FP + f0 + idx % TK] = buf[(idx % TK) * LS + pad(idx / TK)];
    }
  }

  // forward x transform of the line; result in registers at kx = out_index<N,-1>
  static __device__ __forceinline__ void forward(cplx<T> (&v)[E], cplx<T>* L, int t, const TwTables<T>& tw) {
    if constexpr (!DCT) {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(i)]; });
    } else {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(i < N / 2 ? 2 * i : 2 * (N - 1 - i) + 1)]; });
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) L[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          cplx<T> w = tw.d[k];
          v[b * RL + r] = cadd<T>(cmul<T>(L[pad(k)], w), cmul<T>(L[pad((N - k) & (N - 1))], conjg<T>(w)));
        }
    }
  }

  // inverse x transform of register values at kx = out_index<N,-1>; result
  // written to the line in natural x order (caller syncs before reading)
  static __device__ __forceinline__ void inverse_to_line(cplx<T> (&v)[E], cplx<T>* L, int t,
                                                         const TwTables<T>& tw) {
    constexpr int RLI = radix_of<N, +1, Plan<N>::P - 1>();
    if constexpr (!DCT) {
      fft_regs<T, N, +1>(v, L, t, tw.i);
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RLI; ++b)
#pragma unroll
        for (int r = 0; r < RLI; ++r) L[pad(out_index<N, +1>(t, b, r))] = v[b * RLI + r];
    } else {
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) L[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncwarp();
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) {
        cplx<T> a = L[pad(i)];
        cplx<T> u = a;
        if (i != 0) {
          cplx<T> bb = L[pad(N - i)];
          u = mk<T>(a.x + bb.y, a.y - bb.x);
        }
        cplx<T> w = tw.d[i];
        w.y = -w.y;
        return cmul<T>(u, w);
      });
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RLI; ++b)
#pragma unroll
        for (int r = 0; r < RLI; ++r) {
          const int n = out_index<N, +1>(t, b, r);
          L[pad(n < N / 2 ? 2 * n : 2 * (N - 1 - n) + 1)] = v[b * RLI + r];
        }
    }
  }
};

// Spectral multipliers of mode (kx, ky, kz) for replica epsilon ``eps``
template <typename T>
struct Mult {
  T mq2, a_lin, c1, c2;
};
template <typename T>
__device__ __forceinline__ Mult<T> make_mult(T qx, T qy, T qz, T eps, const PointParams& pp) {
  Mult<T> m;
  m.mq2 = qx * qx + qy * qy + qz * qz;
  const T d = m.mq2 - T(pp.q0 * pp.q0);
  const T op_sh = T(pp.alpha) * d * d;
  m.a_lin = eps - op_sh;
  const T h = T(0.5 * pp.dt);
  m.c1 = T(1) + h * m.a_lin;
  m.c2 = T(1) - h * m.a_lin;
  return m;
}

// correctly rounded reciprocal
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }

template <typename T, int N, bool DCT, int MODE>
__global__ void __launch_bounds__(PencilCfg<T, N, DCT>::THREADS)
pencil_kernel(PencilArgs<T> a) {
  using Cfg = PencilCfg<T, N, DCT>;
  using Ops = PencilOps<T, N, DCT>;
  constexpr int E = Cfg::E, G = Cfg::G, TK = Cfg::TK, LS = Cfg::LS, FP = Cfg::FP, RL = Cfg::RL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  double* scratch = reinterpret_cast<double*>(smem_raw + Cfg::RED_OFF);
  const TwTables<T> tw =
      stage_twiddles<T, N>(reinterpret_cast<cplx<T>*>(smem_raw + Cfg::TW_OFF), a.tw, threadIdx.x, Cfg::THREADS);

  const int f0 = blockIdx.x * TK;
  const int rep = blockIdx.y;
  const int line = threadIdx.x / G, t = threadIdx.x % G;
  const int f = f0 + line;
  cplx<T>* L = buf + line * LS;
  const size_t plane_base = size_t(rep) * N * FP;
  cplx<T>* wrow = a.w + (size_t(rep) * FP + f) * N;
  const T eps = T(a.pp.eps[rep]);
  const T scale = T(a.pp.scale);

  // in-plane wavenumber indices of this line
  int ky, kz;
  if (DCT) {
    ky = f / (N / 2);
    kz = 2 * (f % (N / 2));  // the pair holds kz and kz + 1
  } else if (f < N * (N / 2)) {
    ky = f / (N / 2);
    kz = f % (N / 2);
  } else {
    ky = f - N * (N / 2);
    kz = N / 2;
  }
  const T qy = __ldg(&a.q[ky]);
  const T qz0 = __ldg(&a.q[kz]);
  const T qz1 = DCT ? __ldg(&a.q[kz + 1]) : T(0);

  cplx<T> v[E];
  KahanSum acc;
  const bool want_energy = (a.flags & kFlEnergy) != 0;

  if constexpr (MODE == kPencilStep) {
    Ops::load_tile(buf, a.src + plane_base, f0);
    // the state W of this line, fetched while the transform runs
    cplx<T> wreg[E];
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) wreg[b * RL + r] = wrow[out_index<N, -1>(t, b, r)];
    __syncthreads();
    Ops::forward(v, L, t, tw);
    // mode-independent constants of the update; the (ky, kz) part of |q|^2 is
    // fixed for the line
    const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha);
    const T h = T(0.5 * a.pp.dt), h3 = T(1.5 * a.pp.dt), dtT = T(a.pp.dt);
    const T qyz0 = qy * qy + qz0 * qz0 - q02;
    const T qyz1 = qy * qy + qz1 * qz1 - q02;
    const bool cnab2 = a.pp.scheme == kCNAB2;
    bool bad = false;
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kx = out_index<N, -1>(t, b, r);
        const T qx = __ldg(&a.q[kx]);
        const T qx2 = qx * qx;
        cplx<T> wv = wreg[b * RL + r];
        const cplx<T> nh = v[b * RL + r];
        cplx<T> pn;
        // psihat^{n+1} = (W + 3dt/2 Nhat) / C2,  W' = C1 psihat^{n+1} - dt/2 Nhat  (CNAB2)
        // psihat^{n+1} = (psihat + dt Nhat) / (1 - dt aLin),  W' = psihat^{n+1} (IMEX Euler)
        const T d0 = qx2 + qyz0;
        const T a0 = eps - alpha * d0 * d0;
        if (cnab2) {
          const T inv0 = rcp_rn(T(1) - h * a0), c10 = T(1) + h * a0;
          pn.x = (wv.x + h3 * nh.x) * inv0;
          wv.x = c10 * pn.x - h * nh.x;
          if constexpr (!DCT) {
            pn.y = (wv.y + h3 * nh.y) * inv0;
            wv.y = c10 * pn.y - h * nh.y;
          } else {
            const T d1 = qx2 + qyz1;
            const T a1 = eps - alpha * d1 * d1;
            const T inv1 = rcp_rn(T(1) - h * a1);
            pn.y = (wv.y + h3 * nh.y) * inv1;
            wv.y = (T(1) + h * a1) * pn.y - h * nh.y;
          }
        } else {
          const T inv0 = rcp_rn(T(1) - dtT * a0);
          pn.x = (wv.x + dtT * nh.x) * inv0;
          if constexpr (!DCT) {
            pn.y = (wv.y + dtT * nh.y) * inv0;
          } else {
            const T d1 = qx2 + qyz1;
            pn.y = (wv.y + dtT * nh.y) * rcp_rn(T(1) - dtT * (eps - alpha * d1 * d1));
          }
          wv = pn;
        }
        if (want_energy) {
          if constexpr (!DCT) {
            const double d = double(d0);
            const double wgt = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
            acc.add(wgt * d * d * (double(pn.x) * pn.x + double(pn.y) * pn.y));
          } else {
            const double wxy = (kx == 0 ? 0.5 : 1.0) * (ky == 0 ? 0.5 : 1.0);
            const double e0 = double(d0), e1 = double(qx2 + qyz1);
            acc.add(wxy * ((kz == 0 ? 0.5 : 1.0) * e0 * e0 * double(pn.x) * pn.x + e1 * e1 * double(pn.y) * pn.y));
          }
        }
        bad |= !isfinite(pn.x) || !isfinite(pn.y);
        wrow[kx] = wv;
        v[b * RL + r] = cscale<T>(pn, scale);
      }
    if (bad) *a.nonfinite = 1;
  } else if constexpr (MODE == kPencilEnergy) {
    // gradient part of the energy of the current state from its partial P
    Ops::load_tile(buf, a.src + plane_base, f0);
    __syncthreads();
    Ops::forward(v, L, t, tw);
    // P = IDFT_x(scale psihat): its forward x transform is N scale psihat
    // (REDFT10 after REDFT01: 2N scale psihat)
    const double inv = 1.0 / (a.pp.scale * (DCT ? 2 * N : N));
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kx = out_index<N, -1>(t, b, r);
        const T qx = __ldg(&a.q[kx]);
        const double px = double(v[b * RL + r].x) * inv, py = double(v[b * RL + r].y) * inv;
        const double q02 = double(a.pp.q0) * a.pp.q0;
        if constexpr (!DCT) {
          const double d = q02 - double(qx * qx + qy * qy + qz0 * qz0);
          const double wgt = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
          acc.add(wgt * d * d * (px * px + py * py));
        } else {
          const double wxy = (kx == 0 ? 0.5 : 1.0) * (ky == 0 ? 0.5 : 1.0);
          const double d0 = q02 - double(qx * qx + qy * qy + qz0 * qz0);
          const double d1 = q02 - double(qx * qx + qy * qy + qz1 * qz1);
          acc.add(wxy * ((kz == 0 ? 0.5 : 1.0) * d0 * d0 * px * px + d1 * d1 * py * py));
        }
      }
  } else {  // kPencilInit: W^0 from psi^0 and N(psi^0); P^0 from psi^0
    Ops::load_tile(buf, a.src + plane_base, f0);
    __syncthreads();
    Ops::forward(v, L, t, tw);
    cplx<T> vn[E];
    __syncthreads();
    Ops::load_tile(buf, a.src2 + plane_base, f0);
    __syncthreads();
    Ops::forward(vn, L, t, tw);
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kx = out_index<N, -1>(t, b, r);
        const T qx = __ldg(&a.q[kx]);
        const cplx<T> ph = v[b * RL + r], nh = vn[b * RL + r];
        cplx<T> wv;
        const Mult<T> m0 = make_mult<T>(qx, qy, qz0, eps, a.pp);
        const Mult<T> m1 = DCT ? make_mult<T>(qx, qy, qz1, eps, a.pp) : m0;
        if (a.pp.scheme == kCNAB2) {
          wv.x = m0.c1 * ph.x - T(0.5 * a.pp.dt) * nh.x;
          wv.y = m1.c1 * ph.y - T(0.5 * a.pp.dt) * nh.y;
        } else {
          wv = ph;
        }
        wrow[kx] = wv;
        v[b * RL + r] = cscale<T>(ph, scale);
      }
  }

  if constexpr (MODE != kPencilEnergy) {
    Ops::inverse_to_line(v, L, t, tw);
    __syncthreads();
    Ops::store_tile(buf, a.dst + plane_base, f0);
  }

  if (want_energy && MODE != kPencilInit) {
    const double tot = block_sum(acc.s, scratch);
    if (threadIdx.x == 0) a.red[size_t(rep) * gridDim.x + blockIdx.x] = tot;
  }
}

}  // namespace shb
