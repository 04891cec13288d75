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

// warps per SM the FP32 step kernels are register-budgeted for
#ifndef SHB_STEP_WARPS
#define SHB_STEP_WARPS 24
#endif
#ifndef SHB_STEP_WARPS_F64
#define SHB_STEP_WARPS_F64 16
#endif

enum PencilMode : int {
  kPencilStep = 0,
  kPencilInit = 1,
  kPencilEnergy = 2,
  kPencilStepAdv = 3,  // step that also emits extra partials: i q_x psihat and opSH psihat (periodic, advection),
                       // -q_x^2 psihat (Neumann, substrate penalty)
  kPencilInitAdv = 4,
  kPencilStokes = 5,   // Stokes velocity from the stress (periodicFFT/pf3d.cpp:433-447)
  kPencilXMul = 6,     // partial P -> partial of its spectrum times an x-line multiplier (XMul)
  kPencilSpec = 7,     // partial P -> psihat, pencil-major
  kPencilAdjInit = 8,  // adjoint: partial of lambda^T -> lambdahat^T, mu partial
  kPencilAdj = 9,      // adjoint step: lambdahat^n = A lambdahat^{n+1} + ghat^n, mu partial, parameter gradients
  kPencilAdjOut = 10,  // adjoint: lambdahat -> its x-inverse partial (for lambda^0 in real space)
  kPencilStepU64 = 11, // the step of FP32 fields with the CNAB2 multipliers and update in FP64
};
// multiplier of kPencilXMul
enum XMulKind : int {
  kXIqx = 0,     // i q_x (periodic)
  kXNegQx2 = 1,  // -q_x^2
  kXOpSH = 2,    // alpha (|q|^2 - q0^2)^2
  kXSinDx = 3,   // Neumann: x derivative of the cosine series, as the reversed coefficients
                 // -q_{N-k} X[N-k] (0 at k = 0) whose REDFT01 is (-1)^x psi_x
};
// line sets of shared memory a pencil mode uses (FFT scratch, stash, Stokes components)
__host__ __device__ constexpr int pencil_sets(int mode) {
  return mode == kPencilStokes ? 3 : ((mode == kPencilStepAdv || mode == kPencilInitAdv) ? 2 : 1);
}

// TKV: lines per CTA (the tile), 0 = the default of 16 (FP32) or 8 (FP64)
template <typename T, int N, bool DCT, int TKV = 0>
struct PencilCfg {
  static constexpr int E = Plan<N>::E;
  static constexpr int G = N / E;
  static constexpr int TK = TKV > 0 ? TKV : (sizeof(T) == 4 ? 16 : 8);
  static constexpr int THREADS = TK * G;
  static constexpr int LS = line_stride(N);
  static constexpr int FP = DCT ? N * (N / 2) : N * (N / 2 + 1);
  static constexpr int TILES = FP / TK;
  static constexpr int RL = radix_of<N, -1, Plan<N>::P - 1>();
  static constexpr size_t SET_BYTES = size_t(TK) * LS * sizeof(cplx<T>);
  static constexpr size_t tw_off(int mode) { return SET_BYTES * pencil_sets(mode); }
  static constexpr size_t red_off(int mode) { return tw_off(mode) + size_t(tw_staged<N>(DCT)) * sizeof(cplx<T>); }
  // |k| shells of the spectral-power histogram (shell = rint |index vector|):
  // at most sqrt(3) N / 2 + 1 periodic, sqrt(3) (N - 1) + 1 Neumann
  static constexpr int NSHELL = DCT ? 2 * N : N;
  static constexpr size_t shell_off(int mode) { return red_off(mode) + 64 * sizeof(double); }
  static constexpr size_t smem(int mode) {
    return shell_off(mode) + (mode == kPencilEnergy ? size_t(NSHELL) * sizeof(double) : 0);
  }
  // per-CTA shared memory limit of sm_100 (the Stokes mode's three line sets
  // do not fit at 512^3 in FP64)
  static constexpr bool fits(int mode) { return smem(mode) <= size_t(227) * 1024; }
  // The step asks ptxas for a register budget that keeps SHB_STEP_WARPS warps
  // per SM resident in FP32 (three 256-thread CTAs at 256^3, twelve 64-thread
  // CTAs at 64^3) and SHB_STEP_WARPS_F64 in FP64 at N <= 128; every other
  // launch leaves the register budget to ptxas (0).
  // FP64 holds twice the registers per value: only its small CTAs (N <= 128) get a budget
  static constexpr int step_warps() { return sizeof(T) == 4 ? SHB_STEP_WARPS : (THREADS <= 64 ? SHB_STEP_WARPS_F64 : 0); }
  static constexpr int min_blocks(int mode) {
    return ((mode == kPencilStep || mode == kPencilStepU64) && THREADS <= 256 && step_warps() * 32 / THREADS >= 2)
               ? step_warps() * 32 / THREADS
                                                                                      : 0;
  }
  static_assert(FP % TK == 0, "tile must divide the plane");
  static_assert(THREADS % 32 == 0, "pencil CTA must be whole warps");
};

template <typename T>
struct PencilArgs {
  const cplx<T>* src;   // step: partial of N ; init: partial of psi   [rep][x][FP]
  const cplx<T>* src2;  // init: partial of N(psi)
  cplx<T>* w;           // state W [rep][FP][N]
  cplx<T>* dst;         // partial of scale * psihat^{n+1}, x-inverse applied [rep][x][FP]
  cplx<T>* dst_x;       // advection: partial of scale * i q_x psihat^{n+1}
  cplx<T>* dst_sh;      // advection: partial of scale * opSH psihat^{n+1}
  cplx<T>* spec_out;     // kFlSpecOut / kPencilSpec: psihat, pencil-major
  const cplx<T>* spec_a; // adjoint: psihat^n, pencil-major
  const cplx<T>* spec_b; // adjoint: psihat^{n+1}, pencil-major
  const cplx<T>* s3[3]; // Stokes: partial stress components (forward y,z applied)
  cplx<T>* u3[3];       // Stokes: partial velocity components (may alias s3)
  double* red;          // per-CTA spectral energy partial [rep][grid.x]
  double* shell;        // kFlShell: spectral power per |k| shell [rep][NSHELL] (accumulated, FP64)
  int* nonfinite;       // set to 1 when a new coefficient is NaN/Inf
  double coef;          // adjoint: c_{n-1} of the emitted mu combination (0 on the last reverse step)
  int xmul;             // kPencilXMul: XMulKind
  const T* q;           // wavenumber table (N entries)
  const double* qd;     // the same wavenumbers in FP64
  const cplx<T>* tw;    // twiddle table [forward | inverse | quarter-wave]
  PointParams pp;
  int flags;
};

template <typename T, int N, bool DCT, int TKV = 0>
struct PencilOps {
  using Cfg = PencilCfg<T, N, DCT, TKV>;
  static constexpr int E = Cfg::E, G = Cfg::G, TK = Cfg::TK, LS = Cfg::LS, FP = Cfg::FP, RL = Cfg::RL;

  // the TK lines of a tile are consecutive in memory (f0 and TK even: 16-byte pairs)
  static constexpr bool PAIRS = pair_io<T>() && TK % 2 == 0;
  static __device__ __forceinline__ int elem(int e) { return tile_elem<PAIRS>(threadIdx.x, Cfg::THREADS, e); }

  // TK * N == THREADS * E: all E loads of a thread are issued before its stores
  static __device__ __forceinline__ void load_tile(cplx<T>* buf, const cplx<T>* __restrict__ src, int f0) {
    cplx<T> tmp[E];
#pragma unroll
    for (int e = 0; e < E; e += PAIRS ? 2 : 1) {
      const int idx = elem(e);
      const cplx<T>* p = &src[size_t(idx / TK) * FP + f0 + idx % TK];
      if constexpr (PAIRS) ld_pair(p, tmp[e], tmp[e + 1]);
      else tmp[e] = *p;
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = elem(e);
      buf[(idx % TK) * LS + pad(idx / TK)] = tmp[e];
    }
  }
  static __device__ __forceinline__ void store_tile(const cplx<T>* buf, cplx<T>* __restrict__ dst, int f0) {
#pragma unroll
    for (int e = 0; e < E; e += PAIRS ? 2 : 1) {
      const int idx = elem(e);
      cplx<T>* p = &dst[size_t(idx / TK) * FP + f0 + idx % TK];
      if constexpr (PAIRS) st_pair(p, buf[(idx % TK) * LS + pad(idx / TK)], buf[(idx % TK + 1) * LS + pad(idx / TK)]);
      else *p = buf[(idx % TK) * LS + pad(idx / TK)];
    }
  }

  // forward x transform of the line; result in registers at kx = out_index<N,-1>
  static __device__ __forceinline__ void forward(cplx<T> (&v)[E], cplx<T>* L, int t, const TwTables<T>& tw) {
    if constexpr (!DCT) {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(i)]; });
    } else {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(i < N / 2 ? 2 * i : 2 * (N - 1 - i) + 1)]; });
      cplx<T> part[E];  // element (N - k) mod N of every slot
      mirror_partners<T, N, RL>(v, part, t);
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          cplx<T> w = tw.d[k];
          v[b * RL + r] = cadd<T>(cmul<T>(v[b * RL + r], w), cmul<T>(part[b * RL + r], conjg<T>(w)));
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
      // REDFT01 input exp(+i pi i/2N) (X[i] - i X[N-i]), X[N] = 0, formed in
      // registers: the first inverse pass reads element i in the slot where
      // the forward transform left element i
      cplx<T> part[E];
      mirror_partners<T, N, RL>(v, part, t);
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int i = out_index<N, -1>(t, b, r);
          const cplx<T> a = v[b * RL + r];
          cplx<T> u = a;
          if (i != 0) {
            const cplx<T> bb = part[b * RL + r];
            u = mk<T>(a.x + bb.y, a.y - bb.x);
          }
          cplx<T> w = tw.d[i];
          w.y = -w.y;
          v[b * RL + r] = cmul<T>(u, w);
        }
      fft_regs<T, N, +1>(v, L, t, tw.i);
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

template <typename T, int N, bool DCT, int MODE, int TKV = 0>
__global__ void __launch_bounds__(PencilCfg<T, N, DCT, TKV>::THREADS, PencilCfg<T, N, DCT, TKV>::min_blocks(MODE))
pencil_kernel(PencilArgs<T> a) {
  using Cfg = PencilCfg<T, N, DCT, TKV>;
  using Ops = PencilOps<T, N, DCT, TKV>;
  constexpr int E = Cfg::E, G = Cfg::G, TK = Cfg::TK, LS = Cfg::LS, FP = Cfg::FP, RL = Cfg::RL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  double* scratch = reinterpret_cast<double*>(smem_raw + Cfg::red_off(MODE));
  const TwTables<T> tw =
      stage_twiddles<T, N>(reinterpret_cast<cplx<T>*>(smem_raw + Cfg::tw_off(MODE)), a.tw, threadIdx.x, Cfg::THREADS, DCT);
  __syncthreads();  // every staged entry is written before any thread's first transform (kPencilAdjOut starts with one)
  grid_dependency_wait();

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

  if constexpr (MODE == kPencilStep || MODE == kPencilStepU64 || MODE == kPencilStepAdv) {
    // this CTA's rows of W (TK x N complex, contiguous) are read after the forward
    // transform: start bringing them into L2 now
    if (threadIdx.x == 0)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.w + (size_t(rep) * FP + f0) * N),
                   "r"(uint32_t(size_t(TK) * N * sizeof(cplx<T>)))
                   : "memory");
    Ops::load_tile(buf, a.src + plane_base, f0);
    __syncthreads();
    Ops::forward(v, L, t, tw);
    // the state W of this line, loaded after the transform: holding it through
    // the transform costs the registers of a third resident CTA
    cplx<T> wreg[E];
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) wreg[b * RL + r] = wrow[out_index<N, -1>(t, b, r)];
    // mode-independent constants of the update; the (ky, kz) part of |q|^2 is
    // fixed for the line
    const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha);
    const T h = T(0.5 * a.pp.dt), h3 = T(1.5 * a.pp.dt), dtT = T(a.pp.dt);
    const T qyz0 = qy * qy + qz0 * qz0 - q02;
    const T qyz1 = qy * qy + qz1 * qz1 - q02;
    const bool cnab2 = a.pp.scheme == kCNAB2;
    // FP64 values of the FP32 update (see below); the scalars stay kernel parameters
    const double epsd = a.pp.eps[rep];
    double qyz0d = 0.0, qyz1d = 0.0;
    if constexpr (MODE == kPencilStepU64 && sizeof(T) == 4) {
      const double qyd = __ldg(&a.qd[ky]), qz0d = __ldg(&a.qd[kz]);
      qyz0d = qyd * qyd + qz0d * qz0d - a.pp.q0 * a.pp.q0;
      if constexpr (DCT) {
        const double qz1d = __ldg(&a.qd[kz + 1]);
        qyz1d = qyd * qyd + qz1d * qz1d - a.pp.q0 * a.pp.q0;
      }
    }
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
        if constexpr (MODE == kPencilStepU64 && sizeof(T) == 4) {
          // FP32 fields with the per-mode multipliers and the update in FP64 from
          // the FP64 wavenumbers, one rounding of each stored result.  A multiplier
          // rounded to FP32 repeats the same relative error every step, which
          // drifts a mode's amplitude linearly with the step count.
          const double hd = 0.5 * a.pp.dt;
          const double qxd = __ldg(&a.qd[kx]);
          const double e0 = qxd * qxd + qyz0d;
          const double b0 = epsd - a.pp.alpha * e0 * e0;
          if (cnab2) {
            const double i0 = 1.0 / (1.0 - hd * b0), c0 = 1.0 + hd * b0;
            pn.x = T((double(wv.x) + 3.0 * hd * double(nh.x)) * i0);
            wv.x = T(c0 * double(pn.x) - hd * double(nh.x));
            double i1 = i0, c1 = c0;
            if constexpr (DCT) {
              const double e1 = qxd * qxd + qyz1d;
              const double b1 = epsd - a.pp.alpha * e1 * e1;
              i1 = 1.0 / (1.0 - hd * b1);
              c1 = 1.0 + hd * b1;
            }
            pn.y = T((double(wv.y) + 3.0 * hd * double(nh.y)) * i1);
            wv.y = T(c1 * double(pn.y) - hd * double(nh.y));
          } else {
            const double i0 = 1.0 / (1.0 - a.pp.dt * b0);
            pn.x = T((double(wv.x) + a.pp.dt * double(nh.x)) * i0);
            double i1 = i0;
            if constexpr (DCT) {
              const double e1 = qxd * qxd + qyz1d;
              i1 = 1.0 / (1.0 - a.pp.dt * (epsd - a.pp.alpha * e1 * e1));
            }
            pn.y = T((double(wv.y) + a.pp.dt * double(nh.y)) * i1);
            wv = pn;
          }
        } else if (cnab2) {
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
        if (a.flags & kFlSpecOut) a.spec_out[(size_t(rep) * FP + f) * N + kx] = pn;
        wrow[kx] = wv;
        v[b * RL + r] = cscale<T>(pn, scale);
      }
    if (bad) *a.nonfinite = 1;
  } else if constexpr (MODE == kPencilEnergy) {
    // gradient part of the energy of the current state from its partial P,
    // and (kFlShell) its spectral power per |k| shell
    double* hist = reinterpret_cast<double*>(smem_raw + Cfg::shell_off(MODE));
    const bool want_shell = (a.flags & kFlShell) != 0;
    if (want_shell)
      for (int i = threadIdx.x; i < Cfg::NSHELL; i += Cfg::THREADS) hist[i] = 0.0;
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
        if (want_shell) {
          // shell = rint |(ix, iy, iz)|: signed indices (Nyquist +N/2) on the periodic
          // grid, where every kz in (0, N/2) also stands for its conjugate
          if constexpr (!DCT) {
            const int ix = kx <= N / 2 ? kx : kx - N, iy = ky <= N / 2 ? ky : ky - N;
            const int sh = __double2int_rn(sqrt(double(ix * ix + iy * iy + kz * kz)));
            const double wgt = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
            atomicAdd(&hist[sh], wgt * (px * px + py * py));
          } else {
            const double wxy = (kx == 0 ? 0.5 : 1.0) * (ky == 0 ? 0.5 : 1.0);
            const int r2 = kx * kx + ky * ky;
            const int s0 = __double2int_rn(sqrt(double(r2 + kz * kz)));
            const int s1 = __double2int_rn(sqrt(double(r2 + (kz + 1) * (kz + 1))));
            atomicAdd(&hist[s0], wxy * (kz == 0 ? 0.5 : 1.0) * px * px);
            atomicAdd(&hist[s1], wxy * py * py);
          }
        }
      }
    if (want_shell) {
      __syncthreads();
      for (int i = threadIdx.x; i < Cfg::NSHELL; i += Cfg::THREADS)
        if (hist[i] != 0.0) atomicAdd(&a.shell[size_t(rep) * Cfg::NSHELL + i], hist[i]);
    }
  } else if constexpr (MODE == kPencilSpec || MODE == kPencilAdjInit || MODE == kPencilAdj) {
    Ops::load_tile(buf, a.src + plane_base, f0);
    cplx<T> lreg[E];
    if constexpr (MODE == kPencilAdj) {
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) lreg[b * RL + r] = wrow[out_index<N, -1>(t, b, r)];
    }
    __syncthreads();
    Ops::forward(v, L, t, tw);
    if constexpr (MODE == kPencilSpec) {
      // P = IDFT_x(scale psihat): its forward x transform is N scale psihat
      const T inv = T(1.0 / (a.pp.scale * N));
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r)
          a.spec_out[(size_t(rep) * FP + f) * N + out_index<N, -1>(t, b, r)] = cscale<T>(v[b * RL + r], inv);
    } else if constexpr (!DCT) {
      // Discrete adjoint of CNAB2 (reverse of psi^{n+1} = A psi^n + B (c_n N^n - N^{n-1}), c_0 = 2,
      // c_n = 3):
      //   lambdahat^n = A lambdahat^{n+1} + ghat^n,  mu^n = B lambda^n,
      //   g^{n-1} = N'(psi^{n-1}) (c_{n-1} mu^n - mu^{n+1}).
      // The output partial is that combination, scale B (coef lambdahat^n - lambdahat^{n+1}),
      // so the plane pass of step n-1 reads one field.  The parameter gradients
      //   dL/dtheta = sum_n <lambda^{n+1}, dt/2 (psihat^n + psihat^{n+1}) / C2 da/dtheta>
      // are regrouped by psihat^m: step n adds <lambda^{n+1} + [n >= 1] lambda^n, D psihat^n>, and
      // the first reverse step (spec_b set) also <lambda^{n+1}, D psihat^{n+1}>.
      const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha), h = T(0.5 * a.pp.dt);
      const T qyz = qy * qy + qz0 * qz0;
      const double wgt = ((kz == 0 || kz == N / 2) ? 1.0 : 2.0) / (double(N) * N * N);
      const double dadq0 = 4.0 * a.pp.alpha * a.pp.q0;
      const T coef = T(a.coef);
      const bool lam_n = a.coef != 0.0;  // n >= 1
      // a thread's 16 terms are summed plainly (FP64); the per-CTA and
      // per-step totals are combined in a fixed order
      double ge = 0.0, gq = 0.0;
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int kx = out_index<N, -1>(t, b, r);
          const T qx = __ldg(&a.q[kx]);
          const T mq2 = qx * qx + qyz;
          const T d = mq2 - q02;
          const T al = eps - alpha * d * d;
          const T inv2 = rcp_rn(T(1) - h * al);
          const T am = (T(1) + h * al) * inv2, bm = h * inv2;
          cplx<T> lam = v[b * RL + r];
          cplx<T> lnext = mk<T>(T(0), T(0));
          if constexpr (MODE == kPencilAdj) {
            const cplx<T> l1 = lreg[b * RL + r];
            lam = mk<T>(am * l1.x + lam.x, am * l1.y + lam.y);
            const size_t sidx = (size_t(rep) * FP + f) * N + kx;
            const cplx<T> pa = a.spec_a[sidx];
            const double wx = double(l1.x) + (lam_n ? double(lam.x) : 0.0);
            const double wy = double(l1.y) + (lam_n ? double(lam.y) : 0.0);
            double dot = wx * double(pa.x) + wy * double(pa.y);
            if (a.spec_b) {
              const cplx<T> pb = a.spec_b[sidx];
              dot += double(l1.x) * double(pb.x) + double(l1.y) * double(pb.y);
            }
            const double inner = wgt * double(bm) * dot;  // bm = dt/2 / C2
            ge += inner;
            gq += inner * double(d);
            lnext = l1;
          }
          wrow[kx] = lam;
          v[b * RL + r] = cscale<T>(mk<T>(coef * lam.x - lnext.x, coef * lam.y - lnext.y), scale * bm);
        }
      if constexpr (MODE == kPencilAdj) {
        // each CTA accumulates into its own slot over the reverse sweep (fixed order)
        const double te = block_sum(ge, scratch);
        const double tq = block_sum(gq, scratch);
        if (threadIdx.x == 0) {
          double* o = a.red + (size_t(rep) * gridDim.x + blockIdx.x) * 2;
          o[0] += te;
          o[1] += tq * dadq0;
        }
      }
    }
  } else if constexpr (MODE == kPencilAdjOut) {
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) v[b * RL + r] = cscale<T>(wrow[out_index<N, -1>(t, b, r)], scale);
  } else if constexpr (MODE == kPencilXMul) {
    Ops::load_tile(buf, a.src + plane_base, f0);
    __syncthreads();
    Ops::forward(v, L, t, tw);
    // P is the x-inverse of (scale X); its forward x transform is N scale X
    // (2N scale X for REDFT10 after REDFT01): multiply by m(q) / N (/ 2N)
    const T invn = T(1) / T(DCT ? 2 * N : N);
    const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha);
    if constexpr (DCT) {
      if (a.xmul == kXSinDx) {
        // RODFT01(X)[x] = (-1)^x REDFT01(X reversed)[x] (the sine series of
        // d/dx): slot kx takes -q_{N-kx} times coefficient N - kx, the mirror
        // partner of kx; the plane pass applies (-1)^x
        cplx<T> part[E];
        mirror_partners<T, N, RL>(v, part, t);
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int kx = out_index<N, -1>(t, b, r);
            const T w = kx == 0 ? T(0) : -__ldg(&a.q[N - kx]) * invn;
            v[b * RL + r] = cscale<T>(part[b * RL + r], w);
          }
      }
    }
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const T qx = __ldg(&a.q[out_index<N, -1>(t, b, r)]);
        const cplx<T> val = v[b * RL + r];
        if (a.xmul == kXSinDx) {
          // done above
        } else if (a.xmul == kXIqx) {
          v[b * RL + r] = mk<T>(-qx * invn * val.y, qx * invn * val.x);
        } else if (a.xmul == kXNegQx2) {
          v[b * RL + r] = cscale<T>(val, -qx * qx * invn);
        } else {
          const T d0 = qx * qx + qy * qy + qz0 * qz0 - q02;
          const T d1 = DCT ? qx * qx + qy * qy + qz1 * qz1 - q02 : d0;
          v[b * RL + r] = mk<T>(alpha * d0 * d0 * invn * val.x, alpha * d1 * d1 * invn * val.y);
        }
      }
  } else if constexpr (MODE == kPencilStokes) {
    if constexpr (DCT) {
      // Neumann box: the stress came in as the cosine-transform partial of
      // (-1)^(x+y+z) S, whose REDFT10 at index k is the RODFT10 of S at index
      // N-1-k (cosFFT/comet/morphSurfK.cpp:390-418 uses RODFT10/01).  So the
      // sine-wavenumber projector u = CM1 (S - CM2 (Vs . S)) of morphSurfK.cpp:
      // 862-882, Vs(m) = pi (m+1)/L, reads Vs = pi (N-k)/L at index k; the
      // inverse REDFT01 then yields (-1)^(x+y+z) u, unsigned by the plane pass.
      cplx<T>* set[3] = {buf, buf + TK * LS, buf + 2 * TK * LS};
#pragma unroll
      for (int c = 0; c < 3; ++c) Ops::load_tile(set[c], a.s3[c] + plane_base, f0);
      __syncthreads();
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        cplx<T>* Lc = set[c] + line * LS;
        Ops::forward(v, Lc, t, tw);
        __syncwarp();
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) Lc[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      }
      __syncwarp();
      const T q1 = __ldg(&a.q[1]);  // pi / L
      const T sy = T(N - ky) * q1, sz0 = T(N - kz) * q1, sz1 = T(N - kz - 1) * q1;
      const T ce = T(1.0 / a.pp.eta_rho);
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int kx = out_index<N, -1>(t, b, r);
          const T sx = T(N - kx) * q1;
          const int o = line * LS + pad(kx);
          const cplx<T> px = set[0][o], py = set[1][o], pz = set[2][o];
          // .x holds kz, .y holds kz + 1
          const T m0 = sx * sx + sy * sy + sz0 * sz0, m1 = sx * sx + sy * sy + sz1 * sz1;
          const T i0 = T(1) / m0, i1 = T(1) / m1;
          const T c0 = scale * ce * i0, c1 = scale * ce * i1;
          const T d0 = sx * px.x + sy * py.x + sz0 * pz.x;
          const T d1 = sx * px.y + sy * py.y + sz1 * pz.y;
          set[0][o] = mk<T>(c0 * (px.x - sx * i0 * d0), c1 * (px.y - sx * i1 * d1));
          set[1][o] = mk<T>(c0 * (py.x - sy * i0 * d0), c1 * (py.y - sy * i1 * d1));
          set[2][o] = mk<T>(c0 * (pz.x - sz0 * i0 * d0), c1 * (pz.y - sz1 * i1 * d1));
        }
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        cplx<T>* Lc = set[c] + line * LS;
        __syncwarp();
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) v[b * RL + r] = Lc[pad(out_index<N, -1>(t, b, r))];
        Ops::inverse_to_line(v, Lc, t, tw);
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < 3; ++c) Ops::store_tile(set[c], a.u3[c] + plane_base, f0);
    } else {
      // S -> u = scale CM1 (S - CM2 (q.S)),  CM1 = 1/(rho eta |q|^2), CM2 = q/|q|^2, both 0 at q = 0
      cplx<T>* set[3] = {buf, buf + TK * LS, buf + 2 * TK * LS};
#pragma unroll
      for (int c = 0; c < 3; ++c) Ops::load_tile(set[c], a.s3[c] + plane_base, f0);
      __syncthreads();
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx<T>* Lc = set[c] + line * LS;
        Ops::forward(v, Lc, t, tw);
        __syncwarp();
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) Lc[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      }
      __syncwarp();
      const T ce = T(1.0 / a.pp.eta_rho);
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int kx = out_index<N, -1>(t, b, r);
          const T qx = __ldg(&a.q[kx]);
          const T mq2 = qx * qx + qy * qy + qz0 * qz0;
          const int o = line * LS + pad(kx);
          const cplx<T> sx = set[0][o], sy = set[1][o], sz = set[2][o];
          cplx<T> ux = mk<T>(T(0), T(0)), uy = ux, uz = ux;
          if (mq2 != T(0)) {
            const T inv = T(1) / mq2;
            const T cm1 = scale * ce * inv;
            const cplx<T> dot = mk<T>(qx * sx.x + qy * sy.x + qz0 * sz.x, qx * sx.y + qy * sy.y + qz0 * sz.y);
            ux = mk<T>(cm1 * (sx.x - qx * inv * dot.x), cm1 * (sx.y - qx * inv * dot.y));
            uy = mk<T>(cm1 * (sy.x - qy * inv * dot.x), cm1 * (sy.y - qy * inv * dot.y));
            uz = mk<T>(cm1 * (sz.x - qz0 * inv * dot.x), cm1 * (sz.y - qz0 * inv * dot.y));
          }
          set[0][o] = ux;
          set[1][o] = uy;
          set[2][o] = uz;
        }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx<T>* Lc = set[c] + line * LS;
        __syncwarp();
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) v[b * RL + r] = Lc[pad(out_index<N, -1>(t, b, r))];
        Ops::inverse_to_line(v, Lc, t, tw);
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < 3; ++c) Ops::store_tile(set[c], a.u3[c] + plane_base, f0);
    }
  } else {  // kPencilInit(Adv): W^0 from psi^0 and N(psi^0); P^0 from psi^0
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

  if constexpr (MODE == kPencilStep || MODE == kPencilStepU64 || MODE == kPencilInit || MODE == kPencilXMul ||
                MODE == kPencilAdjInit ||
                MODE == kPencilAdj || MODE == kPencilAdjOut) {
    Ops::inverse_to_line(v, L, t, tw);
    __syncthreads();
    Ops::store_tile(buf, a.dst + plane_base, f0);
  } else if constexpr (MODE == kPencilStepAdv || MODE == kPencilInitAdv) {
    if constexpr (DCT) {
      // v = scale psihat^{n+1}; emit the partials of v and, where asked, of
      // -q_x^2 v (the x half of the substrate's in-plane Laplacian) and of
      // opSH v (L psi of the Stokes stress, cosFFT/comet/morphSurfK.cpp:686-696),
      // one inverse x transform each
      cplx<T>* stash = buf + TK * LS + line * LS;
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) stash[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncwarp();
      const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha);
      cplx<T>* outs[3] = {a.dst, a.dst_x, a.dst_sh};
#pragma unroll 1
      for (int o = 0; o < 3; ++o) {
        if (!outs[o]) continue;  // uniform over the CTA
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int kx = out_index<N, -1>(t, b, r);
            const cplx<T> val = stash[pad(kx)];
            const T qx = __ldg(&a.q[kx]);
            if (o == 0) {
              v[b * RL + r] = val;
            } else if (o == 1) {
              v[b * RL + r] = cscale<T>(val, -qx * qx);
            } else {  // the pair holds kz and kz + 1
              const T d0 = qx * qx + qy * qy + qz0 * qz0 - q02;
              const T d1 = qx * qx + qy * qy + qz1 * qz1 - q02;
              v[b * RL + r] = mk<T>(alpha * d0 * d0 * val.x, alpha * d1 * d1 * val.y);
            }
          }
        Ops::inverse_to_line(v, L, t, tw);
        __syncthreads();
        Ops::store_tile(buf, outs[o] + plane_base, f0);
        __syncthreads();
      }
    } else {
      // v = scale psihat^{n+1}; emit the partials of v, i q_x v and opSH v
      // (periodicFFT/pf3d.cpp:404-407), one inverse x transform each
      cplx<T>* stash = buf + TK * LS + line * LS;
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) stash[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncwarp();
      const T q02 = T(a.pp.q0 * a.pp.q0), alpha = T(a.pp.alpha);
      cplx<T>* outs[3] = {a.dst, a.dst_x, a.dst_sh};
#pragma unroll 1
      for (int o = 0; o < 3; ++o) {
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int kx = out_index<N, -1>(t, b, r);
            const cplx<T> val = stash[pad(kx)];
            const T qx = __ldg(&a.q[kx]);
            if (o == 0) {
              v[b * RL + r] = val;
            } else if (o == 1) {
              v[b * RL + r] = mk<T>(-qx * val.y, qx * val.x);
            } else {
              const T d = qx * qx + qy * qy + qz0 * qz0 - q02;
              v[b * RL + r] = cscale<T>(val, alpha * d * d);
            }
          }
        Ops::inverse_to_line(v, L, t, tw);
        __syncthreads();
        Ops::store_tile(buf, outs[o] + plane_base, f0);
        __syncthreads();
      }
    }
  }

  if (want_energy && (MODE == kPencilStep || MODE == kPencilStepU64 || MODE == kPencilStepAdv ||
                      MODE == kPencilEnergy)) {
    const double tot = block_sum(acc.s, scratch);
    if (threadIdx.x == 0) a.red[size_t(rep) * gridDim.x + blockIdx.x] = tot;
  }
}

}  // namespace shb
