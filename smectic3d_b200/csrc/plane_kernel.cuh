// Plane pass: the y and z transforms of one x-plane, fused with the real-space
// pointwise work that sits between an inverse and a forward transform.
//
// One thread-block cluster of CL CTAs owns one x-plane (all replicas in
// blockIdx.y).  The plane is a spectral "partial" (the x transform has already
// been applied by the pencil pass) stored as
//   periodic : [ky][kz]  kz in [0, N/2)  followed by the kz = N/2 column [ky]
//   Neumann  : [y][z] real values, viewed as complex pairs (z even, z odd)
// Each CTA owns NC = N/(2 CL) complex column lines in the column phase and NC
// row-pair lines (2 rows each) in the row phase; the transposes between the
// phases go through distributed shared memory of the cluster.
//
//   column phase   inverse y transform of the owned columns       (registers)
//   -> DSMEM ->    row phase: inverse z transform of two rows packed as one
//                  complex line, real-space pointwise work, forward z transform
//   -> DSMEM ->    column phase: forward y transform, store
//
// Periodic z transforms treat two real rows as the real and imaginary parts of
// one complex N-point transform; the kz = 0 and kz = N/2 columns (real after
// the z transform) travel packed as F0 + i FN through the y transform.  The
// Neumann transforms are REDFT01 / REDFT10 computed as one complex N-point FFT
// with the even/odd permutation and quarter-wave twiddles (Makhoul), applied to
// two real sequences at once (the transform is linear).
#pragma once
#include "sh_common.cuh"

namespace shb {

enum PlaneMode : int { kPlaneStep = 0, kPlaneInit = 1, kPlaneGetPsi = 2 };

template <typename T, int N, int CL, bool DCT>
struct PlaneCfg {
  static constexpr int E = Plan<N>::E;
  static constexpr int G = N / E;
  static constexpr int NC = N / (2 * CL);
  static constexpr int THREADS = NC * G;
  static constexpr int LS = line_stride(N);
  static constexpr int LINES = NC + 1;
  static constexpr int ROWS = N / CL;
  static constexpr int FP = DCT ? N * (N / 2) : N * (N / 2 + 1);
  static constexpr int RL_INV = radix_of<N, +1, Plan<N>::P - 1>();
  static constexpr int RL_FWD = radix_of<N, -1, Plan<N>::P - 1>();
  static constexpr size_t TW_OFF = size_t(LINES) * LS * sizeof(cplx<T>);
  static constexpr size_t RED_OFF = TW_OFF + size_t(tw_total<N>()) * sizeof(cplx<T>);
  static constexpr size_t SMEM = RED_OFF + 64 * sizeof(double);
  static_assert(THREADS % 32 == 0, "plane CTA must be whole warps");
};

template <typename T>
struct PlaneArgs {
  const cplx<T>* src;     // partial spectra in  [rep][x][FP]
  cplx<T>* dst;           // partial spectra out [rep][x][FP]
  cplx<T>* dst2;          // init: partial spectrum of psi
  const double* psi_in;   // init: real psi, dense [rep][x][y][z]
  double* psi_out;        // optional real psi out (dense)
  const double* psi_old;  // optional L1 reference (dense)
  double* red;            // per-CTA partial sums [rep][grid.x][3]
  const cplx<T>* tw;      // twiddle table [forward | inverse | quarter-wave]
  PointParams pp;
  int flags;
};

// Cluster barrier.  RELEASE orders this thread's earlier shared-memory writes
// (local and remote) before the peers' reads; without it the barrier only
// orders execution, which is what a write-after-read hand-over needs.
template <int CL, bool RELEASE>
__device__ __forceinline__ void cluster_sync() {
  if constexpr (CL == 1) {
    __syncthreads();
  } else {
    if constexpr (RELEASE) {
      asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    } else {
      asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
    }
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
}

// Store into element ``off`` of the CTA-``rank`` copy of shared array ``buf``
// (st.shared::cluster on the address mapa gives for that rank).
__device__ __forceinline__ uint32_t dsmem_map(const void* p, int rank) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_dsmem_raw(uint32_t a, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void st_dsmem_raw(uint32_t a, double2 v) {
  asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void st_dsmem_raw(uint32_t a, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void st_dsmem_raw(uint32_t a, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
template <int CL, typename V>
__device__ __forceinline__ void st_dsmem(V* buf, int rank, int off, V val) {
  if constexpr (CL == 1) {
    buf[off] = val;
  } else {
    st_dsmem_raw(dsmem_map(buf + off, rank), val);
  }
}

// z (or y) position of FFT index n in the Makhoul even/odd permutation
template <int N>
__device__ __forceinline__ int mk_perm(int n) { return n < N / 2 ? 2 * n : 2 * (N - 1 - n) + 1; }

// first-pass input of REDFT01 (complex-linear): exp(+i pi i/2N) (X[i] - i X[N-i]), X[N] = 0
template <typename T, int N>
__device__ __forceinline__ cplx<T> dct3_pre(const cplx<T>* L, int i, const cplx<T>* dtw) {
  cplx<T> a = L[pad(i)];
  cplx<T> u = a;
  if (i != 0) {
    cplx<T> b = L[pad(N - i)];
    u = mk<T>(a.x + b.y, a.y - b.x);
  }
  cplx<T> w = dtw[i];
  w.y = -w.y;
  return cmul<T>(u, w);
}

// first-pass input of the two-row C2R: Z = X_a + i X_b with Hermitian extension;
// slot 0 of each half holds (X[0], X[N/2]) packed.
template <typename T, int N>
__device__ __forceinline__ cplx<T> c2r_pre(const cplx<T>* L, int i) {
  if (i == 0) {
    cplx<T> a = L[pad(0)], b = L[pad(N / 2)];
    return mk<T>(a.x, b.x);
  }
  if (i == N / 2) {
    cplx<T> a = L[pad(0)], b = L[pad(N / 2)];
    return mk<T>(a.y, b.y);
  }
  if (i < N / 2) {
    cplx<T> a = L[pad(i)], b = L[pad(N / 2 + i)];
    return mk<T>(a.x - b.y, a.y + b.x);
  }
  const int k = N - i;
  cplx<T> a = L[pad(k)], b = L[pad(N / 2 + k)];
  return mk<T>(a.x + b.y, b.x - a.y);
}

template <typename T, int N, int CL, bool DCT>
struct PlaneOps {
  using Cfg = PlaneCfg<T, N, CL, DCT>;
  static constexpr int E = Cfg::E, G = Cfg::G, NC = Cfg::NC, LS = Cfg::LS, ROWS = Cfg::ROWS;
  static constexpr int THREADS = Cfg::THREADS;

  // ---- column phase, inverse direction ---------------------------------
  static __device__ void col_load(cplx<T>* buf, const cplx<T>* __restrict__ plane, int rank) {
    const int c0 = rank * NC;
    // NC * N == THREADS * E: every thread issues its E loads before any store
    cplx<T> tmp[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + THREADS * e;
      tmp[e] = plane[(idx / NC) * (N / 2) + c0 + idx % NC];
    }
    constexpr int KPT = (N + THREADS - 1) / THREADS;  // ky per thread for the kz=0 / N/2 columns
    cplx<T> nyq[KPT];
    if constexpr (!DCT) {
      if (rank == 0) {
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) nyq[m] = plane[N * (N / 2) + ky];
        }
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + THREADS * e;
      buf[(idx % NC) * LS + pad(idx / NC)] = tmp[e];
    }
    if constexpr (!DCT) {
      if (rank == 0) {
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) buf[NC * LS + pad(ky)] = nyq[m];
        }
      }
    }
    __syncthreads();
    if constexpr (!DCT) {
      if (rank == 0) {
        // Hermitian projection in ky of the kz=0 and kz=N/2 columns (the real
        // part FFTW's c2r keeps on those planes), packed as F0 + i FN.
        cplx<T> out[KPT];
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) {
            const int km = (N - ky) & (N - 1);
            cplx<T> a0 = buf[pad(ky)], a1 = buf[pad(km)];
            cplx<T> b0 = buf[NC * LS + pad(ky)], b1 = buf[NC * LS + pad(km)];
            const T f0x = T(0.5) * (a0.x + a1.x), f0y = T(0.5) * (a0.y - a1.y);
            const T fnx = T(0.5) * (b0.x + b1.x), fny = T(0.5) * (b0.y - b1.y);
            out[m] = mk<T>(f0x - fny, f0y + fnx);
          }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) buf[pad(ky)] = out[m];
        }
        __syncthreads();
      }
    }
  }

  // inverse y transform of the owned columns, then scatter into row layout
  static __device__ void col_inverse_to_rows(cplx<T>* buf, int rank, const TwTables<T>& tw) {
    const int line = threadIdx.x / G, t = threadIdx.x % G;
    cplx<T>* L = buf + line * LS;
    cplx<T> v[E];
    if constexpr (!DCT) {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return L[pad(i)]; });
    } else {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return dct3_pre<T, N>(L, i, tw.d); });
    }
    cluster_sync<CL, false>();
    const int kc = rank * NC + line;  // global complex column
    constexpr int RL = Cfg::RL_INV;
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int n = out_index<N, +1>(t, b, r);
        const cplx<T> val = v[b * RL + r];
        if constexpr (!DCT) {
          const int dest = n / ROWS, yl = n % ROWS;
          st_dsmem<CL>(buf, dest, (yl >> 1) * LS + pad((yl & 1) * (N / 2) + kc), val);
        } else {
          const int y = mk_perm<N>(n);
          const int dest = y / ROWS, yl = y % ROWS;
          T* rb = reinterpret_cast<T*>(buf);
          const int base = (yl >> 1) * LS;
          st_dsmem<CL>(rb, dest, 2 * (base + pad(2 * kc)) + (yl & 1), val.x);
          st_dsmem<CL>(rb, dest, 2 * (base + pad(2 * kc + 1)) + (yl & 1), val.y);
        }
      }
    cluster_sync<CL, true>();
  }

  // ---- row phase -------------------------------------------------------
  // inverse z transform of row pair ``line``; v slot holds psi(y0, z), psi(y0+1, z)
  static __device__ __forceinline__ void row_inverse(cplx<T> (&v)[E], cplx<T>* L, int t,
                                                     const TwTables<T>& tw) {
    if constexpr (!DCT) {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return c2r_pre<T, N>(L, i); });
    } else {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return dct3_pre<T, N>(L, i, tw.d); });
    }
  }

  // z coordinate of register slot (b, r) after row_inverse (== the input slot of
  // the forward z transform)
  static __device__ __forceinline__ int row_z(int t, int b, int r) {
    const int n = out_index<N, +1>(t, b, r);
    if constexpr (DCT) return mk_perm<N>(n);
    return n;
  }

  // forward z transform from registers, then scatter to column layout
  static __device__ void row_forward_to_cols(cplx<T> (&v)[E], cplx<T>* buf, cplx<T>* L, int rank, int line, int t,
                                             const TwTables<T>& tw) {
    fft_regs<T, N, -1>(v, L, t, tw.f);
    constexpr int RL = Cfg::RL_FWD;
    __syncwarp();
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) L[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
    __syncwarp();
    const int y0 = rank * ROWS + 2 * line;  // global y of the real part
    if constexpr (!DCT) {
      // split Z into the two half spectra; slot k < N/2 from register r < RL/2
      cplx<T> oa[E / 2], ob[E / 2];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL / 2; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          const int s = b * (RL / 2) + r;
          if (k == 0) {
            cplx<T> z0 = L[pad(0)], zn = L[pad(N / 2)];
            oa[s] = mk<T>(z0.x, zn.x);
            ob[s] = mk<T>(z0.y, zn.y);
          } else {
            cplx<T> zk = L[pad(k)], zm = L[pad(N - k)];
            oa[s] = mk<T>(T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y));
            ob[s] = mk<T>(T(0.5) * (zk.y + zm.y), T(0.5) * (zm.x - zk.x));
          }
        }
      cluster_sync<CL, false>();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL / 2; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          const int s = b * (RL / 2) + r;
          const int col = (k % NC) * LS;
          st_dsmem<CL>(buf, k / NC, col + pad(y0), oa[s]);
          st_dsmem<CL>(buf, k / NC, col + pad(y0 + 1), ob[s]);
        }
    } else {
      cplx<T> o[E];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          cplx<T> w = tw.d[k];
          cplx<T> a = cmul<T>(L[pad(k)], w);
          cplx<T> bm = cmul<T>(L[pad((N - k) & (N - 1))], conjg<T>(w));
          o[b * RL + r] = cadd<T>(a, bm);
        }
      cluster_sync<CL, false>();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          const int p = k >> 1;
          T* rb = reinterpret_cast<T*>(buf);
          const int col = 2 * (p % NC) * LS;
          st_dsmem<CL>(rb, p / NC, col + 2 * pad(y0) + (k & 1), o[b * RL + r].x);
          st_dsmem<CL>(rb, p / NC, col + 2 * pad(y0 + 1) + (k & 1), o[b * RL + r].y);
        }
    }
    cluster_sync<CL, true>();
  }

  // ---- column phase, forward direction ---------------------------------
  static __device__ void col_forward_store(cplx<T>* buf, cplx<T>* __restrict__ plane, int rank,
                                           const TwTables<T>& tw) {
    const int line = threadIdx.x / G, t = threadIdx.x % G;
    cplx<T>* L = buf + line * LS;
    cplx<T> v[E];
    constexpr int RL = Cfg::RL_FWD;
    if constexpr (!DCT) {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(i)]; });
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) L[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncthreads();
      if (rank == 0) {
        // unpack F0 + i FN of the kz=0 / kz=N/2 columns
        constexpr int KPT = (N + THREADS - 1) / THREADS;
        cplx<T> f0[KPT], fn[KPT];
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) {
            cplx<T> z = buf[pad(ky)], zm = buf[pad((N - ky) & (N - 1))];
            f0[m] = mk<T>(T(0.5) * (z.x + zm.x), T(0.5) * (z.y - zm.y));
            fn[m] = mk<T>(T(0.5) * (z.y + zm.y), T(0.5) * (zm.x - z.x));
          }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) {
            buf[pad(ky)] = f0[m];
            buf[NC * LS + pad(ky)] = fn[m];
          }
        }
        __syncthreads();
      }
    } else {
      fft_line<T, N, -1>(v, L, t, tw.f, [&](int i) { return L[pad(mk_perm<N>(i))]; });
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
      __syncwarp();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) L[pad(out_index<N, -1>(t, b, r))] = v[b * RL + r];
      __syncthreads();
    }
    const int c0 = rank * NC;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = threadIdx.x + THREADS * e;
      plane[(idx / NC) * (N / 2) + c0 + idx % NC] = buf[(idx % NC) * LS + pad(idx / NC)];
    }
    if constexpr (!DCT) {
      if (rank == 0) {
        for (int ky = threadIdx.x; ky < N; ky += THREADS) plane[N * (N / 2) + ky] = buf[NC * LS + pad(ky)];
      }
    }
  }
};

// Real-space pointwise stage of one row pair: nonlinearity (+ pinning penalty
// on the plane z = N/2, periodicFFT/pf3dMorph.cpp:456-467).  ``v`` holds psi
// on entry and N(psi) on exit.
template <typename T, int N, int CL, bool DCT>
__device__ __forceinline__ void row_nonlin(cplx<T> (&v)[Plan<N>::E], cplx<T>* L, int t, const PointParams& pp) {
  using Ops = PlaneOps<T, N, CL, DCT>;
  constexpr int E = Plan<N>::E;
  constexpr int RL = PlaneCfg<T, N, CL, DCT>::RL_INV;
  const T beta = T(pp.beta), gamma = T(pp.gamma);
  if (pp.w_mid != 0.0) {
    __syncwarp();
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) L[pad(Ops::row_z(t, b, r))] = v[b * RL + r];
    __syncwarp();
  }
#pragma unroll
  for (int b = 0; b < E / RL; ++b)
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int z = Ops::row_z(t, b, r);
      cplx<T> p = v[b * RL + r];
      cplx<T> o = mk<T>(nonlin_eval<T>(p.x, beta, gamma, pp.nonlin), nonlin_eval<T>(p.y, beta, gamma, pp.nonlin));
      if (pp.w_mid != 0.0 && z == N / 2) {
        cplx<T> lo = L[pad(z - 1)], hi = L[pad(z + 1)];
        const T c = T(2.0 * pp.w_mid * pp.inv_dz2);
        o.x += c * (lo.x - T(2) * p.x + hi.x);
        o.y += c * (lo.y - T(2) * p.y + hi.y);
      }
      v[b * RL + r] = o;
    }
}

template <typename T, int N, int CL, bool DCT, int MODE>
__global__ void __launch_bounds__(PlaneCfg<T, N, CL, DCT>::THREADS)
plane_kernel(PlaneArgs<T> a) {
  using Cfg = PlaneCfg<T, N, CL, DCT>;
  using Ops = PlaneOps<T, N, CL, DCT>;
  constexpr int E = Cfg::E, G = Cfg::G, LS = Cfg::LS, ROWS = Cfg::ROWS, FP = Cfg::FP;
  constexpr int RL = Cfg::RL_INV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  double* scratch = reinterpret_cast<double*>(smem_raw + Cfg::RED_OFF);
  const TwTables<T> tw =
      stage_twiddles<T, N>(reinterpret_cast<cplx<T>*>(smem_raw + Cfg::TW_OFF), a.tw, threadIdx.x, Cfg::THREADS);

  int rank = 0;
  if constexpr (CL > 1) rank = int(cg::this_cluster().block_rank());
  const int x = blockIdx.x / CL;
  const int rep = blockIdx.y;
  const int line = threadIdx.x / G, t = threadIdx.x % G;
  cplx<T>* L = buf + line * LS;
  const size_t plane_off = (size_t(rep) * N + x) * FP;
  const size_t real_off = (size_t(rep) * N + x) * size_t(N) * N;
  const int y0 = rank * ROWS + 2 * line;
  cplx<T> v[E];

  if constexpr (MODE == kPlaneStep || MODE == kPlaneGetPsi) {
    Ops::col_load(buf, a.src + plane_off, rank);
    Ops::col_inverse_to_rows(buf, rank, tw);
    Ops::row_inverse(v, L, t, tw);

    if (a.flags & (kFlPsiOut | kFlL1 | kFlEnergy)) {
      KahanSum s0, s1, s2;
      const double eps = a.pp.eps[rep];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int z = Ops::row_z(t, b, r);
          const double pa = double(v[b * RL + r].x), pb = double(v[b * RL + r].y);
          const size_t ia = real_off + size_t(y0) * N + z, ib = ia + N;
          if (a.flags & kFlL1) {  // read before a possibly aliased write
            s0.add(fabs(pa - a.psi_old[ia]) + fabs(pb - a.psi_old[ib]));
            s1.add(fabs(pa) + fabs(pb));
          }
          if (a.flags & kFlPsiOut) {
            a.psi_out[ia] = pa;
            a.psi_out[ib] = pb;
          }
          if (a.flags & kFlEnergy) {
            s2.add(local_density(pa, eps, a.pp.beta, a.pp.gamma, a.pp.nonlin) +
                   local_density(pb, eps, a.pp.beta, a.pp.gamma, a.pp.nonlin));
          }
        }
      if (a.flags & (kFlL1 | kFlEnergy)) {
        const double t0 = block_sum(s0.s, scratch);
        const double t1 = block_sum(s1.s, scratch);
        const double t2 = block_sum(s2.s, scratch);
        if (threadIdx.x == 0) {
          double* o = a.red + (size_t(rep) * gridDim.x + blockIdx.x) * 3;
          o[0] = t0;
          o[1] = t1;
          o[2] = t2;
        }
      }
    }
    if constexpr (MODE == kPlaneStep) {
      row_nonlin<T, N, CL, DCT>(v, L, t, a.pp);
      Ops::row_forward_to_cols(v, buf, L, rank, line, t, tw);
      Ops::col_forward_store(buf, a.dst + plane_off, rank, tw);
    }
  } else {  // kPlaneInit: real psi -> partial spectra of psi (dst2) and N(psi) (dst)
    const double* src = a.psi_in + real_off;
    for (int field = 0; field < 2; ++field) {
      __syncthreads();
      constexpr int R0 = radix_of<N, -1, 0>();
      const T beta = T(a.pp.beta), gamma = T(a.pp.gamma);
#pragma unroll
      for (int b = 0; b < E / R0; ++b)
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const int n = in_index<N, -1>(t, b, r);
          const int z = DCT ? mk_perm<N>(n) : n;
          T pa = T(src[size_t(y0) * N + z]), pb = T(src[size_t(y0 + 1) * N + z]);
          if (field == 1) {
            T na = nonlin_eval<T>(pa, beta, gamma, a.pp.nonlin);
            T nb = nonlin_eval<T>(pb, beta, gamma, a.pp.nonlin);
            if (a.pp.w_mid != 0.0 && z == N / 2) {
              const T c = T(2.0 * a.pp.w_mid * a.pp.inv_dz2);
              na += c * (T(src[size_t(y0) * N + z - 1]) - T(2) * pa + T(src[size_t(y0) * N + z + 1]));
              nb += c * (T(src[size_t(y0 + 1) * N + z - 1]) - T(2) * pb + T(src[size_t(y0 + 1) * N + z + 1]));
            }
            pa = na;
            pb = nb;
          }
          v[b * R0 + r] = mk<T>(pa, pb);
        }
      Ops::row_forward_to_cols(v, buf, L, rank, line, t, tw);
      Ops::col_forward_store(buf, (field == 0 ? a.dst2 : a.dst) + plane_off, rank, tw);
    }
  }
}

}  // namespace shb
