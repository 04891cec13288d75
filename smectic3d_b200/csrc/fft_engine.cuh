// In-register / shared-memory FFT building blocks for sm_100a.
//
// A "line" is one 1-D transform of N complex points held in a padded shared
// memory row.  A group of G = N/E consecutive threads (G divides 32, so a group
// never straddles a warp) owns a line; every thread holds E = N/G complex values
// in registers.  The transform is the Stockham autosort formulation (natural
// order in, natural order out) with radix-R butterflies computed in registers:
//
//   pass s (radix R, Ns = product of earlier radices), butterfly j:
//     v[r]   = line[j + r N/R]
//     v[r]  *= w_N^{ (j mod Ns) r N/(Ns R) }
//     v      = DFT_R(v)
//     line[(j/Ns) Ns R + (j mod Ns) + r Ns] = v[r]
//
// The first pass reads through a caller-supplied loader (fusing pre-processing
// such as Hermitian extension, DCT permutation or a pointwise nonlinearity) and
// the last pass leaves its values in registers, so the caller fuses the
// post-processing.  The inverse plan is the forward plan reversed, which makes
// the last forward pass and the first inverse pass use the same register
// layout: a forward transform, a pointwise spectral operation and an inverse
// transform chain without touching shared memory in between.
//
// Shared memory rows are padded with one slot every 16 (pad()), which makes the
// stride-R stores of the first pass and the stride-1 loads of later passes
// bank-conflict free for 8- and 16-byte elements.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace shb {

template <typename T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <typename T> using cplx = typename cvec<T>::type;

template <typename T>
__device__ __forceinline__ cplx<T> mk(T x, T y) { cplx<T> r; r.x = x; r.y = y; return r; }
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && !defined(SHB_NO_F32X2)
// sm_100 packed FP32x2 arithmetic: one instruction for both lanes of a complex
// float, each lane rounded to nearest exactly as the scalar FADD / FSUB
__device__ __forceinline__ unsigned long long pk2(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
template <>
__device__ __forceinline__ float2 cadd<float>(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
template <>
__device__ __forceinline__ float2 csub<float>(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
#endif
template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk<T>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <typename T>
__device__ __forceinline__ cplx<T> cscale(cplx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
template <typename T>
__device__ __forceinline__ cplx<T> conjg(cplx<T> a) { return mk<T>(a.x, -a.y); }

// ---------------------------------------------------------------------------
// Global tile traffic.  The passes move tiles between HBM and shared memory with
// every thread owning E elements.  In FP32 a thread owns consecutive element
// pairs, so that each pair of complex floats moves as one 16-byte access (the
// tiles start on even elements of 16-byte aligned buffers); FP64 complex values
// are 16 bytes already.
// ---------------------------------------------------------------------------
#ifndef SHB_PAIR_IO
#define SHB_PAIR_IO 1
#endif
template <typename T>
__host__ __device__ constexpr bool pair_io() { return SHB_PAIR_IO && sizeof(T) == 4; }
// element index of register slot e (0 <= e < E) of thread tid of nthr
template <bool PAIRS>
__device__ __forceinline__ int tile_elem(int tid, int nthr, int e) {
  if constexpr (PAIRS) return 2 * (tid + nthr * (e >> 1)) + (e & 1);
  else return tid + nthr * e;
}
__device__ __forceinline__ void ld_pair(const float2* p, float2& a, float2& b) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void st_pair(float2* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void ld_pair(const double2*, double2&, double2&) {}
__device__ __forceinline__ void st_pair(double2*, double2, double2) {}

// padded index inside a shared-memory line
__host__ __device__ constexpr int pad(int i) { return i + (i >> 4); }
// line stride in elements (odd spacing between lines of a tile)
__host__ __device__ constexpr int line_stride(int n) { return n + n / 16 + 1; }

// ---------------------------------------------------------------------------
// Radix plans.  E = values per thread; passes are listed forward order.
// ---------------------------------------------------------------------------
template <int N> struct Plan;
template <> struct Plan<16>  { static constexpr int E = 4;  static constexpr int P = 2; static constexpr int R[3] = {4, 4, 1}; };
template <> struct Plan<32>  { static constexpr int E = 8;  static constexpr int P = 2; static constexpr int R[3] = {8, 4, 1}; };
template <> struct Plan<64>  { static constexpr int E = 16; static constexpr int P = 2; static constexpr int R[3] = {16, 4, 1}; };
template <> struct Plan<128> { static constexpr int E = 16; static constexpr int P = 2; static constexpr int R[3] = {16, 8, 1}; };
template <> struct Plan<256> { static constexpr int E = 16; static constexpr int P = 2; static constexpr int R[3] = {16, 16, 1}; };
template <> struct Plan<512> { static constexpr int E = 16; static constexpr int P = 3; static constexpr int R[3] = {16, 16, 2}; };

// radix of pass s in direction DIR (-1 forward, +1 inverse = reversed plan)
template <int N, int DIR, int S>
__host__ __device__ constexpr int radix_of() {
  return DIR < 0 ? Plan<N>::R[S] : Plan<N>::R[Plan<N>::P - 1 - S];
}
template <int N, int DIR, int S>
__host__ __device__ constexpr int ns_of() {
  int ns = 1;
  for (int s = 0; s < S; ++s)
    ns *= (DIR < 0 ? Plan<N>::R[s] : Plan<N>::R[Plan<N>::P - 1 - s]);
  return ns;
}
// Twiddles live in a pass-major table per direction: pass s >= 1 owns
// (R_s - 1) * NS_s entries, entry (r - 1) * NS_s + jm = w_N^{+-jm r N/(NS_s R_s)}
// (the inverse table holds the conjugates), so the G threads of a group read
// consecutive entries.
template <int N, int DIR, int S>
__host__ __device__ constexpr int tw_offset() {
  int off = 0;
  for (int s = 1; s < S; ++s) {
    int ns = 1;
    for (int u = 0; u < s; ++u) ns *= (DIR < 0 ? Plan<N>::R[u] : Plan<N>::R[Plan<N>::P - 1 - u]);
    const int r = DIR < 0 ? Plan<N>::R[s] : Plan<N>::R[Plan<N>::P - 1 - s];
    off += (r - 1) * ns;
  }
  return off;
}
template <int N, int DIR>
__host__ __device__ constexpr int tw_size() { return tw_offset<N, DIR, Plan<N>::P>(); }

// A plan whose radix sequence reads the same both ways (16 = 4 x 4, 256 = 16 x 16)
// has the same pass structure forward and inverse, so its inverse twiddles are
// the conjugates of the forward ones: only the forward table is staged.
template <int N>
__host__ __device__ constexpr bool tw_shared() {
  for (int s = 0; s < Plan<N>::P; ++s)
    if (Plan<N>::R[s] != Plan<N>::R[Plan<N>::P - 1 - s]) return false;
  return true;
}
// entries staged in shared memory: forward table, inverse table unless shared,
// and the quarter-wave table for the cosine transforms
template <int N>
__host__ __device__ constexpr int tw_staged(bool dct) {
  return tw_size<N, -1>() + (tw_shared<N>() ? 0 : tw_size<N, +1>()) + (dct ? N : 0);
}

// Twiddle tables of one transform length, staged in shared memory per CTA:
// forward pass table, inverse pass table, quarter-wave exp(-i pi k / 2N).
template <typename T>
struct TwTables {
  const cplx<T>* f;
  const cplx<T>* i;
  const cplx<T>* d;
};
// total entries of the device table [forward | inverse | quarter-wave]
template <int N>
__host__ __device__ constexpr int tw_total() { return tw_size<N, -1>() + tw_size<N, +1>() + N; }

// Build the device table on the host (long double trigonometry).
template <typename T, int N, class Vec>
void host_twiddles(Vec& out) {
  const long double pi = 3.141592653589793238462643383279502884L;
  out.resize(tw_total<N>());
  int o = 0;
  for (int dir = -1; dir <= 1; dir += 2) {
    for (int s = 1; s < Plan<N>::P; ++s) {
      int ns = 1;
      for (int u = 0; u < s; ++u) ns *= (dir < 0 ? Plan<N>::R[u] : Plan<N>::R[Plan<N>::P - 1 - u]);
      const int r_s = dir < 0 ? Plan<N>::R[s] : Plan<N>::R[Plan<N>::P - 1 - s];
      for (int r = 1; r < r_s; ++r)
        for (int jm = 0; jm < ns; ++jm) {
          const long double a = dir * 2.0L * pi * (long double)(jm * r) / (long double)(ns * r_s);
          out[o].x = T(cosl(a));
          out[o].y = T(sinl(a));
          ++o;
        }
    }
  }
  for (int k = 0; k < N; ++k) {
    const long double b = -pi * k / (2.0L * N);
    out[o].x = T(cosl(b));
    out[o].y = T(sinl(b));
    ++o;
  }
}

// copy the tables a kernel uses (tw_staged entries) from the device table
// [forward | inverse | quarter-wave] into shared memory (caller syncs); the
// periodic transforms need no quarter-wave part
template <typename T, int N>
__device__ __forceinline__ TwTables<T> stage_twiddles(cplx<T>* smem, const cplx<T>* __restrict__ g, int tid, int nthr,
                                                      bool dct) {
  constexpr int nf = tw_size<N, -1>(), ni = tw_size<N, +1>();
  constexpr int nis = tw_shared<N>() ? 0 : ni;
  for (int i = tid; i < nf + nis; i += nthr) smem[i] = __ldg(&g[i]);
  if (dct)
    for (int i = tid; i < N; i += nthr) smem[nf + nis + i] = __ldg(&g[nf + ni + i]);
  TwTables<T> t;
  t.f = smem;
  t.i = smem + (tw_shared<N>() ? 0 : nf);
  t.d = smem + nf + nis;
  return t;
}

// the tables read in place from the device table [forward | inverse | quarter-wave]
template <typename T, int N>
__device__ __forceinline__ TwTables<T> device_twiddles(const cplx<T>* g) {
  constexpr int nf = tw_size<N, -1>(), ni = tw_size<N, +1>();
  TwTables<T> t;
  t.f = g;
  t.i = tw_shared<N>() ? g : g + nf;
  t.d = g + nf + ni;
  return t;
}

// element index held in register slot (b*R + r) after the last pass of
// direction DIR (equivalently: loaded in that slot by the first pass of -DIR)
template <int N, int DIR>
__device__ __forceinline__ int out_index(int t, int b, int r) {
  constexpr int G = N / Plan<N>::E;
  constexpr int RL = radix_of<N, DIR, Plan<N>::P - 1>();
  return t + G * b + r * (N / RL);
}
// element index loaded in register slot (b*R + r) by the first pass of DIR
template <int N, int DIR>
__device__ __forceinline__ int in_index(int t, int b, int r) {
  constexpr int G = N / Plan<N>::E;
  constexpr int R0 = radix_of<N, DIR, 0>();
  return t + G * b + r * (N / R0);
}

// ---------------------------------------------------------------------------
// Small DFTs in registers (decimation in time, compile-time twiddles).
// ---------------------------------------------------------------------------
// cos / sin of 2 pi a / 16
__device__ constexpr double kCos16[8] = {1.0, 0.92387953251128675613, 0.70710678118654752440,
                                          0.38268343236508977173, 0.0, -0.38268343236508977173,
                                          -0.70710678118654752440, -0.92387953251128675613};
__device__ constexpr double kSin16[8] = {0.0, 0.38268343236508977173, 0.70710678118654752440,
                                          0.92387953251128675613, 1.0, 0.92387953251128675613,
                                          0.70710678118654752440, 0.38268343236508977173};

// multiply by w_R^k = exp(DIR * 2 pi i k / R), 0 <= k < R/2
template <typename T, int R, int K, int DIR>
__device__ __forceinline__ cplx<T> twc(cplx<T> v) {
  constexpr int A = K * (16 / R);  // angle in units of 2 pi / 16, < 8
  if constexpr (A == 0) {
    return v;
  } else if constexpr (A == 4) {
    // w = DIR * i
    return DIR < 0 ? mk<T>(v.y, -v.x) : mk<T>(-v.y, v.x);
  } else if constexpr (A == 2 || A == 6) {
    const T h = T(0.70710678118654752440);
    // A==2: w = h (1 + DIR i) ; A==6: w = h (-1 + DIR i)
    if constexpr (A == 2) {
      return DIR < 0 ? mk<T>(h * (v.x + v.y), h * (v.y - v.x)) : mk<T>(h * (v.x - v.y), h * (v.x + v.y));
    } else {
      return DIR < 0 ? mk<T>(h * (v.y - v.x), -h * (v.x + v.y)) : mk<T>(-h * (v.x + v.y), h * (v.x - v.y));
    }
  } else {
    const T c = T(kCos16[A]);
    const T s = DIR < 0 ? T(-kSin16[A]) : T(kSin16[A]);
    return mk<T>(fma(v.x, c, -v.y * s), fma(v.x, s, v.y * c));
  }
}

template <typename T, int R, int DIR> struct DFT;
template <typename T, int DIR> struct DFT<T, 1, DIR> {
  static __device__ __forceinline__ void run(cplx<T>*) {}
};
template <typename T, int DIR> struct DFT<T, 2, DIR> {
  static __device__ __forceinline__ void run(cplx<T>* a) {
    cplx<T> t = a[1];
    a[1] = csub<T>(a[0], t);
    a[0] = cadd<T>(a[0], t);
  }
};
template <typename T, int DIR> struct DFT<T, 4, DIR> {
  static __device__ __forceinline__ void run(cplx<T>* a) {
    cplx<T> s02 = cadd<T>(a[0], a[2]), d02 = csub<T>(a[0], a[2]);
    cplx<T> s13 = cadd<T>(a[1], a[3]), d13 = csub<T>(a[1], a[3]);
    // d13 * (DIR i)
    cplx<T> r13 = DIR < 0 ? mk<T>(d13.y, -d13.x) : mk<T>(-d13.y, d13.x);
    a[0] = cadd<T>(s02, s13);
    a[2] = csub<T>(s02, s13);
    a[1] = cadd<T>(d02, r13);
    a[3] = csub<T>(d02, r13);
  }
};

template <typename T, int R, int DIR, int K>
__device__ __forceinline__ void dft_combine(cplx<T>* a, cplx<T>* e, cplx<T>* o) {
  if constexpr (K < R / 2) {
    cplx<T> t = twc<T, R, K, DIR>(o[K]);
    a[K] = cadd<T>(e[K], t);
    a[K + R / 2] = csub<T>(e[K], t);
    dft_combine<T, R, DIR, K + 1>(a, e, o);
  }
}

template <typename T, int R, int DIR> struct DFT {
  static __device__ __forceinline__ void run(cplx<T>* a) {
    cplx<T> e[R / 2], o[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; ++k) { e[k] = a[2 * k]; o[k] = a[2 * k + 1]; }
    DFT<T, R / 2, DIR>::run(e);
    DFT<T, R / 2, DIR>::run(o);
    dft_combine<T, R, DIR, 0>(a, e, o);
  }
};

// ---------------------------------------------------------------------------
// Stockham passes over a shared-memory line
// ---------------------------------------------------------------------------
template <typename T, int N, int DIR, int S>
__device__ __forceinline__ void pass_compute(cplx<T> (&v)[Plan<N>::E], int t, const cplx<T>* __restrict__ tw) {
  constexpr int E = Plan<N>::E, G = N / E;
  constexpr int R = radix_of<N, DIR, S>();
  constexpr int NS = ns_of<N, DIR, S>();
  constexpr int NB = E / R;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if constexpr (NS > 1) {
      const int jm = (t + G * b) & (NS - 1);
      constexpr int OFF = tw_offset<N, DIR, S>();
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const cplx<T> w = tw[OFF + (r - 1) * NS + jm];
        // a shared table holds the forward twiddles: the inverse uses their conjugates
        v[b * R + r] = cmul<T>(v[b * R + r], (DIR > 0 && tw_shared<N>()) ? conjg<T>(w) : w);
      }
    }
    DFT<T, R, DIR>::run(&v[b * R]);
  }
}

template <typename T, int N, int DIR, int S>
__device__ __forceinline__ void pass_store(cplx<T>* line, const cplx<T> (&v)[Plan<N>::E], int t) {
  constexpr int E = Plan<N>::E, G = N / E;
  constexpr int R = radix_of<N, DIR, S>();
  constexpr int NS = ns_of<N, DIR, S>();
  constexpr int NB = E / R;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + G * b;
    const int base = (j / NS) * NS * R + (j & (NS - 1));
#pragma unroll
    for (int r = 0; r < R; ++r) line[pad(base + r * NS)] = v[b * R + r];
  }
}

template <typename T, int N, int DIR, int S>
__device__ __forceinline__ void pass_load(const cplx<T>* line, cplx<T> (&v)[Plan<N>::E], int t) {
  constexpr int E = Plan<N>::E, G = N / E;
  constexpr int R = radix_of<N, DIR, S>();
  constexpr int NB = E / R;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + G * b;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = line[pad(j + r * (N / R))];
  }
}

template <typename T, int N, int DIR, int S>
__device__ __forceinline__ void passes_from(cplx<T>* line, cplx<T> (&v)[Plan<N>::E], int t,
                                            const cplx<T>* __restrict__ tw) {
  pass_compute<T, N, DIR, S>(v, t, tw);
  if constexpr (S + 1 < Plan<N>::P) {
    __syncwarp();                      // every thread of the group has read the line
    pass_store<T, N, DIR, S>(line, v, t);
    __syncwarp();
    pass_load<T, N, DIR, S + 1>(line, v, t);
    passes_from<T, N, DIR, S + 1>(line, v, t, tw);
  }
}

// Mirror partners in registers.  After a forward transform (and before an
// inverse one) slot b*RL + r of thread t holds element k = t + G b + M r,
// M = N / RL.  part[slot] receives element (N - k) mod N, which thread
// (G - t) mod G holds in a compile-time slot: one warp shuffle per component
// instead of a round trip through shared memory.  Every lane of the warp
// must call it.
template <typename T>
__device__ __forceinline__ cplx<T> shfl_c(cplx<T> v, int src, int width) {
  return mk<T>(__shfl_sync(0xffffffffu, v.x, src, width), __shfl_sync(0xffffffffu, v.y, src, width));
}
template <typename T, int N, int RL>
__device__ __forceinline__ void mirror_partners(const cplx<T> (&v)[Plan<N>::E], cplx<T> (&part)[Plan<N>::E], int t) {
  constexpr int E = Plan<N>::E, G = N / E, NB = E / RL;
  const int src = (G - t) & (G - 1);
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      // t != 0: thread G - t, slot (NB - 1 - b, RL - 1 - r)
      const cplx<T> q = shfl_c<T>(v[(NB - 1 - b) * RL + (RL - 1 - r)], src, G);
      // t == 0: this thread, slot (NB - b, RL - 1 - r), or (0, (RL - r) mod RL) when b = 0
      const int zs = b == 0 ? (RL - r) % RL : (NB - b) * RL + (RL - 1 - r);
      part[b * RL + r] = t == 0 ? v[zs] : q;
    }
}

// Full transform.  The first pass reads element i through ld(i); the result of
// the last pass stays in v (element out_index<N,DIR>(t,b,r) in slot b*R+r).
// ``tw`` is the pass-major twiddle table of direction DIR (shared memory).
// ``line`` is scratch for the intermediate passes (it may be the line that ld
// reads: every read of the first pass happens before the first store).
// First-pass input of a transform of direction DIR: element i through ld(i)
// into its register slot (nothing else is touched, so a caller may order its
// own synchronisation between the loads and the passes).
template <typename T, int N, int DIR, class Loader>
__device__ __forceinline__ void load_first(cplx<T> (&v)[Plan<N>::E], int t, Loader ld) {
  constexpr int E = Plan<N>::E, G = N / E;
  constexpr int R = radix_of<N, DIR, 0>();
#pragma unroll
  for (int b = 0; b < E / R; ++b)
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = ld(t + G * b + r * (N / R));
}

template <typename T, int N, int DIR, class Loader>
__device__ __forceinline__ void fft_line(cplx<T> (&v)[Plan<N>::E], cplx<T>* line, int t,
                                         const cplx<T>* __restrict__ tw, Loader ld) {
  load_first<T, N, DIR>(v, t, ld);
  passes_from<T, N, DIR, 0>(line, v, t, tw);
}

// Transform whose input already sits in registers in the first-pass layout
// (e.g. the output of a transform of the opposite direction).
template <typename T, int N, int DIR>
__device__ __forceinline__ void fft_regs(cplx<T> (&v)[Plan<N>::E], cplx<T>* line, int t,
                                         const cplx<T>* __restrict__ tw) {
  passes_from<T, N, DIR, 0>(line, v, t, tw);
}

}  // namespace shb
