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

enum PlaneMode : int {
  kPlaneStep = 0,
  kPlaneInit = 1,
  kPlaneGetPsi = 2,
  kPlaneInvReal = 3,
  kPlaneAdj = 5,
  kPlaneInvMulFwd = 6,  // inverse of (mult x src) -> real_out; times real_in[0]; forward -> dst
  kPlaneAdvN = 7,       // N(real_in[0]) - sum_c (inverse of src3[c]) real_in[1+c]; forward -> dst
  kPlaneMulFwd = 8,     // real_in[0] real_in[1] (times the signs of sign_axes) forward -> dst
};
// spectral multiplier applied to the partial spectrum as the plane is loaded
// kMulSinDy (Neumann): the sine series of d/dy as reversed coefficients,
// element ky <- -q_{N-ky} X[N-ky] (0 at ky = 0); its REDFT01 is (-1)^y psi_y
enum SpecMult : int { kMulNone = 0, kMulIqy = 1, kMulIqz = 2, kMulNegQy2 = 3, kMulNegQz2 = 4, kMulSinDy = 5 };


template <typename T, int N, int CL, bool DCT>
struct PlaneCfg {
  static constexpr int E = Plan<N>::E;
  static constexpr int G = N / E;
  static constexpr int NC = N / (2 * CL);
  static constexpr int THREADS = NC * G;
  static constexpr int LS = line_stride(N);
  static constexpr int LINES = DCT ? NC : NC + 1;  // periodic: + the kz = N/2 column
  static constexpr int ROWS = N / CL;
  static constexpr int FP = DCT ? N * (N / 2) : N * (N / 2 + 1);
  static constexpr int RL_INV = radix_of<N, +1, Plan<N>::P - 1>();
  static constexpr int RL_FWD = radix_of<N, -1, Plan<N>::P - 1>();
  // Exchange blocks between the CTAs of a cluster (CL > 1), one per
  // (source, destination) pair, padded rows so that both the writer and the
  // reader access shared memory without bank conflicts:
  //   column -> row, periodic : [row yl][column c]        stride NC + 1
  //   column -> row, Neumann  : [row pair q][kz local]    stride 2 NC + 1
  //   row -> column (both)    : [row yl][column c]        stride NC + 1
  static constexpr int SA = DCT ? 2 * NC + 1 : NC + 1;
  static constexpr int SBs = NC + 1;
  static constexpr int BLK_A = DCT ? (ROWS / 2) * (2 * NC + 1) : ROWS * (NC + 1);
  static constexpr int BLK_B = ROWS * (NC + 1);
  static constexpr int BLK = ((BLK_A > BLK_B ? BLK_A : BLK_B) + 1) / 2 * 2;  // even: 16-byte blocks
  static constexpr size_t LB_BYTES = align_up(size_t(LINES) * LS * sizeof(cplx<T>), 128);
  static constexpr size_t XB_RAW = CL > 1 ? align_up(size_t(CL) * BLK * sizeof(cplx<T>), 128) : 0;
  // the periodic transforms need no quarter-wave table
  static constexpr int TW_ENTRIES = tw_staged<N>(DCT);
  // block_sum scratch: one double per warp (at most 16 warps)
  static constexpr int RED_DOUBLES = 16;
  static constexpr size_t TAIL = size_t(TW_ENTRIES) * sizeof(cplx<T>) + 16 + 16 + RED_DOUBLES * sizeof(double);
  // Two exchange variants between the CTAs of a cluster:
  //  - bulk: padded send / receive blocks moved by cp.async.bulk (the default);
  //  - direct: every thread stores its values with st.shared::cluster straight
  //    into the line buffer of the CTA that owns them, between two cluster
  //    barriers.  No send or receive blocks, so it fits where the bulk blocks
  //    do not (FP64 at 512^3: a CTA owns 16 lines of 512 complex doubles).
  static constexpr bool DIRECT = CL > 1 && 2 * (LB_BYTES > XB_RAW ? LB_BYTES : XB_RAW) + TAIL > size_t(227) * 1024;
  // cluster size seen by the bulk-exchange machinery (none in the direct variant)
  static constexpr int XCL = DIRECT ? 1 : CL;
  static constexpr size_t XB_BYTES = DIRECT ? 0 : XB_RAW;
  // With bulk exchanges shared memory holds two regions of max(line buffer,
  // exchange blocks) each: the column-phase line buffer, which the send blocks
  // overlay once the column transforms are done, and the receive blocks, which
  // the scratch lines of the row phase and of the forward column phase overlay
  // once their first pass has read them.  So the send blocks are rewritten only
  // after a whole row phase, and a CTA never waits right after an exchange for
  // its peers to have received its blocks.
  static constexpr bool ALIAS = CL > 1 && !DIRECT;
  static constexpr size_t REGION = LB_BYTES > XB_BYTES ? LB_BYTES : XB_BYTES;
  static constexpr size_t SB_OFF = ALIAS ? 0 : LB_BYTES;
  static constexpr size_t RB_OFF = ALIAS ? REGION : SB_OFF + XB_BYTES;
  static constexpr size_t TW_OFF = RB_OFF + (ALIAS ? REGION : XB_BYTES);
  // CTAs per SM that shared memory admits for a CTA of ``bytes`` (228 KB per
  // SM, 1 KB reserved per CTA)
  static constexpr int ctas_by_smem(size_t bytes) { return int(233472 / (bytes + 1024)); }
  static constexpr size_t smem_with(size_t tw_bytes) {
    return align_up(TW_OFF + tw_bytes, 16) + 16 + RED_DOUBLES * sizeof(double);
  }
  // The twiddle tables are staged in shared memory unless reading them in place
  // from the device table (through L1) lifts a shared-memory-bound CTA count of
  // two or fewer per SM.  That is done for the FP64 cosine transforms only: their
  // 7.9 KB of tables at 256^3 (clusters of 16) are what keeps a third CTA out,
  // and three 128-thread CTAs of that kernel also fit the register file (ptxas:
  // 168 registers); the FP64 periodic plane kernel is register-bound at two
  // (192 registers) and only loses by reading its tables through L1.
  static constexpr bool TW_SMEM =
      !(sizeof(T) == 8 && DCT && ctas_by_smem(smem_with(size_t(TW_ENTRIES) * sizeof(cplx<T>))) <= 2 &&
        ctas_by_smem(smem_with(0)) > ctas_by_smem(smem_with(size_t(TW_ENTRIES) * sizeof(cplx<T>))));
  static constexpr size_t TW_BYTES = TW_SMEM ? size_t(TW_ENTRIES) * sizeof(cplx<T>) : 0;
  static constexpr size_t MB_OFF = align_up(TW_OFF + TW_BYTES, 16);
  static constexpr size_t RED_OFF = MB_OFF + 16;
  static constexpr size_t SMEM = RED_OFF + RED_DOUBLES * sizeof(double);
  static constexpr bool fits = SMEM <= 227 * 1024;  // per-CTA shared memory limit of sm_100
  // FP32: ptxas is asked for a register budget that keeps SHB_STEP_WARPS warps
  // per SM resident, where that many CTAs also fit the 228 KB of shared memory
  // (1 KB reserved per CTA): three 256-thread CTAs in clusters at 256^3, six
  // 128-thread CTAs at 64^3.
#ifndef SHB_PLANE_THREE
#define SHB_PLANE_THREE 1
#endif
#ifndef SHB_STEP_WARPS
#define SHB_STEP_WARPS 24
#endif
  static constexpr int MIN_BLOCKS_RAW = THREADS <= 256 ? SHB_STEP_WARPS * 32 / THREADS : 0;
  static constexpr int MIN_BLOCKS =
      (SHB_PLANE_THREE && sizeof(T) == 4 && MIN_BLOCKS_RAW >= 2 &&
       (SMEM + 1024) * MIN_BLOCKS_RAW <= 233472)
          ? MIN_BLOCKS_RAW
          : 0;
  // kPlaneAdvN keeps an accumulator beside the transform registers: capped for
  // the periodic box (three CTAs per SM, small spills: 256^3 FP32 advected
  // step -19 us), uncapped for the Neumann box, where the cap measured slower
  static constexpr int min_blocks(int mode) { return (mode == kPlaneAdvN && DCT) ? 0 : MIN_BLOCKS; }
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
  int* timeout;           // set when a bounded wait on a cluster exchange gave up
  const cplx<T>* tw;      // twiddle table [forward | inverse | quarter-wave]
  PointParams pp;
  int flags;
  // real-field modes: wavenumber table, multiplier, real inputs / output
  const T* q;
  int mult;
  const T* real_in[4];  // adjoint: [1] psi; stress: [0] L psi; advected N: [0] psi, [1..3] grad psi
  T* real_out;
  // kPlaneInvReal: optional second partial, added after its own multiplier
  const cplx<T>* src2;
  int mult2;
  int real_zn;  // > 0: real_out holds only z < real_zn, layout [rep][x][y][real_zn]
  // Neumann substrate penalty: N += wall[z] * lperp for z < kwall, with lperp
  // the in-plane Laplacian of psi in layout [rep][x][y][kwall]
  const T* wall;
  const T* lperp;
  int kwall;
  // kPlaneAdvN: the three velocity partials
  const cplx<T>* src3[3];
  // Sine transforms on the Neumann box run through the cosine pair with
  // real-space factors (-1)^x, (-1)^y, (-1)^z: on the products kPlaneMulFwd
  // transforms, on the fields kPlaneInvReal and kPlaneAdvN invert.  Bit 0, 1, 2
  // of sign_axes selects x, y, z (the Stokes solve of cosFFT/comet/morphSurfK.cpp
  // uses all three; a spectral derivative the axes it differentiates).
  int sign_axes;
  // kPlaneInvReal, Neumann: the z transform inverts the sine series of d/dz
  // (reversed coefficients -q_{N-k} X[N-k], 0 at k = 0)
  int sin_dz;
  int drop_exchange;  // test hook (see Xchg::drop)
  // > 0: rank 0 of the cluster of plane x starts bringing plane x + pf_dist of
  // the column input into L2 (the plane a cluster of a later wave loads first)
  int pf_dist;
};

// One launch of the plane pass.  The modes that turn independent fields to or
// from real space (kPlaneInvReal, kPlaneInvMulFwd, kPlaneMulFwd) take up to
// kPlaneComps argument sets and run one per blockIdx.z, so that the components
// of a gradient, stress or velocity share one grid (one wave tail instead of
// one per component); every other mode uses set 0.
constexpr int kPlaneComps = 3;
template <typename T>
struct PlaneLaunch {
  PlaneArgs<T> c[kPlaneComps];
};
__host__ __device__ constexpr bool plane_multi(int mode) {
  return mode == kPlaneInvReal || mode == kPlaneInvMulFwd || mode == kPlaneMulFwd;
}

// Cluster barrier halves.  barrier.cluster arrive and wait alternate in every
// thread; Xchg below tracks whether an arrive is outstanding.
template <int CL>
__device__ __forceinline__ void cluster_arrive() {
  if constexpr (CL > 1) asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
template <int CL>
__device__ __forceinline__ void cluster_wait() {
  if constexpr (CL > 1) asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// shared::cluster address of ``p`` in the copy of this CTA's shared memory
// that belongs to cluster rank ``rank``
__device__ __forceinline__ uint32_t dsmem_map(const void* p, int rank) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

// Store into the copy of this CTA's shared memory that belongs to cluster rank
// ``rank`` (the direct exchange variant); a plain store without a cluster.
template <int CL>
__device__ __forceinline__ void st_rank(float* p, float v, int rank) {
  if constexpr (CL == 1) { *p = v; } else {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(dsmem_map(p, rank)), "f"(v) : "memory");
  }
}
template <int CL>
__device__ __forceinline__ void st_rank(double* p, double v, int rank) {
  if constexpr (CL == 1) { *p = v; } else {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(dsmem_map(p, rank)), "d"(v) : "memory");
  }
}
template <int CL>
__device__ __forceinline__ void st_rank(float2* p, float2 v, int rank) {
  if constexpr (CL == 1) { *p = v; } else {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(dsmem_map(p, rank)), "f"(v.x), "f"(v.y) : "memory");
  }
}
template <int CL>
__device__ __forceinline__ void st_rank(double2* p, double2 v, int rank) {
  if constexpr (CL == 1) { *p = v; } else {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(dsmem_map(p, rank)), "d"(v.x), "d"(v.y) : "memory");
  }
}
// Barrier around an in-place transpose of the line buffers: the CTA alone, or
// (direct exchange) the whole cluster, whose release / acquire also orders the
// remote stores before the reads that follow.
template <int CL>
__device__ __forceinline__ void transpose_sync() {
  if constexpr (CL == 1) {
    __syncthreads();
  } else {
    cluster_arrive<CL>();
    cluster_wait<CL>();
  }
}

// Cluster exchange state: send / receive block arrays, two mbarriers (one per
// exchange direction) and their phase parities.
//
// Protocol.  The exchange copies (cp.async.bulk shared::cta -> shared::cluster)
// complete only on the receiver's mbarrier, so a sender learns that its copies
// have finished reading its send blocks only from the receivers.  Every CTA
// arrives at the cluster barrier as soon as its own incoming blocks have landed
// (end of bulk_exchange).  It waits for that phase (settle) only where it
// rewrites its send blocks or the column line buffer they overlay, and before it
// exits; both come after a whole row or column phase, by which time its peers
// have long received.  When a CTA is done with its receive blocks, as data and
// as scratch, and another exchange into them follows, it settles and arrives
// again (xchg_rb_done); the next exchange settles that phase before it copies
// into the peers.  The first exchange settles the arrive that publishes the
// initialised mbarriers.  Arrive and wait strictly alternate in every thread.
template <typename T>
struct Xchg {
  cplx<T>* sb;
  cplx<T>* rb;
  uint64_t* mbar;
  uint32_t phases;
  int* timeout;
  int drop;    // test hook: rank 0 sends nothing in exchange 0, so its peers' bounded waits run out
  bool armed;  // an arrive is outstanding (the next cluster_wait completes it)
};

// The arrives of the bulk protocol carry no memory ordering (.relaxed): what a
// peer waits for is either the completion of copies this CTA has already
// observed on its mbarrier (the copy engine has finished reading the peer's send
// blocks), or the end of this CTA's reads of its receive blocks, whose values
// are already consumed; the data itself is ordered by the mbarrier (complete_tx,
// then try_wait with acquire) and by the async-proxy fence before each copy.  A
// release arrive would add a memory barrier to every phase.  The first arrive
// follows the fence.mbarrier_init.release.cluster of the mbarrier set-up.
template <typename T, int CL>
__device__ __forceinline__ void xchg_arrive(Xchg<T>& x) {
  if constexpr (CL > 1) {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
    x.armed = true;
  }
}
// wait for the outstanding arrive phase, if any
template <typename T, int CL>
__device__ __forceinline__ void xchg_settle(Xchg<T>& x) {
  if constexpr (CL > 1) {
    if (x.armed) {
      cluster_wait<CL>();
      x.armed = false;
    }
  }
}

// This CTA is done with its receive blocks (another exchange into them
// follows): wait for the outstanding phase, then arrive
template <typename T, int CL>
__device__ __forceinline__ void xchg_rb_done(Xchg<T>& x) {
  if constexpr (CL > 1) {
    xchg_settle<T, CL>(x);
    xchg_arrive<T, CL>(x);
  }
}

// Every thread has written its share of the send blocks; copy block d to CTA d
// (cp.async.bulk shared::cta -> shared::cluster, completing on the receiver's
// mbarrier ``which``), wait until all CL incoming blocks have landed, and
// arrive (the senders may reuse their send blocks once every CTA has).  The
// settle before the copies waits for the peers' "receive blocks free" arrive.
template <typename T, int CL>
__device__ __forceinline__ void bulk_exchange(Xchg<T>& x, int which, int rank, int blk) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();         // every thread's send-block writes precede the copies
  xchg_settle<T, CL>(x);   // every peer has arrived: its receive blocks are free, its mbarriers initialised
  // thread d copies block d (a copy may complete on a peer's mbarrier before
  // that peer's expect_tx: the phase completes only once both have happened)
  if (threadIdx.x < CL) {
    const int d = threadIdx.x;
    const uint32_t bytes = uint32_t(blk * sizeof(cplx<T>));
    if (d == 0) {
      const uint32_t mb = smem_u32(&x.mbar[which]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes * CL) : "memory");
    }
    const bool send = !(x.drop && rank == 0 && which == 0);
    if (send) {
      const uint32_t dst = dsmem_map(x.rb + size_t(rank) * blk, d);
      const uint32_t src = smem_u32(x.sb + size_t(d) * blk);
      const uint32_t rmb = dsmem_map(&x.mbar[which], d);
      asm volatile(
          "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
          "r"(src), "r"(bytes), "r"(rmb)
          : "memory");
    }
  }
  mbar_wait_bounded(&x.mbar[which], (x.phases >> which) & 1u, x.timeout);
  x.phases ^= 1u << which;
  xchg_arrive<T, CL>(x);  // this CTA's incoming blocks have landed
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

// (-1)^(x [bit 0] + y [bit 1] + z [bit 2]) of the axes in ``mask``
template <typename T>
__device__ __forceinline__ T axis_sign(int mask, int x, int y, int z) {
  const int e = ((mask & 1) ? x : 0) + ((mask & 2) ? y : 0) + ((mask & 4) ? z : 0);
  return (e & 1) ? T(-1) : T(1);
}

template <typename T, int N, int CL, bool DCT>
struct PlaneOps {
  using Cfg = PlaneCfg<T, N, CL, DCT>;
  static constexpr int E = Cfg::E, G = Cfg::G, NC = Cfg::NC, LS = Cfg::LS, ROWS = Cfg::ROWS;
  static constexpr int THREADS = Cfg::THREADS;
  // a CTA's NC columns of a plane row are consecutive in memory (c0 and NC even:
  // 16-byte pairs)
  static constexpr bool PAIRS = pair_io<T>() && NC % 2 == 0;
  static __device__ __forceinline__ int elem(int e) { return tile_elem<PAIRS>(threadIdx.x, THREADS, e); }

  // ---- column phase, inverse direction ---------------------------------
  // multiply a periodic spectral value at (ky, kz) by i q_y, i q_z or -q_y^2
  static __device__ __forceinline__ cplx<T> apply_mult(cplx<T> v, int mult, const T* q, int ky, int kz) {
    if (mult == kMulNegQz2) {
      if constexpr (DCT) {  // the pair holds kz = 2 kz, 2 kz + 1
        const T qa = __ldg(&q[2 * kz]), qb = __ldg(&q[2 * kz + 1]);
        return mk<T>(-qa * qa * v.x, -qb * qb * v.y);
      } else {
        const T qq = __ldg(&q[kz]);
        return cscale<T>(v, -qq * qq);
      }
    }
    if (mult == kMulIqy || mult == kMulIqz) {
      const T qq = __ldg(&q[mult == kMulIqy ? ky : kz]);
      return mk<T>(-qq * v.y, qq * v.x);
    }
    if (mult == kMulNegQy2) {
      const T qq = __ldg(&q[ky]);
      return cscale<T>(v, -qq * qq);
    }
    if (mult == kMulSinDy) {  // v was loaded from row N - ky (col_load)
      return ky == 0 ? mk<T>(T(0), T(0)) : cscale<T>(v, -__ldg(&q[N - ky]));
    }
    return v;
  }

  // Load this CTA's columns of a partial spectrum (times ``mult``), plus a
  // second partial ``plane2`` times ``mult2`` when given.
  static __device__ void col_load(cplx<T>* buf, const cplx<T>* __restrict__ plane, int rank, int mult = kMulNone,
                                  const T* q = nullptr, const cplx<T>* __restrict__ plane2 = nullptr,
                                  int mult2 = kMulNone) {
    const int c0 = rank * NC;
    // NC * N == THREADS * E: every thread issues its E loads before any store
    cplx<T> tmp[E];
#pragma unroll
    for (int e = 0; e < E; e += PAIRS ? 2 : 1) {
      const int idx = elem(e);
      const int row = mult == kMulSinDy ? (N - idx / NC) & (N - 1) : idx / NC;  // reversed rows for d/dy
      const cplx<T>* p = &plane[row * (N / 2) + c0 + idx % NC];
      if constexpr (PAIRS) ld_pair(p, tmp[e], tmp[e + 1]);
      else tmp[e] = *p;
    }
    if (mult != kMulNone) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int idx = elem(e);
        tmp[e] = apply_mult(tmp[e], mult, q, idx / NC, c0 + idx % NC);
      }
    }
    if (plane2) {
      cplx<T> u[E];
#pragma unroll
      for (int e = 0; e < E; e += PAIRS ? 2 : 1) {
        const int idx = elem(e);
        const cplx<T>* p = &plane2[(idx / NC) * (N / 2) + c0 + idx % NC];
        if constexpr (PAIRS) ld_pair(p, u[e], u[e + 1]);
        else u[e] = *p;
      }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int idx = elem(e);
        tmp[e] = cadd<T>(tmp[e], apply_mult(u[e], mult2, q, idx / NC, c0 + idx % NC));
      }
    }
    constexpr int KPT = (N + THREADS - 1) / THREADS;  // ky per thread for the kz=0 / N/2 columns
    cplx<T> nyq[KPT];
    if constexpr (!DCT) {
      if (rank == 0) {
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) {
            nyq[m] = apply_mult(plane[N * (N / 2) + ky], mult, q, ky, N / 2);
            if (plane2) nyq[m] = cadd<T>(nyq[m], apply_mult(plane2[N * (N / 2) + ky], mult2, q, ky, N / 2));
          }
        }
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = elem(e);
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

  // ---- spectral-slot access of the row and column phases ----------------
  // periodic row phase: slot k of half h (row 2q + h) of row-pair line q
  static __device__ __forceinline__ const cplx<T>& row_slot(const cplx<T>* lb, const Xchg<T>& x, int q, int h, int k) {
    if constexpr (CL == 1 || Cfg::DIRECT) return lb[q * LS + pad(h * (N / 2) + k)];
    else return x.rb[(k / NC) * Cfg::BLK + (2 * q + h) * Cfg::SA + (k % NC)];
  }
  // Neumann row phase: slot kz of row-pair line q
  static __device__ __forceinline__ const cplx<T>& row_pair(const cplx<T>* lb, const Xchg<T>& x, int q, int kz) {
    if constexpr (CL == 1 || Cfg::DIRECT) return lb[q * LS + pad(kz)];
    else return x.rb[(kz / (2 * NC)) * Cfg::BLK + q * Cfg::SA + (kz % (2 * NC))];
  }
  // forward column phase: element ky of column line c
  static __device__ __forceinline__ const cplx<T>& col_in(const cplx<T>* lb, const Xchg<T>& x, int c, int ky) {
    if constexpr (CL == 1 || Cfg::DIRECT) return lb[c * LS + pad(ky)];
    else return x.rb[(ky / ROWS) * Cfg::BLK + (ky % ROWS) * Cfg::SBs + c];
  }

  // inverse y transform of the owned columns, then hand each value to the row
  // phase: in place (CL == 1) or through the cluster exchange
  static __device__ void col_inverse_to_rows(cplx<T>* buf, Xchg<T>& xs, int rank, const TwTables<T>& tw) {
    const int line = threadIdx.x / G, t = threadIdx.x % G;
    cplx<T>* L = buf + line * LS;
    cplx<T> v[E];
    if constexpr (!DCT) {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return L[pad(i)]; });
    } else if constexpr (E / radix_of<N, +1, 0>() == 1) {
      // REDFT01 input exp(+i pi i/2N) (X[i] - i X[N-i]) (as dct3_pre) formed in
      // registers: load the line into the first-pass slots (slot r holds
      // i = t + G r), then take each partner N - i from
      // lane (G - t) mod G, slot E-1-r, by a warp shuffle.  Lane 0 holds its
      // own partners (slot (E - r) mod E), so it pairs slots r+1 and E-1-r in
      // step r; its slot 0 (i = 0, no partner) is already final.  Every slot
      // a shuffle reads is still unmodified in its lane.
      const int src = (G - t) & (G - 1);
#pragma unroll
      for (int r = 0; r < E; ++r) v[r] = L[pad(t + G * r)];
#pragma unroll
      for (int r = 0; r < E / 2; ++r) {
        const int B = E - 1 - r;
        const cplx<T> qB = shfl_c<T>(v[B], src, G);
        const cplx<T> qA = shfl_c<T>(v[r], src, G);
        const bool z = t == 0;
        const int iA = t + G * (r + (z ? 1 : 0)), iB = t + G * B;
        const cplx<T> aA = z ? v[r + 1] : v[r];
        const cplx<T> pB = z ? v[r + 1] : qA;
        const cplx<T> aB = v[B];
        cplx<T> wA = tw.d[iA], wB = tw.d[iB];
        wA.y = -wA.y;
        wB.y = -wB.y;
        const cplx<T> oA = cmul<T>(mk<T>(aA.x + qB.y, aA.y - qB.x), wA);  // iA, iB > 0
        const cplx<T> oB = cmul<T>(mk<T>(aB.x + pB.y, aB.y - pB.x), wB);
        if (z) v[r + 1] = oA;
        else v[r] = oA;
        v[B] = oB;
      }
      fft_regs<T, N, +1>(v, L, t, tw.i);
    } else {
      fft_line<T, N, +1>(v, L, t, tw.i, [&](int i) { return dct3_pre<T, N>(L, i, tw.d); });
    }
    constexpr int RL = Cfg::RL_INV;
    if constexpr (CL == 1 || Cfg::DIRECT) {
      // in place: row y of global column kc goes to the line buffer of the CTA
      // that owns row y (this one without a cluster), row-pair line (y mod ROWS)/2
      transpose_sync<CL>();
      const int kc = rank * NC + line;
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int n = out_index<N, +1>(t, b, r);
          const cplx<T> val = v[b * RL + r];
          if constexpr (!DCT) {
            const int yl = n % ROWS;
            st_rank<CL>(&buf[(yl >> 1) * LS + pad((yl & 1) * (N / 2) + kc)], val, n / ROWS);
          } else {
            const int y = mk_perm<N>(n);
            const int yl = y % ROWS;
            T* rb = reinterpret_cast<T*>(buf);
            const int base = (yl >> 1) * LS;
            st_rank<CL>(&rb[2 * (base + pad(2 * kc)) + (yl & 1)], val.x, y / ROWS);
            st_rank<CL>(&rb[2 * (base + pad(2 * kc + 1)) + (yl & 1)], val.y, y / ROWS);
          }
        }
      transpose_sync<CL>();
    } else {
      if constexpr (Cfg::ALIAS) __syncthreads();  // every line has left the scratch the send blocks overlay
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int n = out_index<N, +1>(t, b, r);
          const cplx<T> val = v[b * RL + r];
          if constexpr (!DCT) {
            const int dest = n / ROWS, yl = n % ROWS;
            xs.sb[dest * Cfg::BLK + yl * Cfg::SA + line] = val;
          } else {
            const int y = mk_perm<N>(n);
            const int dest = y / ROWS, yl = y % ROWS;
            T* sb = reinterpret_cast<T*>(xs.sb + dest * Cfg::BLK + (yl >> 1) * Cfg::SA + 2 * line);
            sb[yl & 1] = val.x;
            sb[2 + (yl & 1)] = val.y;
          }
        }
      bulk_exchange<T, Cfg::XCL>(xs, 0, rank, Cfg::BLK);
    }
  }

  // ---- row phase -------------------------------------------------------
  // inverse z transform of row pair ``line``; v slot holds psi(y0, z), psi(y0+1, z)
  static __device__ __forceinline__ void row_inverse(cplx<T> (&v)[E], const cplx<T>* buf, Xchg<T>& xs,
                                                     cplx<T>* L, int q, int t, const TwTables<T>& tw,
                                                     const T* qt = nullptr, bool sin_dz = false) {
    // the first pass reads the row pair into registers; the passes after it use
    // the scratch L (for bulk exchanges a line of the receive-block region)
    if constexpr (!DCT) {
      // Z = X_a + i X_b with Hermitian extension; slot 0 holds (X[0], X[N/2])
      load_first<T, N, +1>(v, t, [&](int i) {
        if (i == 0 || i == N / 2) {
          const cplx<T> a = row_slot(buf, xs, q, 0, 0), b = row_slot(buf, xs, q, 1, 0);
          return i == 0 ? mk<T>(a.x, b.x) : mk<T>(a.y, b.y);
        }
        const int k = i < N / 2 ? i : N - i;
        const cplx<T> a = row_slot(buf, xs, q, 0, k), b = row_slot(buf, xs, q, 1, k);
        return i < N / 2 ? mk<T>(a.x - b.y, a.y + b.x) : mk<T>(a.x + b.y, b.x - a.y);
      });
    } else {
      // REDFT01 input: exp(+i pi i/2N) (X[i] - i X[N-i]), X[N] = 0; for the
      // sine series of d/dz X[k] is -q_{N-k} times coefficient N - k (0 at k = 0)
      auto X = [&](int k) -> cplx<T> {
        if (!sin_dz) return row_pair(buf, xs, q, k);
        if (k == 0) return mk<T>(T(0), T(0));
        return cscale<T>(row_pair(buf, xs, q, N - k), -__ldg(&qt[N - k]));
      };
      load_first<T, N, +1>(v, t, [&](int i) {
        const cplx<T> a = X(i);
        cplx<T> u = a;
        if (i != 0) {
          const cplx<T> b = X(N - i);
          u = mk<T>(a.x + b.y, a.y - b.x);
        }
        cplx<T> w = tw.d[i];
        w.y = -w.y;
        return cmul<T>(u, w);
      });
    }
    // bulk exchanges: the scratch L overlays the receive blocks, which every
    // line's first pass has read once the CTA has synchronised
    if constexpr (Cfg::ALIAS) __syncthreads();
    fft_regs<T, N, +1>(v, L, t, tw.i);
  }

  // z coordinate of register slot (b, r) after row_inverse (== the input slot of
  // the forward z transform)
  static __device__ __forceinline__ int row_z(int t, int b, int r) {
    const int n = out_index<N, +1>(t, b, r);
    if constexpr (DCT) return mk_perm<N>(n);
    return n;
  }

  // forward z transform from registers, then hand the spectra to the column
  // owners (in place or through the cluster exchange)
  static __device__ void row_forward_to_cols(cplx<T> (&v)[E], cplx<T>* buf, Xchg<T>& xs, cplx<T>* L, int rank,
                                             int line, int t, const TwTables<T>& tw) {
    fft_regs<T, N, -1>(v, L, t, tw.f);
    constexpr int RL = Cfg::RL_FWD;
    cplx<T> part[E];  // element (N - k) mod N of every slot
    mirror_partners<T, N, RL>(v, part, t);
    if constexpr (!DCT) {
      // split Z into the two half spectra; slot k < N/2 from register r < RL/2
      cplx<T> oa[E / 2], ob[E / 2];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL / 2; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          const int s = b * (RL / 2) + r;
          const cplx<T> zk = v[b * RL + r];
          if (k == 0) {
            const cplx<T> zn = v[RL / 2];  // k = N/2 sits in slot (0, RL/2) of the same thread
            oa[s] = mk<T>(zk.x, zn.x);
            ob[s] = mk<T>(zk.y, zn.y);
          } else {
            const cplx<T> zm = part[b * RL + r];
            oa[s] = mk<T>(T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y));
            ob[s] = mk<T>(T(0.5) * (zk.y + zm.y), T(0.5) * (zm.x - zk.x));
          }
        }
      if constexpr (CL == 1 || Cfg::DIRECT) {
        // in place: column k goes to the line buffer of the CTA that owns it
        transpose_sync<CL>();
        const int y0 = rank * ROWS + 2 * line;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL / 2; ++r) {
            const int k = out_index<N, -1>(t, b, r);
            const int s = b * (RL / 2) + r;
            cplx<T>* col = buf + (k % NC) * LS;
            st_rank<CL>(&col[pad(y0)], oa[s], k / NC);
            st_rank<CL>(&col[pad(y0 + 1)], ob[s], k / NC);
          }
        transpose_sync<CL>();
      } else {
        xchg_rb_done<T, Cfg::XCL>(xs);  // the row scratch overlays the receive blocks
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL / 2; ++r) {
            const int k = out_index<N, -1>(t, b, r);
            const int s = b * (RL / 2) + r;
            cplx<T>* blk = xs.sb + (k / NC) * Cfg::BLK + (k % NC);
            blk[(2 * line) * Cfg::SBs] = oa[s];
            blk[(2 * line + 1) * Cfg::SBs] = ob[s];
          }
        bulk_exchange<T, Cfg::XCL>(xs, 1, rank, Cfg::BLK);
      }
    } else {
      cplx<T>(&o)[E] = v;  // REDFT10 output, in place
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          cplx<T> w = tw.d[k];
          cplx<T> a = cmul<T>(v[b * RL + r], w);
          cplx<T> bm = cmul<T>(part[b * RL + r], conjg<T>(w));
          o[b * RL + r] = cadd<T>(a, bm);
        }
      if constexpr (CL == 1 || Cfg::DIRECT) {
        transpose_sync<CL>();
        const int y0 = rank * ROWS + 2 * line;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int k = out_index<N, -1>(t, b, r);
            const int pk = k >> 1;
            T* cb = reinterpret_cast<T*>(buf + (pk % NC) * LS);
            st_rank<CL>(&cb[2 * pad(y0) + (k & 1)], o[b * RL + r].x, pk / NC);
            st_rank<CL>(&cb[2 * pad(y0 + 1) + (k & 1)], o[b * RL + r].y, pk / NC);
          }
        transpose_sync<CL>();
      } else {
        xchg_rb_done<T, Cfg::XCL>(xs);  // the row scratch overlays the receive blocks
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int k = out_index<N, -1>(t, b, r);
            const int p = k >> 1;
            T* blk = reinterpret_cast<T*>(xs.sb + (p / NC) * Cfg::BLK + (p % NC));
            blk[2 * (2 * line) * Cfg::SBs + (k & 1)] = o[b * RL + r].x;
            blk[2 * (2 * line + 1) * Cfg::SBs + (k & 1)] = o[b * RL + r].y;
          }
        bulk_exchange<T, Cfg::XCL>(xs, 1, rank, Cfg::BLK);
      }
    }
  }

  // ---- column phase, forward direction ---------------------------------
  static __device__ void col_forward_store(cplx<T>* buf, Xchg<T>& xs, cplx<T>* __restrict__ plane, int rank,
                                           const TwTables<T>& tw) {
    const int line = threadIdx.x / G, t = threadIdx.x % G;
    // bulk exchanges: the column lines are built in the receive-block region once
    // every first pass has read it; the send blocks (still being read by the
    // peers' copies) stay untouched
    cplx<T>* cb = Cfg::ALIAS ? xs.rb : buf;
    cplx<T>* L = cb + line * LS;
    cplx<T> v[E];
    constexpr int RL = Cfg::RL_FWD;
    if constexpr (!DCT) {
      load_first<T, N, -1>(v, t, [&](int i) { return col_in(buf, xs, line, i); });
      if constexpr (Cfg::ALIAS) __syncthreads();
      fft_regs<T, N, -1>(v, L, t, tw.f);
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
            cplx<T> z = cb[pad(ky)], zm = cb[pad((N - ky) & (N - 1))];
            f0[m] = mk<T>(T(0.5) * (z.x + zm.x), T(0.5) * (z.y - zm.y));
            fn[m] = mk<T>(T(0.5) * (z.y + zm.y), T(0.5) * (zm.x - z.x));
          }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < KPT; ++m) {
          const int ky = threadIdx.x + m * THREADS;
          if (ky < N) {
            cb[pad(ky)] = f0[m];
            cb[NC * LS + pad(ky)] = fn[m];
          }
        }
        __syncthreads();
      }
    } else {
      load_first<T, N, -1>(v, t, [&](int i) { return col_in(buf, xs, line, mk_perm<N>(i)); });
      if constexpr (Cfg::ALIAS) __syncthreads();
      fft_regs<T, N, -1>(v, L, t, tw.f);
      // REDFT10 post-processing, one slot at a time: the partner (N - k) mod N
      // of each slot comes from lane (G - t) mod G by a warp shuffle (lane 0
      // holds its own partners, as in mirror_partners), and the result goes
      // straight to the line; v is only read, so no partner array is held
      __syncwarp();  // every lane of the line has finished reading it in the last pass
      constexpr int NB = E / RL;
      const int src = (G - t) & (G - 1);
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int k = out_index<N, -1>(t, b, r);
          const cplx<T> q = shfl_c<T>(v[(NB - 1 - b) * RL + (RL - 1 - r)], src, G);
          const int zs = b == 0 ? (RL - r) % RL : (NB - b) * RL + (RL - 1 - r);
          const cplx<T> pm = t == 0 ? v[zs] : q;
          const cplx<T> w = tw.d[k];
          L[pad(k)] = cadd<T>(cmul<T>(v[b * RL + r], w), cmul<T>(pm, conjg<T>(w)));
        }
      __syncthreads();
    }
    const int c0 = rank * NC;
#pragma unroll
    for (int e = 0; e < E; e += PAIRS ? 2 : 1) {
      const int idx = elem(e);
      cplx<T>* p = &plane[(idx / NC) * (N / 2) + c0 + idx % NC];
      if constexpr (PAIRS) st_pair(p, cb[(idx % NC) * LS + pad(idx / NC)], cb[(idx % NC + 1) * LS + pad(idx / NC)]);
      else *p = cb[(idx % NC) * LS + pad(idx / NC)];
    }
    if constexpr (!DCT) {
      if (rank == 0) {
        for (int ky = threadIdx.x; ky < N; ky += THREADS) plane[N * (N / 2) + ky] = cb[NC * LS + pad(ky)];
      }
    }
  }
};

// Real-space pointwise stage of one row pair: nonlinearity (+ pinning penalty
// on the plane z = N/2, periodicFFT/pf3dMorph.cpp:456-467).  ``v`` holds psi
// on entry and N(psi) on exit.
template <typename T, int N, int CL, bool DCT>
__device__ __forceinline__ void row_nonlin(cplx<T> (&v)[Plan<N>::E], cplx<T>* L, int t, const PointParams& pp,
                                           const T* wall = nullptr, const T* lp0 = nullptr, int kwall = 0) {
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
      if (z < kwall) {  // substrate penalty (cosFFT/comet/cosNoAdvMorph.cpp:591-623)
        const T w = wall[z];
        o.x += w * lp0[z];
        o.y += w * lp0[kwall + z];
      }
      v[b * RL + r] = o;
    }
}

template <typename T, int N, int CL, bool DCT, int MODE>
__global__ void __launch_bounds__(PlaneCfg<T, N, CL, DCT>::THREADS, PlaneCfg<T, N, CL, DCT>::min_blocks(MODE))
plane_kernel(const __grid_constant__ PlaneLaunch<T> pl) {
  const PlaneArgs<T>& a = pl.c[plane_multi(MODE) ? blockIdx.z : 0];
  using Cfg = PlaneCfg<T, N, CL, DCT>;
  using Ops = PlaneOps<T, N, CL, DCT>;
  constexpr int E = Cfg::E, G = Cfg::G, LS = Cfg::LS, ROWS = Cfg::ROWS, FP = Cfg::FP;
  constexpr int RL = Cfg::RL_INV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  double* scratch = reinterpret_cast<double*>(smem_raw + Cfg::RED_OFF);
  const TwTables<T> tw =
      Cfg::TW_SMEM
          ? stage_twiddles<T, N>(reinterpret_cast<cplx<T>*>(smem_raw + Cfg::TW_OFF), a.tw, threadIdx.x, Cfg::THREADS, DCT)
          : device_twiddles<T, N>(a.tw);
  // every staged entry is written before any thread's first transform (the
  // passes that start with a row transform read them right away)
  if constexpr (Cfg::TW_SMEM) __syncthreads();

  int rank = 0;
  if constexpr (CL > 1) rank = int(cg::this_cluster().block_rank());
  Xchg<T> xs{};
  if constexpr (CL > 1 && !Cfg::DIRECT) {
    xs.sb = reinterpret_cast<cplx<T>*>(smem_raw + Cfg::SB_OFF);
    xs.rb = reinterpret_cast<cplx<T>*>(smem_raw + Cfg::RB_OFF);
    xs.mbar = reinterpret_cast<uint64_t*>(smem_raw + Cfg::MB_OFF);
    xs.phases = 0;
    xs.timeout = a.timeout;
    xs.drop = a.drop_exchange;
    xs.armed = false;
    if (threadIdx.x == 0) {
      // peers see the initialised barriers once they have waited on the arrive below
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&xs.mbar[0])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&xs.mbar[1])) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // publishes the initialised mbarriers (and, for the passes that start with
    // a column phase, the free receive blocks); matched by the settle of the first
    // exchange.  The passes that start with a row phase use the receive blocks as
    // scratch first and arrive in xchg_rb_done.
    if constexpr (MODE != kPlaneInit && MODE != kPlaneMulFwd) xchg_arrive<T, Cfg::XCL>(xs);
  }
  grid_dependency_wait();
  const int x = blockIdx.x / CL;
  if (a.pf_dist > 0 && rank == 0 && threadIdx.x == 0 && x + a.pf_dist < N) {
    const size_t off = (size_t(blockIdx.y) * N + x + a.pf_dist) * FP;
    const uint32_t bytes = uint32_t(size_t(FP) * sizeof(cplx<T>));
    if constexpr (MODE == kPlaneStep || MODE == kPlaneGetPsi || MODE == kPlaneInvReal || MODE == kPlaneAdj ||
                  MODE == kPlaneInvMulFwd) {
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.src + off), "r"(bytes) : "memory");
    } else if constexpr (MODE == kPlaneAdvN) {
      for (int c = 0; c < 3; ++c)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.src3[c] + off), "r"(bytes) : "memory");
    }
  }
  const int rep = blockIdx.y;
  const int line = threadIdx.x / G, t = threadIdx.x % G;
  // row-phase scratch line: the column line buffer without a cluster or with
  // direct exchanges, a line of the receive-block region with bulk exchanges
  cplx<T>* L;
  if constexpr (Cfg::ALIAS) L = xs.rb + line * LS;
  else L = buf + line * LS;
  const size_t plane_off = (size_t(rep) * N + x) * FP;
  const size_t real_off = (size_t(rep) * N + x) * size_t(N) * N;
  const int y0 = rank * ROWS + 2 * line;
  cplx<T> v[E];

  if constexpr (MODE == kPlaneStep || MODE == kPlaneGetPsi || MODE == kPlaneInvReal || MODE == kPlaneAdj ||
                MODE == kPlaneInvMulFwd) {
    if constexpr (MODE == kPlaneInvReal || MODE == kPlaneInvMulFwd) {
      Ops::col_load(buf, a.src + plane_off, rank, a.mult, a.q, a.src2 ? a.src2 + plane_off : nullptr, a.mult2);
    } else {
      Ops::col_load(buf, a.src + plane_off, rank);
    }
    Ops::col_inverse_to_rows(buf, xs, rank, tw);
    Ops::row_inverse(v, buf, xs, L, line, t, tw, a.q, DCT && MODE == kPlaneInvReal && a.sin_dz);
    // done with the receive blocks; the step and the adjoint exchange once more
    if constexpr (MODE == kPlaneInvReal) {
      if (a.sign_axes) {  // the sine transforms' real-space signs (rows y0, y0 + 1)
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
          for (int r = 0; r < RL; ++r) {
            const int z = Ops::row_z(t, b, r);
            v[b * RL + r] = mk<T>(axis_sign<T>(a.sign_axes, x, y0, z) * v[b * RL + r].x,
                                  axis_sign<T>(a.sign_axes, x, y0 + 1, z) * v[b * RL + r].y);
          }
      }
    }

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
    if (MODE == kPlaneInvReal && a.real_zn > 0) {
      // only the planes z < real_zn, compact
      const int zn = a.real_zn;
      T* o0 = a.real_out + ((size_t(rep) * N + x) * N + y0) * zn;
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int z = Ops::row_z(t, b, r);
          if (z < zn) {
            o0[z] = v[b * RL + r].x;
            o0[zn + z] = v[b * RL + r].y;
          }
        }
    } else if (MODE == kPlaneInvReal || MODE == kPlaneInvMulFwd || (MODE == kPlaneStep && (a.flags & kFlRealOut))) {
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const size_t ia = real_off + size_t(y0) * N + Ops::row_z(t, b, r);
          a.real_out[ia] = v[b * RL + r].x;
          a.real_out[ia + N] = v[b * RL + r].y;
        }
    }
    if constexpr (MODE == kPlaneAdj) {
      // g^n = N'(psi^n) (c_n mu^{n+1} - mu^{n+2}); v holds the bracket (its
      // partial is what the pencil pass of step n+1 emitted)
      const T beta = T(a.pp.beta), gamma = T(a.pp.gamma);
      const T* psi = a.real_in[1];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const size_t ia = real_off + size_t(y0) * N + Ops::row_z(t, b, r);
          const cplx<T> m = v[b * RL + r];
          v[b * RL + r] = mk<T>(nonlin_deriv<T>(psi[ia], beta, gamma, a.pp.nonlin) * m.x,
                                nonlin_deriv<T>(psi[ia + N], beta, gamma, a.pp.nonlin) * m.y);
        }
      Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
      Ops::col_forward_store(buf, xs, a.dst + plane_off, rank, tw);
    }
    if constexpr (MODE == kPlaneInvMulFwd) {
      // stress component S_c = (L psi) d_c psi (periodicFFT/pf3d.cpp:417-429), formed
      // from the derivative just written and sent forward in the same pass
      const T* f = a.real_in[0];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const size_t ia = real_off + size_t(y0) * N + Ops::row_z(t, b, r);
          v[b * RL + r] = mk<T>(v[b * RL + r].x * f[ia], v[b * RL + r].y * f[ia + N]);
        }
      Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
      Ops::col_forward_store(buf, xs, a.dst + plane_off, rank, tw);
    }
    if constexpr (MODE == kPlaneStep) {
      const T* lp0 = a.kwall > 0 ? a.lperp + ((size_t(rep) * N + x) * N + y0) * a.kwall : nullptr;
      row_nonlin<T, N, CL, DCT>(v, L, t, a.pp, a.wall, lp0, a.kwall);
      Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
      Ops::col_forward_store(buf, xs, a.dst + plane_off, rank, tw);
    }
  } else if constexpr (MODE == kPlaneAdvN) {
    // N = beta psi^3 - gamma psi^5 (+ pinning) - u . grad psi (periodicFFT/pf3d.cpp:455-467):
    // the velocity components come in as partials and are inverted here one
    // after the other, u_c d_c psi accumulating in registers
    cplx<T> acc[E];
#pragma unroll
    for (int e = 0; e < E; ++e) acc[e] = mk<T>(T(0), T(0));
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      if (c > 0) __syncthreads();  // every line has left the line buffer
      Ops::col_load(buf, a.src3[c] + plane_off, rank);
      Ops::col_inverse_to_rows(buf, xs, rank, tw);
      Ops::row_inverse(v, buf, xs, L, line, t, tw);
      if (c < 2) xchg_rb_done<T, Cfg::XCL>(xs);  // done with the receive blocks; another exchange follows
      const T* d = a.real_in[1 + c];
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int z = Ops::row_z(t, b, r);
          const size_t ia = real_off + size_t(y0) * N + z;
          // Neumann: the partials carry (-1)^(x+y+z) u (rows y0, y0 + 1)
          const T sg = axis_sign<T>(a.sign_axes, x, y0, z), sb = axis_sign<T>(a.sign_axes, x, y0 + 1, z);
          acc[b * RL + r].x = fma(sg * v[b * RL + r].x, d[ia], acc[b * RL + r].x);
          acc[b * RL + r].y = fma(sb * v[b * RL + r].y, d[ia + N], acc[b * RL + r].y);
        }
    }
    const T beta = T(a.pp.beta), gamma = T(a.pp.gamma);
    const T cpen = T(2.0 * a.pp.w_mid * a.pp.inv_dz2);
    const T* ps = a.real_in[0];
#pragma unroll
    for (int b = 0; b < E / RL; ++b)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int z = Ops::row_z(t, b, r);
        const size_t ia = real_off + size_t(y0) * N + z, ib = ia + N;
        const T pa = ps[ia], pb = ps[ib];
        T oa = nonlin_eval<T>(pa, beta, gamma, a.pp.nonlin);
        T ob = nonlin_eval<T>(pb, beta, gamma, a.pp.nonlin);
        if (a.pp.w_mid != 0.0 && z == N / 2) {
          oa += cpen * (ps[ia - 1] - T(2) * pa + ps[ia + 1]);
          ob += cpen * (ps[ib - 1] - T(2) * pb + ps[ib + 1]);
        }
        v[b * RL + r] = mk<T>(oa - acc[b * RL + r].x, ob - acc[b * RL + r].y);
      }
    Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
    Ops::col_forward_store(buf, xs, a.dst + plane_off, rank, tw);
  } else if constexpr (MODE == kPlaneMulFwd) {
    // stress component S_c = (L psi) d_c psi of the Neumann Stokes solve
    // (cosFFT/comet/morphSurfK.cpp:760-770), signed for the sine transform
    const T* f0 = a.real_in[0];
    const T* f1 = a.real_in[1];
    constexpr int R0 = radix_of<N, -1, 0>();
#pragma unroll
    for (int b = 0; b < E / R0; ++b)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int n = in_index<N, -1>(t, b, r);
        const int z = DCT ? mk_perm<N>(n) : n;
        const size_t ia = real_off + size_t(y0) * N + z, ib = ia + N;
        const T sg = axis_sign<T>(a.sign_axes, x, y0, z), sb = axis_sign<T>(a.sign_axes, x, y0 + 1, z);
        v[b * R0 + r] = mk<T>(sg * f0[ia] * f1[ia], sb * f0[ib] * f1[ib]);
      }
    Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
    Ops::col_forward_store(buf, xs, a.dst + plane_off, rank, tw);
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
            if (z < a.kwall) {  // substrate penalty of psi^0
              const T* lp0 = a.lperp + ((size_t(rep) * N + x) * N + y0) * a.kwall;
              na += a.wall[z] * lp0[z];
              nb += a.wall[z] * lp0[a.kwall + z];
            }
            pa = na;
            pb = nb;
          }
          v[b * R0 + r] = mk<T>(pa, pb);
        }
      Ops::row_forward_to_cols(v, buf, xs, L, rank, line, t, tw);
      Ops::col_forward_store(buf, xs, (field == 0 ? a.dst2 : a.dst) + plane_off, rank, tw);
    }
  }
  // every peer has received this CTA's last blocks (and this CTA its own): no
  // copy still reads its shared memory or is on its way into it
  xchg_settle<T, Cfg::XCL>(xs);
}

}  // namespace shb
