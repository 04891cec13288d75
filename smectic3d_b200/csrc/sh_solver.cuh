// Host-side solver: owns the device state of one handle and sequences the
// plane and pencil passes of each time step.
#pragma once
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smectic_b200.h"
#include "pencil_kernel.cuh"
#include "plane_kernel.cuh"
#include "surface_kernel.cuh"

namespace shb {

// Device allocations of the library go through here.  Test hook: while the
// countdown is armed (only inside sh_create, from SMECTIC_B200_TEST_FAIL_ALLOC=k),
// the k-th allocation fails as out of memory, which exercises the clean-up and
// SH_ENOMEM paths without exhausting the GPU.
inline int& alloc_fail_countdown() {
  static thread_local int n = 0;
  return n;
}
inline cudaError_t dev_malloc(void** ptr, size_t bytes) {
  int& c = alloc_fail_countdown();
  if (c > 0 && --c == 0) {
    *ptr = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(ptr, bytes);
}
template <class P>
inline cudaError_t dev_malloc(P** ptr, size_t bytes) {
  return dev_malloc(reinterpret_cast<void**>(ptr), bytes);
}

#define SHB_CUDA(expr)                                                        \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      err = std::string(#expr) + ": " + cudaGetErrorString(e_);               \
      return SH_ECUDA;                                                        \
    }                                                                         \
  } while (0)

// Deterministic FP64 reduction of per-CTA partials, one block per replica.
// what = 0: energy dv (local + alpha/2 norm spec); what = 1: L1 = A / (dt B)
__global__ void finalize_kernel(const double* red_plane, int nbp, const double* red_spec, int nbs, int what,
                                double dv, double spec_norm, double alpha, double dt, double* out);
// Sums the per-CTA (eps, q0) gradient slots of the reverse sweep into
// acc[rep][4] = {g_eps, 0, g_q0, 0}.
__global__ void adj_reduce_kernel(const double* red, int nblocks, double* acc);
// dst[i] = double(src[i])
template <typename T>
__global__ void to_double_kernel(const T* __restrict__ src, double* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = double(src[i]);
}
// out[rep] = dq * (the shell >= 1 of largest power in shell[rep][nshell]; the
// lowest such shell on a tie)
__global__ void shell_argmax_kernel(const double* shell, int nshell, double dq, double* out);

struct SolverBase {
  sh_params p{};
  std::vector<double> eps;
  cudaStream_t stream = nullptr;
  std::string err;
  long long steps = 0;
  long long launches = 0;
  int* d_flag = nullptr;       // [0] non-finite state, [1] cluster-exchange timeout
  double* d_psi = nullptr;     // batch * N^3 doubles (dense)
  double* d_stash = nullptr;   // L1 reference psi
  double* d_eps = nullptr;
  double* d_red_plane = nullptr;
  double* d_red_spec = nullptr;
  double* d_scalar = nullptr;  // batch doubles
  double* d_trace = nullptr;   // energy trace of the current chunk
  double* d_amp[2] = {nullptr, nullptr};  // local-amplitude map work fields (allocated on first use)
  double* d_shell = nullptr;               // spectral power per |k| shell (allocated on first use)
  int trace_cap = 0;
  std::vector<double> energy_trace;  // host copy, steps * batch
  std::vector<double> l1_last;
  int l1_count = 0;
  bool ready = false;
  bool psi0_valid = false;  // d_psi holds psi^0 exactly as uploaded
  // Test hook for the timeout path, from SMECTIC_B200_TEST_DROP_EXCHANGE=1 at
  // sh_create: the first exchange of every plane pass of a cluster loses rank
  // 0's copies, the bounded waits expire (about 1 s) and the call returns
  // SH_ETIMEOUT.  Never set otherwise.
  int drop_exchange = 0;

  virtual ~SolverBase() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_flag);
    cudaFree(d_psi);
    cudaFree(d_stash);
    cudaFree(d_eps);
    cudaFree(d_red_plane);
    cudaFree(d_red_spec);
    cudaFree(d_scalar);
    cudaFree(d_trace);
    cudaFree(d_amp[0]);
    cudaFree(d_amp[1]);
    cudaFree(d_shell);
    for (auto& e : prof_ev)
      if (e) cudaEventDestroy(e);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (stream) cudaStreamDestroy(stream);
  }
  size_t n3() const { return size_t(p.n) * p.n * p.n; }
  virtual int setup() = 0;
  virtual int init_from_psi() = 0;     // d_psi holds psi^0
  virtual int step_async(int n) = 0;
  virtual int build_graph() = 0;       // instantiate the replayed step graph ahead of time
  // per-launch event timing of the two passes (nullptr: off)
  double* prof_ms = nullptr;
  cudaEvent_t prof_ev[3] = {nullptr, nullptr, nullptr};
  // CUDA graph of kGraphChunk plain steps (replayed when no per-step host
  // bookkeeping is needed: no energy trace, L1 monitor, profiling or history)
  static constexpr int kGraphChunk = 16;
  cudaGraphExec_t graph_exec = nullptr;
  bool use_graphs = true;
  virtual int psi_to_dpsi() = 0;       // current psi -> d_psi
  virtual int energy_now(double* host) = 0;
  virtual int dominant_wavenumber(double* host) = 0;
  virtual int velocity(double* ux, double* uy, double* uz) = 0;
  virtual size_t state_bytes() const = 0;
  virtual int save_state(void* host) = 0;
  virtual int load_state(const void* host) = 0;
  virtual int surface_step(int* z, double* vn, double* hh, double* kk) = 0;
  // forward sweep from host psi0 keeping a checkpoint every ckpt_every steps,
  // then (adjoint_backward) the recompute and reverse sweep from those checkpoints
  virtual int adjoint_forward(const double* psi0, int nsteps, int ckpt_every) = 0;
  virtual int adjoint_backward(const double* dl_dpsi_t, double* g_eps, double* g_q0, double* g_psi0) = 0;
  int adjoint(const double* psi0, int nsteps, const double* dl_dpsi_t, int ckpt_every, double* g_eps, double* g_q0,
              double* g_psi0) {
    const int rc = adjoint_forward(psi0, nsteps, ckpt_every);
    return rc ? rc : adjoint_backward(dl_dpsi_t, g_eps, g_q0, g_psi0);
  }
  // the checkpoints of the last adjoint_forward, valid while the state is the
  // one that forward sweep ended in
  int adj_nsteps = 0, adj_k = 0;
  long long adj_end = -1;
  bool adj_last_hist = false;  // the history buffers hold the last segment's states
  virtual int residency(int* out) = 0;
};

template <typename T, int N, int CL, bool DCT, int TKV = 0>
struct Solver final : SolverBase {
  using PC = PlaneCfg<T, N, CL, DCT>;
  using QC = PencilCfg<T, N, DCT, TKV>;
  static constexpr int FP = PC::FP;
  // step kernels may start while the previous kernel drains (SMECTIC_B200_NO_PDL=1: off)
  bool use_pdl = getenv("SMECTIC_B200_NO_PDL") == nullptr;

  cplx<T>* W = nullptr;
  cplx<T>* P = nullptr;
  cplx<T>* Nt = nullptr;
  cplx<T>* tw = nullptr;  // [forward | inverse | quarter-wave] twiddle table
  // Stokes advection (periodic): partials of i q_x psihat and opSH psihat, the
  // three stress / velocity partials, and the real fields
  // psi, d_x psi, d_y psi, d_z psi, L psi (then u_x), u_y, u_z
  cplx<T>* Px = nullptr;
  cplx<T>* PSH = nullptr;
  cplx<T>* S3[3] = {nullptr, nullptr, nullptr};
  T* R[8] = {};      // psi, d_x psi, d_y psi, d_z psi, L psi, u_x, u_y, u_z of the current state
  T* SR[4] = {};     // surface pass: psi_xx, psi_yy, psi_xy, H-numerator (allocated on first use)
  int* d_zout = nullptr;
  double* d_surf[3] = {nullptr, nullptr, nullptr};
  // Neumann substrate penalty (sub_sigma != 0): partial of -q_x^2 scale psihat,
  // the in-plane Laplacian of psi on the planes z < kwall ([rep][x][y][kwall])
  // and wall(z) on those planes
  cplx<T>* Pxx = nullptr;
  T* Lp = nullptr;
  T* d_wall = nullptr;
  int kwall = 0;
  // Neumann curvature pass: psi, psi_xx, psi_yy, psi_zz, L psi and a scratch partial;
  // with the spectral option also psi_x, psi_y, psi_z, psi_xy, psi_xz, psi_yz
  T* CR[5] = {};
  T* CSP[6] = {};
  cplx<T>* Psc = nullptr;
  bool real_fields_current = false;
  bool u_real_current = false;
  // adjoint work buffers, kept for the handle's lifetime once allocated
  struct AdjBufs {
    cplx<T>* ck = nullptr;   // checkpoints: nseg states x {W, P, Nt}
    cplx<T>* hs = nullptr;   // (k+1) psihat of a segment, pencil-major
    T* hr = nullptr;         // (k+1) psi of a segment
    cplx<T>* lam = nullptr;  // lambdahat, pencil-major
    cplx<T>* gp = nullptr;   // partial of g
    cplx<T>* mp = nullptr;   // partial of c_n mu^{n+1} - mu^{n+2}
    double* red = nullptr;   // per-CTA gradient sums of the reverse sweep
    double* acc = nullptr;
    cplx<T>* fin = nullptr;  // {W, P, Nt} of the state the forward sweep ended in
    int nseg = 0, k = 0;
    ~AdjBufs() {
      cudaFree(ck); cudaFree(hs); cudaFree(hr); cudaFree(lam); cudaFree(gp); cudaFree(mp);
      cudaFree(red); cudaFree(acc); cudaFree(fin);
    }
  } adj;
  // adjoint: per-step history of a recomputed segment (psihat pencil-major, psi real)
  cplx<T>* hist_spec = nullptr;
  T* hist_real = nullptr;
  int hist_pos = 0;
  T* q = nullptr;
  double* qd = nullptr;  // the wavenumbers in FP64 (the FP32 spectral update uses them)

  ~Solver() override {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(W);
    cudaFree(P);
    cudaFree(Nt);
    cudaFree(tw);
    cudaFree(q);
    cudaFree(qd);
    cudaFree(Px);
    cudaFree(PSH);
    for (auto* p3 : S3) cudaFree(p3);
    for (auto* r : R) cudaFree(r);
    for (auto* r : SR) cudaFree(r);
    cudaFree(d_zout);
    for (auto* d : d_surf) cudaFree(d);
    cudaFree(Pxx);
    cudaFree(Lp);
    cudaFree(d_wall);
    for (auto* r : CR) cudaFree(r);
    for (auto* r : CSP) cudaFree(r);
    cudaFree(Psc);
  }

  size_t field_elems() const { return size_t(p.batch) * N * FP; }

  PointParams point_params() const {
    PointParams pp;
    pp.dt = p.dt;
    pp.beta = p.beta;
    pp.gamma = p.gamma;
    pp.alpha = p.alpha;
    pp.q0 = p.q0;
    pp.eta_rho = p.eta * p.rho;
    pp.w_mid = p.w_mid;
    pp.inv_dz2 = 1.0 / (p.dx * p.dx);
    pp.scale = DCT ? 0.125 / (double(N) * N * N) : 1.0 / (double(N) * N * N);
    pp.nonlin = p.nonlinearity;
    pp.scheme = p.scheme;
    pp.eps = d_eps;
    return pp;
  }

  template <int MODE>
  static constexpr auto plane_fn() { return &plane_kernel<T, N, CL, DCT, MODE>; }
  template <int MODE>
  static constexpr auto pencil_fn() { return &pencil_kernel<T, N, DCT, MODE, TKV>; }

  template <class K>
  int set_attrs(K kern, size_t smem, bool cluster) {
    SHB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if (cluster && CL > 8) SHB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return SH_OK;
  }

  // the plain step's pencil pass: FP32 fields take their CNAB2 multipliers in
  // FP64 when the handle asks for it (SH_FP32_UPDATE64)
  int launch_pencil_step(const PencilArgs<T>& b, int reps = 0) {
    if (sizeof(T) == 4 && p.precision == SH_FP32_UPDATE64) return launch_pencil<kPencilStepU64>(b, reps);
    return launch_pencil<kPencilStep>(b, reps);
  }

  // a pencil mode whose shared memory does not fit a CTA is never launched
  template <int MODE>
  int set_pencil_attrs() {
    if constexpr (QC::fits(MODE)) return set_attrs(pencil_fn<MODE>(), QC::smem(MODE), false);
    return SH_OK;
  }

  int setup() override {
    const size_t fe = field_elems();
    if (p.advection && !QC::fits(kPencilStokes)) {
      err = "Stokes advection is not built for this size and precision (its pencil pass does not fit a CTA)";
      return SH_EUNSUPPORTED;
    }
    SHB_CUDA(dev_malloc(&W, fe * sizeof(cplx<T>)));
    SHB_CUDA(dev_malloc(&P, fe * sizeof(cplx<T>)));
    SHB_CUDA(dev_malloc(&Nt, fe * sizeof(cplx<T>)));
    if (p.advection) {
      // periodic: partials of psi, i q_x psi and opSH psi; Neumann: of psi and
      // opSH psi (its gradient is a difference stencil in real space)
      if (DCT && p.sub_sigma != 0.0) {
        err = "advection and the substrate penalty are not combined";
        return SH_EUNSUPPORTED;
      }
      if (!DCT) SHB_CUDA(dev_malloc(&Px, fe * sizeof(cplx<T>)));
      SHB_CUDA(dev_malloc(&PSH, fe * sizeof(cplx<T>)));
      for (auto& p3 : S3) SHB_CUDA(dev_malloc(&p3, fe * sizeof(cplx<T>)));
      for (auto& r : R) SHB_CUDA(dev_malloc(&r, size_t(p.batch) * N * N * N * sizeof(T)));
    }
    if (p.sub_sigma != 0.0) {
      if constexpr (!DCT) {
        err = "the substrate penalty is defined for the Neumann boundary only";
        return SH_EINVAL;
      } else {
        // wall(z) = sigma exp(-z / z0) (cosFFT/comet/cosNoAdvMorph.cpp:67-74), kept on the planes
        // where it is at least 1e-30 |sigma|; below that its term is under the FP64 rounding of N
        std::vector<T> hw;
        for (int k = 0; k < N; ++k) {
          const double w = p.sub_sigma * std::exp(-double(k) / p.sub_z0);
          if (std::fabs(w) < 1e-30 * std::fabs(p.sub_sigma)) break;
          hw.push_back(T(w));
        }
        kwall = int(hw.size());
        SHB_CUDA(dev_malloc(&Pxx, fe * sizeof(cplx<T>)));
        SHB_CUDA(dev_malloc(&Lp, size_t(p.batch) * N * N * kwall * sizeof(T)));
        SHB_CUDA(dev_malloc(&d_wall, kwall * sizeof(T)));
        SHB_CUDA(cudaMemcpy(d_wall, hw.data(), kwall * sizeof(T), cudaMemcpyHostToDevice));
      }
    }
    SHB_CUDA(dev_malloc(&tw, tw_total<N>() * sizeof(cplx<T>)));
    SHB_CUDA(dev_malloc(&q, N * sizeof(T)));
    SHB_CUDA(dev_malloc(&qd, N * sizeof(double)));
    SHB_CUDA(dev_malloc(&d_red_plane, size_t(p.batch) * N * CL * 3 * sizeof(double)));
    SHB_CUDA(dev_malloc(&d_red_spec, size_t(p.batch) * QC::TILES * sizeof(double)));
    std::vector<cplx<T>> htw;
    host_twiddles<T, N>(htw);
    std::vector<T> hq(N);
    std::vector<double> hqd(N);
    if (!DCT) {
      // periodicFFT/pf3d.cpp:166-190 (Nyquist entry +pi/dx)
      for (int i = 0; i < N; ++i)
        hqd[i] = i < N / 2 + 1 ? 2.0 * M_PI * i / (p.dx * N) : -(N - i) * 2.0 * M_PI / (p.dx * N);
    } else {
      // cosFFT/mesabi/cosNoAdvMorph.cpp:216-231
      for (int i = 0; i < N; ++i) hqd[i] = M_PI * i / (p.dx * N);
    }
    for (int i = 0; i < N; ++i) hq[i] = T(hqd[i]);
    SHB_CUDA(cudaMemcpy(qd, hqd.data(), N * sizeof(double), cudaMemcpyHostToDevice));
    SHB_CUDA(cudaMemcpy(tw, htw.data(), htw.size() * sizeof(cplx<T>), cudaMemcpyHostToDevice));
    SHB_CUDA(cudaMemcpy(q, hq.data(), N * sizeof(T), cudaMemcpyHostToDevice));
    int rc;
    if ((rc = set_attrs(plane_fn<kPlaneStep>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneInit>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneGetPsi>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneInvReal>(), PC::SMEM, true))) return rc;
    if ((rc = set_pencil_attrs<kPencilStep>())) return rc;
    if ((rc = set_pencil_attrs<kPencilStepU64>())) return rc;
    if ((rc = set_pencil_attrs<kPencilInit>())) return rc;
    if ((rc = set_pencil_attrs<kPencilEnergy>())) return rc;
    if ((rc = set_pencil_attrs<kPencilStepAdv>())) return rc;
    if ((rc = set_pencil_attrs<kPencilInitAdv>())) return rc;
    if ((rc = set_pencil_attrs<kPencilStokes>())) return rc;
    if ((rc = set_pencil_attrs<kPencilXMul>())) return rc;
    if ((rc = set_pencil_attrs<kPencilSpec>())) return rc;
    if ((rc = set_pencil_attrs<kPencilAdjInit>())) return rc;
    if ((rc = set_pencil_attrs<kPencilAdj>())) return rc;
    if ((rc = set_pencil_attrs<kPencilAdjOut>())) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneAdj>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneInvMulFwd>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneAdvN>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneMulFwd>(), PC::SMEM, true))) return rc;
    return SH_OK;
  }

  template <int MODE>
  int launch_plane(const PlaneArgs<T>& a, int reps = 0) {
    return launch_plane_sets<MODE>(&a, 1, reps);
  }
  // ``ncomp`` argument sets in one grid (blockIdx.z), for the modes that take several
  template <int MODE>
  int launch_plane_sets(const PlaneArgs<T>* as, int ncomp, int reps = 0) {
    if (ncomp < 1 || ncomp > kPlaneComps || (ncomp > 1 && !plane_multi(MODE))) {
      err = "plane pass: unsupported number of argument sets";
      return SH_EINVAL;
    }
    PlaneLaunch<T> pl{};
    for (int i = 0; i < ncomp; ++i) pl.c[i] = as[i];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(N * CL, reps > 0 ? reps : p.batch, ncomp);
    cfg.blockDim = dim3(PC::THREADS, 1, 1);
    cfg.dynamicSmemBytes = PC::SMEM;
    cfg.stream = stream;
    cudaLaunchAttribute attr[2];
    unsigned na = 0;
    if (CL > 1) {
      attr[na].id = cudaLaunchAttributeClusterDimension;
      attr[na].val.clusterDim.x = CL;
      attr[na].val.clusterDim.y = 1;
      attr[na].val.clusterDim.z = 1;
      ++na;
    }
    if (use_pdl) {
      attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[na].val.programmaticStreamSerializationAllowed = 1;
      ++na;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    SHB_CUDA(cudaLaunchKernelEx(&cfg, plane_fn<MODE>(), pl));
    ++launches;
    return SH_OK;
  }

  template <int MODE>
  int launch_pencil(const PencilArgs<T>& a, int reps = 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(QC::TILES, reps > 0 ? reps : p.batch, 1);
    cfg.blockDim = dim3(QC::THREADS, 1, 1);
    cfg.dynamicSmemBytes = QC::smem(MODE);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = use_pdl ? 1 : 0;
    SHB_CUDA(cudaLaunchKernelEx(&cfg, pencil_fn<MODE>(), a));
    ++launches;
    return SH_OK;
  }

  // CTAs per SM of the step kernels and, for the clustered plane pass, the
  // clusters the GPU holds at once (its GPCs place whole clusters only)
  int residency(int* out) override {
    int dev = 0, sms = 0, pb = 0, qb = 0, nc = 0;
    SHB_CUDA(cudaGetDevice(&dev));
    SHB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SHB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pb, plane_fn<kPlaneStep>(), PC::THREADS, PC::SMEM));
    SHB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&qb, pencil_fn<kPencilStep>(), QC::THREADS,
                                                           QC::smem(kPencilStep)));
    if (CL > 1) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(N * CL, p.batch, 1);
      cfg.blockDim = dim3(PC::THREADS, 1, 1);
      cfg.dynamicSmemBytes = PC::SMEM;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = CL;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      SHB_CUDA(cudaOccupancyMaxActiveClusters(&nc, plane_fn<kPlaneStep>(), &cfg));
    } else {
      nc = pb * sms;
    }
    out[0] = pb;
    out[1] = nc;
    out[2] = CL;
    out[3] = N * CL * p.batch;
    out[4] = qb;
    out[5] = QC::TILES * p.batch;
    out[6] = sms;
    return SH_OK;
  }

#ifndef SHB_PLANE_PF
#define SHB_PLANE_PF 16
#endif
  PlaneArgs<T> plane_args() const {
    PlaneArgs<T> a{};
    // clustered plane passes run in several waves: prefetch a later wave's planes
    a.pf_dist = CL > 1 ? SHB_PLANE_PF : 0;
    a.tw = tw;
    a.pp = point_params();
    a.red = d_red_plane;
    a.timeout = d_flag + 1;
    a.drop_exchange = drop_exchange;
    a.q = q;
    return a;
  }
  PencilArgs<T> pencil_args() const {
    PencilArgs<T> a{};
    a.tw = tw;
    a.q = q;
    a.qd = qd;
    a.pp = point_params();
    a.red = d_red_spec;
    a.nonfinite = d_flag;
    return a;
  }

  int finalize(int what, double* out) {
    const double dv = p.dx * p.dx * p.dx;
    const double norm = DCT ? 1.0 / (8.0 * double(N) * N * N) : 1.0 / (double(N) * N * N);
    finalize_kernel<<<p.batch, 256, 0, stream>>>(d_red_plane, N * CL, d_red_spec, QC::TILES, what, dv, norm,
                                                  p.alpha, p.dt, out);
    SHB_CUDA(cudaGetLastError());
    ++launches;
    return SH_OK;
  }

  // In-plane Laplacian of the current psi on the substrate planes:
  // Lp = IDCT_yz(partial of -q_x^2 scale psihat  -  q_y^2 x partial of scale psihat)
  int substrate_lperp() {
    PlaneArgs<T> a = plane_args();
    a.src = Pxx;
    a.src2 = P;
    a.mult2 = kMulNegQy2;
    a.real_out = Lp;
    a.real_zn = kwall;
    return launch_plane<kPlaneInvReal>(a);
  }
  PlaneArgs<T> plane_args_step() const {
    PlaneArgs<T> a = plane_args();
    a.wall = d_wall;
    a.lperp = Lp;
    a.kwall = kwall;
    return a;
  }

  int init_from_psi() override {
    int rc;
    adj_end = -1;
    PlaneArgs<T> a = plane_args();
    a.psi_in = d_psi;
    a.dst2 = P;   // partial of psi^0 (consumed by the init pencil, then overwritten)
    a.dst = Nt;   // partial of N(psi^0): the first Nhat (Euler start)
    PencilArgs<T> b = pencil_args();
    b.src = P;
    b.src2 = Nt;
    b.w = W;
    b.dst = P;
    if (kwall > 0) {
      // N(psi^0) carries the substrate term of psi^0 (cosFFT/comet/cosNoAdvMorph.cpp:486-529):
      // a first pass yields psi^0's partials, hence its in-plane Laplacian; the second
      // pass builds N-hat^{-1} and W^0 with it
      if ((rc = launch_plane<kPlaneInit>(a))) return rc;
      b.dst_x = Pxx;
      if ((rc = launch_pencil<kPencilInitAdv>(b))) return rc;
      if ((rc = substrate_lperp())) return rc;
      a = plane_args_step();
      a.psi_in = d_psi;
      a.dst2 = P;
      a.dst = Nt;
      if ((rc = launch_plane<kPlaneInit>(a))) return rc;
      if ((rc = launch_pencil<kPencilInitAdv>(b))) return rc;
    } else {
      if ((rc = launch_plane<kPlaneInit>(a))) return rc;
      if (p.advection) {
        b.dst_x = DCT ? nullptr : Px;
        b.dst_sh = PSH;
        if ((rc = launch_pencil<kPencilInitAdv>(b))) return rc;
        // the first advected N (N-hat^{-1} above discards advection, pf3d.cpp:363-374,
        // cosFFT/comet/morphSurfK.cpp:629-636)
        if ((rc = adv_nonlinear(0))) return rc;
      } else {
        if ((rc = launch_pencil<kPencilInit>(b))) return rc;
      }
    }
    if (p.l1_interval > 0)
      SHB_CUDA(cudaMemcpyAsync(d_stash, d_psi, size_t(p.batch) * n3() * sizeof(double), cudaMemcpyDeviceToDevice,
                               stream));
    steps = 0;
    psi0_valid = true;
    l1_count = 0;
    energy_trace.clear();
    ready = true;
    return SH_OK;
  }

  // plain steps are replayed from a CUDA graph when no per-step host
  // bookkeeping is needed (with the L1 monitor on: between its steps)
  bool graph_eligible() const {
    return use_graphs && !prof_ms && !hist_spec && !p.energy_trace && (p.l1_interval == 0 || !blocked());
  }
  // with the L1 monitor on, a replayed chunk of kGraphChunk steps after step
  // count s0 must hold neither a monitored step (count % l1_interval == 0) nor the
  // step before one, which keeps psi for the difference
  bool chunk_unmonitored(long long s0) const {
    const int li = p.l1_interval;
    if (li <= 0) return true;
    for (long long c = s0 + 1; c <= s0 + kGraphChunk; ++c)
      if (c % li == 0 || (c + 1) % li == 0) return false;
    return true;
  }
  // Replica blocks (batched plain steps, replica_block = g > 0): the graph
  // advances replicas [0, g) by kGraphChunk steps, then [g, 2g), and so on, so
  // a block's W, P and N-hat (3 fields per replica) stay in L2 across its steps
  // and the passes read and write L2 instead of HBM
  bool blocked() const {
    return p.replica_block > 0 && p.replica_block < p.batch && !p.advection && kwall == 0;
  }
  // n plain steps of replicas [r0, r0 + g) only: every per-replica pointer of the
  // two passes is offset to the block (no diagnostics, no history)
  int step_window(int r0, int g, int n) {
    int rc;
    const size_t off = size_t(r0) * N * FP;
    for (int s = 0; s < n; ++s) {
      PencilArgs<T> b = pencil_args();
      b.src = Nt + off;
      b.w = W + off;
      b.dst = P + off;
      b.pp.eps = d_eps + r0;
      if ((rc = launch_pencil_step(b, g))) return rc;
      PlaneArgs<T> a = plane_args_step();
      a.src = P + off;
      a.dst = Nt + off;
      a.pp.eps = d_eps + r0;
      if ((rc = launch_plane<kPlaneStep>(a, g))) return rc;
    }
    return SH_OK;
  }

  // capture kGraphChunk steps once (nothing runs; the steps counter is restored)
  int build_graph() override {
    if (graph_exec || !graph_eligible()) return SH_OK;
    cudaGraph_t g;
    const long long s0 = steps, l0 = launches;
    // the graph holds plain steps only: the L1 monitor's steps run outside it
    const int li = p.l1_interval;
    p.l1_interval = 0;
    SHB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int rc = SH_OK;
    if (blocked()) {
      for (int r0 = 0; r0 < p.batch && !rc; r0 += p.replica_block) {
        const int gsz = r0 + p.replica_block <= p.batch ? p.replica_block : p.batch - r0;
        rc = step_window(r0, gsz, kGraphChunk);
      }
      steps += kGraphChunk;
      hist_pos += kGraphChunk;
    } else {
      rc = step_direct(kGraphChunk);
    }
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    p.l1_interval = li;
    steps = s0;
    hist_pos -= kGraphChunk;
    graph_launches = launches - l0;
    launches = l0;
    if (rc) return rc;
    SHB_CUDA(e);
    e = cudaGraphInstantiate(&graph_exec, g, 0);
    cudaGraphDestroy(g);
    SHB_CUDA(e);
    return SH_OK;
  }

  int step_async(int n) override {
    if (graph_eligible() && n >= kGraphChunk) {
      int rc;
      if ((rc = build_graph())) return rc;
      if (p.l1_interval <= 0) {
        const int chunks = n / kGraphChunk;
        for (int c = 0; c < chunks; ++c) {
          SHB_CUDA(cudaGraphLaunch(graph_exec, stream));
          steps += kGraphChunk;
          launches += graph_launches;
        }
        return step_direct(n - chunks * kGraphChunk);
      }
      // L1 monitor on (the reference's loop): replay the graph over the chunks
      // that hold no monitored step, take the steps around each one directly
      while (n > 0) {
        if (n >= kGraphChunk && chunk_unmonitored(steps)) {
          SHB_CUDA(cudaGraphLaunch(graph_exec, stream));
          steps += kGraphChunk;
          launches += graph_launches;
          n -= kGraphChunk;
        } else {
          if ((rc = step_direct(1))) return rc;
          --n;
        }
      }
      return SH_OK;
    }
    return step_direct(n);
  }
  long long graph_launches = 0;

  int step_direct(int n) {
    int rc;
    const bool trace = p.energy_trace != 0;
    if (trace && n > trace_cap) {
      cudaFree(d_trace);
      d_trace = nullptr;
      SHB_CUDA(dev_malloc(&d_trace, size_t(n) * p.batch * sizeof(double)));
      trace_cap = n;
    }
    for (int s = 0; s < n; ++s) {
      const long long count = steps + 1;  // index of the state this step produces
      const int li = p.l1_interval;
      const bool l1_now = li > 0 && count % li == 0;
      const bool stash_now = li > 0 && (count + 1) % li == 0;
      PencilArgs<T> b = pencil_args();
      b.src = Nt;
      b.w = W;
      b.dst = P;
      b.flags = trace ? kFlEnergy : 0;
      if (hist_spec) {  // adjoint recompute: keep psihat^{n+1}
        b.flags |= kFlSpecOut;
        b.spec_out = hist_spec + size_t(hist_pos + 1) * field_elems();
      }
      if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[0], stream));
      const int diag = (trace ? kFlEnergy : 0) | (l1_now ? kFlL1 : 0) | (stash_now ? kFlPsiOut : 0);
      if (p.advection) {
        b.dst_x = DCT ? nullptr : Px;
        b.dst_sh = PSH;
        if ((rc = launch_pencil<kPencilStepAdv>(b))) return rc;
        if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[1], stream));
        if ((rc = adv_nonlinear(diag))) return rc;
      } else {
        if (kwall > 0) {  // Neumann substrate: also the -q_x^2 partial, then the in-plane Laplacian
          b.dst_x = Pxx;
          if ((rc = launch_pencil<kPencilStepAdv>(b))) return rc;
          if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[1], stream));
          if ((rc = substrate_lperp())) return rc;
        } else {
          if ((rc = launch_pencil_step(b))) return rc;
          if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[1], stream));
        }
        PlaneArgs<T> a = plane_args_step();
        a.src = P;
        a.dst = Nt;
        a.flags = diag;
        a.psi_old = d_stash;
        a.psi_out = d_stash;
        if (hist_real) {  // adjoint recompute: keep psi^{n+1}
          a.flags |= kFlRealOut;
          a.real_out = hist_real + size_t(hist_pos + 1) * size_t(p.batch) * N * N * N;
        }
        if ((rc = launch_plane<kPlaneStep>(a))) return rc;
      }
      if (prof_ms) {
        float t0, t1;
        SHB_CUDA(cudaEventRecord(prof_ev[2], stream));
        SHB_CUDA(cudaEventSynchronize(prof_ev[2]));
        SHB_CUDA(cudaEventElapsedTime(&t0, prof_ev[0], prof_ev[1]));
        SHB_CUDA(cudaEventElapsedTime(&t1, prof_ev[1], prof_ev[2]));
        prof_ms[0] += t0;
        prof_ms[1] += t1;
      }
      if (trace && (rc = finalize(0, d_trace + size_t(s) * p.batch))) return rc;
      if (l1_now) {
        if ((rc = finalize(1, d_scalar))) return rc;
        ++l1_count;
      }
      ++steps;
      ++hist_pos;
    }
    return SH_OK;
  }

  // Nonlinear term with Stokes advection of the state held in P, Px, PSH
  // (periodicFFT/pf3d.cpp:397-465): psi, grad psi and L psi in real space,
  // stress S = (L psi) grad psi, Stokes velocity u, then
  // N = beta psi^3 - gamma psi^5 (+ penalty) - u.grad psi, forward y,z -> Nt.
  int adv_nonlinear(int diag) {
    if constexpr (DCT) {
      // Neumann box (cosFFT/comet/morphSurfK.cpp:686-898): psi and L psi to real
      // space, grad psi by the wall stencil, S_c = (L psi) d_c psi through the
      // sine transform (signed cosine pair), the projector in the pencil pass,
      // then N = beta psi^3 - gamma psi^5 - u . grad psi forward -> Nt
      int rc;
      if ((rc = psi_lpsi_real(diag))) return rc;
      grad_wall_kernel<T><<<dim3(4 * 148, p.batch), 256, 0, stream>>>(R[0], R[1], R[2], R[3], N,
                                                                        T(0.5 / p.dx));
      SHB_CUDA(cudaGetLastError());
      ++launches;
      PlaneArgs<T> st[3];
      for (int c = 0; c < 3; ++c) {
        st[c] = plane_args();
        st[c].real_in[0] = R[4];
        st[c].real_in[1] = R[1 + c];
        st[c].sign_axes = 7;
        st[c].dst = S3[c];
      }
      if ((rc = launch_plane_sets<kPlaneMulFwd>(st, 3))) return rc;
      PencilArgs<T> b = pencil_args();
      for (int c = 0; c < 3; ++c) {
        b.s3[c] = S3[c];
        b.u3[c] = S3[c];
      }
      if ((rc = launch_pencil<kPencilStokes>(b))) return rc;
      PlaneArgs<T> a = plane_args();
      for (int i = 0; i < 4; ++i) a.real_in[i] = R[i];
      for (int c = 0; c < 3; ++c) a.src3[c] = S3[c];
      a.sign_axes = 7;
      a.dst = Nt;
      if ((rc = launch_plane<kPlaneAdvN>(a))) return rc;
      real_fields_current = true;
      u_real_current = false;
      return SH_OK;
    } else {
      int rc;
      if ((rc = psi_lpsi_real(diag))) return rc;
      // grad psi to real space, and in the same pass the stress S_c = (L psi) d_c psi forward
      const cplx<T>* dsrc[3] = {Px, P, P};
      const int dmult[3] = {kMulNone, kMulIqy, kMulIqz};
      PlaneArgs<T> st[3];
      for (int c = 0; c < 3; ++c) {
        st[c] = plane_args();
        st[c].src = dsrc[c];
        st[c].mult = dmult[c];
        st[c].real_out = R[1 + c];
        st[c].real_in[0] = R[4];
        st[c].dst = S3[c];
      }
      if ((rc = launch_plane_sets<kPlaneInvMulFwd>(st, 3))) return rc;
      PencilArgs<T> b = pencil_args();
      for (int c = 0; c < 3; ++c) {
        b.s3[c] = S3[c];
        b.u3[c] = S3[c];
      }
      if ((rc = launch_pencil<kPencilStokes>(b))) return rc;
      // N = beta psi^3 - gamma psi^5 - u . grad psi, the velocity inverted inside the pass
      PlaneArgs<T> a = plane_args();
      for (int i = 0; i < 4; ++i) a.real_in[i] = R[i];
      for (int c = 0; c < 3; ++c) a.src3[c] = S3[c];
      a.dst = Nt;
      if ((rc = launch_plane<kPlaneAdvN>(a))) return rc;
      real_fields_current = true;
      u_real_current = false;  // the velocity stays spectral (S3) unless a surface pass needs it
      return SH_OK;
    }
  }
  // psi and L psi of the state held in P, PSH to real space (R[0], R[4]), one
  // grid; the diagnostics ``diag`` (L1 monitor, psi stash) ride on psi
  int psi_lpsi_real(int diag) {
    PlaneArgs<T> st[2] = {plane_args(), plane_args()};
    st[0].src = P;
    st[0].real_out = R[0];
    st[0].flags = diag;
    st[0].psi_old = d_stash;
    st[0].psi_out = d_stash;
    st[1].src = PSH;
    st[1].real_out = R[4];
    return launch_plane_sets<kPlaneInvReal>(st, 2);
  }
  // velocity of the current state in real space (R[5..7]) from its partials in S3
  int velocity_real() {
    int rc;
    PlaneArgs<T> st[3];
    for (int c = 0; c < 3; ++c) {
      st[c] = plane_args();
      st[c].src = S3[c];
      st[c].real_out = R[5 + c];
      st[c].sign_axes = DCT ? 7 : 0;  // Neumann: the partials carry (-1)^(x+y+z) u
    }
    if ((rc = launch_plane_sets<kPlaneInvReal>(st, 3))) return rc;
    u_real_current = true;
    return SH_OK;
  }

  // Stokes velocity of the current state in FP64 (batch * N^3 per component)
  int velocity(double* ux, double* uy, double* uz) override {
    if (!p.advection) {
      err = "the velocity is computed by advected handles (advection = 1)";
      return SH_EINVAL;
    }
    int rc;
    if (!real_fields_current && (rc = adv_nonlinear(0))) return rc;
    if (!u_real_current && (rc = velocity_real())) return rc;
    const size_t nr = size_t(p.batch) * N * N * N;
    double* outs[3] = {ux, uy, uz};
    for (int c = 0; c < 3; ++c) {
      to_double_kernel<T><<<4 * 148, 256, 0, stream>>>(R[5 + c], d_psi, (long long)nr);
      SHB_CUDA(cudaGetLastError());
      ++launches;
      SHB_CUDA(cudaMemcpyAsync(outs[c], d_psi, nr * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaStreamSynchronize(stream));
    }
    psi0_valid = false;  // d_psi was used as scratch
    return SH_OK;
  }

  int psi_to_dpsi() override {
    if (steps == 0 && psi0_valid) return SH_OK;  // d_psi still holds the uploaded psi^0
    psi0_valid = false;
    return plane_getpsi(true, false);
  }

  int plane_getpsi(bool write_psi, bool energy) {
    PlaneArgs<T> a = plane_args();
    a.src = P;
    a.psi_out = d_psi;
    a.flags = (write_psi ? kFlPsiOut : 0) | (energy ? kFlEnergy : 0);
    return launch_plane<kPlaneGetPsi>(a);
  }

  int energy_now(double* host) override {
    int rc;
    if ((rc = plane_getpsi(false, true))) return rc;
    PencilArgs<T> b = pencil_args();
    b.src = P;
    b.flags = kFlEnergy;
    if ((rc = launch_pencil<kPencilEnergy>(b))) return rc;
    if ((rc = finalize(0, d_scalar))) return rc;
    SHB_CUDA(cudaMemcpyAsync(host, d_scalar, p.batch * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaStreamSynchronize(stream));
    return SH_OK;
  }

  // |q| of the shell holding the most spectral power of the current state,
  // DC excluded (the dominant layer wavenumber): one pencil pass over the
  // partial P that builds the per-shell power in FP64, then an argmax per replica
  int dominant_wavenumber(double* host) override {
    int rc;
    const size_t nb = size_t(p.batch) * QC::NSHELL;
    if (!d_shell) SHB_CUDA(dev_malloc(&d_shell, nb * sizeof(double)));
    SHB_CUDA(cudaMemsetAsync(d_shell, 0, nb * sizeof(double), stream));
    PencilArgs<T> b = pencil_args();
    b.src = P;
    b.flags = kFlShell;
    b.shell = d_shell;
    if ((rc = launch_pencil<kPencilEnergy>(b))) return rc;
    const double dq = (DCT ? M_PI : 2.0 * M_PI) / (double(N) * p.dx);
    shell_argmax_kernel<<<p.batch, 256, 0, stream>>>(d_shell, QC::NSHELL, dq, d_scalar);
    SHB_CUDA(cudaGetLastError());
    ++launches;
    SHB_CUDA(cudaMemcpyAsync(host, d_scalar, p.batch * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaStreamSynchronize(stream));
    return SH_OK;
  }

  size_t state_bytes() const override { return (p.advection ? 5 : 3) * field_elems() * sizeof(cplx<T>); }
  int save_state(void* host) override {
    const size_t fb = field_elems() * sizeof(cplx<T>);
    char* h = static_cast<char*>(host);
    SHB_CUDA(cudaMemcpyAsync(h, W, fb, cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaMemcpyAsync(h + fb, P, fb, cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaMemcpyAsync(h + 2 * fb, Nt, fb, cudaMemcpyDeviceToHost, stream));
    if (p.advection) {
      SHB_CUDA(cudaMemcpyAsync(h + 3 * fb, Px, fb, cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(h + 4 * fb, PSH, fb, cudaMemcpyDeviceToHost, stream));
    }
    SHB_CUDA(cudaStreamSynchronize(stream));
    return SH_OK;
  }
  int load_state(const void* host) override {
    adj_end = -1;
    const size_t fb = field_elems() * sizeof(cplx<T>);
    const char* h = static_cast<const char*>(host);
    SHB_CUDA(cudaMemcpyAsync(W, h, fb, cudaMemcpyHostToDevice, stream));
    SHB_CUDA(cudaMemcpyAsync(P, h + fb, fb, cudaMemcpyHostToDevice, stream));
    SHB_CUDA(cudaMemcpyAsync(Nt, h + 2 * fb, fb, cudaMemcpyHostToDevice, stream));
    if (p.advection) {
      SHB_CUDA(cudaMemcpyAsync(Px, h + 3 * fb, fb, cudaMemcpyHostToDevice, stream));
      SHB_CUDA(cudaMemcpyAsync(PSH, h + 4 * fb, fb, cudaMemcpyHostToDevice, stream));
    }
    SHB_CUDA(cudaStreamSynchronize(stream));
    ready = true;
    psi0_valid = false;
    real_fields_current = false;
    return SH_OK;
  }

  // Discrete adjoint of the plain periodic CNAB2 loop (reverse sweep
  // lambda^n = A lambda^{n+1} + N'(psi^n)(c_n B lambda^{n+1} - B lambda^{n+2}),
  // c_n = 3, c_0 = 2) for a loss whose gradient with respect to psi^T is
  // dl_dpsi_t.  The forward states are checkpointed every ckpt_every steps and
  // recomputed segment by segment; the (eps, q0) gradients accumulate in FP64.
  // the adjoint covers the plain periodic CNAB2 step
  int adjoint_supported() {
    if constexpr (DCT) {
      err = "the adjoint is built for the periodic boundary";
      return SH_EUNSUPPORTED;
    } else {
      if (p.advection || p.scheme != kCNAB2 || p.w_mid != 0.0) {
        err = "the adjoint covers the plain CNAB2 step without advection or penalty";
        return SH_EUNSUPPORTED;
      }
      return SH_OK;
    }
  }

#define ADJ_CUDA(expr)                                                           \
  do {                                                                           \
    cudaError_t e_ = (expr);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      err = std::string(#expr) + ": " + cudaGetErrorString(e_);                  \
      restore();                                                                 \
      return e_ == cudaErrorMemoryAllocation ? SH_ENOMEM : SH_ECUDA;             \
    }                                                                            \
  } while (0)
#define ADJ_RC(expr)       \
  do {                     \
    if ((rc = (expr))) {   \
      restore();           \
      return rc;           \
    }                      \
  } while (0)

  // Forward sweep of the discrete adjoint: psi0 from the host, nsteps plain
  // steps, a checkpoint (W, P, Nt) at s = 0, K, 2K, ...  The handle then holds
  // psi^T as after sh_run, and adjoint_backward can use the checkpoints.
  int adjoint_forward(const double* psi0, int nsteps, int K) override {
    int rc;
    if ((rc = adjoint_supported())) return rc;
    if (nsteps < 1 || K < 1) {
      err = "nsteps and ckpt_every must be >= 1";
      return SH_EINVAL;
    }
    const size_t fe = field_elems();
    const size_t nr = size_t(p.batch) * N * N * N;
    const int nseg = (nsteps + K - 1) / K;
    const bool saved_trace = p.energy_trace != 0;
    const int saved_l1 = p.l1_interval;
    p.energy_trace = 0;
    p.l1_interval = 0;
    AdjBufs& bf = adj;
    auto restore = [&]() { p.energy_trace = saved_trace; p.l1_interval = saved_l1; };
    // buffers persist across calls; they grow when nsteps / ckpt_every need more
    if (bf.nseg < nseg) {
      cudaFree(bf.ck);
      bf.ck = nullptr;
      bf.nseg = 0;
      ADJ_CUDA(dev_malloc(&bf.ck, size_t(nseg) * 3 * fe * sizeof(cplx<T>)));
      bf.nseg = nseg;
    }
    if (bf.k < K) {
      cudaFree(bf.hs);
      cudaFree(bf.hr);
      bf.hs = nullptr;
      bf.hr = nullptr;
      bf.k = 0;
      ADJ_CUDA(dev_malloc(&bf.hs, size_t(K + 1) * fe * sizeof(cplx<T>)));
      ADJ_CUDA(dev_malloc(&bf.hr, size_t(K + 1) * nr * sizeof(T)));
      bf.k = K;
    }
    const size_t fb = fe * sizeof(cplx<T>);
    ADJ_CUDA(cudaMemcpyAsync(d_psi, psi0, nr * sizeof(double), cudaMemcpyHostToDevice, stream));
    ADJ_RC(init_from_psi());
    for (int sg = 0; sg < nseg; ++sg) {
      cplx<T>* c = bf.ck + size_t(sg) * 3 * fe;
      ADJ_CUDA(cudaMemcpyAsync(c, W, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(c + fe, P, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(c + 2 * fe, Nt, fb, cudaMemcpyDeviceToDevice, stream));
      const int s1 = (sg + 1) * K < nsteps ? (sg + 1) * K : nsteps;
      if (sg == nseg - 1) {
        // the last segment keeps its states (psihat^n pencil-major, psi^n real) as
        // the reverse sweep needs them, so the backward does not recompute it
        PencilArgs<T> b = pencil_args();
        b.src = P;
        b.spec_out = bf.hs;
        ADJ_RC(launch_pencil<kPencilSpec>(b));
        PlaneArgs<T> a = plane_args();
        a.src = P;
        a.real_out = bf.hr;
        ADJ_RC(launch_plane<kPlaneInvReal>(a));
        hist_spec = bf.hs;
        hist_real = bf.hr;
        hist_pos = 0;
        rc = step_async(s1 - sg * K);
        hist_spec = nullptr;
        hist_real = nullptr;
        ADJ_RC(rc);
      } else {
        ADJ_RC(step_async(s1 - sg * K));
      }
    }
    restore();
    psi0_valid = false;
    adj_nsteps = nsteps;
    adj_k = K;
    adj_end = steps;
    adj_last_hist = true;
    return SH_OK;
  }

  // Reverse sweep from the checkpoints of the last adjoint_forward (the
  // handle must still hold the state that sweep ended in): lambda^T from
  // dl_dpsi_t, then per segment in reverse the recomputed states and the
  // adjoint steps.  Leaves the handle's state at psi^T.
  int adjoint_backward(const double* dl_dpsi_t, double* g_eps, double* g_q0, double* g_psi0) override {
    if constexpr (DCT) {
      return adjoint_supported();
    } else {
      int rc;
      if ((rc = adjoint_supported())) return rc;
      if (adj_end < 0 || adj_end != steps) {
        err = "no forward sweep with checkpoints ends at the current state (call sh_adjoint_forward first)";
        return SH_ESTATE;
      }
      const int nsteps = adj_nsteps, K = adj_k;
      const size_t fe = field_elems();
      const size_t nr = size_t(p.batch) * N * N * N;
      const int nseg = (nsteps + K - 1) / K;
      const bool saved_trace = p.energy_trace != 0;
      const int saved_l1 = p.l1_interval;
      p.energy_trace = 0;
      p.l1_interval = 0;
      AdjBufs& bf = adj;
      // the state at psi^T, restored at the end: the last checkpoint's segment is recomputed over it
      auto restore = [&]() { p.energy_trace = saved_trace; p.l1_interval = saved_l1; hist_spec = nullptr; hist_real = nullptr; };
      if (bf.k < K) {
        cudaFree(bf.hs);
        cudaFree(bf.hr);
        bf.hs = nullptr;
        bf.hr = nullptr;
        bf.k = 0;
        ADJ_CUDA(dev_malloc(&bf.hs, size_t(K + 1) * fe * sizeof(cplx<T>)));
        ADJ_CUDA(dev_malloc(&bf.hr, size_t(K + 1) * nr * sizeof(T)));
        bf.k = K;
      }
      if (!bf.lam) {
        ADJ_CUDA(dev_malloc(&bf.lam, fe * sizeof(cplx<T>)));
        ADJ_CUDA(dev_malloc(&bf.gp, fe * sizeof(cplx<T>)));
        ADJ_CUDA(dev_malloc(&bf.mp, fe * sizeof(cplx<T>)));
        ADJ_CUDA(dev_malloc(&bf.red, size_t(p.batch) * QC::TILES * 2 * sizeof(double)));
        ADJ_CUDA(dev_malloc(&bf.acc, size_t(p.batch) * 4 * sizeof(double)));
        ADJ_CUDA(dev_malloc(&bf.fin, 3 * fe * sizeof(cplx<T>)));
      }
      ADJ_CUDA(cudaMemsetAsync(bf.red, 0, size_t(p.batch) * QC::TILES * 2 * sizeof(double), stream));
      const size_t fb = fe * sizeof(cplx<T>);
      const long long end_steps = steps;
      // keep the final state (the recompute overwrites W, P, Nt)
      ADJ_CUDA(cudaMemcpyAsync(bf.fin, W, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(bf.fin + fe, P, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(bf.fin + 2 * fe, Nt, fb, cudaMemcpyDeviceToDevice, stream));
      // ---- lambda^T -> lambdahat^T and the partial of mu^T = B lambda^T
      ADJ_CUDA(cudaMemcpyAsync(d_psi, dl_dpsi_t, nr * sizeof(double), cudaMemcpyHostToDevice, stream));
      {
        PlaneArgs<T> a = plane_args();
        a.psi_in = d_psi;
        a.dst2 = bf.gp;   // partial of lambda^T
        a.dst = bf.mp;    // (the N of lambda^T, unused scratch)
        ADJ_RC(launch_plane<kPlaneInit>(a));
        PencilArgs<T> b = pencil_args();
        b.src = bf.gp;
        b.w = bf.lam;
        b.dst = bf.mp;  // partial of c_{T-1} mu^T
        b.coef = nsteps - 1 >= 1 ? 3.0 : 2.0;
        ADJ_RC(launch_pencil<kPencilAdjInit>(b));
      }
      // ---- reverse sweep, one recomputed segment at a time
      for (int sg = nseg - 1; sg >= 0; --sg) {
        const int s0 = sg * K;
        const int s1 = (sg + 1) * K < nsteps ? (sg + 1) * K : nsteps;
        if (!(sg == nseg - 1 && adj_last_hist)) {  // the forward sweep kept the last segment's states
          adj_last_hist = false;                    // this recompute overwrites them
          const cplx<T>* c = bf.ck + size_t(sg) * 3 * fe;
          ADJ_CUDA(cudaMemcpyAsync(W, c, fb, cudaMemcpyDeviceToDevice, stream));
          ADJ_CUDA(cudaMemcpyAsync(P, c + fe, fb, cudaMemcpyDeviceToDevice, stream));
          ADJ_CUDA(cudaMemcpyAsync(Nt, c + 2 * fe, fb, cudaMemcpyDeviceToDevice, stream));
          {  // psihat^{s0} and psi^{s0} of the segment's first state
            PencilArgs<T> b = pencil_args();
            b.src = P;
            b.spec_out = bf.hs;
            ADJ_RC(launch_pencil<kPencilSpec>(b));
            PlaneArgs<T> a = plane_args();
            a.src = P;
            a.real_out = bf.hr;
            ADJ_RC(launch_plane<kPlaneInvReal>(a));
          }
          hist_spec = bf.hs;
          hist_real = bf.hr;
          hist_pos = 0;
          ADJ_RC(step_async(s1 - s0));
          hist_spec = nullptr;
          hist_real = nullptr;
        }
        for (int n = s1 - 1; n >= s0; --n) {
          const int j = n - s0;
          PlaneArgs<T> a = plane_args();
          a.src = bf.mp;                       // partial of c_n mu^{n+1} - mu^{n+2}
          a.real_in[1] = bf.hr + size_t(j) * nr;               // psi^n
          a.dst = bf.gp;                       // partial of g^n
          ADJ_RC(launch_plane<kPlaneAdj>(a));
          PencilArgs<T> b = pencil_args();
          b.src = bf.gp;
          b.w = bf.lam;                        // lambdahat^{n+1} -> lambdahat^n
          b.spec_a = bf.hs + size_t(j) * fe;   // psihat^n
          b.spec_b = n == nsteps - 1 ? bf.hs + size_t(j + 1) * fe : nullptr;  // psihat^T, once
          b.coef = n >= 1 ? (n - 1 >= 1 ? 3.0 : 2.0) : 0.0;
          b.dst = bf.mp;                       // partial of c_{n-1} mu^n - mu^{n+1}
          b.red = bf.red;
          ADJ_RC(launch_pencil<kPencilAdj>(b));
        }
      }
      adj_reduce_kernel<<<p.batch, 256, 0, stream>>>(bf.red, QC::TILES, bf.acc);
      ADJ_CUDA(cudaGetLastError());
      launches += 1;
      // ---- lambda^0 = dL/dpsi^0 in real space
      {
        PencilArgs<T> b = pencil_args();
        b.w = bf.lam;
        b.dst = bf.gp;
        ADJ_RC(launch_pencil<kPencilAdjOut>(b));
        PlaneArgs<T> a = plane_args();
        a.src = bf.gp;
        a.psi_out = d_psi;
        a.flags = kFlPsiOut;
        ADJ_RC(launch_plane<kPlaneGetPsi>(a));
      }
      std::vector<double> acc(size_t(p.batch) * 4);
      ADJ_CUDA(cudaMemcpyAsync(acc.data(), bf.acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
      ADJ_CUDA(cudaMemcpyAsync(g_psi0, d_psi, nr * sizeof(double), cudaMemcpyDeviceToHost, stream));
      // back to the state the forward sweep ended in
      ADJ_CUDA(cudaMemcpyAsync(W, bf.fin, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(P, bf.fin + fe, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaMemcpyAsync(Nt, bf.fin + 2 * fe, fb, cudaMemcpyDeviceToDevice, stream));
      ADJ_CUDA(cudaStreamSynchronize(stream));
      for (int r = 0; r < p.batch; ++r) {
        g_eps[r] = acc[size_t(r) * 4 + 0];
        g_q0[r] = acc[size_t(r) * 4 + 2];
      }
      steps = end_steps;
      psi0_valid = false;
      restore();
      return SH_OK;
    }
  }
#undef ADJ_CUDA
#undef ADJ_RC

  // surfTrack pass (periodicFFT/surfTrack.cpp:592-626, 744-806): one advected
  // step; the crossing of psi^{n+1} per (x, y) column with v_n, H, K from the
  // fields of state n.
  int surface_step(int* z, double* vn, double* hh, double* kk) override {
    if constexpr (DCT) {
      if (p.advection) {
        // d_t psi of cosNoAdvMorphCurv has no u . grad psi term
        err = "the Neumann curvature pass is defined for handles without advection";
        return SH_EUNSUPPORTED;
      }
      // curvature pass of cosFFT/comet/cosNoAdvMorphCurv.cpp:742-965 at state n, then one step
      int rc;
      const size_t nr = size_t(p.batch) * N * N * N, nc = size_t(p.batch) * N * N;
      if (!CR[0]) {
        for (auto& r : CR) SHB_CUDA(dev_malloc(&r, nr * sizeof(T)));
        SHB_CUDA(dev_malloc(&Psc, field_elems() * sizeof(cplx<T>)));
        SHB_CUDA(dev_malloc(&d_zout, nc * sizeof(int)));
        for (auto& d : d_surf) SHB_CUDA(dev_malloc(&d, nc * sizeof(double)));
      }
      CurvArgs<T> ca{};
      if (p.curvature == SH_CURV_SPECTRAL) {
        // exact first and mixed derivatives of the cosine series: d/dx, d/dy, d/dz
        // turn the cosine series along that axis into a sine series, inverted as the
        // REDFT01 of reversed coefficients times (-1)^index (sign_axes)
        if (!CSP[0])
          for (auto& r : CSP) SHB_CUDA(dev_malloc(&r, nr * sizeof(T)));
        PencilArgs<T> b = pencil_args();
        b.src = P;
        b.dst = Psc;
        b.xmul = kXSinDx;
        if ((rc = launch_pencil<kPencilXMul>(b))) return rc;
        struct D { const cplx<T>* src; int mult, sin_dz, sign; };
        const D d[6] = {{Psc, kMulNone, 0, 1}, {P, kMulSinDy, 0, 2}, {P, kMulNone, 1, 4},
                        {Psc, kMulSinDy, 0, 3}, {Psc, kMulNone, 1, 5}, {P, kMulSinDy, 1, 6}};
        for (int i = 0; i < 6; ++i) {
          PlaneArgs<T> a = plane_args();
          a.src = d[i].src;
          a.mult = d[i].mult;
          a.sin_dz = d[i].sin_dz;
          a.sign_axes = d[i].sign;
          a.real_out = CSP[i];
          if ((rc = launch_plane<kPlaneInvReal>(a))) return rc;
          ca.spec[i] = CSP[i];
        }
      }
      // psi, psi_yy, psi_zz from the partial of psi; psi_xx and L psi through an x multiplier
      const int mult[3] = {kMulNone, kMulNegQy2, kMulNegQz2};
      T* outs[3] = {CR[0], CR[2], CR[3]};
      PlaneArgs<T> st[3];
      for (int i = 0; i < 3; ++i) {
        st[i] = plane_args();
        st[i].src = P;
        st[i].mult = mult[i];
        st[i].real_out = outs[i];
      }
      if ((rc = launch_plane_sets<kPlaneInvReal>(st, 3))) return rc;
      const int xm[2] = {kXNegQx2, kXOpSH};
      T* xo[2] = {CR[1], CR[4]};
      for (int i = 0; i < 2; ++i) {
        PencilArgs<T> b = pencil_args();
        b.src = P;
        b.dst = Psc;
        b.xmul = xm[i];
        if ((rc = launch_pencil<kPencilXMul>(b))) return rc;
        PlaneArgs<T> a = plane_args();
        a.src = Psc;
        a.real_out = xo[i];
        if ((rc = launch_plane<kPlaneInvReal>(a))) return rc;
      }
      ca.psi = CR[0];
      ca.dxx = CR[1];
      ca.dyy = CR[2];
      ca.dzz = CR[3];
      ca.lpsi = CR[4];
      ca.wall = d_wall;
      ca.lperp = Lp;
      ca.kwall = kwall;
      ca.pp = point_params();
      ca.n = N;
      ca.dx = p.dx;
      ca.zout = d_zout;
      ca.vn = d_surf[0];
      ca.hh = d_surf[1];
      ca.kk = d_surf[2];
      curv_scan_kernel<T><<<dim3((N * N + 127) / 128, p.batch), 128, 0, stream>>>(ca);
      SHB_CUDA(cudaGetLastError());
      ++launches;
      if ((rc = step_async(1))) return rc;
      SHB_CUDA(cudaMemcpyAsync(z, d_zout, nc * sizeof(int), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(vn, d_surf[0], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(hh, d_surf[1], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(kk, d_surf[2], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaStreamSynchronize(stream));
      return SH_OK;
    } else {
      if (!p.advection) {
        err = "surface tracking runs the advected step (advection = 1)";
        return SH_EINVAL;
      }
      int rc;
      const size_t nr = size_t(p.batch) * N * N * N, nc = size_t(p.batch) * N * N;
      if (!SR[0]) {
        for (auto& r : SR) SHB_CUDA(dev_malloc(&r, nr * sizeof(T)));
        SHB_CUDA(dev_malloc(&d_zout, nc * sizeof(int)));
        for (auto& d : d_surf) SHB_CUDA(dev_malloc(&d, nc * sizeof(double)));
      }
      if (!real_fields_current && (rc = adv_nonlinear(0))) return rc;
      if (!u_real_current && (rc = velocity_real())) return rc;
      // second derivatives of psi^n: psi_xx = C2R(-q_x^2 psihat), psi_yy, psi_xy
      PencilArgs<T> b = pencil_args();
      b.src = Px;
      b.dst = S3[0];
      if ((rc = launch_pencil<kPencilXMul>(b))) return rc;
      const cplx<T>* src[3] = {S3[0], P, Px};
      const int mult[3] = {kMulNone, kMulNegQy2, kMulIqy};
      PlaneArgs<T> st[3];
      for (int i = 0; i < 3; ++i) {
        st[i] = plane_args();
        st[i].src = src[i];
        st[i].mult = mult[i];
        st[i].real_out = SR[i];
      }
      if ((rc = launch_plane_sets<kPlaneInvReal>(st, 3))) return rc;
      SurfArgs<T> sa;
      sa.psi = R[0];
      sa.gx = R[1];
      sa.gy = R[2];
      sa.gz = R[3];
      sa.lpsi = R[4];
      sa.ux = R[5];
      sa.uy = R[6];
      sa.uz = R[7];
      sa.dxx = SR[0];
      sa.dyy = SR[1];
      sa.dxy = SR[2];
      sa.hnum = SR[3];
      sa.pp = point_params();
      sa.n3 = (long long)N * N * N;
      sa.n = N;
      surface_prep_kernel<T><<<dim3(592, p.batch), 256, 0, stream>>>(sa);
      SHB_CUDA(cudaGetLastError());
      ++launches;
      if ((rc = step_async(1))) return rc;  // R[0] now holds psi^{n+1}
      surface_scan_kernel<T><<<dim3((N * N + 127) / 128, p.batch), 128, 0, stream>>>(
          R[0], SR[0], SR[1], SR[3], SR[2], N, d_zout, d_surf[0], d_surf[1], d_surf[2]);
      SHB_CUDA(cudaGetLastError());
      ++launches;
      SHB_CUDA(cudaMemcpyAsync(z, d_zout, nc * sizeof(int), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(vn, d_surf[0], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(hh, d_surf[1], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaMemcpyAsync(kk, d_surf[2], nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      SHB_CUDA(cudaStreamSynchronize(stream));
      return SH_OK;
    }
  }
};

// factories: one per (precision, boundary, size), defined in the
// instantiation units sh_inst_<precision>_<boundary>_<size>.cu
#define SHB_DECLARE_FACTORIES(P, B)                                                                  \
  SolverBase* make_solver_##P##_##B##_n16(int cl, int tile);                                         \
  SolverBase* make_solver_##P##_##B##_n32(int cl, int tile);                                         \
  SolverBase* make_solver_##P##_##B##_n64(int cl, int tile);                                         \
  SolverBase* make_solver_##P##_##B##_n128(int cl, int tile);                                        \
  SolverBase* make_solver_##P##_##B##_n256(int cl, int tile);                                        \
  SolverBase* make_solver_##P##_##B##_n512(int cl, int tile);                                        \
  inline SolverBase* make_solver_##P##_##B(int n, int variant, int tile) {                           \
    switch (n) {                                                                                      \
      case 16: return make_solver_##P##_##B##_n16(variant, tile);                                    \
      case 32: return make_solver_##P##_##B##_n32(variant, tile);                                    \
      case 64: return make_solver_##P##_##B##_n64(variant, tile);                                    \
      case 128: return make_solver_##P##_##B##_n128(variant, tile);                                  \
      case 256: return make_solver_##P##_##B##_n256(variant, tile);                                  \
      case 512: return make_solver_##P##_##B##_n512(variant, tile);                                  \
      default: return nullptr;                                                                        \
    }                                                                                                 \
  }
SHB_DECLARE_FACTORIES(f32, periodic)
SHB_DECLARE_FACTORIES(f64, periodic)
SHB_DECLARE_FACTORIES(f32, neumann)
SHB_DECLARE_FACTORIES(f64, neumann)
#undef SHB_DECLARE_FACTORIES

}  // namespace shb
