// Host-side solver: owns the device state of one handle and sequences the
// plane and pencil passes of each time step.
#pragma once
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smectic_b200.h"
#include "pencil_kernel.cuh"
#include "plane_kernel.cuh"

namespace shb {

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
  int trace_cap = 0;
  std::vector<double> energy_trace;  // host copy, steps * batch
  std::vector<double> l1_last;
  int l1_count = 0;
  bool ready = false;
  bool psi0_valid = false;  // d_psi holds psi^0 exactly as uploaded

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
    for (auto& e : prof_ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  size_t n3() const { return size_t(p.n) * p.n * p.n; }
  virtual int setup() = 0;
  virtual int init_from_psi() = 0;     // d_psi holds psi^0
  virtual int step_async(int n) = 0;
  // per-launch event timing of the two passes (nullptr: off)
  double* prof_ms = nullptr;
  cudaEvent_t prof_ev[3] = {nullptr, nullptr, nullptr};
  virtual int psi_to_dpsi() = 0;       // current psi -> d_psi
  virtual int energy_now(double* host) = 0;
  virtual size_t state_bytes() const = 0;
  virtual int save_state(void* host) = 0;
  virtual int load_state(const void* host) = 0;
};

template <typename T, int N, int CL, bool DCT>
struct Solver final : SolverBase {
  using PC = PlaneCfg<T, N, CL, DCT>;
  using QC = PencilCfg<T, N, DCT>;
  static constexpr int FP = PC::FP;

  cplx<T>* W = nullptr;
  cplx<T>* P = nullptr;
  cplx<T>* Nt = nullptr;
  cplx<T>* tw = nullptr;  // [forward | inverse | quarter-wave] twiddle table
  T* q = nullptr;

  ~Solver() override {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(W);
    cudaFree(P);
    cudaFree(Nt);
    cudaFree(tw);
    cudaFree(q);
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
  static constexpr auto pencil_fn() { return &pencil_kernel<T, N, DCT, MODE>; }

  template <class K>
  int set_attrs(K kern, size_t smem, bool cluster) {
    SHB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if (cluster && CL > 8) SHB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return SH_OK;
  }

  int setup() override {
    const size_t fe = field_elems();
    SHB_CUDA(cudaMalloc(&W, fe * sizeof(cplx<T>)));
    SHB_CUDA(cudaMalloc(&P, fe * sizeof(cplx<T>)));
    SHB_CUDA(cudaMalloc(&Nt, fe * sizeof(cplx<T>)));
    SHB_CUDA(cudaMalloc(&tw, tw_total<N>() * sizeof(cplx<T>)));
    SHB_CUDA(cudaMalloc(&q, N * sizeof(T)));
    SHB_CUDA(cudaMalloc(&d_red_plane, size_t(p.batch) * N * CL * 3 * sizeof(double)));
    SHB_CUDA(cudaMalloc(&d_red_spec, size_t(p.batch) * QC::TILES * sizeof(double)));
    std::vector<cplx<T>> htw;
    host_twiddles<T, N>(htw);
    std::vector<T> hq(N);
    if (!DCT) {
      // periodicFFT/pf3d.cpp:166-190 (Nyquist entry +pi/dx)
      for (int i = 0; i < N; ++i)
        hq[i] = T(i < N / 2 + 1 ? 2.0 * M_PI * i / (p.dx * N) : -(N - i) * 2.0 * M_PI / (p.dx * N));
    } else {
      // cosFFT/mesabi/cosNoAdvMorph.cpp:216-231
      for (int i = 0; i < N; ++i) hq[i] = T(M_PI * i / (p.dx * N));
    }
    SHB_CUDA(cudaMemcpy(tw, htw.data(), htw.size() * sizeof(cplx<T>), cudaMemcpyHostToDevice));
    SHB_CUDA(cudaMemcpy(q, hq.data(), N * sizeof(T), cudaMemcpyHostToDevice));
    int rc;
    if ((rc = set_attrs(plane_fn<kPlaneStep>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneInit>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(plane_fn<kPlaneGetPsi>(), PC::SMEM, true))) return rc;
    if ((rc = set_attrs(pencil_fn<kPencilStep>(), QC::SMEM, false))) return rc;
    if ((rc = set_attrs(pencil_fn<kPencilInit>(), QC::SMEM, false))) return rc;
    if ((rc = set_attrs(pencil_fn<kPencilEnergy>(), QC::SMEM, false))) return rc;
    return SH_OK;
  }

  template <int MODE>
  int launch_plane(const PlaneArgs<T>& a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(N * CL, p.batch, 1);
    cfg.blockDim = dim3(PC::THREADS, 1, 1);
    cfg.dynamicSmemBytes = PC::SMEM;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = CL > 1 ? 1 : 0;
    SHB_CUDA(cudaLaunchKernelEx(&cfg, plane_fn<MODE>(), a));
    ++launches;
    return SH_OK;
  }

  template <int MODE>
  int launch_pencil(const PencilArgs<T>& a) {
    pencil_fn<MODE>()<<<dim3(QC::TILES, p.batch, 1), QC::THREADS, QC::SMEM, stream>>>(a);
    SHB_CUDA(cudaGetLastError());
    ++launches;
    return SH_OK;
  }

  PlaneArgs<T> plane_args() const {
    PlaneArgs<T> a{};
    a.tw = tw;
    a.pp = point_params();
    a.red = d_red_plane;
    a.timeout = d_flag + 1;
    return a;
  }
  PencilArgs<T> pencil_args() const {
    PencilArgs<T> a{};
    a.tw = tw;
    a.q = q;
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

  int init_from_psi() override {
    int rc;
    PlaneArgs<T> a = plane_args();
    a.psi_in = d_psi;
    a.dst2 = P;   // partial of psi^0 (consumed by the init pencil, then overwritten)
    a.dst = Nt;   // partial of N(psi^0): the first Nhat (Euler start)
    if ((rc = launch_plane<kPlaneInit>(a))) return rc;
    PencilArgs<T> b = pencil_args();
    b.src = P;
    b.src2 = Nt;
    b.w = W;
    b.dst = P;
    if ((rc = launch_pencil<kPencilInit>(b))) return rc;
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

  int step_async(int n) override {
    int rc;
    const bool trace = p.energy_trace != 0;
    if (trace && n > trace_cap) {
      cudaFree(d_trace);
      d_trace = nullptr;
      SHB_CUDA(cudaMalloc(&d_trace, size_t(n) * p.batch * sizeof(double)));
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
      if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[0], stream));
      if ((rc = launch_pencil<kPencilStep>(b))) return rc;
      if (prof_ms) SHB_CUDA(cudaEventRecord(prof_ev[1], stream));
      PlaneArgs<T> a = plane_args();
      a.src = P;
      a.dst = Nt;
      a.flags = (trace ? kFlEnergy : 0) | (l1_now ? kFlL1 : 0) | (stash_now ? kFlPsiOut : 0);
      a.psi_old = d_stash;
      a.psi_out = d_stash;
      if ((rc = launch_plane<kPlaneStep>(a))) return rc;
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
    }
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

  size_t state_bytes() const override { return 3 * field_elems() * sizeof(cplx<T>); }
  int save_state(void* host) override {
    const size_t fb = field_elems() * sizeof(cplx<T>);
    char* h = static_cast<char*>(host);
    SHB_CUDA(cudaMemcpyAsync(h, W, fb, cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaMemcpyAsync(h + fb, P, fb, cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaMemcpyAsync(h + 2 * fb, Nt, fb, cudaMemcpyDeviceToHost, stream));
    SHB_CUDA(cudaStreamSynchronize(stream));
    return SH_OK;
  }
  int load_state(const void* host) override {
    const size_t fb = field_elems() * sizeof(cplx<T>);
    const char* h = static_cast<const char*>(host);
    SHB_CUDA(cudaMemcpyAsync(W, h, fb, cudaMemcpyHostToDevice, stream));
    SHB_CUDA(cudaMemcpyAsync(P, h + fb, fb, cudaMemcpyHostToDevice, stream));
    SHB_CUDA(cudaMemcpyAsync(Nt, h + 2 * fb, fb, cudaMemcpyHostToDevice, stream));
    SHB_CUDA(cudaStreamSynchronize(stream));
    ready = true;
    psi0_valid = false;
    return SH_OK;
  }
};

// factory: defined per precision / boundary in the instantiation units
SolverBase* make_solver_f32_periodic(int n, int variant);
SolverBase* make_solver_f64_periodic(int n, int variant);
SolverBase* make_solver_f32_neumann(int n, int variant);
SolverBase* make_solver_f64_neumann(int n, int variant);

}  // namespace shb
