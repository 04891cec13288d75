// C-ABI of the smectic3d_b200 solver (declarations in include/smectic_b200.h).
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "amplitude_kernel.cuh"
#include "sh_solver.cuh"

using namespace shb;

struct sh_handle {
  SolverBase* s = nullptr;
};

static thread_local std::string g_err;

// NVTX range over one public call (named after the entry point), so that a
// timeline profiler shows the library's calls; without a tool attached the
// push and pop are no-ops.
struct ApiRange {
  explicit ApiRange(const char* name) { nvtxRangePushA(name); }
  ~ApiRange() { nvtxRangePop(); }
};

namespace shb {
void set_global_error(const std::string& msg) { g_err = msg; }
}  // namespace shb

namespace shb {

__global__ void finalize_kernel(const double* red_plane, int nbp, const double* red_spec, int nbs, int what,
                                double dv, double spec_norm, double alpha, double dt, double* out) {
  __shared__ double scratch[32];
  const int rep = blockIdx.x;
  KahanSum s0, s1;
  if (what == 0) {
    for (int b = threadIdx.x; b < nbp; b += blockDim.x) s0.add(red_plane[(size_t(rep) * nbp + b) * 3 + 2]);
    for (int b = threadIdx.x; b < nbs; b += blockDim.x) s1.add(red_spec[size_t(rep) * nbs + b]);
    const double local = block_sum(s0.s, scratch);
    const double spec = block_sum(s1.s, scratch);
    if (threadIdx.x == 0) out[rep] = dv * (local + 0.5 * alpha * spec_norm * spec);
  } else {
    for (int b = threadIdx.x; b < nbp; b += blockDim.x) {
      s0.add(red_plane[(size_t(rep) * nbp + b) * 3 + 0]);
      s1.add(red_plane[(size_t(rep) * nbp + b) * 3 + 1]);
    }
    const double a = block_sum(s0.s, scratch);
    const double b = block_sum(s1.s, scratch);
    if (threadIdx.x == 0) out[rep] = a / (dt * b);
  }
}

// Sum of the per-CTA adjoint gradient slots (red[rep][blk][2]) into
// acc[rep] = {g_eps, 0, g_q0, 0}, compensated, in a fixed order.
__global__ void adj_reduce_kernel(const double* red, int nblocks, double* acc) {
  __shared__ double scratch[32];
  const int rep = blockIdx.x;
  KahanSum s0, s1;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    s0.add(red[(size_t(rep) * nblocks + b) * 2 + 0]);
    s1.add(red[(size_t(rep) * nblocks + b) * 2 + 1]);
  }
  const double te = block_sum(s0.s, scratch);
  const double tq = block_sum(s1.s, scratch);
  if (threadIdx.x == 0) {
    double* a = acc + size_t(rep) * 4;
    a[0] = te;
    a[1] = 0.0;
    a[2] = tq;
    a[3] = 0.0;
  }
}

__global__ void shell_argmax_kernel(const double* shell, int nshell, double dq, double* out) {
  __shared__ double bv[256];
  __shared__ int bi[256];
  const double* s = shell + size_t(blockIdx.x) * nshell;
  double best = -1.0;
  int idx = 0;
  for (int i = 1 + threadIdx.x; i < nshell; i += blockDim.x)
    if (s[i] > best) {  // strided ascending: the first maximum of this thread
      best = s[i];
      idx = i;
    }
  bv[threadIdx.x] = best;
  bi[threadIdx.x] = idx;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      const double ov = bv[threadIdx.x + h];
      const int oi = bi[threadIdx.x + h];
      if (ov > bv[threadIdx.x] || (ov == bv[threadIdx.x] && oi < bi[threadIdx.x] && oi > 0)) {
        bv[threadIdx.x] = ov;
        bi[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = bi[0] * dq;
}

}  // namespace shb

#define API_CUDA(h, expr)                                                        \
  do {                                                                           \
    cudaError_t e_ = (expr);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      (h)->s->err = std::string(#expr) + ": " + cudaGetErrorString(e_);          \
      return SH_ECUDA;                                                           \
    }                                                                            \
  } while (0)

static int fail(sh_handle* h, int code, const std::string& msg) {
  if (h && h->s) h->s->err = msg;
  g_err = msg;
  return code;
}

static bool supported_n(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512; }

// Dense <-> padded host layouts (padded: (i*N + j) * 2(N/2+1) + k)
static void to_dense(const double* src, double* dst, int n, int batch, int layout) {
  const size_t n3 = size_t(n) * n * n;
  if (layout == SH_LAYOUT_DENSE) {
    std::memcpy(dst, src, n3 * batch * sizeof(double));
    return;
  }
  const size_t pz = 2 * (n / 2 + 1);
  for (int r = 0; r < batch; ++r)
    for (size_t ij = 0; ij < size_t(n) * n; ++ij)
      std::memcpy(dst + r * n3 + ij * n, src + (r * size_t(n) * n + ij) * pz, n * sizeof(double));
}
static void from_dense(const double* src, double* dst, int n, int batch, int layout) {
  const size_t n3 = size_t(n) * n * n;
  if (layout == SH_LAYOUT_DENSE) {
    std::memcpy(dst, src, n3 * batch * sizeof(double));
    return;
  }
  const size_t pz = 2 * (n / 2 + 1);
  for (int r = 0; r < batch; ++r)
    for (size_t ij = 0; ij < size_t(n) * n; ++ij) {
      double* d = dst + (r * size_t(n) * n + ij) * pz;
      std::memcpy(d, src + r * n3 + ij * n, n * sizeof(double));
      d[n] = 0.0;
      d[n + 1] = 0.0;
    }
}

extern "C" {

const char* sh_version(void) { return "smectic3d_b200 0.1 (sm_100a)"; }

int sh_default_params(sh_params* p) {
  if (!p) return SH_EINVAL;
  std::memset(p, 0, sizeof(*p));
  p->n = 128;
  p->batch = 1;
  p->boundary = SH_PERIODIC;
  p->advection = 0;
  p->nonlinearity = SH_QUINTIC;
  p->scheme = SH_CNAB2;
  p->precision = SH_FP64;
  p->l1_interval = 0;
  p->energy_trace = 0;
  p->dx = 2.0 * M_PI / 8.0;
  p->dt = 0.05;
  p->eps = -0.75;
  p->beta = 2.0;
  p->gamma = 1.0;
  p->alpha = 1.0;
  p->q0 = 1.0;
  p->eta = 1.0;
  p->rho = 1.0;
  p->w_mid = 0.0;
  p->sub_sigma = 0.0;
  p->sub_z0 = 1e-4;
  p->eps_per_replica = nullptr;
  p->curvature = SH_CURV_DIFFERENCE;
  p->replica_block = 0;
  p->pencil_tile = 0;
  return SH_OK;
}

int sh_create(const sh_params* p, sh_handle** out) {
  ApiRange range_("sh_create");
  if (!p || !out) return fail(nullptr, SH_EINVAL, "null argument");
  *out = nullptr;
  if (!supported_n(p->n)) return fail(nullptr, SH_EUNSUPPORTED, "n must be one of 16, 32, 64, 128, 256, 512");
  if (p->batch < 1 || p->batch > 65535) return fail(nullptr, SH_EINVAL, "batch must be in [1, 65535]");
  if (p->boundary != SH_PERIODIC && p->boundary != SH_NEUMANN) return fail(nullptr, SH_EINVAL, "bad boundary");
  if (p->precision != SH_FP64 && p->precision != SH_FP32 && p->precision != SH_FP32_UPDATE64)
    return fail(nullptr, SH_EINVAL, "bad precision");
  if (p->nonlinearity != SH_QUINTIC && p->nonlinearity != SH_QUAD_CUBIC) return fail(nullptr, SH_EINVAL, "bad nonlinearity");
  if (p->scheme != SH_CNAB2 && p->scheme != SH_IMEX_EULER) return fail(nullptr, SH_EINVAL, "bad scheme");
  if (!(p->dx > 0) || !(p->dt > 0)) return fail(nullptr, SH_EINVAL, "dx and dt must be positive");
  if (p->l1_interval < 0) return fail(nullptr, SH_EINVAL, "l1_interval must be >= 0");
  if (p->sub_sigma != 0.0) {
    if (p->boundary != SH_NEUMANN) return fail(nullptr, SH_EUNSUPPORTED, "the substrate penalty is defined for the Neumann boundary");
    if (p->advection) return fail(nullptr, SH_EUNSUPPORTED, "advection and the substrate penalty are not combined");
    if (!(p->sub_z0 > 0.0)) return fail(nullptr, SH_EINVAL, "sub_z0 must be > 0");
  }
  if (p->variant < 0) return fail(nullptr, SH_EINVAL, "variant must be >= 0");
  if (p->curvature != SH_CURV_DIFFERENCE && p->curvature != SH_CURV_SPECTRAL)
    return fail(nullptr, SH_EINVAL, "bad curvature");
  if (p->replica_block < 0) return fail(nullptr, SH_EINVAL, "replica_block must be >= 0");
  if (p->pencil_tile != 0 && p->pencil_tile != 8 && p->pencil_tile != 16 && p->pencil_tile != 32)
    return fail(nullptr, SH_EINVAL, "pencil_tile must be 0, 8, 16 or 32");

  SolverBase* s = nullptr;
  const bool f32 = p->precision != SH_FP64;
  const int tile = p->pencil_tile;
  if (p->boundary == SH_PERIODIC)
    s = f32 ? make_solver_f32_periodic(p->n, p->variant, tile) : make_solver_f64_periodic(p->n, p->variant, tile);
  else
    s = f32 ? make_solver_f32_neumann(p->n, p->variant, tile) : make_solver_f64_neumann(p->n, p->variant, tile);
  if (!s) return fail(nullptr, SH_EUNSUPPORTED, "this size / variant is not built");
  std::unique_ptr<sh_handle> h(new sh_handle);
  h->s = s;
  s->p = *p;
  s->p.eps_per_replica = nullptr;
  s->eps.assign(p->batch, p->eps);
  if (p->eps_per_replica)
    for (int r = 0; r < p->batch; ++r) s->eps[r] = p->eps_per_replica[r];
  const size_t n3 = s->n3();
  auto bad = [&](const char* what) {
    g_err = std::string(what) + ": " + s->err;
    delete s;
    h->s = nullptr;
    return SH_ECUDA;
  };
  {
    const char* fa = getenv("SMECTIC_B200_TEST_FAIL_ALLOC");
    alloc_fail_countdown() = fa ? atoi(fa) : 0;
  }
  struct Disarm {
    ~Disarm() { alloc_fail_countdown() = 0; }
  } disarm;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    s->err = cudaGetErrorString(e);
    return bad("stream");
  }
  if ((e = dev_malloc(&s->d_flag, 2 * sizeof(int))) != cudaSuccess ||
      (e = dev_malloc(&s->d_psi, n3 * p->batch * sizeof(double))) != cudaSuccess ||
      (e = dev_malloc(&s->d_eps, p->batch * sizeof(double))) != cudaSuccess ||
      (e = dev_malloc(&s->d_scalar, p->batch * sizeof(double))) != cudaSuccess) {
    s->err = cudaGetErrorString(e);
    delete s;
    h->s = nullptr;
    g_err = std::string("device allocation: ") + cudaGetErrorString(e);
    return SH_ENOMEM;
  }
  if (p->l1_interval > 0 && (e = dev_malloc(&s->d_stash, n3 * p->batch * sizeof(double))) != cudaSuccess) {
    delete s;
    h->s = nullptr;
    g_err = std::string("device allocation: ") + cudaGetErrorString(e);
    return SH_ENOMEM;
  }
  cudaMemset(s->d_flag, 0, 2 * sizeof(int));
  {
    const char* drop = getenv("SMECTIC_B200_TEST_DROP_EXCHANGE");
    s->drop_exchange = (drop && drop[0] == '1') ? 1 : 0;
  }
  cudaMemcpy(s->d_eps, s->eps.data(), p->batch * sizeof(double), cudaMemcpyHostToDevice);
  s->l1_last.assign(p->batch, 0.0);
  int rc = s->setup();
  if (rc) {
    const int code = (s->err.find("out of memory") != std::string::npos) ? SH_ENOMEM : rc;
    g_err = s->err;
    delete s;
    h->s = nullptr;
    return code;
  }
  *out = h.release();
  return SH_OK;
}

int sh_destroy(sh_handle* h) {
  if (!h) return SH_EINVAL;
  delete h->s;
  delete h;
  return SH_OK;
}

int sh_set_psi_device(sh_handle* h, const double* dev_psi) {
  ApiRange range_("sh_set_psi_device");
  if (!h || !h->s || !dev_psi) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  if (dev_psi != s->d_psi)
    API_CUDA(h, cudaMemcpyAsync(s->d_psi, dev_psi, s->n3() * s->p.batch * sizeof(double), cudaMemcpyDeviceToDevice,
                                s->stream));
  API_CUDA(h, cudaMemsetAsync(s->d_flag, 0, 2 * sizeof(int), s->stream));
  return s->init_from_psi();
}

int sh_set_psi(sh_handle* h, const double* host_psi, int layout) {
  ApiRange range_("sh_set_psi");
  if (!h || !h->s || !host_psi) return fail(h, SH_EINVAL, "null argument");
  if (layout != SH_LAYOUT_DENSE && layout != SH_LAYOUT_PADDED) return fail(h, SH_EINVAL, "bad layout");
  SolverBase* s = h->s;
  const size_t bytes = s->n3() * s->p.batch * sizeof(double);
  if (layout == SH_LAYOUT_DENSE) {
    API_CUDA(h, cudaMemcpyAsync(s->d_psi, host_psi, bytes, cudaMemcpyHostToDevice, s->stream));
  } else {
    std::vector<double> tmp(s->n3() * s->p.batch);
    to_dense(host_psi, tmp.data(), s->p.n, s->p.batch, layout);
    API_CUDA(h, cudaMemcpyAsync(s->d_psi, tmp.data(), bytes, cudaMemcpyHostToDevice, s->stream));
    API_CUDA(h, cudaStreamSynchronize(s->stream));
  }
  return sh_set_psi_device(h, s->d_psi);
}

int sh_get_psi_device(sh_handle* h, double* dev_psi) {
  ApiRange range_("sh_get_psi_device");
  if (!h || !h->s || !dev_psi) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  if (!s->ready) return fail(h, SH_ESTATE, "psi was never set");
  int rc = s->psi_to_dpsi();
  if (rc) return rc;
  if (dev_psi != s->d_psi)
    API_CUDA(h, cudaMemcpyAsync(dev_psi, s->d_psi, s->n3() * s->p.batch * sizeof(double), cudaMemcpyDeviceToDevice,
                                s->stream));
  return SH_OK;
}

int sh_get_psi(sh_handle* h, double* host_psi, int layout) {
  ApiRange range_("sh_get_psi");
  if (!h || !h->s || !host_psi) return fail(h, SH_EINVAL, "null argument");
  if (layout != SH_LAYOUT_DENSE && layout != SH_LAYOUT_PADDED) return fail(h, SH_EINVAL, "bad layout");
  SolverBase* s = h->s;
  if (!s->ready) return fail(h, SH_ESTATE, "psi was never set");
  int rc = s->psi_to_dpsi();
  if (rc) return rc;
  const size_t bytes = s->n3() * s->p.batch * sizeof(double);
  if (layout == SH_LAYOUT_DENSE) {
    API_CUDA(h, cudaMemcpyAsync(host_psi, s->d_psi, bytes, cudaMemcpyDeviceToHost, s->stream));
    API_CUDA(h, cudaStreamSynchronize(s->stream));
  } else {
    std::vector<double> tmp(s->n3() * s->p.batch);
    API_CUDA(h, cudaMemcpyAsync(tmp.data(), s->d_psi, bytes, cudaMemcpyDeviceToHost, s->stream));
    API_CUDA(h, cudaStreamSynchronize(s->stream));
    from_dense(tmp.data(), host_psi, s->p.n, s->p.batch, layout);
  }
  return SH_OK;
}

int sh_local_amplitude(sh_handle* h, int nw, double* out) {
  ApiRange range_("sh_local_amplitude");
  if (!h || !h->s || !out) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  if (!s->ready) return fail(h, SH_ESTATE, "psi was never set");
  const int n = s->p.n, nl = nw / 2;
  if (nw < 2 || 3 * nl > n - 1) return fail(h, SH_EINVAL, "nw must satisfy 2 <= nw and 3 (nw / 2) <= n - 1");
  int rc = s->psi_to_dpsi();
  if (rc) return rc;
  const size_t bytes = s->n3() * s->p.batch * sizeof(double);
  for (auto& b : s->d_amp)
    if (!b) API_CUDA(h, dev_malloc(&b, bytes));
  const dim3 lines((unsigned)((size_t(n) * n + 255) / 256), s->p.batch);
  const double dx = s->p.dx;
  // psi^2 -> x window -> y window -> z window (morphSurfAmp.cpp:1076-1107)
  amp_window_kernel<<<lines, 256, 0, s->stream>>>(s->d_psi, s->d_amp[0], n, 0, nl, dx, 1);
  amp_window_kernel<<<lines, 256, 0, s->stream>>>(s->d_amp[0], s->d_amp[1], n, 1, nl, dx, 0);
  amp_window_kernel<<<lines, 256, 0, s->stream>>>(s->d_amp[1], s->d_amp[0], n, 2, nl, dx, 0);
  const double lam = 2.0 * M_PI / s->p.q0;
  amp_normalise_kernel<<<dim3(592, s->p.batch), 256, 0, s->stream>>>(s->d_amp[0], s->d_amp[1], n, nl, dx,
                                                                      lam * lam * lam);
  API_CUDA(h, cudaGetLastError());
  s->launches += 4;
  API_CUDA(h, cudaMemcpyAsync(out, s->d_amp[1], bytes, cudaMemcpyDeviceToHost, s->stream));
  API_CUDA(h, cudaStreamSynchronize(s->stream));
  return SH_OK;
}

int sh_step_async(sh_handle* h, int nsteps) {
  ApiRange range_("sh_step_async");
  if (!h || !h->s) return fail(h, SH_EINVAL, "null handle");
  if (nsteps < 0) return fail(h, SH_EINVAL, "nsteps must be >= 0");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->step_async(nsteps);
}

int sh_prepare(sh_handle* h) {
  ApiRange range_("sh_prepare");
  if (!h || !h->s) return fail(h, SH_EINVAL, "null handle");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->build_graph();
}

int sh_step(sh_handle* h, int nsteps) {
  ApiRange range_("sh_step");
  int rc = sh_step_async(h, nsteps);
  if (rc) return rc;
  SolverBase* s = h->s;
  int flag[2] = {0, 0};
  API_CUDA(h, cudaMemcpyAsync(flag, s->d_flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (s->p.energy_trace && nsteps > 0) {
    const size_t old = s->energy_trace.size();
    s->energy_trace.resize(old + size_t(nsteps) * s->p.batch);
    API_CUDA(h, cudaMemcpyAsync(s->energy_trace.data() + old, s->d_trace, size_t(nsteps) * s->p.batch * sizeof(double),
                                cudaMemcpyDeviceToHost, s->stream));
  }
  if (s->p.l1_interval > 0)
    API_CUDA(h, cudaMemcpyAsync(s->l1_last.data(), s->d_scalar, s->p.batch * sizeof(double), cudaMemcpyDeviceToHost,
                                s->stream));
  API_CUDA(h, cudaStreamSynchronize(s->stream));
  if (flag[1]) return fail(h, SH_ETIMEOUT, "a cluster exchange wait gave up (results invalid)");
  if (flag[0]) return fail(h, SH_ENONFINITE, "psi became non-finite");
  return SH_OK;
}

int sh_run(sh_handle* h, const double* host_psi0, int nsteps, double* host_psi_out, int layout) {
  ApiRange range_("sh_run");
  int rc = sh_set_psi(h, host_psi0, layout);
  if (rc) return rc;
  if ((rc = sh_step(h, nsteps))) return rc;
  return sh_get_psi(h, host_psi_out, layout);
}

int sh_energy(sh_handle* h, double* out) {
  ApiRange range_("sh_energy");
  if (!h || !h->s || !out) return fail(h, SH_EINVAL, "null argument");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->energy_now(out);
}

int sh_dominant_wavenumber(sh_handle* h, double* out) {
  ApiRange range_("sh_dominant_wavenumber");
  if (!h || !h->s || !out) return fail(h, SH_EINVAL, "null argument");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->dominant_wavenumber(out);
}

int sh_velocity(sh_handle* h, double* ux, double* uy, double* uz) {
  ApiRange range_("sh_velocity");
  if (!h || !h->s || !ux || !uy || !uz) return fail(h, SH_EINVAL, "null argument");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->velocity(ux, uy, uz);
}

int sh_energy_trace(sh_handle* h, double* out, int max_steps, int* count) {
  if (!h || !h->s) return fail(h, SH_EINVAL, "null handle");
  SolverBase* s = h->s;
  const int avail = int(s->energy_trace.size() / s->p.batch);
  if (count) *count = avail;
  if (out && max_steps > 0) {
    const int m = avail < max_steps ? avail : max_steps;
    std::memcpy(out, s->energy_trace.data(), size_t(m) * s->p.batch * sizeof(double));
  }
  return SH_OK;
}

int sh_l1(sh_handle* h, double* out, int* count) {
  if (!h || !h->s) return fail(h, SH_EINVAL, "null handle");
  SolverBase* s = h->s;
  if (count) *count = s->l1_count;
  if (out) std::memcpy(out, s->l1_last.data(), s->p.batch * sizeof(double));
  return SH_OK;
}

int sh_surface_step(sh_handle* h, int* z, double* vn, double* hmean, double* kgauss) {
  ApiRange range_("sh_surface_step");
  if (!h || !h->s || !z || !vn || !hmean || !kgauss) return fail(h, SH_EINVAL, "null argument");
  if (!h->s->ready) return fail(h, SH_ESTATE, "psi was never set");
  return h->s->surface_step(z, vn, hmean, kgauss);
}

int sh_adjoint(sh_handle* h, const double* psi0, int nsteps, const double* dl_dpsi_t, int ckpt_every, double* g_eps,
               double* g_q0, double* g_psi0) {
  ApiRange range_("sh_adjoint");
  if (!h || !h->s || !psi0 || !dl_dpsi_t || !g_eps || !g_q0 || !g_psi0) return fail(h, SH_EINVAL, "null argument");
  int rc = h->s->adjoint(psi0, nsteps, dl_dpsi_t, ckpt_every, g_eps, g_q0, g_psi0);
  if (rc == SH_OK) h->s->ready = true;
  return rc;
}

int sh_adjoint_forward(sh_handle* h, const double* psi0, int nsteps, int ckpt_every) {
  ApiRange range_("sh_adjoint_forward");
  if (!h || !h->s || !psi0) return fail(h, SH_EINVAL, "null argument");
  int rc = h->s->adjoint_forward(psi0, nsteps, ckpt_every);
  if (rc == SH_OK) h->s->ready = true;
  return rc;
}

int sh_adjoint_backward(sh_handle* h, const double* dl_dpsi_t, double* g_eps, double* g_q0, double* g_psi0) {
  ApiRange range_("sh_adjoint_backward");
  if (!h || !h->s || !dl_dpsi_t || !g_eps || !g_q0 || !g_psi0) return fail(h, SH_EINVAL, "null argument");
  return h->s->adjoint_backward(dl_dpsi_t, g_eps, g_q0, g_psi0);
}

int sh_checkpoint_save(sh_handle* h, void* buf, size_t* bytes) {
  ApiRange range_("sh_checkpoint_save");
  if (!h || !h->s || !bytes) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  const size_t need = sizeof(sh_params) + sizeof(long long) + s->state_bytes();
  if (!buf) {
    *bytes = need;
    return SH_OK;
  }
  if (*bytes < need) return fail(h, SH_EINVAL, "checkpoint buffer too small");
  if (!s->ready) return fail(h, SH_ESTATE, "psi was never set");
  char* c = static_cast<char*>(buf);
  std::memcpy(c, &s->p, sizeof(sh_params));
  std::memcpy(c + sizeof(sh_params), &s->steps, sizeof(long long));
  *bytes = need;
  return s->save_state(c + sizeof(sh_params) + sizeof(long long));
}

int sh_checkpoint_load(sh_handle* h, const void* buf, size_t bytes) {
  ApiRange range_("sh_checkpoint_load");
  if (!h || !h->s || !buf) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  const size_t need = sizeof(sh_params) + sizeof(long long) + s->state_bytes();
  if (bytes != need) return fail(h, SH_EINVAL, "checkpoint size does not match this solver");
  const char* c = static_cast<const char*>(buf);
  sh_params q;
  std::memcpy(&q, c, sizeof(sh_params));
  if (q.n != s->p.n || q.batch != s->p.batch || q.boundary != s->p.boundary || q.precision != s->p.precision)
    return fail(h, SH_EINVAL, "checkpoint was written by a solver of another shape");
  std::memcpy(&s->steps, c + sizeof(sh_params), sizeof(long long));
  return s->load_state(c + sizeof(sh_params) + sizeof(long long));
}

int sh_host_alloc(size_t bytes, void** out) {
  if (!out) return SH_EINVAL;
  cudaError_t e = cudaMallocHost(out, bytes);
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    *out = nullptr;
    return SH_ENOMEM;
  }
  return SH_OK;
}

int sh_host_free(void* p) {
  cudaError_t e = cudaFreeHost(p);
  return e == cudaSuccess ? SH_OK : SH_ECUDA;
}

int sh_profile_steps(sh_handle* h, int nsteps, double* ms_pencil, double* ms_plane) {
  ApiRange range_("sh_profile_steps");
  if (!h || !h->s || !ms_pencil || !ms_plane) return fail(h, SH_EINVAL, "null argument");
  SolverBase* s = h->s;
  if (!s->ready) return fail(h, SH_ESTATE, "psi was never set");
  for (auto& e : s->prof_ev)
    if (!e) API_CUDA(h, cudaEventCreate(&e));
  double ms[2] = {0.0, 0.0};
  s->prof_ms = ms;
  int rc = s->step_async(nsteps);
  s->prof_ms = nullptr;
  if (rc) return rc;
  API_CUDA(h, cudaStreamSynchronize(s->stream));
  *ms_pencil = ms[0];
  *ms_plane = ms[1];
  return SH_OK;
}

int sh_synchronize(sh_handle* h) {
  if (!h || !h->s) return SH_EINVAL;
  API_CUDA(h, cudaStreamSynchronize(h->s->stream));
  return SH_OK;
}

void* sh_stream(sh_handle* h) { return (h && h->s) ? static_cast<void*>(h->s->stream) : nullptr; }

long long sh_steps_taken(sh_handle* h) { return (h && h->s) ? h->s->steps : -1; }

int sh_residency(sh_handle* h, int* out) {
  ApiRange range_("sh_residency");
  if (!h || !h->s || !out) return fail(h, SH_EINVAL, "null argument");
  return h->s->residency(out);
}

int sh_kernel_launches(sh_handle* h, long long* count) {
  if (!h || !h->s || !count) return SH_EINVAL;
  *count = h->s->launches;
  return SH_OK;
}

const char* sh_last_error(sh_handle* h) {
  if (h && h->s) return h->s->err.c_str();
  return g_err.c_str();
}

}  // extern "C"
