// L1 relaxation monitor that allocates no device memory.
//
// sh_l1_noalloc computes the same value as the handle-based monitor behind
// sh_l1: L1 = sum|psi_new - psi_old| / (dt sum|psi_new|). The handle-based
// monitor accumulates the per-CTA partial sums in device buffers that
// sh_create allocates. This variant keeps those partial sums in a fixed
// file-scope device array instead. Some callers cannot let a library allocate:
//  - a host that owns device memory through its own pool allocator;
//  - a real-time loop that cannot afford the implicit device synchronisation
//    of cudaMalloc/cudaFree.
// Such a caller passes its own input fields and output buffer, and the call
// uses no other memory.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/smectic_b200.h"
#include "sh_common.cuh"

namespace shb {
void set_global_error(const std::string& msg);  // defined with the C-ABI (sh_api.cu)
}

namespace {

// Partial sums: kL1BlocksPerReplica blocks per replica, two sums per block.
constexpr int kL1BlocksPerReplica = 128;
constexpr int kL1ThreadsPerBlock = 256;
constexpr int kL1MaxReplicas = SH_L1_NOALLOC_MAX_BATCH;
constexpr int kL1ScratchDoubles = 2 * kL1BlocksPerReplica * kL1MaxReplicas;  // 32768 doubles = 256 KiB

// Scratch of the partial sums. Every GPU that loads the library holds it until
// the process exits. Host code must not pass the symbol itself to a kernel:
// on the host it names a host-side stand-in, so the kernel gets the device
// address returned by cudaGetSymbolAddress.
static __device__ __align__(256) double g_l1_scratch[kL1ScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

__global__ void l1_partial_kernel(const double* __restrict__ psi_new, const double* __restrict__ psi_old,
                                  long long n3, double* __restrict__ scratch) {
  __shared__ double red[32];
  const int rep = blockIdx.y;
  const double* a = psi_new + size_t(rep) * n3;
  const double* b = psi_old + size_t(rep) * n3;
  shb::KahanSum s0, s1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x) {
    const double x = a[i];
    s0.add(fabs(x - b[i]));
    s1.add(fabs(x));
  }
  const double t0 = shb::block_sum(s0.s, red);
  const double t1 = shb::block_sum(s1.s, red);
  if (threadIdx.x == 0) {
    // every slot this call reads is written here first: nothing needs zeroing
    double* o = scratch + (size_t(rep) * gridDim.x + blockIdx.x) * 2;
    o[0] = t0;
    o[1] = t1;
  }
}

__global__ void l1_finalize_kernel(const double* __restrict__ scratch, int nblocks, double dt, double* __restrict__ out) {
  __shared__ double red[32];
  const int rep = blockIdx.x;
  shb::KahanSum s0, s1;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    s0.add(scratch[(size_t(rep) * nblocks + b) * 2 + 0]);
    s1.add(scratch[(size_t(rep) * nblocks + b) * 2 + 1]);
  }
  const double a = shb::block_sum(s0.s, red);
  const double b = shb::block_sum(s1.s, red);
  if (threadIdx.x == 0) out[rep] = a / (dt * b);
}

int fail_noalloc(int code, const std::string& msg) {
  shb::set_global_error(msg);
  return code;
}

// Device address of the scratch on the current device; looked up on the first
// call on each device (with that device current) and cached.
int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_noalloc(SH_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail_noalloc(SH_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_l1_scratch);
    if (e != cudaSuccess || !p)
      return fail_noalloc(SH_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SH_OK;
}

}  // namespace

extern "C" {

int sh_l1_noalloc(const double* dev_psi_new, const double* dev_psi_old, long long n3, int batch, double dt,
                  double* dev_out, void* stream) {
  if (!dev_psi_new || !dev_psi_old || !dev_out) return fail_noalloc(SH_EINVAL, "null argument");
  if (n3 <= 0 || !(dt > 0)) return fail_noalloc(SH_EINVAL, "n3 must be positive and dt > 0");
  if (batch < 1 || batch > kL1MaxReplicas)
    return fail_noalloc(SH_EINVAL, "batch must be in [1, " + std::to_string(kL1MaxReplicas) +
                                       "]: the fixed scratch holds the partial sums of at most that many replicas");
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  l1_partial_kernel<<<dim3(kL1BlocksPerReplica, batch), kL1ThreadsPerBlock, 0, st>>>(dev_psi_new, dev_psi_old, n3,
                                                                                      scratch);
  l1_finalize_kernel<<<batch, kL1ThreadsPerBlock, 0, st>>>(scratch, kL1BlocksPerReplica, dt, dev_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_noalloc(SH_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  return SH_OK;
}

}  // extern "C"
