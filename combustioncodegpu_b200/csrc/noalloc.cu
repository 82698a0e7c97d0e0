// Residual reduction that allocates nothing: cc_residual_rms_noalloc.
//
// Some callers cannot call cudaMalloc at the point where they need the
// residual norms -- for example a host application that runs the solver
// inside its own memory pool or allocation-free real-time loop, or code that
// runs while another component owns the device allocator.  For them this
// entry point reduces caller-provided device arrays using a fixed scratch
// array that lives in the library image itself.
//
// The scratch is the file-scope array below (64 KiB).  Every GPU that loads
// the library holds it until the process exits.  Host code must not take its
// address directly: in host code the symbol is only a stand-in, so the first
// call on each device looks up the device address with cudaGetSymbolAddress
// (that first call should therefore come before any stream capture).  The
// address belongs to the device's current context: if that context is
// destroyed and a new one made (cudaDeviceReset, or a host application that
// resets the device), the module is loaded again at another address, so the
// cached address is keyed on the context's unique id and looked up again when
// the id changes.  Every call shares the array and it keeps the previous
// call's contents; each call writes every partial it later reads, so nothing
// needs clearing, but two calls whose work overlaps on the GPU race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cc_b200.h"

void ccb_set_last_error(const std::string &msg);  // api.cu: message returned by cc_last_error

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;                                   // points per thread
constexpr int64_t kPointsPerCta = (int64_t)kThreads * kItems;  // 4096
constexpr int kMaxPartials = CC_NOALLOC_MAX_POINTS / (int)kPointsPerCta;

static __device__ __align__(256) double g_partials[4 * kMaxPartials];

__global__ void k_partials(const double *__restrict__ cur, const double *__restrict__ last, int64_t n,
                           double *partials) {
  double acc[4] = {0, 0, 0, 0};
  const int64_t base = (int64_t)blockIdx.x * kPointsPerCta;
  for (int it = 0; it < kItems; ++it) {
    const int64_t g = base + (int64_t)it * kThreads + threadIdx.x;
    if (g < n)
      for (int l = 0; l < 4; ++l) {
        const double d = cur[l * n + g] - last[l * n + g];
        acc[l] += d * d;
      }
  }
  __shared__ double sh[4][kThreads];
  for (int l = 0; l < 4; ++l) sh[l][threadIdx.x] = acc[l];
  __syncthreads();
  for (int st = kThreads / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int l = 0; l < 4; ++l) sh[l][threadIdx.x] += sh[l][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int l = 0; l < 4; ++l) partials[4 * blockIdx.x + l] = sh[l][0];
}

__global__ void k_final(const double *partials, int n_partials, int64_t n, double *out) {
  if (threadIdx.x != 0) return;
  double r[4] = {0, 0, 0, 0};
  for (int b = 0; b < n_partials; ++b)
    for (int l = 0; l < 4; ++l) r[l] += partials[4 * b + l];
  for (int l = 0; l < 4; ++l) out[l] = sqrt(r[l] / (double)n);
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Scratch {
  unsigned long long ctx_id;  // context the address belongs to
  double *ptr;
};
Scratch g_scratch[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context (0 when it cannot be
// read).  The driver entry points are looked up once.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(fn);
    looked_up = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

int fail(int code, const std::string &msg) {
  ccb_set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int cc_residual_rms_noalloc(const double *cur, const double *last, int64_t n, double *out,
                                       void *stream) {
  if (!cur || !last || !out) return fail(CC_ERR_ARG, "cc_residual_rms_noalloc: null pointer");
  if (n <= 0 || n > CC_NOALLOC_MAX_POINTS)
    return fail(CC_ERR_ARG, "cc_residual_rms_noalloc: n = " + std::to_string(n) + " outside [1, " +
                                std::to_string(CC_NOALLOC_MAX_POINTS) +
                                "]: the fixed scratch holds one partial sum per 4096 points");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(CC_ERR_CUDA, std::string("cc_residual_rms_noalloc: no current device: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(CC_ERR_ARG, "cc_residual_rms_noalloc: device index " + std::to_string(dev) + " is not below " +
                                std::to_string(kMaxDevices) + ", the devices this entry point keeps an address for");
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long id = current_context_id();
    Scratch &sc = g_scratch[dev];
    if (!sc.ptr || id == 0 || sc.ctx_id != id) {
      // once per device and context, with that device current: the device
      // address of the static array (its host-side name is not a device
      // address)
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_partials);
      if (e != cudaSuccess || !p)
        return fail(CC_ERR_CUDA,
                    std::string("cc_residual_rms_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      sc.ptr = static_cast<double *>(p);
      sc.ctx_id = id;
    }
    scratch = sc.ptr;
  }
  const int grid = (int)((n + kPointsPerCta - 1) / kPointsPerCta);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_partials<<<grid, kThreads, 0, s>>>(cur, last, n, scratch);
  k_final<<<1, 32, 0, s>>>(scratch, grid, n, out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(CC_ERR_CUDA, std::string("cc_residual_rms_noalloc: launch failed: ") + cudaGetErrorString(e));
  return CC_OK;
}
