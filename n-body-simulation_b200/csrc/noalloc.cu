// noalloc.cu -- the FP64 direct-sum check for callers that cannot allocate
// device memory.
//
// nbx_direct_fp64 (diag.cu, api.cu) keeps its partial sums in memory the
// handle allocates with cudaMalloc on first use.  Some callers cannot do
// that: their device memory belongs to another allocator (a framework's
// caching pool) or is budgeted once at start-up, or they run a loop that
// must not pay cudaMalloc's device-wide synchronisation (an interactive
// viewer, a solver step in a latency-bound pipeline).  They already hold
// the bodies and the outputs in device memory of their own.
//
// nbx_direct_fp64_noalloc serves them: it takes device pointers for every
// input and output and keeps its partial sums in `g_partial`, a file-scope
// __device__ array of fixed size (kNoallocMaxTargets targets x
// kNoallocChunks source chunks x 16 bytes = 4 MiB), which every GPU that
// loads this library holds until the process exits.  It calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// Notes for users:
//  * host code cannot use the array's name as a device address; the first
//    call on each device looks the address up (cudaGetSymbolAddress, with
//    that device current) and caches it.  Make that first call before any
//    stream capture on the device;
//  * all calls on a device share the one array.  Every partial sum is
//    written before it is read, so nothing needs to start at zero, but two
//    calls whose kernels overlap on the GPU (different streams, or
//    different host threads) race on it: order them on one stream;
//  * more than kNoallocMaxTargets targets is rejected with NBX_ERR_CAPACITY
//    before anything is launched;
//  * a target index outside 0..n-1 is never read through: its outputs are
//    NaN (the targets live in device memory, so the host cannot check them);
//  * it sums the tree law m d / (|d| (d^2 + eps^2)) over all n bodies it is
//    given (one contiguous body set), like nbx_direct_fp64 on a
//    single-instance handle with force_law 0; it has no Plummer law and no
//    per-instance source ranges;
//  * the cached address does not survive cudaDeviceReset: a process that
//    resets a device must not call it on that device again;
//  * launch failures are taken from the launch calls themselves, so an
//    error left pending by the caller's earlier CUDA calls is neither
//    reported as this call's nor cleared.
#include "nbx.h"

#include <cuda_runtime.h>

#include <mutex>

namespace {

constexpr uint32_t kNoallocMaxTargets = 4096;
constexpr int kNoallocChunks = 64;
constexpr int kThreads = 128;

static __device__ __align__(256) double2
    g_partial[kNoallocChunks * kNoallocMaxTargets];

// Partial FP64 sums of the tree force law for targets
// blockIdx.x*128 .. +127 over the sources of chunk blockIdx.y
// (exactTreeLawForces, CheckCuda.cu:453-475; the same summation as
// nbx_direct_fp64).
__global__ void __launch_bounds__(kThreads)
    k_noalloc_partial(const float *__restrict__ x, const float *__restrict__ y,
                      const float *__restrict__ m, uint32_t n,
                      const uint32_t *__restrict__ targets, uint32_t nt,
                      double eSq, double2 *__restrict__ partial) {
  __shared__ float4 src[kThreads];
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t ti = t < nt ? targets[t] : 0u;
  // an index outside the body array is not read through (its sums are
  // replaced by NaN below)
  const bool inRange = ti < n;
  const bool valid = t < nt && inRange;
  const double px = valid ? (double)x[ti] : 0.0;
  const double py = valid ? (double)y[ti] : 0.0;
  const uint32_t chunk = (n + gridDim.y - 1) / gridDim.y;
  const uint32_t j0 = blockIdx.y * chunk;
  const uint32_t j1 = min(n, j0 + chunk);
  double ax = 0.0, ay = 0.0;
  for (uint32_t base = j0; base < j1; base += kThreads) {
    const uint32_t j = base + threadIdx.x;
    __syncthreads();
    if (j < j1) src[threadIdx.x] = make_float4(x[j], y[j], m[j], __uint_as_float(j));
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kThreads, j1 - base);
    if (valid) {
      for (uint32_t k = 0; k < cnt; ++k) {
        const float4 s = src[k];
        if (__float_as_uint(s.w) == ti) continue;
        const double dx = (double)s.x - px;
        const double dy = (double)s.y - py;
        const double dSq = dx * dx + dy * dy;
        if (dSq == 0.0) continue;
        const double f = (double)s.z / (sqrt(dSq) * (dSq + eSq));
        ax += dx * f;
        ay += dy * f;
      }
    }
  }
  if (t < nt) {
    const double bad = __longlong_as_double(0x7ff8000000000000ll); // quiet NaN
    partial[(size_t)blockIdx.y * nt + t] =
        inRange ? make_double2(ax, ay) : make_double2(bad, bad);
  }
}

__global__ void k_noalloc_reduce(const double2 *__restrict__ partial, uint32_t nt,
                                 double *ax, double *ay) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double sx = 0.0, sy = 0.0;
  for (int c = 0; c < kNoallocChunks; ++c) {
    const double2 v = partial[(size_t)c * nt + t];
    sx += v.x;
    sy += v.y;
  }
  ax[t] = sx;
  ay[t] = sy;
}

// Per-device address of g_partial, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_setupLock;
void *g_partialAddr[kMaxDevices] = {};

int partial_address(int device, double2 **out) {
  if (device < 0 || device >= kMaxDevices) return NBX_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setupLock);
  if (!g_partialAddr[device]) {
    void *p = nullptr;
    // the device is current here (the caller's current device)
    if (cudaGetSymbolAddress(&p, g_partial) != cudaSuccess || !p)
      return NBX_ERR_CUDA;
    g_partialAddr[device] = p;
  }
  *out = static_cast<double2 *>(g_partialAddr[device]);
  return NBX_OK;
}

} // namespace

extern "C" int nbx_direct_fp64_noalloc(const float *x, const float *y,
                                       const float *mass, uint32_t n,
                                       const uint32_t *targets, uint32_t m,
                                       double epsilon, double *ax, double *ay,
                                       void *stream) {
  if (m == 0) return NBX_OK;
  if (!x || !y || !mass || !targets || !ax || !ay) return NBX_ERR_ARG;
  if (m > kNoallocMaxTargets) return NBX_ERR_CAPACITY;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return NBX_ERR_CUDA;
  double2 *partial = nullptr;
  const int rc = partial_address(device, &partial);
  if (rc != NBX_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // each launch's own return code: an error the caller left pending is not
  // this call's to report or to clear
  double eSq = epsilon * epsilon;
  void *argsPartial[] = {(void *)&x, (void *)&y, (void *)&mass, (void *)&n,
                         (void *)&targets, (void *)&m, (void *)&eSq,
                         (void *)&partial};
  if (cudaLaunchKernel((const void *)k_noalloc_partial,
                       dim3((m + kThreads - 1) / kThreads, kNoallocChunks),
                       dim3(kThreads), argsPartial, 0, s) != cudaSuccess)
    return NBX_ERR_CUDA;
  const double2 *part = partial;
  void *argsReduce[] = {(void *)&part, (void *)&m, (void *)&ax, (void *)&ay};
  if (cudaLaunchKernel((const void *)k_noalloc_reduce, dim3((m + 255) / 256),
                       dim3(256), argsReduce, 0, s) != cudaSuccess)
    return NBX_ERR_CUDA;
  return NBX_OK;
}
