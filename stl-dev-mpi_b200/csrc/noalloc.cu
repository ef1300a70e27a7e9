// Allocation-free mean / var coefficients of maps already on the device.
//
// stlp_mean_var_noalloc is a variant of the level-0 mean / var sums of the
// coefficient products (k_products with the input maps, then
// k_reduce_partials): the per-block partial sums live in a fixed device
// array of this file instead of an engine buffer, and the call allocates no
// device or host memory (no cudaMalloc / cudaFree, no library routine that
// allocates).  It serves callers that must not allocate device memory at the
// point of the call: a host framework whose caching allocator has already
// reserved the device memory (a cudaMalloc there fails or makes the pool
// release cached blocks), and callers that keep a stream running without
// host synchronisation, for which cudaMalloc / cudaFree can add an implicit
// device-wide synchronisation.
//
// Coefficients, as the engine's MEAN and VAR families: mean = <x>,
// var = <x^2> over the pixels of each map, summed in FP64 in a fixed order
// (results are bit-reproducible run to run).
//
// Scratch: g_noalloc_partials holds kNoAllocMaxMaps x kNoAllocBlocks x 2
// doubles (296 KiB).  Every block writes its own partial before the final
// pass reads it, so nothing in the scratch has to start at zero and no
// clearing pass runs.  The scratch is one per device: two calls in flight at
// the same time on one device (overlapping streams, or host threads) race on
// it; order them on one stream or with events.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

namespace {

typedef int64_t i64;

constexpr int kNoAllocMaxMaps = 64;   // maps per call
constexpr int kNoAllocBlocks = 296;   // partial sums per map (2 blocks per SM)
constexpr int kNoAllocThreads = 256;
constexpr size_t kNoAllocScratch = (size_t)kNoAllocMaxMaps * kNoAllocBlocks * 2;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocScratch];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// per device: the context the address was looked up in, and the address
void* g_ctx[kMaxDevices] = {};
double* g_partials[kMaxDevices] = {};

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// The driver's current context (cuCtxGetCurrent through the runtime's entry
// point table, so the library needs no link to the driver library).  A
// device reset destroys the device's primary context, and the runtime makes
// a new one at the next call: the scratch then has another address.
void* current_context() {
  typedef int (*GetCtx)(void**);
  static GetCtx get = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCtx>(f);
  }();
  void* ctx = nullptr;
  if (!get || get(&ctx) != 0) throw std::runtime_error("cuCtxGetCurrent failed");
  return ctx;
}

// Device address of the scratch on the current device, looked up once per
// device and context (cudaGetSymbolAddress may load the module on that
// device).  The first call on a device -- and the first after a reset of
// the device -- therefore does this set-up; when the call is to be recorded
// in a stream capture, make one call on that device before the capture
// starts.
double* partials_on_current_device() {
  int dev = -1;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
  void* ctx = current_context();  // null before the runtime first binds a context on this thread
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_partials[dev] || !ctx || g_ctx[dev] != ctx) {
    void* p = nullptr;
    // binds the device's primary context when none is current
    check(cudaGetSymbolAddress(&p, g_noalloc_partials), "cudaGetSymbolAddress of the fixed scratch");
    g_partials[dev] = static_cast<double*>(p);
    g_ctx[dev] = current_context();
  }
  return g_partials[dev];
}

// block (j, b): sum x and x^2 of the pixels j T + t + i kNoAllocBlocks T of
// map b, then a fixed-order tree over the block's threads
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_mv_partials(const T* __restrict__ x, i64 n,
                                                                 double* __restrict__ part) {
  __shared__ double a1[kNoAllocThreads], a2[kNoAllocThreads];
  const int b = blockIdx.y, t = threadIdx.x;
  const T* xb = x + (i64)b * n;
  double s1 = 0.0, s2 = 0.0;
  for (i64 i = (i64)blockIdx.x * kNoAllocThreads + t; i < n; i += (i64)kNoAllocBlocks * kNoAllocThreads) {
    const double v = (double)xb[i];
    s1 += v;
    s2 = fma(v, v, s2);
  }
  a1[t] = s1;
  a2[t] = s2;
  __syncthreads();
  for (int h = kNoAllocThreads / 2; h > 0; h >>= 1) {
    if (t < h) {
      a1[t] += a1[t + h];
      a2[t] += a2[t + h];
    }
    __syncthreads();
  }
  if (t == 0) {
    double* p = part + ((i64)b * kNoAllocBlocks + blockIdx.x) * 2;
    p[0] = a1[0];
    p[1] = a2[0];
  }
}

// one warp per map: lane-strided sums of the partials, then a fixed
// butterfly; out[b] = (mean, var)
__global__ void k_mv_final(const double* __restrict__ part, i64 n, double* __restrict__ out) {
  const int b = blockIdx.x, lane = threadIdx.x;
  double s1 = 0.0, s2 = 0.0;
  for (int j = lane; j < kNoAllocBlocks; j += 32) {
    s1 += part[((i64)b * kNoAllocBlocks + j) * 2];
    s2 += part[((i64)b * kNoAllocBlocks + j) * 2 + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    out[2 * b] = s1 / (double)n;
    out[2 * b + 1] = s2 / (double)n;
  }
}

}  // namespace

extern "C" int stlp_mean_var_noalloc(uint64_t x, size_t n_pix, size_t batch, int f32, uint64_t out,
                                     uint64_t stream) {
  try {
    if (x == 0 || out == 0) throw std::runtime_error("null device pointer");
    if (n_pix == 0 || batch == 0) throw std::runtime_error("empty maps");
    if (batch > (size_t)kNoAllocMaxMaps)
      throw std::runtime_error("batch " + std::to_string(batch) + " exceeds the " +
                               std::to_string(kNoAllocMaxMaps) + " maps the fixed device scratch holds");
    if (n_pix > (size_t)INT64_MAX / batch) throw std::runtime_error("map size out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int dev = -1, sdev = -1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaStreamGetDevice(s, &sdev), "cudaStreamGetDevice");
    if (sdev != dev)
      throw std::runtime_error("the stream belongs to device " + std::to_string(sdev) + ", the current device is " +
                               std::to_string(dev) + ": make the stream's device current before the call");
    double* part = partials_on_current_device();
    const dim3 grid(kNoAllocBlocks, (unsigned)batch);
    if (f32)
      k_mv_partials<float><<<grid, kNoAllocThreads, 0, s>>>(reinterpret_cast<const float*>(x), (i64)n_pix, part);
    else
      k_mv_partials<double><<<grid, kNoAllocThreads, 0, s>>>(reinterpret_cast<const double*>(x), (i64)n_pix, part);
    check(cudaGetLastError(), "launch of the partial sums");
    k_mv_final<<<(unsigned)batch, 32, 0, s>>>(part, (i64)n_pix, reinterpret_cast<double*>(out));
    check(cudaGetLastError(), "launch of the final sums");
    return 0;
  } catch (const std::exception& e) {
    stl::set_error(e.what());
  } catch (...) {
    stl::set_error("unknown native failure");
  }
  return -1;
}
