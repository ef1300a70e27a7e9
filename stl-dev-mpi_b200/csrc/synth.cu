// Map synthesis with every vector on the device: L-BFGS (the steps of
// lbfgs.hpp) of the loss sum_k w_k |S_k(x) - T_k|^2 over maps x held in
// device memory, the objective evaluated by the engine on its own stream.
// This is the loop of the reference's synthesis (crates/stl-mpi/src/
// synthesis.rs:207-316: weighted squared residual of the statistics, its
// gradient by the VJP, L-BFGS of crates/stl-core/src/lbfgs.rs:250-470)
// with the iterate, gradients and curvature pairs resident in HBM instead of
// host memory, so an iteration moves no map across PCIe.
//
// Vector operations are FP64.  Reductions (dots, |.|_1, |.|_inf) split the
// vector into a fixed number of equal ranges, sum each range in a fixed
// order and add the ranges in index order: results do not depend on launch
// timing.  Each reduction returns its scalar to the host (the line search
// branches on it); the vectors stay on the device.
#include <cmath>
#include <stdexcept>
#include <vector>

#include "engine.cuh"
#include "lbfgs.hpp"
#include "scatcov.hpp"

namespace stl {

namespace {

constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 512;
constexpr int kVecThreads = 256;

__global__ void k_vec_neg(double* __restrict__ o, const double* __restrict__ a, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = -a[i];
}
__global__ void k_vec_sub(double* __restrict__ o, const double* __restrict__ a, const double* __restrict__ b,
                          i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = a[i] - b[i];
}
__global__ void k_vec_scale(double* __restrict__ o, const double* __restrict__ a, double c, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = a[i] * c;
}
__global__ void k_vec_fma3(double* __restrict__ o, const double* __restrict__ d, double t,
                           const double* __restrict__ x0, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = fma(d[i], t, x0[i]);
}
// p = fma(u, a, p); p may not alias u
__global__ void k_vec_axpy(double* __restrict__ p, double a, const double* __restrict__ u, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = fma(u[i], a, p[i]);
}

enum { RED_DOT = 0, RED_ABS_SUM = 1, RED_ABS_MAX = 2, RED_NONFINITE = 3 };

template <int OP>
__device__ __forceinline__ double red_term(const double* a, const double* b, i64 i) {
  if (OP == RED_DOT) return a[i] * b[i];
  if (OP == RED_ABS_SUM || OP == RED_ABS_MAX) return fabs(a[i]);
  return isfinite(a[i]) ? 0.0 : 1.0;
}
template <int OP>
__device__ __forceinline__ double red_join(double x, double y) {
  return OP == RED_ABS_MAX ? fmax(x, y) : x + y;
}

// range k = [k chunk, (k + 1) chunk) of [0, n): thread-strided terms in
// order, then a tree over the block, in a fixed order
template <int OP>
__global__ void __launch_bounds__(kRedThreads) k_vec_reduce(const double* __restrict__ a,
                                                            const double* __restrict__ b, i64 n, i64 chunk,
                                                            double* __restrict__ part) {
  __shared__ double red[kRedThreads];
  const i64 lo = (i64)blockIdx.x * chunk, hi = min(n, lo + chunk);
  double s = 0.0;
  for (i64 i = lo + threadIdx.x; i < hi; i += kRedThreads) s = red_join<OP>(s, red_term<OP>(a, b, i));
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kRedThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] = red_join<OP>(red[threadIdx.x], red[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

template <int OP>
__global__ void k_vec_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k < np; ++k) s = red_join<OP>(s, part[k]);
  *out = s;
}

unsigned vec_blocks(size_t n) { return (unsigned)((n + kVecThreads - 1) / kVecThreads); }

// Device vectors of one length from a pool: a vector returns its buffer to
// the pool when it dies, so the steps of an iteration allocate nothing.
struct Pool {
  size_t n = 0;
  std::vector<DevMem> owned;
  std::vector<double*> free;
  double* get() {
    if (free.empty()) {
      owned.emplace_back(sizeof(double) * n);
      return owned.back().as<double>();
    }
    double* p = free.back();
    free.pop_back();
    return p;
  }
  void put(double* p) { free.push_back(p); }
};

struct DVec {
  double* p = nullptr;
  Pool* pool = nullptr;
  DVec() = default;
  DVec(double* q, Pool* o) : p(q), pool(o) {}
  DVec(const DVec&) = delete;
  DVec& operator=(const DVec&) = delete;
  DVec(DVec&& o) noexcept : p(o.p), pool(o.pool) { o.p = nullptr; }
  DVec& operator=(DVec&& o) noexcept {
    if (this != &o) {
      if (p && pool) pool->put(p);
      p = o.p;
      pool = o.pool;
      o.p = nullptr;
    }
    return *this;
  }
  ~DVec() {
    if (p && pool) pool->put(p);
  }
};

struct DeviceOps {
  typedef DVec Vec;
  Pool pool;
  cudaStream_t s = nullptr;
  DevMem part{sizeof(double) * kRedBlocks}, res{sizeof(double)};
  explicit DeviceOps(size_t n, cudaStream_t st) : s(st) { pool.n = n; }
  size_t n() const { return pool.n; }
  Vec make(size_t n_) {
    if (n_ != pool.n) throw std::runtime_error("device vector of another length");
    return DVec(pool.get(), &pool);
  }
  // a view of caller memory (not returned to the pool)
  Vec view(double* p) { return DVec(p, nullptr); }
  void copy(Vec& dst, const Vec& src) {
    STL_CUDA(cudaMemcpyAsync(dst.p, src.p, sizeof(double) * n(), cudaMemcpyDeviceToDevice, s));
  }
  void neg(Vec& o, const Vec& a) { k_vec_neg<<<vec_blocks(n()), kVecThreads, 0, s>>>(o.p, a.p, (i64)n()); check(); }
  void sub(Vec& o, const Vec& a, const Vec& b) {
    k_vec_sub<<<vec_blocks(n()), kVecThreads, 0, s>>>(o.p, a.p, b.p, (i64)n());
    check();
  }
  void scale(Vec& o, const Vec& a, double c) {
    k_vec_scale<<<vec_blocks(n()), kVecThreads, 0, s>>>(o.p, a.p, c, (i64)n());
    check();
  }
  void fma3(Vec& o, const Vec& d, double t, const Vec& x0) {
    k_vec_fma3<<<vec_blocks(n()), kVecThreads, 0, s>>>(o.p, d.p, t, x0.p, (i64)n());
    check();
  }
  void axpy(Vec& p, double a, const Vec& u) {
    k_vec_axpy<<<vec_blocks(n()), kVecThreads, 0, s>>>(p.p, a, u.p, (i64)n());
    check();
  }
  template <int OP>
  double reduce(const double* a, const double* b) {
    const i64 chunk = ((i64)n() + kRedBlocks - 1) / kRedBlocks;
    k_vec_reduce<OP><<<kRedBlocks, kRedThreads, 0, s>>>(a, b, (i64)n(), chunk, part.as<double>());
    k_vec_final<OP><<<1, 32, 0, s>>>(part.as<double>(), kRedBlocks, res.as<double>());
    check();
    double h = 0.0;
    STL_CUDA(cudaMemcpyAsync(&h, res.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    return h;
  }
  double dot(const Vec& a, const Vec& b) { return reduce<RED_DOT>(a.p, b.p); }
  double abs_sum(const Vec& a) { return reduce<RED_ABS_SUM>(a.p, a.p); }
  double abs_max(const Vec& a) { return reduce<RED_ABS_MAX>(a.p, a.p); }
  double nonfinite(const double* a) { return reduce<RED_NONFINITE>(a, a); }
  static void check() { STL_CUDA(cudaGetLastError()); }
};

// loss sum_i w_(i mod np) |S_i(x) - T_i|^2 and its gradient, both from the
// engine (maps loaded from device memory, cotangent 2 w (S - T))
struct SynthObjective {
  Engine& e;
  DeviceOps& ops;
  const double* target;   // complex interleaved [values]
  const double* weights;  // [np] or null
  size_t nv = 0, np = 0;
  std::vector<double> values, cot;
  std::vector<double>* losses;
  double operator()(const DVec& x, DVec& g) {
    e.load_device(x.p, false);
    e.forward(false, values.data(), nullptr);
    double loss = 0.0;
    for (size_t i = 0; i < nv; ++i) {
      const double w = weights ? weights[i % np] : 1.0;
      const double rr = values[2 * i] - target[2 * i], ri = values[2 * i + 1] - target[2 * i + 1];
      loss += w * (rr * rr + ri * ri);
      cot[2 * i] = 2.0 * w * rr;
      cot[2 * i + 1] = 2.0 * w * ri;
    }
    e.reverse_device(cot.data(), g.p, false);
    if (!std::isfinite(loss) || ops.nonfinite(g.p) != 0.0)
      throw std::runtime_error("non-finite synthesis loss or gradient");
    if (losses) losses->push_back(loss);
    return loss;
  }
};

}  // namespace

long long synthesize_device(Engine& e, double* x, size_t n, const double* target, const double* weights,
                            const lbfgs::Options& o, std::vector<double>* losses) {
  const size_t np = e.plan().size();
  const size_t nv = (size_t)e.options().B * std::max(1, e.nmasks()) * np;
  if (n != (size_t)e.options().B * (size_t)e.npix(0)) throw std::runtime_error("synthesis: map shape mismatch");
  DeviceOps ops(n, e.stream());
  SynthObjective obj{e, ops, target, weights, nv, np, std::vector<double>(2 * nv), std::vector<double>(2 * nv),
                     losses};
  DVec xv = ops.view(x);
  const long long evals = lbfgs::minimize(ops, xv, n, o, obj);
  STL_CUDA(cudaStreamSynchronize(e.stream()));
  return evals;
}

}  // namespace stl
