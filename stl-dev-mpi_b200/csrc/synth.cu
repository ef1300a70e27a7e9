// Map synthesis with every vector on the device: L-BFGS (the steps of
// lbfgs.hpp) of the loss sum_k w_k |S_k(x) - T_k|^2 over maps x held in
// device memory, the objective evaluated by the engine on the device
// (Engine::objective: forward, loss, cotangents and reverse sweep with no
// host round trip).  This is the loop of the reference's synthesis
// (crates/stl-mpi/src/synthesis.rs:207-316: weighted squared residual of the
// statistics, its gradient by the VJP, L-BFGS of
// crates/stl-core/src/lbfgs.rs:250-470) with the iterate, gradients and
// curvature pairs resident in HBM instead of host memory.
//
// Vector operations are FP64.  Reductions (dots, |.|_1, |.|_inf) split the
// vector into a fixed number of equal ranges, sum each range in a fixed
// order and add the ranges in index order: results do not depend on launch
// timing.
//
// Graph mode (the default): iteration 1 runs step by step; every later
// iteration is one CUDA graph launch -- the new curvature pair (kept when
// y.s > 1e-10), the two-loop recursion over a ring of history + 1 pair slots
// with every scalar (rho, alpha, beta, the scaling y.s / y.y) in device
// memory, g.d, the first trial point x0 + lr d, its objective, gradient
// slope, |g|_inf and finiteness -- followed by one copy of those scalars to
// the host.  The host runs the strong Wolfe test on them; only when the
// first trial fails does the search continue step by step.  The arithmetic
// is that of the step-by-step path (same reductions, same order, products
// rounded before they are added), so both give the same iterates.
#include <cmath>
#include <cstring>
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

// loss and gradient from the engine's device objective: one copy of the
// loss, the gradient's finiteness and the error flag to the host per call
struct SynthObjective {
  Engine& e;
  DeviceOps& ops;
  double* sc;      // device: loss, non-finite count
  PinnedMem& pin;  // host: the same, then the error flag
  std::vector<double>* losses;
  double operator()(const DVec& x, DVec& g) {
    cudaStream_t s = ops.s;
    e.objective(x.p, g.p, sc);
    const i64 chunk = ((i64)ops.n() + kRedBlocks - 1) / kRedBlocks;
    k_vec_reduce<RED_NONFINITE><<<kRedBlocks, kRedThreads, 0, s>>>(g.p, g.p, (i64)ops.n(), chunk,
                                                                   ops.part.as<double>());
    k_vec_final<RED_NONFINITE><<<1, 32, 0, s>>>(ops.part.as<double>(), kRedBlocks, sc + 1);
    DeviceOps::check();
    double* h = static_cast<double*>(pin.p);
    STL_CUDA(cudaMemcpyAsync(h, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaMemcpyAsync(h + 2, e.error_flag(), sizeof(int), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    int err = 0;
    std::memcpy(&err, h + 2, sizeof(int));
    if (err) {
      STL_CUDA(cudaMemsetAsync(e.error_flag(), 0, sizeof(int), s));
      throw std::runtime_error(wait_timeout_message(err, "the synthesis objective"));
    }
    const double loss = h[0];
    if (!std::isfinite(loss) || h[1] != 0.0) throw std::runtime_error("non-finite synthesis loss or gradient");
    if (losses) losses->push_back(loss);
    return loss;
  }
};

// ---- graph mode ---------------------------------------------------------------
// device scalars of an iteration
enum { SC_T = 0, SC_YS, SC_YY, SC_HDIAG, SC_GTD, SC_FNEW, SC_GTDNEW, SC_DNORM, SC_GMAX, SC_NONFIN, SC_COEF, SC_N };

// slot of the j-th newest pair (mode 0), the j-th oldest (1), or the next
// free slot (2) of a ring of P slots holding ring[0] pairs, next free at ring[1]
__device__ __forceinline__ int ring_slot(const int* ring, int j, int mode, int P) {
  const int count = ring[0], head = ring[1];
  if (mode == 2) return head;
  return mode == 0 ? (head - 1 - j + 2 * P) % P : (head - count + j + 2 * P) % P;
}

// partial dots of the ring vector a (slot of (j, mode)) with b (a ring
// vector of the same slot when b_ring), as k_vec_reduce; nothing when pair j
// does not exist
__global__ void __launch_bounds__(kRedThreads) k_ring_dot(const double* __restrict__ A, const double* __restrict__ Bv,
                                                          int b_ring, i64 n, i64 chunk, const int* __restrict__ ring,
                                                          int j, int mode, int P, double* __restrict__ part) {
  if (mode != 2 && j >= ring[0]) return;
  const i64 off = (i64)ring_slot(ring, j, mode, P) * n;
  const double* a = A + off;
  const double* b = b_ring ? Bv + off : Bv;
  __shared__ double red[kRedThreads];
  const i64 lo = (i64)blockIdx.x * chunk, hi = min(n, lo + chunk);
  double s = 0.0;
  for (i64 i = lo + threadIdx.x; i < hi; i += kRedThreads) s = red_join<RED_DOT>(s, red_term<RED_DOT>(a, b, i));
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kRedThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] = red_join<RED_DOT>(red[threadIdx.x], red[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// alpha of the j-th newest pair: (s . q) rho
__global__ void k_ring_alpha(const double* __restrict__ part, int np, const int* __restrict__ ring, int j, int P,
                             const double* __restrict__ ro, double* __restrict__ al) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || j >= ring[0]) return;
  double s = 0.0;
  for (int k = 0; k < np; ++k) s = red_join<RED_DOT>(s, part[k]);
  const int slot = ring_slot(ring, j, 0, P);
  al[slot] = __dmul_rn(s, ro[slot]);
}

// alpha - beta of the j-th oldest pair, beta = (y . d) rho rounded before
// the subtraction (no fused multiply-add), as the step-by-step path does
__global__ void k_ring_beta(const double* __restrict__ part, int np, const int* __restrict__ ring, int j, int P,
                            const double* __restrict__ ro, const double* __restrict__ al, double* __restrict__ sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || j >= ring[0]) return;
  double s = 0.0;
  for (int k = 0; k < np; ++k) s = red_join<RED_DOT>(s, part[k]);
  const int slot = ring_slot(ring, j, 1, P);
  sc[SC_COEF] = __dsub_rn(al[slot], __dmul_rn(s, ro[slot]));
}

// q = fma(y, -alpha, q) for the j-th newest pair
__global__ void k_ring_axpy_alpha(double* __restrict__ q, const double* __restrict__ Y, i64 n,
                                  const int* __restrict__ ring, int j, int P, const double* __restrict__ al) {
  if (j >= ring[0]) return;
  const int slot = ring_slot(ring, j, 0, P);
  const double a = -al[slot];
  const double* y = Y + (i64)slot * n;
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) q[i] = fma(y[i], a, q[i]);
}

// d = fma(s, alpha - beta, d) for the j-th oldest pair
__global__ void k_ring_axpy_coef(double* __restrict__ d, const double* __restrict__ S, i64 n,
                                 const int* __restrict__ ring, int j, int P, const double* __restrict__ sc) {
  if (j >= ring[0]) return;
  const int slot = ring_slot(ring, j, 1, P);
  const double a = sc[SC_COEF];
  const double* sv = S + (i64)slot * n;
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = fma(sv[i], a, d[i]);
}

// the candidate pair into the free slot: y = g - g_prev, s = d t
__global__ void k_ring_write(double* __restrict__ Y, double* __restrict__ S, const double* __restrict__ g,
                             const double* __restrict__ g_prev, const double* __restrict__ d,
                             const double* __restrict__ sc, const int* __restrict__ ring, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const i64 off = (i64)ring[1] * n;
  Y[off + i] = g[i] - g_prev[i];
  S[off + i] = d[i] * sc[SC_T];
}

// keep the candidate when y.s > 1e-10: rho = 1 / y.s, scaling y.s / y.y;
// the oldest pair leaves when m are held
__global__ void k_ring_commit(int* __restrict__ ring, double* __restrict__ ro, double* __restrict__ sc, int P, int m) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double ys = sc[SC_YS];
  if (ys > 1e-10) {
    const int head = ring[1];
    ro[head] = 1.0 / ys;
    sc[SC_HDIAG] = ys / sc[SC_YY];
    ring[1] = (head + 1) % P;
    ring[0] = min(ring[0] + 1, m);
  }
}

// o = a c[0]
__global__ void k_vec_scale_dev(double* __restrict__ o, const double* __restrict__ a, const double* __restrict__ c,
                                i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = a[i] * c[0];
}

// Buffers and the captured graph of one synthesis run.
struct GraphIteration {
  size_t n = 0;
  int m = 0, P = 0;
  DevMem ring_y, ring_s, ring, ro, al, sc;
  DevMem g, g_prev, d, q, x0, xt, g_new;
  PinnedMem param, out;  // host: t; the scalars, then the error flag
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GraphIteration(size_t n_, int m_) : n(n_), m(m_), P(m_ + 1) {
    ring_y.alloc(sizeof(double) * P * n);
    ring_s.alloc(sizeof(double) * P * n);
    ring.alloc(2 * sizeof(int));
    ro.alloc(sizeof(double) * P);
    al.alloc(sizeof(double) * P);
    sc.alloc(sizeof(double) * SC_N);
    for (DevMem* v : {&g, &g_prev, &d, &q, &x0, &xt, &g_new}) v->alloc(sizeof(double) * n);
    param.alloc(sizeof(double));
    out.alloc(sizeof(double) * SC_N + sizeof(int));
  }
  ~GraphIteration() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  double* scal(int i) { return sc.as<double>() + i; }
  const double* host() const { return static_cast<const double*>(out.p); }

  void reset(cudaStream_t s) {
    STL_CUDA(cudaMemsetAsync(ring.p, 0, 2 * sizeof(int), s));
    const double one = 1.0;  // the initial scaling
    STL_CUDA(cudaMemcpyAsync(scal(SC_HDIAG), &one, sizeof(double), cudaMemcpyHostToDevice, s));
    STL_CUDA(cudaStreamSynchronize(s));
  }

  // the launches of one iteration (it >= 2), x the iterate, lr the step
  void record(Engine& e, DeviceOps& ops, double* x, double lr) {
    cudaStream_t s = ops.s;
    const i64 N = (i64)n, chunk = (N + kRedBlocks - 1) / kRedBlocks;
    double* part = ops.part.as<double>();
    const int* rg = ring.as<int>();
    const unsigned vb = vec_blocks(n);
    auto dot_to = [&](const double* a, const double* b, int slot_sc) {
      k_vec_reduce<RED_DOT><<<kRedBlocks, kRedThreads, 0, s>>>(a, b, N, chunk, part);
      k_vec_final<RED_DOT><<<1, 32, 0, s>>>(part, kRedBlocks, scal(slot_sc));
    };
    auto max_to = [&](const double* a, int slot_sc) {
      k_vec_reduce<RED_ABS_MAX><<<kRedBlocks, kRedThreads, 0, s>>>(a, a, N, chunk, part);
      k_vec_final<RED_ABS_MAX><<<1, 32, 0, s>>>(part, kRedBlocks, scal(slot_sc));
    };
    STL_CUDA(cudaMemcpyAsync(scal(SC_T), param.p, sizeof(double), cudaMemcpyHostToDevice, s));
    // the curvature pair of the last step
    k_ring_write<<<vb, kVecThreads, 0, s>>>(ring_y.as<double>(), ring_s.as<double>(), g.as<double>(),
                                            g_prev.as<double>(), d.as<double>(), sc.as<double>(), rg, N);
    k_ring_dot<<<kRedBlocks, kRedThreads, 0, s>>>(ring_y.as<double>(), ring_s.as<double>(), 1, N, chunk, rg, 0, 2, P,
                                                  part);
    k_vec_final<RED_DOT><<<1, 32, 0, s>>>(part, kRedBlocks, scal(SC_YS));
    k_ring_dot<<<kRedBlocks, kRedThreads, 0, s>>>(ring_y.as<double>(), ring_y.as<double>(), 1, N, chunk, rg, 0, 2, P,
                                                  part);
    k_vec_final<RED_DOT><<<1, 32, 0, s>>>(part, kRedBlocks, scal(SC_YY));
    k_ring_commit<<<1, 32, 0, s>>>(ring.as<int>(), ro.as<double>(), sc.as<double>(), P, m);
    // two-loop recursion
    k_vec_neg<<<vb, kVecThreads, 0, s>>>(q.as<double>(), g.as<double>(), N);
    for (int j = 0; j < m; ++j) {
      k_ring_dot<<<kRedBlocks, kRedThreads, 0, s>>>(ring_s.as<double>(), q.as<double>(), 0, N, chunk, rg, j, 0, P,
                                                    part);
      k_ring_alpha<<<1, 32, 0, s>>>(part, kRedBlocks, rg, j, P, ro.as<double>(), al.as<double>());
      k_ring_axpy_alpha<<<vb, kVecThreads, 0, s>>>(q.as<double>(), ring_y.as<double>(), N, rg, j, P, al.as<double>());
    }
    k_vec_scale_dev<<<vb, kVecThreads, 0, s>>>(d.as<double>(), q.as<double>(), scal(SC_HDIAG), N);
    for (int j = 0; j < m; ++j) {
      k_ring_dot<<<kRedBlocks, kRedThreads, 0, s>>>(ring_y.as<double>(), d.as<double>(), 0, N, chunk, rg, j, 1, P,
                                                    part);
      k_ring_beta<<<1, 32, 0, s>>>(part, kRedBlocks, rg, j, P, ro.as<double>(), al.as<double>(), sc.as<double>());
      k_ring_axpy_coef<<<vb, kVecThreads, 0, s>>>(d.as<double>(), ring_s.as<double>(), N, rg, j, P, sc.as<double>());
    }
    STL_CUDA(cudaMemcpyAsync(g_prev.p, g.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    dot_to(g.as<double>(), d.as<double>(), SC_GTD);
    STL_CUDA(cudaMemcpyAsync(x0.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    // the first trial of the line search
    max_to(d.as<double>(), SC_DNORM);
    k_vec_fma3<<<vb, kVecThreads, 0, s>>>(xt.as<double>(), d.as<double>(), lr, x0.as<double>(), N);
    e.objective(xt.as<double>(), g_new.as<double>(), scal(SC_FNEW));
    dot_to(g_new.as<double>(), d.as<double>(), SC_GTDNEW);
    max_to(g_new.as<double>(), SC_GMAX);
    k_vec_reduce<RED_NONFINITE><<<kRedBlocks, kRedThreads, 0, s>>>(g_new.as<double>(), g_new.as<double>(), N, chunk,
                                                                   part);
    k_vec_final<RED_NONFINITE><<<1, 32, 0, s>>>(part, kRedBlocks, scal(SC_NONFIN));
    STL_CUDA(cudaMemcpyAsync(out.p, sc.p, sizeof(double) * SC_N, cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaMemcpyAsync(static_cast<char*>(out.p) + sizeof(double) * SC_N, e.error_flag(), sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    DeviceOps::check();
  }

  void capture(Engine& e, DeviceOps& ops, double* x, double lr) {
    STL_CUDA(cudaStreamBeginCapture(ops.s, cudaStreamCaptureModeThreadLocal));
    try {
      record(e, ops, x, lr);
    } catch (...) {
      cudaGraph_t g_ = nullptr;
      cudaStreamEndCapture(ops.s, &g_);
      if (g_) cudaGraphDestroy(g_);
      throw;
    }
    STL_CUDA(cudaStreamEndCapture(ops.s, &graph));
    STL_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  }

  // one iteration from the previous step t; the scalars are then on the host
  void launch(cudaStream_t s, double t) {
    *static_cast<double*>(param.p) = t;
    STL_CUDA(cudaGraphLaunch(exec, s));
    STL_CUDA(cudaStreamSynchronize(s));
  }
  int err() const {
    int v = 0;
    std::memcpy(&v, static_cast<const char*>(out.p) + sizeof(double) * SC_N, sizeof(int));
    return v;
  }
};

// lbfgs::minimize with iterations 2 on from the graph (same steps and
// arithmetic); x: the iterate (device)
long long minimize_graph(Engine& e, DeviceOps& ops, SynthObjective& obj, double* x, size_t n,
                         const lbfgs::Options& o) {
  using lbfgs::py_min;
  const long long max_eval = o.max_eval >= 0 ? o.max_eval : o.max_iter * 5 / 4;
  GraphIteration G(n, (int)o.history);
  G.reset(ops.s);
  DVec xv = ops.view(x), g = ops.view(G.g.as<double>()), d = ops.view(G.d.as<double>());
  DVec prev_g = ops.view(G.g_prev.as<double>()), x0 = ops.view(G.x0.as<double>());
  double loss = obj(xv, g);
  long long evals = 1;
  if (ops.abs_max(g) <= o.tol_grad) return evals;
  // iteration 1, step by step
  ops.neg(d, g);
  ops.copy(prev_g, g);
  double t = py_min(1.0, 1.0 / ops.abs_sum(g)) * o.lr;
  double gtd = ops.dot(g, d);
  if (gtd > -o.tol_change) return evals;
  ops.copy(x0, xv);
  {
    const double prev_loss = loss;
    lbfgs::LineResult<DVec> r = lbfgs::strong_wolfe(ops, obj, x0, d, t, loss, g, gtd, max_eval - evals, n);
    loss = r.f;
    ops.copy(g, r.g);
    t = r.t;
    ops.fma3(xv, d, t, x0);
    evals += r.evals;
    const bool opt = ops.abs_max(g) <= o.tol_grad;
    if (o.max_iter == 1 || evals >= max_eval || opt) return evals;
    if (ops.abs_max(d) * std::fabs(t) <= o.tol_change) return evals;
    if (std::fabs(loss - prev_loss) < o.tol_change) return evals;
  }
  // iterations 2 on: one graph launch each
  G.capture(e, ops, x, o.lr);
  DVec g_new = ops.view(G.g_new.as<double>());
  for (long long it = 2; it <= o.max_iter; ++it) {
    G.launch(ops.s, t);
    const double* h = G.host();
    if (const int err = G.err()) {
      STL_CUDA(cudaMemsetAsync(e.error_flag(), 0, sizeof(int), ops.s));
      throw std::runtime_error(wait_timeout_message(err, "the synthesis objective"));
    }
    const double prev_loss = loss;
    gtd = h[SC_GTD];
    if (gtd > -o.tol_change) break;  // before any trial: the speculative one is not counted
    if (!std::isfinite(h[SC_FNEW]) || h[SC_NONFIN] != 0.0)
      throw std::runtime_error("non-finite synthesis loss or gradient");
    if (obj.losses) obj.losses->push_back(h[SC_FNEW]);
    const lbfgs::FirstTrial<DVec> first{h[SC_FNEW], h[SC_GTDNEW], h[SC_DNORM], &g_new};
    const double d_norm = h[SC_DNORM], gmax_first = h[SC_GMAX];
    lbfgs::LineResult<DVec> r =
        lbfgs::strong_wolfe(ops, obj, x0, d, o.lr, loss, g, gtd, max_eval - evals, n, &first);
    loss = r.f;
    ops.copy(g, r.g);
    const bool first_taken = r.evals == 1 && r.t == o.lr;  // then g is the trial's gradient
    t = r.t;
    ops.fma3(xv, d, t, x0);
    evals += r.evals;
    const bool opt = (first_taken ? gmax_first : ops.abs_max(g)) <= o.tol_grad;
    if (it == o.max_iter || evals >= max_eval || opt) break;
    if (d_norm * std::fabs(t) <= o.tol_change) break;
    if (std::fabs(loss - prev_loss) < o.tol_change) break;
  }
  return evals;
}

}  // namespace

long long synthesize_device(Engine& e, double* x, size_t n, const double* target, const double* weights,
                            const lbfgs::Options& o, std::vector<double>* losses) {
  if (n != (size_t)e.options().B * (size_t)e.npix(0)) throw std::runtime_error("synthesis: map shape mismatch");
  // a stream of its own (a graph is captured from it), profiling off
  cudaStream_t s = nullptr, prev = e.stream();
  STL_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const bool prof = e.profiling();
  e.set_profiling(false);
  e.set_stream(s);
  long long evals = 0;
  try {
    e.set_objective(target, weights);
    DeviceOps ops(n, s);
    DevMem sc(2 * sizeof(double));
    PinnedMem pin;
    pin.alloc(2 * sizeof(double) + sizeof(int));
    SynthObjective obj{e, ops, sc.as<double>(), pin, losses};
    if (o.graph) {
      evals = minimize_graph(e, ops, obj, x, n, o);
    } else {
      DVec xv = ops.view(x);
      evals = lbfgs::minimize(ops, xv, n, o, obj);
    }
    STL_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    e.set_stream(prev);
    e.set_profiling(prof);
    cudaStreamDestroy(s);
    throw;
  }
  e.set_stream(prev);
  e.set_profiling(prof);
  STL_CUDA(cudaStreamDestroy(s));
  return evals;
}

}  // namespace stl
