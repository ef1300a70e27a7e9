// L-BFGS with the strong Wolfe line search over a host callback, behind
// stlp_lbfgs; the steps are those of lbfgs.hpp (torch.optim.LBFGS with
// strong Wolfe, crates/stl-core/src/lbfgs.rs:250-470, lib.rs:711-741).
//
// Vector operations run over chunks of kChunk elements on the host threads
// (STL_THREADS, else the hardware concurrency); a reduction adds the
// chunks' sums in chunk order, so results do not depend on the number of
// threads.  p += a u is a fused multiply-add.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "json.hpp"
#include "lbfgs.hpp"
#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

namespace {

typedef std::vector<double> Vec;
constexpr size_t kChunk = size_t(1) << 16;

int host_threads() {
  static const int n = [] {
    if (const char* e = std::getenv("STL_THREADS")) {
      const int v = std::atoi(e);
      if (v > 0) return v;
    }
    const unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
  }();
  return n;
}

// f(chunk index, lo, hi) for every chunk of [0, n), spread over the threads
template <typename F>
void for_chunks(size_t n, F&& f) {
  const size_t chunks = std::max<size_t>(1, (n + kChunk - 1) / kChunk);
  const size_t t = std::min<size_t>((size_t)host_threads(), chunks);
  auto run = [&](size_t c0, size_t c1) {
    for (size_t c = c0; c < c1; ++c) f(c, c * kChunk, std::min(n, (c + 1) * kChunk));
  };
  if (t <= 1) {
    run(0, chunks);
    return;
  }
  const size_t per = (chunks + t - 1) / t;
  std::vector<std::thread> pool;
  for (size_t k = 0; k < t; ++k) {
    const size_t c0 = std::min(chunks, k * per), c1 = std::min(chunks, (k + 1) * per);
    if (c0 < c1) pool.emplace_back(run, c0, c1);
  }
  for (auto& th : pool) th.join();
}

// sum over chunks (in chunk order) of f(lo, hi)
template <typename F>
double chunk_sum(size_t n, F&& f) {
  const size_t chunks = std::max<size_t>(1, (n + kChunk - 1) / kChunk);
  std::vector<double> part(chunks, 0.0);
  for_chunks(n, [&](size_t c, size_t lo, size_t hi) { part[c] = f(lo, hi); });
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}

template <typename F>
double chunk_max(size_t n, F&& f) {
  const size_t chunks = std::max<size_t>(1, (n + kChunk - 1) / kChunk);
  std::vector<double> part(chunks, 0.0);
  for_chunks(n, [&](size_t c, size_t lo, size_t hi) { part[c] = f(lo, hi); });
  double m = 0.0;
  for (double v : part) m = std::max(m, v);
  return m;
}

double vdot(const Vec& a, const Vec& b) {
  return chunk_sum(a.size(), [&](size_t lo, size_t hi) {
    double s = 0.0;
    for (size_t i = lo; i < hi; ++i) s += a[i] * b[i];
    return s;
  });
}

double vabs_max(const Vec& a) {
  return chunk_max(a.size(), [&](size_t lo, size_t hi) {
    double m = 0.0;
    for (size_t i = lo; i < hi; ++i) m = std::max(m, std::fabs(a[i]));
    return m;
  });
}

double vabs_sum(const Vec& a) {
  return chunk_sum(a.size(), [&](size_t lo, size_t hi) {
    double s = 0.0;
    for (size_t i = lo; i < hi; ++i) s += std::fabs(a[i]);
    return s;
  });
}

// host vectors: the chunked, threaded operations above
struct HostOps {
  typedef Vec Vec;
  Vec make(size_t n) { return Vec(n); }
  void copy(Vec& dst, const Vec& src) { dst = src; }
  template <typename F>
  void fill(Vec& out, F&& f) {
    for_chunks(out.size(), [&](size_t, size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) out[i] = f(i);
    });
  }
  void neg(Vec& out, const Vec& a) { fill(out, [&](size_t i) { return -a[i]; }); }
  void sub(Vec& out, const Vec& a, const Vec& b) { fill(out, [&](size_t i) { return a[i] - b[i]; }); }
  void scale(Vec& out, const Vec& a, double c) { fill(out, [&](size_t i) { return a[i] * c; }); }
  void fma3(Vec& out, const Vec& d, double t, const Vec& x0) {
    fill(out, [&](size_t i) { return std::fma(d[i], t, x0[i]); });
  }
  void axpy(Vec& p, double a, const Vec& u) {
    for_chunks(p.size(), [&](size_t, size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) p[i] = std::fma(u[i], a, p[i]);
    });
  }
  double dot(const Vec& a, const Vec& b) { return vdot(a, b); }
  double abs_max(const Vec& a) { return vabs_max(a); }
  double abs_sum(const Vec& a) { return vabs_sum(a); }
};

struct Objective {
  stlp_callback cb;
  void* ctx;
  long long evals = 0;
  double operator()(const Vec& x, Vec& g) {
    g.assign(x.size(), 0.0);
    const double loss = cb(x.data(), x.size(), g.data(), ctx);
    ++evals;
    bool finite = std::isfinite(loss);
    if (finite) finite = chunk_max(g.size(), [&](size_t lo, size_t hi) {
                           for (size_t i = lo; i < hi; ++i)
                             if (!std::isfinite(g[i])) return 1.0;
                           return 0.0;
                         }) == 0.0;
    if (!finite) throw std::runtime_error("non-finite objective or gradient (or a callback exception)");
    return loss;
  }
};

}  // namespace

namespace stl {
namespace lbfgs {
Options parse_options(const char* json) {
  const stl::Json v = stl::Json::parse(json && *json ? json : "{}");
  Options o;
  o.lr = v.real("lr", 1.0);
  o.max_iter = v.integer("max_iter", 20);
  o.max_eval = v.has("max_eval") ? v.integer("max_eval", 0) : -1;
  o.tol_grad = v.real("tolerance_grad", 1e-12);
  o.tol_change = v.real("tolerance_change", 1e-15);
  o.history = v.integer("history_size", 10);
  o.graph = v.boolean("graph", true);
  if (o.history <= 0 || !(o.lr > 0.0) || !std::isfinite(o.lr)) throw std::runtime_error("invalid L-BFGS options");
  return o;
}
}  // namespace lbfgs
}  // namespace stl

extern "C" int64_t stlp_lbfgs(double* x, size_t n, const char* options, stlp_callback callback, void* ctx) {
  try {
    if (!x || !callback) throw std::runtime_error("null argument");
    const stl::lbfgs::Options o = stl::lbfgs::parse_options(options);
    Vec xv(x, x + n);
    Objective obj{callback, ctx};
    long long evals = 0;
    try {
      HostOps ops;
      evals = stl::lbfgs::minimize(ops, xv, n, o, obj);
    } catch (...) {
      std::copy(xv.begin(), xv.end(), x);  // the iterate reached, as an in-place update leaves it
      throw;
    }
    std::copy(xv.begin(), xv.end(), x);
    return evals;
  } catch (const std::exception& e) {
    stl::set_error(e.what());
  } catch (...) {
    stl::set_error("unknown native failure");
  }
  return -1;
}
