// L-BFGS with the strong Wolfe line search, behind stlp_lbfgs.
//
// The algorithm is torch.optim.LBFGS with line_search_fn="strong_wolfe"
// (two-loop recursion over the last history_size pairs, H0 = (s.y / y.y) I,
// first step min(1, 1 / |g|_1) lr; the line search of lswolfe.lua with
// c1 = 1e-4, c2 = 0.9, its own tolerance_change 1e-9 and cubic
// interpolation), the optimiser the reference's synthesis ports
// (crates/stl-core/src/lbfgs.rs:250-470, driven by stlp_lbfgs in
// crates/stl-bridge/src/lib.rs:711-741): the line search may use the
// evaluations left, max_eval - evaluations so far.  Python's min / max keep
// the first argument on ties, as here.
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

double dot(const Vec& a, const Vec& b) {
  return chunk_sum(a.size(), [&](size_t lo, size_t hi) {
    double s = 0.0;
    for (size_t i = lo; i < hi; ++i) s += a[i] * b[i];
    return s;
  });
}

double abs_max(const Vec& a) {
  return chunk_max(a.size(), [&](size_t lo, size_t hi) {
    double m = 0.0;
    for (size_t i = lo; i < hi; ++i) m = std::max(m, std::fabs(a[i]));
    return m;
  });
}

double abs_sum(const Vec& a) {
  return chunk_sum(a.size(), [&](size_t lo, size_t hi) {
    double s = 0.0;
    for (size_t i = lo; i < hi; ++i) s += std::fabs(a[i]);
    return s;
  });
}

// out[i] = f(i)
template <typename F>
void fill(Vec& out, F&& f) {
  for_chunks(out.size(), [&](size_t, size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) out[i] = f(i);
  });
}

void axpy(Vec& p, double a, const Vec& u) {
  for_chunks(p.size(), [&](size_t, size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) p[i] = std::fma(u[i], a, p[i]);
  });
}

double py_min(double a, double b) { return b < a ? b : a; }
double py_max(double a, double b) { return b > a ? b : a; }

// minimiser of the cubic through (x1, f1, g1), (x2, f2, g2), clamped to
// [lo, hi] (default: the interval between x1 and x2)
double cubic_min(double x1, double f1, double g1, double x2, double f2, double g2, const double* bounds) {
  const double lo = bounds ? bounds[0] : (x1 <= x2 ? x1 : x2);
  const double hi = bounds ? bounds[1] : (x1 <= x2 ? x2 : x1);
  const double d1 = g1 + g2 - 3.0 * (f1 - f2) / (x1 - x2);
  const double d2sq = d1 * d1 - g1 * g2;
  if (d2sq >= 0.0) {
    const double d2 = std::sqrt(d2sq);
    const double m = x1 <= x2 ? x2 - (x2 - x1) * ((g2 + d2 - d1) / (g2 - g1 + 2.0 * d2))
                              : x1 - (x1 - x2) * ((g1 + d2 - d1) / (g1 - g2 + 2.0 * d2));
    return std::min(std::max(m, lo), hi);
  }
  return (lo + hi) / 2.0;
}

struct Options {
  double lr = 1.0;
  long long max_iter = 20, max_eval = -1, history = 10;
  double tol_grad = 1e-12, tol_change = 1e-15;
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

struct LineResult {
  double f, t;
  Vec g;
  long long evals;
};

// strong Wolfe search along d from x0 (loss f, gradient g, g.d = gtd)
LineResult strong_wolfe(Objective& obj, const Vec& x0, const Vec& d, double t, double f, const Vec& g, double gtd,
                        long long max_ls) {
  const double c1 = 1e-4, c2 = 0.9, tol = 1e-9;
  max_ls = std::max(max_ls, 0LL);
  long long evals = 0;
  Vec xt(x0.size());
  auto eval = [&](double step, Vec& gout) {
    fill(xt, [&](size_t i) { return std::fma(d[i], step, x0[i]); });
    ++evals;
    return obj(xt, gout);
  };
  const double d_norm = abs_max(d);
  Vec g_new;
  double f_new = eval(t, g_new);
  double gtd_new = dot(g_new, d);
  double t_prev = 0.0, f_prev = f, gtd_prev = gtd;
  Vec g_prev = g;
  bool done = false;
  long long ls = 0;
  std::vector<double> br, br_f, br_gtd;
  std::vector<Vec> br_g;
  while (ls < max_ls) {
    if (f_new > f + c1 * t * gtd || (ls > 1 && f_new >= f_prev)) {
      br = {t_prev, t}; br_f = {f_prev, f_new}; br_g = {g_prev, g_new}; br_gtd = {gtd_prev, gtd_new};
      break;
    }
    if (std::fabs(gtd_new) <= -c2 * gtd) {
      br = {t}; br_f = {f_new}; br_g = {g_new};
      done = true;
      break;
    }
    if (gtd_new >= 0.0) {
      br = {t_prev, t}; br_f = {f_prev, f_new}; br_g = {g_prev, g_new}; br_gtd = {gtd_prev, gtd_new};
      break;
    }
    const double bounds[2] = {t + 0.01 * (t - t_prev), t * 10.0};
    const double tmp = t;
    t = cubic_min(t_prev, f_prev, gtd_prev, t, f_new, gtd_new, bounds);
    t_prev = tmp;
    f_prev = f_new;
    g_prev = g_new;
    gtd_prev = gtd_new;
    f_new = eval(t, g_new);
    gtd_new = dot(g_new, d);
    ++ls;
  }
  if (ls == max_ls) {
    br = {0.0, t}; br_f = {f, f_new}; br_g = {g, g_new};
  }
  // zoom
  bool insuf = false;
  int low = br_f.front() <= br_f.back() ? 0 : 1, high = 1 - low;
  while (!done && ls < max_ls) {
    if (std::fabs(br[1] - br[0]) * d_norm < tol) break;
    t = cubic_min(br[0], br_f[0], br_gtd[0], br[1], br_f[1], br_gtd[1], nullptr);
    const double bmax = py_max(br[0], br[1]), bmin = py_min(br[0], br[1]);
    const double eps = 0.1 * (bmax - bmin);
    if (py_min(bmax - t, t - bmin) < eps) {
      if (insuf || t >= bmax || t <= bmin) {
        t = std::fabs(t - bmax) < std::fabs(t - bmin) ? bmax - eps : bmin + eps;
        insuf = false;
      } else {
        insuf = true;
      }
    } else {
      insuf = false;
    }
    f_new = eval(t, g_new);
    gtd_new = dot(g_new, d);
    ++ls;
    if (f_new > f + c1 * t * gtd || f_new >= br_f[low]) {
      br[high] = t; br_f[high] = f_new; br_g[high] = g_new; br_gtd[high] = gtd_new;
      low = br_f[0] <= br_f[1] ? 0 : 1;
      high = 1 - low;
    } else {
      if (std::fabs(gtd_new) <= -c2 * gtd) {
        done = true;
      } else if (gtd_new * (br[high] - br[low]) >= 0.0) {
        br[high] = br[low]; br_f[high] = br_f[low]; br_g[high] = br_g[low]; br_gtd[high] = br_gtd[low];
      }
      br[low] = t; br_f[low] = f_new; br_g[low] = g_new; br_gtd[low] = gtd_new;
    }
  }
  low = std::min(low, (int)br.size() - 1);
  return LineResult{br_f[low], br[low], std::move(br_g[low]), evals};
}

long long minimize(Vec& x, const Options& o, Objective& obj) {
  const long long max_eval = o.max_eval >= 0 ? o.max_eval : o.max_iter * 5 / 4;
  Vec g;
  double loss = obj(x, g);
  long long evals = 1;
  if (abs_max(g) <= o.tol_grad) return evals;
  const size_t n = x.size();
  Vec d, prev_g;
  double t = 0.0, h_diag = 1.0;
  std::vector<Vec> dirs, stps;  // y and s pairs, oldest first
  std::vector<double> ro;
  std::vector<double> al((size_t)o.history, 0.0);
  long long it = 0;
  while (it < o.max_iter) {
    ++it;
    if (it == 1) {
      d.assign(n, 0.0);
      fill(d, [&](size_t i) { return -g[i]; });
    } else {
      Vec y(n), s(n);
      fill(y, [&](size_t i) { return g[i] - prev_g[i]; });
      fill(s, [&](size_t i) { return d[i] * t; });
      const double ys = dot(y, s);
      if (ys > 1e-10) {
        if ((long long)dirs.size() == o.history) {
          dirs.erase(dirs.begin());
          stps.erase(stps.begin());
          ro.erase(ro.begin());
        }
        h_diag = ys / dot(y, y);
        dirs.push_back(std::move(y));
        stps.push_back(std::move(s));
        ro.push_back(1.0 / ys);
      }
      const int m = (int)dirs.size();
      Vec q(n);
      fill(q, [&](size_t i) { return -g[i]; });
      for (int i = m - 1; i >= 0; --i) {
        al[i] = dot(stps[i], q) * ro[i];
        axpy(q, -al[i], dirs[i]);
      }
      fill(d, [&](size_t i) { return q[i] * h_diag; });
      for (int i = 0; i < m; ++i) {
        const double be = dot(dirs[i], d) * ro[i];
        axpy(d, al[i] - be, stps[i]);
      }
    }
    prev_g = g;
    const double prev_loss = loss;
    t = it == 1 ? py_min(1.0, 1.0 / abs_sum(g)) * o.lr : o.lr;
    const double gtd = dot(g, d);
    if (gtd > -o.tol_change) break;
    const Vec x0 = x;
    LineResult r = strong_wolfe(obj, x0, d, t, loss, g, gtd, max_eval - evals);
    loss = r.f;
    g = std::move(r.g);
    t = r.t;
    fill(x, [&](size_t i) { return std::fma(d[i], t, x0[i]); });
    evals += r.evals;
    const bool opt = abs_max(g) <= o.tol_grad;
    if (it == o.max_iter || evals >= max_eval || opt) break;
    const double step = chunk_max(n, [&](size_t lo, size_t hi) {
      double mm = 0.0;
      for (size_t i = lo; i < hi; ++i) mm = std::max(mm, std::fabs(d[i] * t));
      return mm;
    });
    if (step <= o.tol_change) break;
    if (std::fabs(loss - prev_loss) < o.tol_change) break;
  }
  return evals;
}

}  // namespace

extern "C" int64_t stlp_lbfgs(double* x, size_t n, const char* options, stlp_callback callback, void* ctx) {
  try {
    if (!x || !callback) throw std::runtime_error("null argument");
    const stl::Json v = stl::Json::parse(options && *options ? options : "{}");
    Options o;
    o.lr = v.real("lr", 1.0);
    o.max_iter = v.integer("max_iter", 20);
    o.max_eval = v.has("max_eval") ? v.integer("max_eval", 0) : -1;
    o.tol_grad = v.real("tolerance_grad", 1e-12);
    o.tol_change = v.real("tolerance_change", 1e-15);
    o.history = v.integer("history_size", 10);
    if (o.history <= 0 || !(o.lr > 0.0) || !std::isfinite(o.lr)) throw std::runtime_error("invalid L-BFGS options");
    Vec xv(x, x + n);
    Objective obj{callback, ctx};
    long long evals = 0;
    try {
      evals = minimize(xv, o, obj);
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
