// L-BFGS with the strong Wolfe line search, written once over a vector
// policy so that the same steps run on host vectors (stlp_lbfgs) and on
// device vectors (stlp_synthesize_device).
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
// A policy Ops provides: typedef Vec (movable), Vec make(n), copy(dst, src),
// neg(out, a) = -a, sub(out, a, b) = a - b, scale(out, a, c) = a c,
// fma3(out, d, t, x0) = fma(d, t, x0), axpy(p, a, u): p = fma(u, a, p),
// dot, abs_max, abs_sum.  The objective obj(x, g) returns the loss, writes
// the gradient and throws on a non-finite loss or gradient.
#pragma once
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

namespace stl {
namespace lbfgs {

inline double py_min(double a, double b) { return b < a ? b : a; }
inline double py_max(double a, double b) { return b > a ? b : a; }

// minimiser of the cubic through (x1, f1, g1), (x2, f2, g2), clamped to
// [lo, hi] (default: the interval between x1 and x2)
inline double cubic_min(double x1, double f1, double g1, double x2, double f2, double g2, const double* bounds) {
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
  bool graph = true;  // device synthesis: iterations 2 on as one CUDA graph launch each
};
// options JSON (lr, max_iter, max_eval, tolerance_grad, tolerance_change,
// history_size, graph), validated; throws on invalid values
Options parse_options(const char* json);

template <typename Vec>
struct LineResult {
  double f, t;
  Vec g;
  long long evals;
};

// the search's first evaluation when the caller made it already: loss f and
// gradient g at x0 + t d, g.d = gtd, and max |d_i| = d_norm
template <typename Vec>
struct FirstTrial {
  double f, gtd, d_norm;
  const Vec* g;
};

// strong Wolfe search along d from x0 (loss f, gradient g, g.d = gtd)
template <typename Ops, typename Obj>
LineResult<typename Ops::Vec> strong_wolfe(Ops& ops, Obj& obj, const typename Ops::Vec& x0,
                                           const typename Ops::Vec& d, double t, double f,
                                           const typename Ops::Vec& g, double gtd, long long max_ls, size_t n,
                                           const FirstTrial<typename Ops::Vec>* first = nullptr) {
  typedef typename Ops::Vec Vec;
  const double c1 = 1e-4, c2 = 0.9, tol = 1e-9;
  max_ls = std::max(max_ls, 0LL);
  long long evals = 0;
  Vec xt = ops.make(n);
  auto eval = [&](double step, Vec& gout) {
    ops.fma3(xt, d, step, x0);
    ++evals;
    return obj(xt, gout);
  };
  const double d_norm = first ? first->d_norm : ops.abs_max(d);
  Vec g_new = ops.make(n);
  double f_new, gtd_new;
  if (first) {
    ++evals;
    f_new = first->f;
    ops.copy(g_new, *first->g);
    gtd_new = first->gtd;
  } else {
    f_new = eval(t, g_new);
    gtd_new = ops.dot(g_new, d);
  }
  double t_prev = 0.0, f_prev = f, gtd_prev = gtd;
  Vec g_prev = ops.make(n);
  ops.copy(g_prev, g);
  bool done = false;
  long long ls = 0;
  // the bracket: nb points (t, f, gradient, g.d)
  int nb = 0;
  double br[2] = {0.0, 0.0}, br_f[2] = {0.0, 0.0}, br_gtd[2] = {0.0, 0.0};
  Vec br_g[2] = {ops.make(n), ops.make(n)};
  auto bracket2 = [&](double ta, double fa, const Vec& ga, double da, double tb, double fb, const Vec& gb,
                      double db) {
    nb = 2;
    br[0] = ta; br_f[0] = fa; ops.copy(br_g[0], ga); br_gtd[0] = da;
    br[1] = tb; br_f[1] = fb; ops.copy(br_g[1], gb); br_gtd[1] = db;
  };
  while (ls < max_ls) {
    if (f_new > f + c1 * t * gtd || (ls > 1 && f_new >= f_prev)) {
      bracket2(t_prev, f_prev, g_prev, gtd_prev, t, f_new, g_new, gtd_new);
      break;
    }
    if (std::fabs(gtd_new) <= -c2 * gtd) {
      nb = 1;
      br[0] = t; br_f[0] = f_new; ops.copy(br_g[0], g_new);
      done = true;
      break;
    }
    if (gtd_new >= 0.0) {
      bracket2(t_prev, f_prev, g_prev, gtd_prev, t, f_new, g_new, gtd_new);
      break;
    }
    const double bounds[2] = {t + 0.01 * (t - t_prev), t * 10.0};
    const double tmp = t;
    t = cubic_min(t_prev, f_prev, gtd_prev, t, f_new, gtd_new, bounds);
    t_prev = tmp;
    f_prev = f_new;
    ops.copy(g_prev, g_new);
    gtd_prev = gtd_new;
    f_new = eval(t, g_new);
    gtd_new = ops.dot(g_new, d);
    ++ls;
  }
  if (ls == max_ls) {  // the slopes of this bracket are not read: no zoom follows
    nb = 2;
    br[0] = 0.0; br_f[0] = f; ops.copy(br_g[0], g);
    br[1] = t; br_f[1] = f_new; ops.copy(br_g[1], g_new);
  }
  // zoom
  bool insuf = false;
  int low = br_f[0] <= br_f[nb - 1] ? 0 : 1, high = 1 - low;
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
    gtd_new = ops.dot(g_new, d);
    ++ls;
    if (f_new > f + c1 * t * gtd || f_new >= br_f[low]) {
      br[high] = t; br_f[high] = f_new; ops.copy(br_g[high], g_new); br_gtd[high] = gtd_new;
      low = br_f[0] <= br_f[1] ? 0 : 1;
      high = 1 - low;
    } else {
      if (std::fabs(gtd_new) <= -c2 * gtd) {
        done = true;
      } else if (gtd_new * (br[high] - br[low]) >= 0.0) {
        br[high] = br[low]; br_f[high] = br_f[low]; ops.copy(br_g[high], br_g[low]); br_gtd[high] = br_gtd[low];
      }
      br[low] = t; br_f[low] = f_new; ops.copy(br_g[low], g_new); br_gtd[low] = gtd_new;
    }
  }
  low = std::min(low, nb - 1);
  return LineResult<Vec>{br_f[low], br[low], std::move(br_g[low]), evals};
}

// minimises obj from x (updated in place); returns the evaluations made
template <typename Ops, typename Obj>
long long minimize(Ops& ops, typename Ops::Vec& x, size_t n, const Options& o, Obj& obj) {
  typedef typename Ops::Vec Vec;
  const long long max_eval = o.max_eval >= 0 ? o.max_eval : o.max_iter * 5 / 4;
  Vec g = ops.make(n);
  double loss = obj(x, g);
  long long evals = 1;
  if (ops.abs_max(g) <= o.tol_grad) return evals;
  Vec d = ops.make(n), prev_g = ops.make(n), q = ops.make(n), x0 = ops.make(n);
  double t = 0.0, h_diag = 1.0;
  std::vector<Vec> dirs, stps;  // y and s pairs, oldest first
  std::vector<Vec> spare;       // buffers of dropped pairs, reused
  std::vector<double> ro;
  std::vector<double> al((size_t)o.history, 0.0);
  auto take = [&]() {
    if (spare.empty()) return ops.make(n);
    Vec v = std::move(spare.back());
    spare.pop_back();
    return v;
  };
  long long it = 0;
  while (it < o.max_iter) {
    ++it;
    if (it == 1) {
      ops.neg(d, g);
    } else {
      Vec y = take(), s = take();
      ops.sub(y, g, prev_g);
      ops.scale(s, d, t);
      const double ys = ops.dot(y, s);
      if (ys > 1e-10) {
        if ((long long)dirs.size() == o.history) {
          spare.push_back(std::move(dirs.front()));
          spare.push_back(std::move(stps.front()));
          dirs.erase(dirs.begin());
          stps.erase(stps.begin());
          ro.erase(ro.begin());
        }
        h_diag = ys / ops.dot(y, y);
        dirs.push_back(std::move(y));
        stps.push_back(std::move(s));
        ro.push_back(1.0 / ys);
      } else {
        spare.push_back(std::move(y));
        spare.push_back(std::move(s));
      }
      const int m = (int)dirs.size();
      ops.neg(q, g);
      for (int i = m - 1; i >= 0; --i) {
        al[i] = ops.dot(stps[i], q) * ro[i];
        ops.axpy(q, -al[i], dirs[i]);
      }
      ops.scale(d, q, h_diag);
      for (int i = 0; i < m; ++i) {
        const double be = ops.dot(dirs[i], d) * ro[i];
        ops.axpy(d, al[i] - be, stps[i]);
      }
    }
    ops.copy(prev_g, g);
    const double prev_loss = loss;
    t = it == 1 ? py_min(1.0, 1.0 / ops.abs_sum(g)) * o.lr : o.lr;
    const double gtd = ops.dot(g, d);
    if (gtd > -o.tol_change) break;
    ops.copy(x0, x);
    LineResult<Vec> r = strong_wolfe(ops, obj, x0, d, t, loss, g, gtd, max_eval - evals, n);
    loss = r.f;
    std::swap(g, r.g);
    t = r.t;
    ops.fma3(x, d, t, x0);
    evals += r.evals;
    const bool opt = ops.abs_max(g) <= o.tol_grad;
    if (it == o.max_iter || evals >= max_eval || opt) break;
    // max |d_i t| = (max |d_i|) |t|: rounding is monotonic
    const double step = ops.abs_max(d) * std::fabs(t);
    if (step <= o.tol_change) break;
    if (std::fabs(loss - prev_loss) < o.tol_change) break;
  }
  return evals;
}

}  // namespace lbfgs
}  // namespace stl
