// CPU FP64 restatement of the reference's spin-2 front end
// (crates/stl-core/src/spin.rs): the transported mean of the four NESTED
// children, and the local operator -(d_x - i d_y)^2 on the pixels within
// `rings` rings with weights exact on the polynomials of degree 2 rings.
//
// TEST INFRASTRUCTURE ONLY: the engine never links this file.  Operation
// order follows spin.rs so that the weights agree with the reference's to a
// few ulps (libm's exp / sin / cos / atan2 are the same glibc functions the
// reference's Rust build calls on Linux).
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "healpix_ops.hpp"

namespace orc {
namespace {

struct cx {  // num_complex::Complex64 arithmetic, written out
  double re = 0.0, im = 0.0;
};
inline cx cmul(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cx cscale(cx a, double s) { return {a.re * s, a.im * s}; }
inline cx cadd(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
inline cx csub(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
inline cx cdivr(cx a, double s) { return {a.re / s, a.im / s}; }
inline cx cpolar(double r, double t) { return {r * std::cos(t), r * std::sin(t)}; }

using V3 = std::array<double, 3>;
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

// x^n by binary powering (LLVM's powi lowering for a run-time exponent)
double powi(double a, int b) {
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return r;
}

// centre, e_theta, e_phi of a NESTED pixel (spin.rs:46-50)
void frame(i64 pix, i64 nside, V3& c, V3& et, V3& ep) {
  double t, p;
  pix2ang_nest(pix, nside, t, p);
  const double st = std::sin(t), ct = std::cos(t), sp = std::sin(p), cp = std::cos(p);
  c = {st * cp, st * sp, ct};
  et = {ct * cp, ct * sp, -st};
  ep = {-sp, cp, 0.0};
}

// angle in the frame of m of the tangent vector v at a carried along the
// geodesic to the centre of m (spin.rs:55-74)
double transported_angle(const V3& a, const V3& v, i64 m, i64 nside) {
  V3 b, et, ep;
  frame(m, nside, b, et, ep);
  const V3 axis = cross(a, b);
  const double s = std::sqrt(dot(axis, axis));
  const double c = dot(a, b);
  V3 w;
  if (s < 1e-15) {
    w = v;
  } else {
    const V3 k = {axis[0] / s, axis[1] / s, axis[2] / s};
    const V3 kv = cross(k, v);
    const double kd = dot(k, v);
    for (int i = 0; i < 3; ++i) w[i] = v[i] * c + kv[i] * s + k[i] * kd * (1.0 - c);
  }
  return std::atan2(dot(w, ep), dot(w, et));
}

// e^{-2 i psi} (spin.rs:80-83)
inline cx spin_rotation(double psi) { return cpolar(1.0, -2.0 * psi); }

struct Mono {
  int a, b;
  cx image;
};
// x^a y^b with a + b <= degree, by total degree then a descending, and their
// image under -(d_x - i d_y)^2 at the origin (spin.rs:214-231)
std::vector<Mono> monomials(int degree) {
  std::vector<Mono> out;
  for (int t = 0; t <= degree; ++t)
    for (int a = t; a >= 0; --a) {
      const int b = t - a;
      cx img;
      if (a == 2 && b == 0) img = {-2.0, 0.0};
      else if (a == 0 && b == 2) img = {2.0, 0.0};
      else if (a == 1 && b == 1) img = {0.0, 2.0};
      out.push_back({a, b, img});
    }
  return out;
}

// Cholesky solve of the SPD a x = b, false when not positive definite
// (spin.rs:235-272)
bool cholesky_solve(std::vector<double>& a, int n, std::vector<cx>& y) {
  for (int j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    if (d <= 1e-12 * std::max(std::fabs(a[j * n + j]), 1e-300)) return false;
    d = std::sqrt(d);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = a[i * n + j];
      for (int k = 0; k < j; ++k) v -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = v / d;
    }
  }
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k) y[i] = csub(y[i], cscale(y[k], a[i * n + k]));
    y[i] = cdivr(y[i], a[i * n + i]);
  }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k) y[i] = csub(y[i], cscale(y[k], a[k * n + i]));
    y[i] = cdivr(y[i], a[i * n + i]);
  }
  return true;
}

// the cells the stencil of p reads (spin.rs:276-284)
std::vector<i64> stencil_pixels(i64 p, i64 nside, int rings) {
  if ((i64)rings < nside) return kth_neighbourhood_set(p, nside, rings);
  V3 c, et, ep;
  frame(p, nside, c, et, ep);
  const double h = std::sqrt(4.0 * PI / (double)npix(nside));
  const double cut = std::cos(std::min(((double)rings + 1.0) * h, 1.2));
  std::vector<i64> out;
  for (i64 m = 0; m < npix(nside); ++m) {
    V3 v, a, b;
    frame(m, nside, v, a, b);
    if (dot(v, c) >= cut) out.push_back(m);
  }
  return out;
}

}  // namespace

// Complex sparse rows out[r] = sum_e w[e] P[col[e]] and their transpose
// (spin.rs:88-157)
struct SpinCsr {
  i64 n_in = 0;
  std::vector<i64> ptr, col;
  std::vector<double> w;  // re, im per entry
  std::vector<i64> t_ptr, t_row;
  std::vector<double> t_w;

  void finish() {
    const i64 nnz = (i64)col.size();
    std::vector<i64> count(n_in + 1, 0);
    for (i64 c : col) count[c + 1] += 1;
    for (i64 i = 0; i < n_in; ++i) count[i + 1] += count[i];
    t_ptr = count;
    t_row.assign(nnz, 0);
    t_w.assign(2 * nnz, 0.0);
    const i64 rows = (i64)ptr.size() - 1;
    for (i64 r = 0; r < rows; ++r)
      for (i64 e = ptr[r]; e < ptr[r + 1]; ++e) {
        i64& slot = count[col[e]];
        t_row[slot] = r;
        t_w[2 * slot] = w[2 * e];
        t_w[2 * slot + 1] = -w[2 * e + 1];
        ++slot;
      }
  }
  i64 rows() const { return (i64)ptr.size() - 1; }

  // [R, 2, n_in] -> [R, 2, rows] (or the transpose: [R, 2, rows] -> [R, 2, n_in])
  void apply(const double* x, i64 R, double* out, bool adjoint) const {
    const std::vector<i64>& P = adjoint ? t_ptr : ptr;
    const std::vector<i64>& C = adjoint ? t_row : col;
    const std::vector<double>& W = adjoint ? t_w : w;
    const i64 nr = (i64)P.size() - 1, ni = adjoint ? rows() : n_in;
    for (i64 r = 0; r < R; ++r) {
      const double* q = x + r * 2 * ni;
      const double* u = q + ni;
      double* oq = out + r * 2 * nr;
      double* ou = oq + nr;
      parallel_chunks(nr, [&](i64 k0, i64 k1, int) {
        for (i64 k = k0; k < k1; ++k) {
          cx acc;
          for (i64 e = P[k]; e < P[k + 1]; ++e) {
            const i64 c = C[e];
            acc = cadd(acc, cmul({W[2 * e], W[2 * e + 1]}, {q[c], u[c]}));
          }
          oq[k] = acc.re;
          ou[k] = acc.im;
        }
      });
    }
  }
};

// transported mean of the four NESTED children, level nside_fine -> its
// parents (spin.rs:193-210)
SpinCsr spin_decimation(i64 nside_fine) {
  SpinCsr s;
  s.n_in = npix(nside_fine);
  const i64 nc = npix(nside_fine / 2);
  s.ptr.resize(nc + 1);
  s.col.resize(4 * nc);
  s.w.resize(8 * nc);
  parallel_chunks(nc, [&](i64 p0, i64 p1, int) {
    for (i64 p = p0; p < p1; ++p) {
      V3 c, et, ep;
      frame(p, nside_fine / 2, c, et, ep);
      for (int k = 0; k < 4; ++k) {
        const i64 child = 4 * p + k;
        const cx v = cscale(spin_rotation(transported_angle(c, et, child, nside_fine)), 0.25);
        // 0.25 * e^{-2 i psi}: the real factor on the left (Complex64 scalar product)
        s.col[4 * p + k] = child;
        s.w[2 * (4 * p + k)] = v.re;
        s.w[2 * (4 * p + k) + 1] = v.im;
      }
    }
  });
  for (i64 p = 0; p <= nc; ++p) s.ptr[p] = 4 * p;
  s.finish();
  return s;
}

// -(d_x - i d_y)^2 at nside in pixel units, one row per pixel
// (spin.rs:294-338)
SpinCsr eth_bar2(i64 nside, int kernel_sz) {
  if (kernel_sz % 2 != 1 || kernel_sz < 3 || kernel_sz > 9)
    throw std::runtime_error("spin stencil: kernel 3, 5, 7 or 9");
  const int rings = kernel_sz / 2;
  const i64 n = npix(nside);
  const double h = std::sqrt(4.0 * PI / (double)n);
  std::vector<std::vector<std::pair<i64, cx>>> rows(n);
  std::vector<i64> singular(num_threads() + 1, -1);
  parallel_chunks(n, [&](i64 p0, i64 p1, int worker) {
    for (i64 p = p0; p < p1 && singular[worker] < 0; ++p) {
      V3 c, et, ep;
      frame(p, nside, c, et, ep);
      std::vector<i64> cells = stencil_pixels(p, nside, rings);
      std::sort(cells.begin(), cells.end());
      const size_t M = cells.size();
      std::vector<double> px(M), py(M), wt(M);
      for (size_t m = 0; m < M; ++m) {
        V3 v, a, b;
        frame(cells[m], nside, v, a, b);
        const double z = dot(v, c);
        px[m] = dot(v, et) / z / h;
        py[m] = dot(v, ep) / z / h;
        wt[m] = std::exp(-(px[m] * px[m] + py[m] * py[m]) / (double)(rings * rings));
      }
      int degree = 2 * rings;
      std::vector<cx> wm;
      for (;;) {
        const auto mono = monomials(degree);
        const int k = (int)mono.size();
        std::vector<double> A((size_t)k * M);
        for (int i = 0; i < k; ++i)
          for (size_t m = 0; m < M; ++m) A[i * M + m] = powi(px[m], mono[i].a) * powi(py[m], mono[i].b);
        std::vector<double> g((size_t)k * k);
        for (int i = 0; i < k; ++i)
          for (int j = 0; j <= i; ++j) {
            double v = 0.0;
            for (size_t m = 0; m < M; ++m) v += A[i * M + m] * wt[m] * A[j * M + m];
            g[i * k + j] = v;
            g[j * k + i] = v;
          }
        std::vector<cx> l(k);
        for (int i = 0; i < k; ++i) l[i] = mono[i].image;
        if (cholesky_solve(g, k, l)) {
          wm.resize(M);
          for (size_t m = 0; m < M; ++m) {
            cx s;
            for (int i = 0; i < k; ++i) s = cadd(s, cscale(l[i], A[i * M + m]));
            wm[m] = cscale(s, wt[m]);
          }
          break;
        }
        if (degree <= 2) break;  // singular at degree 2 as well
        degree = 2;
      }
      if (wm.empty()) {
        singular[worker] = p;
        break;
      }
      auto& row = rows[p];
      row.resize(M);
      for (size_t m = 0; m < M; ++m)
        row[m] = {cells[m], cmul(wm[m], spin_rotation(transported_angle(c, et, cells[m], nside)))};
    }
  });
  for (i64 p : singular)
    if (p >= 0) throw std::runtime_error("spin stencil: singular system at pixel " + std::to_string(p));
  SpinCsr s;
  s.n_in = n;
  s.ptr.assign(1, 0);
  for (auto& row : rows) {
    for (auto& e : row) {
      s.col.push_back(e.first);
      s.w.push_back(e.second.re);
      s.w.push_back(e.second.im);
    }
    s.ptr.push_back((i64)s.col.size());
  }
  s.finish();
  return s;
}

}  // namespace orc

using orc::SpinCsr;
using orc::i64;

static thread_local std::string g_spin_err;

extern "C" {

const char* or_spin_last_error() { return g_spin_err.c_str(); }

// eth_bar2 (kind 0, nside, kernel) or the transported decimation of the
// level nside (kind 1; rows: the parents); null on failure
void* or_spin_new(int kind, i64 nside, int kernel) {
  try {
    return new SpinCsr(kind == 0 ? orc::eth_bar2(nside, kernel) : orc::spin_decimation(nside));
  } catch (const std::exception& ex) {
    g_spin_err = ex.what();
    return nullptr;
  }
}
void or_spin_free(void* h) { delete static_cast<SpinCsr*>(h); }
// rows, inputs and entries
void or_spin_shape(void* h, i64* rows, i64* n_in, i64* nnz) {
  auto* s = static_cast<SpinCsr*>(h);
  *rows = s->rows();
  *n_in = s->n_in;
  *nnz = (i64)s->col.size();
}
// the rows: ptr [rows + 1], col [nnz], w [nnz][2]
void or_spin_export(void* h, i64* ptr, i64* col, double* w) {
  auto* s = static_cast<SpinCsr*>(h);
  std::memcpy(ptr, s->ptr.data(), s->ptr.size() * sizeof(i64));
  std::memcpy(col, s->col.data(), s->col.size() * sizeof(i64));
  std::memcpy(w, s->w.data(), s->w.size() * sizeof(double));
}
void or_spin_apply(void* h, const double* x, i64 R, double* out, int adjoint) {
  static_cast<SpinCsr*>(h)->apply(x, R, out, adjoint != 0);
}

}  // extern "C"
