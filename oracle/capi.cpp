// C entry points of the oracle, for ctypes (oracle/oracle.py).
// TEST INFRASTRUCTURE ONLY: the engine never links this library.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>

#include "engine.hpp"

using namespace orc;

static thread_local std::string g_err;

#define GUARD(fail, body)                 \
  try {                                   \
    body                                  \
  } catch (const std::exception& ex) {    \
    g_err = ex.what();                    \
    return fail;                          \
  }

extern "C" {

const char* or_last_error() { return g_err.c_str(); }
void or_set_threads(int n) { set_num_threads(n); }
int or_get_threads() { return num_threads(); }

void or_centres(i64 nside, i64 n, const i64* ids, i64* ix, i64* iy, i64* face, double* theta, double* phi,
                double* lon, double* lat) {
  int order = order_of(nside);
  for (i64 i = 0; i < n; ++i) {
    nest2xyf(ids[i], order, ix[i], iy[i], face[i]);
    xyf2ang(ix[i], iy[i], face[i], nside, theta[i], phi[i]);
    centre_lonlat(ids[i], nside, lon[i], lat[i]);
  }
}

void or_ring2nest(int order, i64 n, const i64* ring, i64* nest) {
  for (i64 i = 0; i < n; ++i) nest[i] = ring2nest(ring[i], order);
}

void or_interp_ring(i64 nside, i64 n, const double* theta, const double* phi, i64* pix, double* w) {
  for (i64 i = 0; i < n; ++i) get_interpol_ring(theta[i], phi[i], nside, pix + 4 * i, w + 4 * i);
}

void or_interp_nested(int order, i64 n, const double* vecs, i64* pix, double* w) {
  for (i64 i = 0; i < n; ++i) interp_weights_nested(vecs + 3 * i, order, pix + 4 * i, w + 4 * i);
}

void or_rotations(i64 n, const double* theta, const double* phi, int G, int gauge, double* out) {
  for (i64 k = 0; k < n; ++k) {
    auto r = rotation_matrices(theta[k], phi[k], G, (Gauge)gauge);
    for (int g = 0; g < G; ++g)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[((k * G + g) * 3 + i) * 3 + j] = r[g][i][j];
  }
}

void or_kernel_grid(int ksz, i64 nside, double* out) {
  auto v = local_kernel_grid(ksz, nside);
  for (size_t i = 0; i < v.size(); ++i)
    for (int j = 0; j < 3; ++j) out[3 * i + j] = v[i][j];
}

void or_wavelet_weights(int ksz, double* out) {
  auto w = wavelet_weights(ksz);
  std::memcpy(out, w.data(), w.size() * sizeof(double));
}

// Bound stencils of the rows `grid` on the grid `grid`, in the reference's
// layout ((n * G + g) * K + k) * P + p (conv.rs:18-22).
int or_bind(const i64* grid, i64 ngrid, i64 nside, int ksz, int G, int gauge, double eps, i64* pos, double* w,
            uint8_t* complete) {
  GUARD(-1, {
    Bound b;
    bind_rows(grid, ngrid, grid, ngrid, nside, ksz, G, (Gauge)gauge, eps, b);
    int P = ksz * ksz;
    for (i64 k = 0; k < ngrid; ++k) {
      complete[k] = b.complete[k];
      for (int g = 0; g < G; ++g)
        for (int p = 0; p < P; ++p)
          for (int n = 0; n < 4; ++n) {
            size_t src = (((size_t)k * G + g) * P + p) * 4 + n;
            size_t dst = (((size_t)n * G + g) * ngrid + k) * P + p;
            pos[dst] = b.pos[src];
            w[dst] = b.w[src];
          }
    }
    return 0;
  })
}

// The sorted distinct cells of nonzero weight each row reads, bound on the
// whole sky (conv.rs rows_eps with every cell present): out [nrows][width]
// padded with -1, wmax [nrows][width] the cell's largest bound weight over
// the gauges and taps, counts [nrows]; -1 when a row has more than width
// cells.
typedef std::pair<i64, double> CellWeight;

int or_row_cells(const i64* rows, i64 nrows, i64 nside, int ksz, int G, int gauge, i64* out, double* wmax,
                 i64 width, i64* counts) {
  GUARD(-1, {
    Bound b;
    bind_rows(nullptr, 12 * nside * nside, rows, nrows, nside, ksz, G, (Gauge)gauge, 0.0, b);
    const int P = ksz * ksz;
    for (i64 k = 0; k < nrows; ++k) {
      std::vector<CellWeight> c;
      for (int g = 0; g < G; ++g)
        for (int p = 0; p < P; ++p)
          for (int n = 0; n < 4; ++n) {
            const size_t e = (((size_t)k * G + g) * P + p) * 4 + n;
            if (b.w[e] != 0.0) c.push_back({b.pos[e], std::fabs(b.w[e])});
          }
      std::sort(c.begin(), c.end());
      std::vector<CellWeight> m;
      for (const auto& e : c) {
        if (!m.empty() && m.back().first == e.first) m.back().second = std::max(m.back().second, e.second);
        else m.push_back(e);
      }
      if ((i64)m.size() > width) throw std::runtime_error("a row reads more cells than the width");
      counts[k] = (i64)m.size();
      for (i64 j = 0; j < width; ++j) {
        out[k * width + j] = j < (i64)m.size() ? m[j].first : -1;
        wmax[k * width + j] = j < (i64)m.size() ? m[j].second : 0.0;
      }
    }
    return 0;
  })
}

// Convolution of x [R, ngrid] on the grid (rows = grid) with the wavelet of
// `ksz` taps (or the weights [2, P] given): y [R, G * 2, ngrid].  grid nullptr:
// the whole sky.
int or_conv_forward(const i64* grid, i64 ngrid, i64 nside, int ksz, int G, int gauge, double eps,
                    const double* weights, const double* x, i64 R, double* y) {
  GUARD(-1, {
    ConvOp op;
    std::vector<i64> g;
    if (grid) g.assign(grid, grid + ngrid);
    op.init(g, {}, nside, ksz, G, (Gauge)gauge, eps, 0);
    int P = ksz * ksz;
    auto ker = shared_kernel(weights ? std::vector<double>(weights, weights + 2 * P) : wavelet_weights(ksz), G, P);
    op.forward(ker, x, R, y);
    return 0;
  })
}

int or_conv_adjoint(const i64* grid, i64 ngrid, i64 nside, int ksz, int G, int gauge, double eps,
                    const double* weights, const double* gy, i64 R, double* gx) {
  GUARD(-1, {
    ConvOp op;
    std::vector<i64> g;
    if (grid) g.assign(grid, grid + ngrid);
    op.init(g, {}, nside, ksz, G, (Gauge)gauge, eps, 0);
    int P = ksz * ksz;
    auto ker = shared_kernel(weights ? std::vector<double>(weights, weights + 2 * P) : wavelet_weights(ksz), G, P);
    std::memset(gx, 0, sizeof(double) * R * op.n_in);
    op.adjoint_add(ker, gy, R, gx);
    return 0;
  })
}

i64 or_kth_neighbourhood(i64 id, i64 nside, int k, i64* out) {
  auto v = kth_neighbourhood_set(id, nside, k);
  std::memcpy(out, v.data(), v.size() * sizeof(i64));
  return (i64)v.size();
}

struct DownH {
  std::vector<i64> coarse;
  Csr csr;
};

void* or_down_new(const i64* ids, i64 n, i64 nside) {
  GUARD(nullptr, {
    auto* h = new DownH;
    h->coarse = smooth_decimation(ids, n, nside, h->csr);
    return (void*)h;
  })
}
i64 or_down_nrows(void* h) { return ((DownH*)h)->csr.n_rows; }
i64 or_down_nnz(void* h) { return (i64)((DownH*)h)->csr.values.size(); }
void or_down_get(void* hv, i64* coarse, i64* indptr, i64* indices, double* values) {
  auto* h = (DownH*)hv;
  std::memcpy(coarse, h->coarse.data(), h->coarse.size() * sizeof(i64));
  std::memcpy(indptr, h->csr.indptr.data(), h->csr.indptr.size() * sizeof(i64));
  std::memcpy(indices, h->csr.indices.data(), h->csr.indices.size() * sizeof(i64));
  std::memcpy(values, h->csr.values.data(), h->csr.values.size() * sizeof(double));
}
void or_down_free(void* h) { delete (DownH*)h; }

// plan rows (family, native, c1, c2, j1, j2, j3, l1, l2, l3) of dg(j) = j;
// returns the count (rows written only when it fits in cap)
i64 or_build_plan(int J, int L, int C, int cross_only, int* out, i64 cap) {
  std::vector<int> dg(J);
  for (int j = 0; j < J; ++j) dg[j] = j;
  auto plan = build_plan(J, L, dg, C, cross_only != 0);
  if ((i64)plan.size() <= cap)
    for (size_t i = 0; i < plan.size(); ++i) {
      const Coef& c = plan[i];
      int v[10] = {c.family, c.native, c.c1, c.c2, c.j1, c.j2, c.j3, c.l1, c.l2, c.l3};
      std::memcpy(out + 10 * i, v, sizeof(v));
    }
  return (i64)plan.size();
}

// -- engine ----------------------------------------------------------------
struct EngineH {
  Engine e;
  std::vector<std::vector<double>> mg;
};

void* or_engine_new(i64 nside, int J, int L, int ksz, int gauge, int B, int C, int fewer, const int* j_to_dg,
                    int cross_only, double cache_gb) {
  GUARD(nullptr, {
    auto* h = new EngineH;
    std::vector<int> dg;
    if (j_to_dg) dg.assign(j_to_dg, j_to_dg + J);
    h->e.init(nside, J, L, ksz, (Gauge)gauge, B, C, fewer != 0, dg, cross_only != 0, (size_t)(cache_gb * 1e9));
    return (void*)h;
  })
}
void or_engine_free(void* h) { delete (EngineH*)h; }
i64 or_engine_ncoeff(void* h) { return (i64)((EngineH*)h)->e.plan.size(); }
int or_engine_levels(void* h) { return ((EngineH*)h)->e.levels; }
void or_engine_plan(void* hv, int* out) {
  auto& p = ((EngineH*)hv)->e.plan;
  for (size_t i = 0; i < p.size(); ++i) {
    const Coef& c = p[i];
    int v[10] = {c.family, c.native, c.c1, c.c2, c.j1, c.j2, c.j3, c.l1, c.l2, c.l3};
    std::memcpy(out + 10 * i, v, sizeof(v));
  }
}
int or_engine_set_masks(void* hv, const double* w, i64 K) {
  GUARD(-1, {
    ((EngineH*)hv)->e.set_masks(w, K);
    return 0;
  })
}
int or_engine_set_mask_levels(void* hv, const double* w, i64 K) {
  GUARD(-1, {
    ((EngineH*)hv)->e.set_mask_levels(w, K);
    return 0;
  })
}
i64 or_engine_native_pixels(void* hv, i64* out) {
  auto& e = ((EngineH*)hv)->e;
  i64 np = (i64)e.plan.size();
  for (int k = 0; k < e.K(); ++k)
    for (i64 i = 0; i < np; ++i)
      out[k * np + i] = e.has_masks ? e.masks.counts[k][e.plan[i].native] : e.npix(e.plan[i].native);
  return 0;
}

static void put_values(const std::vector<cplx>& v, double* out) {
  for (size_t i = 0; i < v.size(); ++i) { out[2 * i] = v[i].real(); out[2 * i + 1] = v[i].imag(); }
}

// values: 2 * B * K * ncoeff (re, im interleaved); var: B * K * ncoeff when moments
int or_engine_forward(void* hv, const double* x, int moments, double* values, double* var) {
  GUARD(-1, {
    auto& e = ((EngineH*)hv)->e;
    e.load(x);
    std::vector<cplx> v;
    std::vector<double> second;
    e.forward(v, moments ? &second : nullptr);
    put_values(v, values);
    if (moments)
      for (size_t i = 0; i < v.size(); ++i) var[i] = std::max(second[i] - std::norm(v[i]), 0.0);
    return 0;
  })
}

int or_engine_forward_levels(void* hv, const double* x, double* values) {
  GUARD(-1, {
    auto& e = ((EngineH*)hv)->e;
    e.load_levels(x);
    std::vector<cplx> v;
    e.forward(v, nullptr);
    put_values(v, values);
    return 0;
  })
}

int or_engine_get_map(void* hv, int d, double* out) {
  auto& e = ((EngineH*)hv)->e;
  if (d < 0 || d >= (int)e.maps.size()) return -1;
  std::memcpy(out, e.maps[d].data(), e.maps[d].size() * sizeof(double));
  return 0;
}

int or_engine_get_m(void* hv, int d, int n, double* out) {
  auto& e = ((EngineH*)hv)->e;
  auto it = e.m.find({d, n});
  if (it == e.m.end()) return -1;
  std::memcpy(out, it->second.data(), it->second.size() * sizeof(double));
  return 0;
}

// z of level n: [BC][L][N] complex interleaved
int or_engine_get_z(void* hv, int n, double* out) {
  auto& e = ((EngineH*)hv)->e;
  if (n < 0 || n >= (int)e.z.size()) return -1;
  put_values(e.z[n], out);
  return 0;
}

// maps cotangent of every level (concatenated) after a forward
int or_engine_reverse(void* hv, const double* cot, double* out_levels) {
  GUARD(-1, {
    auto* h = (EngineH*)hv;
    auto& e = h->e;
    size_t n = (size_t)e.B * e.K() * e.plan.size();
    std::vector<cplx> c(n);
    for (size_t i = 0; i < n; ++i) c[i] = cplx(cot[2 * i], cot[2 * i + 1]);
    h->mg = e.reverse(c);
    double* o = out_levels;
    for (auto& v : h->mg) { std::memcpy(o, v.data(), v.size() * sizeof(double)); o += v.size(); }
    return 0;
  })
}

// after or_engine_reverse: level-0 map cotangent and the band cotangents
int or_engine_analysis(void* hv, double* g0, double* bands) {
  GUARD(-1, {
    auto* h = (EngineH*)hv;
    std::vector<double> g;
    std::vector<std::vector<double>> b;
    h->e.analysis_vjp(h->mg, g, b);
    std::memcpy(g0, g.data(), g.size() * sizeof(double));
    double* o = bands;
    for (auto& v : b) { std::memcpy(o, v.data(), v.size() * sizeof(double)); o += v.size(); }
    return 0;
  })
}

}  // extern "C"
