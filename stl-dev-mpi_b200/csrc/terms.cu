// Objective terms of the synthesis on the device (the extra loss terms of
// stl-synth after the statistics): the kappa transform through a monotone
// cubic table, the 4-children pyramid of NESTED rows with the moments of
// its details and the level-power and kurtosis gradients, the stable sort
// of a row in f64 total order with the pixel-marginal term, and g += a b.
// Counterpart of the reference's crates/stl-gpu/src/terms.rs (kernels in
// crates/stl-gpu/src/kernels.cu:1454-1707), reached through the stlp_terms_*
// entry points of include/stl_b200.h.
//
// This file is compiled with --fmad=false: every product is rounded on its
// own and the element-wise expressions run in the order of the host code,
// so the transform, the pyramid and the gradients equal the host's bit for
// bit.  Sums over pixels (moments, the marginal's loss) go by chunks of
// kTermsChunk cells, each in a fixed tree, the chunks added in order: the
// results are deterministic and equal to sequential sums to rounding.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.cuh"
#include "json.hpp"
#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

namespace stl {
namespace {

constexpr i64 kTermsChunk = 1 << 16;  // cells per partial sum
constexpr int kSumThreads = 256;

inline unsigned blocks_of(i64 n, int t) { return (unsigned)((n + t - 1) / t); }

// ---- kappa ----------------------------------------------------------------------
// k = (f(x gs + gm) - km) / ks and dk = f'(x gs + gm) gs / ks, f the cubic
// Hermite interpolant of knots kx (increasing), values ky and slopes kd,
// continued linearly outside the knots; the interval is the last knot <= t.
__global__ void k_kappa(const double* __restrict__ x, i64 n, const double* __restrict__ kx,
                        const double* __restrict__ ky, const double* __restrict__ kd, int nk, double gm, double gs,
                        double km, double ks, double* __restrict__ k, double* __restrict__ dk) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double t = x[i] * gs + gm;
  double v, dv;
  if (t <= kx[0]) {
    v = ky[0] + kd[0] * (t - kx[0]);
    dv = kd[0];
  } else if (t >= kx[nk - 1]) {
    v = ky[nk - 1] + kd[nk - 1] * (t - kx[nk - 1]);
    dv = kd[nk - 1];
  } else {
    int a = 0, b = nk - 1;  // kx[a] <= t < kx[b]
    while (b - a > 1) {
      const int m = (a + b) >> 1;
      if (kx[m] <= t) a = m; else b = m;
    }
    const double h = kx[a + 1] - kx[a];
    const double u = (t - kx[a]) / h;
    const double y0 = ky[a], y1 = ky[a + 1], d0 = kd[a] * h, d1 = kd[a + 1] * h;
    const double u2 = u * u, u3 = u * u * u;
    v = (2.0 * u3 - 3.0 * u2 + 1.0) * y0 + (u3 - 2.0 * u2 + u) * d0 + (3.0 * u2 - 2.0 * u3) * y1 + (u3 - u2) * d1;
    const double w = (6.0 * u2 - 6.0 * u) * (y0 - y1) + (3.0 * u2 - 4.0 * u + 1.0) * d0 + (3.0 * u2 - 2.0 * u) * d1;
    dv = w / h;
  }
  k[i] = (v - km) / ks;
  dk[i] = dv * gs / ks;
}

// ---- pyramid ------------------------------------------------------------------------
// parent j of row r: (((c0 + c1) + c2) + c3) / 4 over x[r xs + 4 j + .]
__global__ void k_quad_parents(const double* __restrict__ x, i64 xs, i64 m, int rows, double* __restrict__ out) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m * rows) return;
  const i64 r = t / m, j = t - r * m;
  const double2* c = reinterpret_cast<const double2*>(x + r * xs + 4 * j);
  const double2 a = c[0], b = c[1];
  out[t] = (((a.x + a.y) + b.x) + b.y) / 4.0;
}

// partial (sum d^2, sum d^4) of the details d_j = a[j] - p[j / 4] of row
// blockIdx.y over chunk blockIdx.x of kTermsChunk cells, in a fixed tree:
// part[(r nch + c) 2 + {0, 1}]
__global__ void __launch_bounds__(kSumThreads) k_detail_sums(const double* __restrict__ a, i64 as,
                                                            const double* __restrict__ p, i64 ps, i64 m,
                                                            double* __restrict__ part) {
  __shared__ double s2[kSumThreads], s4[kSumThreads];
  const int r = blockIdx.y, tid = threadIdx.x;
  const i64 c = blockIdx.x, nch = gridDim.x;
  const i64 lo = c * kTermsChunk, hi = min(lo + kTermsChunk, m);
  const double* ar = a + (i64)r * as;
  const double* pr = p + (i64)r * ps;
  double t2 = 0.0, t4 = 0.0;
  for (i64 j = lo + tid; j < hi; j += kSumThreads) {
    const double d = ar[j] - pr[j >> 2];
    t2 += d * d;
    t4 += d * d * d * d;
  }
  s2[tid] = t2;
  s4[tid] = t4;
  __syncthreads();
  for (int h = kSumThreads / 2; h > 0; h >>= 1) {
    if (tid < h) {
      s2[tid] += s2[tid + h];
      s4[tid] += s4[tid + h];
    }
    __syncthreads();
  }
  if (tid == 0) {
    part[((i64)r * nch + c) * 2] = s2[0];
    part[((i64)r * nch + c) * 2 + 1] = s4[0];
  }
}

// out[(r D + n) w + k] = sum over the chunks, in order, of part[(r nch + c) w + k]
__global__ void k_chunk_totals(const double* __restrict__ part, int rows, i64 nch, int w, int D, int n,
                               double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * w) return;
  const int r = i / w, k = i - r * w;
  double s = 0.0;
  for (i64 c = 0; c < nch; ++c) s += part[((i64)r * nch + c) * w + k];
  out[((i64)r * D + n) * w + k] = s;
}

// level address table: lv[n] (n = 0 the maps), row strides ls[n]
struct Levels {
  const double* lv[32];
  i64 ls[32];
};

// g[r, i] += sum_{n < L} coef[r L + n] (lv[n][r, i >> 2n] - lv[n + 1][r, i >> 2(n + 1)]),
// the sum from 0 in level order, added to g last
__global__ void k_level_power_grad(Levels lv, int L, const double* __restrict__ coef, i64 len, int rows,
                                   double* __restrict__ g) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len * rows) return;
  const i64 r = t / len, i = t - r * len;
  double acc = 0.0;
  for (int n = 0; n < L; ++n) {
    const double d = lv.lv[n][r * lv.ls[n] + (i >> (2 * n))] - lv.lv[n + 1][r * lv.ls[n + 1] + (i >> (2 * n + 2))];
    acc = acc + coef[r * L + n] * d;
  }
  g[t] = g[t] + acc;
}

// g[r, i] += (dk[r, i]) sum_k cf0 (d^3 - c - (cf1 cf2) d) over the levels
// lev[k], d the level's detail of pixel i and c the mean of the cubes of
// its four siblings' details, cf [r][T][3]
__global__ void k_kurtosis_grad(Levels lv, const int* __restrict__ lev, int T, const double* __restrict__ cf, i64 len,
                                int rows, const double* __restrict__ dk, double* __restrict__ g) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len * rows) return;
  const i64 r = t / len, i = t - r * len;
  double acc = 0.0;
  for (int k = 0; k < T; ++k) {
    const int n = lev[k];
    const double* a = lv.lv[n] + r * lv.ls[n];
    const i64 j = i >> (2 * n), j0 = j & ~i64(3);
    const double pv = lv.lv[n + 1][r * lv.ls[n + 1] + (j >> 2)];
    const double e0 = a[j0] - pv, e1 = a[j0 + 1] - pv, e2 = a[j0 + 2] - pv, e3 = a[j0 + 3] - pv;
    const double c = (((e0 * e0 * e0 + e1 * e1 * e1) + e2 * e2 * e2) + e3 * e3 * e3) / 4.0;
    const double d = a[j] - pv;
    const double* q = cf + (r * T + k) * 3;
    const double kv = q[1] * q[2];
    acc = acc + q[0] * (((d * d * d) - c) - kv * d);
  }
  g[t] = g[t] + (dk ? acc * dk[t] : acc);
}

// g += a b (b null: g += a)
__global__ void k_add_product(double* __restrict__ g, const double* __restrict__ a, const double* __restrict__ b,
                              i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  g[i] = g[i] + (b ? a[i] * b[i] : a[i]);
}

// ---- stable sort in f64 total order -------------------------------------------------
// LSD radix sort of u64 keys (8 passes of 8-bit digits) with the positions
// as payload.  Per pass: per-tile digit counts, their exclusive scan in
// (digit, tile) order, then a stable scatter in which each tile first sorts
// its keys by digit in shared memory (warp-level ranks in index order:
// rounds of 32 keys, __match_any_sync on the digit) and then writes every
// digit's run contiguously, so the global stores are coalesced.
constexpr int kSortThreads = 512;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;    // 4096 keys
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kWarpKeys = kSortTile / kSortWarps;       // 256 keys per warp, in index order
constexpr size_t kSortSmem = (sizeof(uint64_t) + sizeof(uint32_t)) * kSortTile;

// keys ordering as f64 total order: negative values have every bit flipped,
// the others the sign bit set
__global__ void k_sort_init(const double* __restrict__ x, i64 n, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ vals) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t b = (uint64_t)__double_as_longlong(x[i]);
  keys[i] = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
  vals[i] = (uint32_t)i;
}

// counts[d * ntiles + tile]: keys of the tile with digit d
__global__ void __launch_bounds__(kSortThreads) k_sort_count(const uint64_t* __restrict__ keys, i64 n, int shift,
                                                             uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[256];
  const int tid = threadIdx.x;
  const i64 tile = blockIdx.x, ntiles = gridDim.x;
  if (tid < 256) h[tid] = 0;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const i64 i = tile * kSortTile + (i64)k * kSortThreads + tid;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1u);
  }
  __syncthreads();
  if (tid < 256) counts[(i64)tid * ntiles + tile] = h[tid];
}

// exclusive scan of counts [256][ntiles] in (digit, tile) order, one block
// of 256 threads: thread d scans its digit's row, then the digit totals
__global__ void __launch_bounds__(256) k_sort_scan(uint32_t* __restrict__ counts, i64 ntiles) {
  __shared__ uint32_t tot[256];
  const int d = threadIdx.x;
  uint32_t* row = counts + (i64)d * ntiles;
  uint32_t s = 0;
  for (i64 t = 0; t < ntiles; ++t) {
    const uint32_t c = row[t];
    row[t] = s;
    s += c;
  }
  tot[d] = s;
  __syncthreads();
  if (d == 0) {
    uint32_t acc = 0;
    for (int k = 0; k < 256; ++k) {
      const uint32_t c = tot[k];
      tot[k] = acc;
      acc += c;
    }
  }
  __syncthreads();
  const uint32_t base = tot[d];
  for (i64 t = 0; t < ntiles; ++t) row[t] += base;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const uint64_t* __restrict__ kin,
                                                               const uint32_t* __restrict__ vin, i64 n, int shift,
                                                               const uint32_t* __restrict__ offs,
                                                               uint64_t* __restrict__ kout,
                                                               uint32_t* __restrict__ vout) {
  extern __shared__ __align__(16) unsigned char sort_smem[];  // keys [kSortTile] u64, then positions [kSortTile] u32
  uint64_t* sk = reinterpret_cast<uint64_t*>(sort_smem);
  uint32_t* sv = reinterpret_cast<uint32_t*>(sort_smem + sizeof(uint64_t) * kSortTile);
  __shared__ uint32_t wcount[kSortWarps][257];  // per warp: keys of each digit; then exclusive per digit over warps
  __shared__ uint32_t dstart[257];              // tile-local start of each digit's run
  __shared__ uint32_t gbase[256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const i64 tile = blockIdx.x, ntiles = gridDim.x;
  for (int i = tid; i < kSortWarps * 257; i += kSortThreads) (&wcount[0][0])[i] = 0;
  if (tid < 256) gbase[tid] = offs[(i64)tid * ntiles + tile];
  __syncthreads();
  // ranks within the warp's 256 keys (index order), by rounds of 32
  uint64_t key[kSortItems];
  uint32_t val[kSortItems];
  int dig[kSortItems], rank[kSortItems];
  const i64 w0 = tile * kSortTile + (i64)warp * kWarpKeys;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const i64 i = w0 + k * 32 + lane;
    const bool ok = i < n;
    key[k] = ok ? kin[i] : 0;
    val[k] = ok ? vin[i] : 0;
    dig[k] = ok ? (int)((key[k] >> shift) & 255) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, dig[k]);
    const int below = __popc(peers & ((1u << lane) - 1u));
    rank[k] = (int)wcount[warp][dig[k]] + below;
    __syncwarp();
    if (below == 0) wcount[warp][dig[k]] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit: exclusive prefix over the warps, and the digit totals' prefix
  if (tid < 257) {
    uint32_t s = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = wcount[w][tid];
      wcount[w][tid] = s;
      s += c;
    }
    dstart[tid] = s;  // the digit's total, scanned below
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t acc = 0;
    for (int d = 0; d < 257; ++d) {
      const uint32_t c = dstart[d];
      dstart[d] = acc;
      acc += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const int pos = (int)(dstart[dig[k]] + wcount[warp][dig[k]]) + rank[k];
    sk[pos] = key[k];
    sv[pos] = val[k];
  }
  __syncthreads();
  const int valid = (int)min((i64)kSortTile, n - tile * kSortTile);
  for (int p = tid; p < valid; p += kSortThreads) {
    const uint64_t k = sk[p];
    const int d = (int)((k >> shift) & 255);
    const uint32_t dst = gbase[d] + (uint32_t)(p - (int)dstart[d]);
    kout[dst] = k;
    vout[dst] = sv[p];
  }
}

// the marginal of one row: d_q = x[perm[q]] - t[q], g[perm[q]] += coef d_q,
// part[c] = sum of d_q^2 over chunk c of positions (fixed tree)
__global__ void __launch_bounds__(kSumThreads) k_marginal(const double* __restrict__ x,
                                                         const uint32_t* __restrict__ perm,
                                                         const double* __restrict__ ts, i64 n, double coef,
                                                         double* __restrict__ g, double* __restrict__ part) {
  __shared__ double s[kSumThreads];
  const int tid = threadIdx.x;
  const i64 c = blockIdx.x;
  const i64 lo = c * kTermsChunk, hi = min(lo + kTermsChunk, n);
  double acc = 0.0;
  for (i64 q = lo + tid; q < hi; q += kSumThreads) {
    const uint32_t p = perm[q];
    const double d = x[p] - ts[q];
    acc += d * d;
    g[p] = g[p] + coef * d;
  }
  s[tid] = acc;
  __syncthreads();
  for (int h = kSumThreads / 2; h > 0; h >>= 1) {
    if (tid < h) s[tid] += s[tid + h];
    __syncthreads();
  }
  if (tid == 0) part[c] = s[0];
}

}  // namespace
}  // namespace stl

using namespace stl;

struct StlpTerms {
  int device = 0;
  cudaStream_t stream = nullptr;
  i64 rows = 0, len = 0;
  int depth = 0;
  i64 sort_max = 0;
  bool have_pyramid = false;
  std::vector<DevMem> levels;  // levels 1..depth: [rows][len >> 2n]
  DevMem kx, ky, kd;
  int nk = 0;
  DevMem part;                 // chunk partial sums
  DevMem totals;               // [rows][depth][2]
  DevMem coef;                 // [rows][depth]
  DevMem cf;                   // [rows][depth][3]
  DevMem lev;                  // [depth] int
  DevMem keys[2], vals[2], counts;
  Levels table(uint64_t x) const {
    Levels t{};
    t.lv[0] = reinterpret_cast<const double*>(x);
    t.ls[0] = len;
    for (int n = 1; n <= depth; ++n) {
      t.lv[n] = levels[n - 1].as<double>();
      t.ls[n] = len >> (2 * n);
    }
    return t;
  }
};

namespace {

template <typename R, typename F>
R guard(R fail, F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    stl::set_error(e.what());
  } catch (...) {
    stl::set_error("unknown native failure");
  }
  return fail;
}

void need(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

void check_launch() { STL_CUDA(cudaGetLastError()); }

// the stream's work, then the host: a checked wait
void wait(StlpTerms* h) { STL_CUDA(cudaStreamSynchronize(h->stream)); }

void set_device(StlpTerms* h) { STL_CUDA(cudaSetDevice(h->device)); }

}  // namespace

extern "C" {

StlpTerms* stlp_terms_new(const char* config) {
  return guard<StlpTerms*>(nullptr, [&] {
    need(config != nullptr, "null configuration");
    Json v = Json::parse(config);
    auto h = std::make_unique<StlpTerms>();
    h->rows = v.integer("rows", 1);
    h->len = v.integer("len", 0);
    h->depth = (int)v.integer("depth", 0);
    h->sort_max = v.integer("sort", 0);
    h->device = (int)v.integer("device", 0);
    need(h->rows >= 1 && h->len >= 0 && h->depth >= 0 && h->sort_max >= 0, "terms sizes must not be negative");
    need(h->depth <= 30, "pyramid depth above 30");
    need(h->depth == 0 || (h->len > 0 && h->len % ((i64)1 << (2 * h->depth)) == 0),
         "rows not aligned on the pyramid: len must be a multiple of 4^depth");
    need(h->sort_max < (i64)UINT32_MAX, "sort size above 2^32 - 1");
    set_device(h.get());
    for (int n = 1; n <= h->depth; ++n) h->levels.emplace_back(sizeof(double) * h->rows * (h->len >> (2 * n)));
    const i64 nch = std::max<i64>((std::max(h->len, h->sort_max) + kTermsChunk - 1) / kTermsChunk, 1);
    h->part.alloc(sizeof(double) * 2 * h->rows * nch);
    h->totals.alloc(sizeof(double) * 2 * h->rows * std::max(h->depth, 1));
    h->coef.alloc(sizeof(double) * h->rows * std::max(h->depth, 1));
    h->cf.alloc(sizeof(double) * 3 * h->rows * std::max(h->depth, 1));
    h->lev.alloc(sizeof(int) * std::max(h->depth, 1));
    if (h->sort_max > 0) {
      for (int b = 0; b < 2; ++b) {
        h->keys[b].alloc(sizeof(uint64_t) * h->sort_max);
        h->vals[b].alloc(sizeof(uint32_t) * h->sort_max);
      }
      h->counts.alloc(sizeof(uint32_t) * 256 * ((h->sort_max + kSortTile - 1) / kSortTile));
    }
    return h.release();
  });
}

void stlp_terms_free(StlpTerms* h) { delete h; }

int stlp_terms_set_stream(StlpTerms* h, uint64_t stream) {
  return guard<int>(-1, [&] {
    need(h != nullptr, "null handle");
    h->stream = reinterpret_cast<cudaStream_t>(stream);
    return 0;
  });
}

int stlp_terms_kappa_table(StlpTerms* h, const double* x, const double* y, const double* d, size_t nk) {
  return guard<int>(-1, [&] {
    need(h && x && y && d, "null argument");
    need(nk >= 2, "the kappa table needs at least two knots");
    for (size_t i = 0; i + 1 < nk; ++i) need(x[i] < x[i + 1], "kappa knots must increase");
    set_device(h);
    h->kx.alloc(8 * nk);
    h->ky.alloc(8 * nk);
    h->kd.alloc(8 * nk);
    STL_CUDA(cudaMemcpyAsync(h->kx.p, x, 8 * nk, cudaMemcpyHostToDevice, h->stream));
    STL_CUDA(cudaMemcpyAsync(h->ky.p, y, 8 * nk, cudaMemcpyHostToDevice, h->stream));
    STL_CUDA(cudaMemcpyAsync(h->kd.p, d, 8 * nk, cudaMemcpyHostToDevice, h->stream));
    wait(h);
    h->nk = (int)nk;
    return 0;
  });
}

int stlp_terms_kappa(StlpTerms* h, uint64_t x, size_t n, double gm, double gs, double km, double ks, uint64_t k,
                     uint64_t dk) {
  return guard<int>(-1, [&] {
    need(h && x && k && dk, "null argument");
    need(h->nk >= 2, "no kappa table (stlp_terms_kappa_table)");
    set_device(h);
    if (n)
      k_kappa<<<blocks_of((i64)n, 256), 256, 0, h->stream>>>(
          reinterpret_cast<const double*>(x), (i64)n, h->kx.as<double>(), h->ky.as<double>(), h->kd.as<double>(),
          h->nk, gm, gs, km, ks, reinterpret_cast<double*>(k), reinterpret_cast<double*>(dk));
    check_launch();
    return 0;
  });
}

int stlp_terms_pyramid(StlpTerms* h, uint64_t x) {
  return guard<int>(-1, [&] {
    need(h && x, "null argument");
    set_device(h);
    for (int n = 1; n <= h->depth; ++n) {
      const i64 m = h->len >> (2 * n);
      const double* src = n == 1 ? reinterpret_cast<const double*>(x) : h->levels[n - 2].as<double>();
      const i64 xs = n == 1 ? h->len : 4 * m;
      k_quad_parents<<<blocks_of(m * h->rows, 256), 256, 0, h->stream>>>(src, xs, m, (int)h->rows,
                                                                         h->levels[n - 1].as<double>());
      check_launch();
    }
    h->have_pyramid = true;
    return 0;
  });
}

int stlp_terms_moments(StlpTerms* h, uint64_t x, double* out) {
  return guard<int>(-1, [&] {
    need(h && x && out, "null argument");
    need(h->have_pyramid, "no pyramid (stlp_terms_pyramid)");
    set_device(h);
    const Levels t = h->table(x);
    for (int n = 0; n < h->depth; ++n) {
      const i64 m = h->len >> (2 * n);
      const i64 nch = (m + kTermsChunk - 1) / kTermsChunk;
      k_detail_sums<<<dim3((unsigned)nch, (unsigned)h->rows), kSumThreads, 0, h->stream>>>(
          t.lv[n], t.ls[n], t.lv[n + 1], t.ls[n + 1], m, h->part.as<double>());
      check_launch();
      k_chunk_totals<<<blocks_of(2 * h->rows, 64), 64, 0, h->stream>>>(h->part.as<double>(), (int)h->rows, nch, 2,
                                                                      h->depth, n, h->totals.as<double>());
      check_launch();
    }
    if (h->depth)
      STL_CUDA(cudaMemcpyAsync(out, h->totals.p, sizeof(double) * 2 * h->rows * h->depth, cudaMemcpyDeviceToHost,
                               h->stream));
    wait(h);
    return 0;
  });
}

int stlp_terms_level_power_grad(StlpTerms* h, uint64_t x, const double* coef, size_t L, uint64_t g) {
  return guard<int>(-1, [&] {
    need(h && x && g && (coef || L == 0), "null argument");
    need(h->have_pyramid, "no pyramid (stlp_terms_pyramid)");
    need((int)L <= h->depth, "more level-power levels than the pyramid holds");
    set_device(h);
    if (L)
      STL_CUDA(cudaMemcpyAsync(h->coef.p, coef, sizeof(double) * h->rows * L, cudaMemcpyHostToDevice, h->stream));
    k_level_power_grad<<<blocks_of(h->len * h->rows, 256), 256, 0, h->stream>>>(
        h->table(x), (int)L, h->coef.as<double>(), h->len, (int)h->rows, reinterpret_cast<double*>(g));
    check_launch();
    wait(h);  // the coefficients' staging buffer is reused by the next call
    return 0;
  });
}

int stlp_terms_kurtosis_grad(StlpTerms* h, uint64_t x, const int* levels, size_t T, const double* cf, uint64_t dk,
                             uint64_t g) {
  return guard<int>(-1, [&] {
    need(h && x && g && ((levels && cf) || T == 0), "null argument");
    need(h->have_pyramid, "no pyramid (stlp_terms_pyramid)");
    need((int)T <= h->depth, "more kurtosis levels than the pyramid holds");
    for (size_t k = 0; k < T; ++k) need(levels[k] >= 0 && levels[k] < h->depth, "kurtosis level outside the pyramid");
    set_device(h);
    if (T) {
      STL_CUDA(cudaMemcpyAsync(h->lev.p, levels, sizeof(int) * T, cudaMemcpyHostToDevice, h->stream));
      STL_CUDA(cudaMemcpyAsync(h->cf.p, cf, sizeof(double) * 3 * h->rows * T, cudaMemcpyHostToDevice, h->stream));
    }
    k_kurtosis_grad<<<blocks_of(h->len * h->rows, 256), 256, 0, h->stream>>>(
        h->table(x), h->lev.as<int>(), (int)T, h->cf.as<double>(), h->len, (int)h->rows,
        reinterpret_cast<const double*>(dk), reinterpret_cast<double*>(g));
    check_launch();
    wait(h);
    return 0;
  });
}

int stlp_terms_add_product(StlpTerms* h, uint64_t g, uint64_t a, uint64_t b, size_t n) {
  return guard<int>(-1, [&] {
    need(h && g && a, "null argument");
    set_device(h);
    if (n)
      k_add_product<<<blocks_of((i64)n, 256), 256, 0, h->stream>>>(reinterpret_cast<double*>(g),
                                                                   reinterpret_cast<const double*>(a),
                                                                   reinterpret_cast<const double*>(b), (i64)n);
    check_launch();
    return 0;
  });
}

int stlp_terms_sort(StlpTerms* h, uint64_t x, size_t n, uint64_t perm) {
  return guard<int>(-1, [&] {
    need(h && x && perm, "null argument");
    need((i64)n <= h->sort_max, "more values than the handle's sort size");
    set_device(h);
    if (n == 0) return 0;
    const i64 nn = (i64)n, tiles = (nn + kSortTile - 1) / kSortTile;
    allow_dynamic_smem(k_sort_scatter);
    k_sort_init<<<blocks_of(nn, 256), 256, 0, h->stream>>>(reinterpret_cast<const double*>(x), nn,
                                                           h->keys[0].as<uint64_t>(), h->vals[0].as<uint32_t>());
    check_launch();
    for (int pass = 0; pass < 8; ++pass) {
      const int a = pass & 1, b = a ^ 1, shift = 8 * pass;
      uint32_t* vout = pass == 7 ? reinterpret_cast<uint32_t*>(perm) : h->vals[b].as<uint32_t>();
      k_sort_count<<<(unsigned)tiles, kSortThreads, 0, h->stream>>>(h->keys[a].as<uint64_t>(), nn, shift,
                                                                      h->counts.as<uint32_t>());
      check_launch();
      k_sort_scan<<<1, 256, 0, h->stream>>>(h->counts.as<uint32_t>(), tiles);
      check_launch();
      k_sort_scatter<<<(unsigned)tiles, kSortThreads, kSortSmem, h->stream>>>(
          h->keys[a].as<uint64_t>(), h->vals[a].as<uint32_t>(), nn, shift, h->counts.as<uint32_t>(),
          h->keys[b].as<uint64_t>(), vout);
      check_launch();
    }
    return 0;
  });
}

int stlp_terms_marginal(StlpTerms* h, uint64_t x, uint64_t perm, uint64_t t_sorted, size_t n, double coef,
                        uint64_t g, double* sum_sq) {
  return guard<int>(-1, [&] {
    need(h && x && perm && t_sorted && g && sum_sq, "null argument");
    need((i64)n <= std::max(h->len, h->sort_max), "more values than the handle holds");
    set_device(h);
    *sum_sq = 0.0;
    if (n == 0) return 0;
    const i64 nch = ((i64)n + kTermsChunk - 1) / kTermsChunk;
    k_marginal<<<(unsigned)nch, kSumThreads, 0, h->stream>>>(
        reinterpret_cast<const double*>(x), reinterpret_cast<const uint32_t*>(perm),
        reinterpret_cast<const double*>(t_sorted), (i64)n, coef, reinterpret_cast<double*>(g), h->part.as<double>());
    check_launch();
    k_chunk_totals<<<1, 64, 0, h->stream>>>(h->part.as<double>(), 1, nch, 1, 1, 0, h->totals.as<double>());
    check_launch();
    STL_CUDA(cudaMemcpyAsync(sum_sq, h->totals.p, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    wait(h);
    return 0;
  });
}

}  // extern "C"
