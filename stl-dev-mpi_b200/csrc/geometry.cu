// Device builders of the engine's operators, in FP64.
//
// build_conv: for every output row, the G rotated ksz x ksz stencils are
// interpolated bilinearly on the RING grid, bound to the input grid with
// renormalised weights (crates/stl-core/src/conv.rs:73-135, including the
// central-tap fallback and the eps threshold of disc patches), and folded
// with the f32-rounded wavelet kernel into one coefficient per (cell read,
// gauge, re/im) -- the per-row form of the reference's DIA coefficients
// (crates/stl-core/src/dia.rs:213-238), kept as a list of cells instead of
// face-frame diagonals so the same operator serves every level (nside 1
// included) and partial grids.
//
// build_dec: the smooth decimation rows (crates/stl-core/src/decimation.rs):
// candidates are the children of the 2-ring coarse neighbourhood (all fine
// pixels below coarse nside 4), Gaussian weights of the haversine distance
// within 3 fine pixels, l1-normalised, zeros dropped; then the transpose.
#include <algorithm>
#include <cstring>

#include "engine.cuh"
#include "healpix.cuh"

namespace stl {

namespace {

constexpr int kFoldCap = 128;  // distinct cells one row may read
constexpr int kDecCap = 256;   // candidates of one decimation row
constexpr uint32_t kSentinel = 0xFFFFFFFFu;

__device__ __forceinline__ i64 grid_find(const i64* grid, i64 n, i64 v) {
  if (!grid) return (v >= 0 && v < n) ? v : -1;
  i64 lo = 0, hi = n;
  while (lo < hi) {
    i64 mid = (lo + hi) >> 1;
    if (grid[mid] < v) lo = mid + 1; else hi = mid;
  }
  return (lo < n && grid[lo] == v) ? lo : -1;
}

struct FoldArgs {
  i64 nside;
  int order, ksz, P, G, gauge, p_ref;
  double eps;
  const i64* grid;
  i64 n_in;
  const i64* rows;
  i64 n_rows;
  const double* stencil;  // [P][3]
  const double* kernel;   // [G][2][P]
};

// One thread per output row: bind and fold.  Pass 1 (cell == nullptr)
// only counts the distinct cells; pass 2 writes the S slots.
template <typename T>
__global__ void k_fold(FoldArgs a, int* counts, int S, int32_t* cell, T* coef, int* overflow) {
  i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n_rows) return;
  i64 id = a.rows ? a.rows[k] : (a.grid ? a.grid[k] : k);
  double theta, phi;
  pix2ang_nest(id, a.nside, theta, phi);
  theta = deg2rad(90.0 - rad2deg(kPi / 2.0 - theta));
  phi = deg2rad(rad2deg(phi));
  int32_t cells[kFoldCap];
  double acc[kFoldCap][8];
  int n = 0;
  bool over = false;
  for (int g = 0; g < a.G; ++g) {
    double R[9];
    rotation_matrix(theta, phi, g, a.G, a.gauge, R);
    i64 ref_pix[4];
    double ref_w[4];
    {
      const double* v = a.stencil + 3 * a.p_ref;
      double u[3] = {R[0] * v[0] + R[1] * v[1] + R[2] * v[2], R[3] * v[0] + R[4] * v[1] + R[5] * v[2],
                     R[6] * v[0] + R[7] * v[1] + R[8] * v[2]};
      interp_weights_nested(u, a.order, ref_pix, ref_w);
    }
    for (int t = 0; t < a.P; ++t) {
      const double* v = a.stencil + 3 * t;
      double u[3] = {R[0] * v[0] + R[1] * v[1] + R[2] * v[2], R[3] * v[0] + R[4] * v[1] + R[5] * v[2],
                     R[6] * v[0] + R[7] * v[1] + R[8] * v[2]};
      i64 ipx[4];
      double iw[4];
      interp_weights_nested(u, a.order, ipx, iw);
      i64 found[4];
      const i64* ix = ipx;
      const double* wx = iw;
      for (int q = 0; q < 4; ++q) {
        found[q] = grid_find(a.grid, a.n_in, ix[q]);
        if (a.eps > 0.0 && wx[q] <= a.eps) found[q] = -1;
      }
      if (found[0] < 0 && found[1] < 0 && found[2] < 0 && found[3] < 0) {  // empty tap: central tap
        ix = ref_pix;
        wx = ref_w;
        for (int q = 0; q < 4; ++q) {
          found[q] = grid_find(a.grid, a.n_in, ix[q]);
          if (a.eps > 0.0 && wx[q] <= a.eps) found[q] = -1;
        }
      }
      double w[4];
      for (int q = 0; q < 4; ++q) w[q] = wx[q] * (found[q] >= 0 ? 1.0 : 0.0);
      double colsum = w[0] + w[1] + w[2] + w[3];
      if (colsum == 0.0) {
        w[0] = found[0] >= 0 ? 1.0 : 0.0;
        colsum = w[0] + w[1] + w[2] + w[3];
      }
      double inv = colsum > 1e-12 ? colsum : 1e-12;
      for (int q = 0; q < 4; ++q) {
        double wn = w[q] / inv;
        if (wn == 0.0 || found[q] < 0) continue;
        int32_t c = (int32_t)found[q];
        int slot = -1;
        for (int j = 0; j < n; ++j)
          if (cells[j] == c) { slot = j; break; }
        if (slot < 0) {
          if (n >= kFoldCap) { over = true; continue; }
          slot = n++;
          cells[slot] = c;
          for (int o = 0; o < 8; ++o) acc[slot][o] = 0.0;
        }
        if (cell) {
          acc[slot][2 * g + 0] += a.kernel[(g * 2 + 0) * a.P + t] * wn;
          acc[slot][2 * g + 1] += a.kernel[(g * 2 + 1) * a.P + t] * wn;
        }
      }
    }
  }
  if (over) atomicExch(overflow, 1);
  counts[k] = n;
  if (!cell) return;
  int32_t pad = n > 0 ? cells[0] : 0;
  for (int s = 0; s < S; ++s) {
    i64 e = (i64)s * a.n_rows + k;
    cell[e] = s < n ? cells[s] : pad;
    for (int o = 0; o < 2 * a.G; ++o) coef[e * (2 * a.G) + o] = (T)(s < n ? acc[s][o] : 0.0);
  }
}

__global__ void k_max_int(const int* v, i64 n, int* out) {
  int m = 0;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) m = max(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// transposed table of a slot-major ELL: entries (row << shift | slot) per column
__global__ void k_tcount(const int32_t* cell, const int* counts, i64 n_rows, int S, int* tcount) {
  i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_rows) return;
  int n = counts ? counts[k] : S;
  for (int s = 0; s < n; ++s) atomicAdd(&tcount[cell[(i64)s * n_rows + k]], 1);
}

__global__ void k_tfill(const int32_t* cell, const int* counts, i64 n_rows, int S, int shift, i64 n_in, int* tfill,
                        uint32_t* tent) {
  i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_rows) return;
  int n = counts ? counts[k] : S;
  for (int s = 0; s < n; ++s) {
    int32_t c = cell[(i64)s * n_rows + k];
    int pos = atomicAdd(&tfill[c], 1);
    tent[(i64)pos * n_in + c] = (uint32_t)(((uint64_t)k << shift) | (uint64_t)s);
  }
}

__global__ void k_tsort(uint32_t* tent, const int* tcount, i64 n_in, int ST) {
  i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_in) return;
  int n = tcount[c];
  for (int i = 1; i < n; ++i) {  // insertion sort: a fixed order of the gathered sums
    uint32_t v = tent[(i64)i * n_in + c];
    int j = i - 1;
    while (j >= 0 && tent[(i64)j * n_in + c] > v) {
      tent[(i64)(j + 1) * n_in + c] = tent[(i64)j * n_in + c];
      --j;
    }
    tent[(i64)(j + 1) * n_in + c] = v;
  }
  for (int i = n; i < ST; ++i) tent[(i64)i * n_in + c] = kSentinel;
}

// ---- decimation ------------------------------------------------------------
struct DecArgs {
  i64 nside;      // fine
  int order, corder;
  const i64* ids;  // fine grid (nullptr: whole sky)
  i64 n_in;
  const i64* out;  // coarse rows (nullptr: whole sky)
  i64 n_out;
  double radius, sigma;
};

__device__ __forceinline__ double haversine(double lat1, double lon1, double lat2, double lon2) {
  double dlat = 0.5 * (lat2 - lat1);
  double dlon = 0.5 * (lon2 - lon1);
  double sa = sin(dlat), so = sin(dlon);
  double a = sa * sa + cos(lat1) * cos(lat2) * (so * so);
  a = a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a);
  return 2.0 * asin(sqrt(a));
}

template <typename T>
__global__ void k_dec_rows(DecArgs a, int* counts, int W, int32_t* col, T* wout, int* overflow) {
  i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.n_out) return;
  i64 c = a.out ? a.out[r] : r;
  i64 cn = a.nside / 2;
  i64 cand[kDecCap];
  int n = 0;
  bool over = false;
  auto push = [&](i64 fine) {
    i64 q = grid_find(a.ids, a.n_in, fine);
    if (q < 0) return;
    if (n >= kDecCap) { over = true; return; }
    cand[n++] = q;
  };
  if (cn >= 4) {
    i64 x, y, f;
    nest2xyf(c, a.corder, x, y, f);
    for (int dy = -2; dy <= 2; ++dy)
      for (int dx = -2; dx <= 2; ++dx) {
        i64 v;
        if (ext_pix(f, x + dx, y + dy, cn, a.corder, v))
          for (int ch = 0; ch < 4; ++ch) push(4 * v + ch);
      }
  } else {
    for (i64 v = 0; v < npix_of(a.nside); ++v) push(v);
  }
  for (int i = 1; i < n; ++i) {  // sort the fine positions, then dedup
    i64 v = cand[i];
    int j = i - 1;
    while (j >= 0 && cand[j] > v) { cand[j + 1] = cand[j]; --j; }
    cand[j + 1] = v;
  }
  int m = 0;
  for (int i = 0; i < n; ++i)
    if (m == 0 || cand[m - 1] != cand[i]) cand[m++] = cand[i];
  n = m;
  double lon_c, lat_c;
  centre_lonlat(c, cn, lon_c, lat_c);
  double w[kDecCap];
  double row_sum = 0.0;
  for (int i = 0; i < n; ++i) {
    i64 fine = a.ids ? a.ids[cand[i]] : cand[i];
    double lon_f, lat_f;
    centre_lonlat(fine, a.nside, lon_f, lat_f);
    double gamma = haversine(lat_c, lon_c, lat_f, lon_f);
    double t = gamma / a.sigma;
    w[i] = gamma > a.radius ? 0.0 : exp(-0.5 * (t * t));
    row_sum += w[i];
  }
  if (row_sum <= 0.0 && n > 0) {  // every candidate cut: uniform
    double u = 1.0 / (double)n;
    row_sum = 0.0;
    for (int i = 0; i < n; ++i) { w[i] = u; row_sum += u; }
  }
  double scale = row_sum > 1e-300 ? row_sum : 1e-300;
  int k = 0;
  for (int i = 0; i < n; ++i) {
    double v = w[i] / scale;
    if (v == 0.0) continue;
    if (col && k < W) {
      col[(i64)k * a.n_out + r] = (int32_t)cand[i];
      wout[(i64)k * a.n_out + r] = (T)v;
    }
    ++k;
  }
  if (over) atomicExch(overflow, 1);
  counts[r] = k;
  if (col)
    for (int j = k; j < W; ++j) {
      col[(i64)j * a.n_out + r] = 0;
      wout[(i64)j * a.n_out + r] = (T)0;
    }
}

// transpose of an ELL (col, w) [W][n_out] -> (tcol, tw) [WT][n_in], entries of a
// fine column in increasing coarse row (decimation.rs:70-91)
template <typename T>
__global__ void k_dec_tfill(const int32_t* col, const T* w, const int* counts, i64 n_out, i64 n_in, int* tfill,
                            int32_t* tcol, T* tw) {
  i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_out) return;
  for (int k = 0; k < counts[r]; ++k) {
    int32_t c = col[(i64)k * n_out + r];
    int pos = atomicAdd(&tfill[c], 1);
    tcol[(i64)pos * n_in + c] = (int32_t)r;
    tw[(i64)pos * n_in + c] = w[(i64)k * n_out + r];
  }
}

template <typename T>
__global__ void k_dec_tsort(int32_t* tcol, T* tw, const int* tcount, i64 n_in, int WT) {
  i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_in) return;
  int n = tcount[c];
  for (int i = 1; i < n; ++i) {
    int32_t v = tcol[(i64)i * n_in + c];
    T vw = tw[(i64)i * n_in + c];
    int j = i - 1;
    while (j >= 0 && tcol[(i64)j * n_in + c] > v) {
      tcol[(i64)(j + 1) * n_in + c] = tcol[(i64)j * n_in + c];
      tw[(i64)(j + 1) * n_in + c] = tw[(i64)j * n_in + c];
      --j;
    }
    tcol[(i64)(j + 1) * n_in + c] = v;
    tw[(i64)(j + 1) * n_in + c] = vw;
  }
  for (int i = n; i < WT; ++i) {
    tcol[(i64)i * n_in + c] = 0;
    tw[(i64)i * n_in + c] = (T)0;
  }
}

int device_max(const int* d, i64 n, cudaStream_t s) {
  DevMem m(sizeof(int));
  STL_CUDA(cudaMemsetAsync(m.p, 0, sizeof(int), s));
  int blocks = (int)std::min<i64>((n + 255) / 256, 4096);
  if (n > 0) k_max_int<<<std::max(blocks, 1), 256, 0, s>>>(d, n, m.as<int>());
  STL_CUDA(cudaGetLastError());
  int h = 0;
  STL_CUDA(cudaMemcpyAsync(&h, m.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  return h;
}

int read_flag(const DevMem& f, cudaStream_t s) {
  int h = 0;
  STL_CUDA(cudaMemcpyAsync(&h, f.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  return h;
}

inline unsigned nblocks(i64 n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Tangent stencil of ksz x ksz taps at the north pole (stencil.rs:33-47).
static std::vector<double> kernel_grid(int ksz, i64 nside) {
  std::vector<double> out;
  i64 half = ksz / 2;
  double ns = (double)nside;
  double alpha_pix = std::sqrt(4.0 * kPi / (12.0 * ns * ns));
  for (i64 i = 0; i < ksz; ++i)
    for (i64 j = 0; j < ksz; ++j) {
      i64 x = j - half, y = i - half;
      double dtheta = std::sqrt((double)(x * x + y * y)) * alpha_pix;
      double dphi = std::atan2((double)y, (double)x);
      out.push_back(std::sin(dtheta) * std::cos(dphi));
      out.push_back(std::sin(dtheta) * std::sin(dphi));
      out.push_back(std::cos(dtheta));
    }
  return out;
}

template <typename T>
static void build_conv_t(const ConvSpec& sp, const std::vector<double>& kernel, ConvOp& op, cudaStream_t s) {
  const int P = sp.ksz * sp.ksz;
  if (sp.G != 4) throw std::runtime_error("the engine's convolution is built for L = 4 orientations");
  std::vector<double> st = kernel_grid(sp.ksz, sp.nside);
  DevMem d_st(st.size() * 8), d_ker(kernel.size() * 8);
  STL_CUDA(cudaMemcpyAsync(d_st.p, st.data(), st.size() * 8, cudaMemcpyHostToDevice, s));
  STL_CUDA(cudaMemcpyAsync(d_ker.p, kernel.data(), kernel.size() * 8, cudaMemcpyHostToDevice, s));
  FoldArgs a;
  a.nside = sp.nside; a.order = order_of(sp.nside); a.ksz = sp.ksz; a.P = P; a.G = sp.G; a.gauge = sp.gauge;
  a.p_ref = (sp.ksz / 2) * (sp.ksz + 1); a.eps = sp.eps;
  a.grid = sp.d_grid; a.n_in = sp.d_grid ? sp.n_in : npix_of(sp.nside);
  a.rows = sp.d_rows; a.n_rows = sp.d_rows ? sp.n_rows : a.n_in;
  a.stencil = d_st.as<double>(); a.kernel = d_ker.as<double>();
  op.n_rows = a.n_rows; op.n_in = a.n_in; op.G = sp.G;
  op.dtype = sizeof(T) == 8 ? DType::F64 : DType::F32;
  DevMem counts(sizeof(int) * std::max<i64>(a.n_rows, 1)), flag(sizeof(int));
  STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  const int TB = 64;
  k_fold<T><<<nblocks(a.n_rows, TB), TB, 0, s>>>(a, counts.as<int>(), 0, nullptr, nullptr, flag.as<int>());
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) throw std::runtime_error("a wavelet stencil reads more cells than the builder holds");
  op.S = std::max(1, device_max(counts.as<int>(), a.n_rows, s));
  op.cell.alloc(sizeof(int32_t) * op.S * a.n_rows);
  op.coef.alloc(sizeof(T) * 2 * sp.G * op.S * a.n_rows);
  k_fold<T><<<nblocks(a.n_rows, TB), TB, 0, s>>>(a, counts.as<int>(), op.S, op.cell.as<int32_t>(), op.coef.as<T>(),
                                                flag.as<int>());
  STL_CUDA(cudaGetLastError());
  // transposed gather table
  op.shift = 1;
  while ((1 << op.shift) < op.S) ++op.shift;
  if ((uint64_t)(a.n_rows - 1) >= ((uint64_t)1 << (32 - op.shift)) - 1)
    throw std::runtime_error("level too large for the 32-bit transposed table");
  DevMem tcount(sizeof(int) * a.n_in), tfill(sizeof(int) * a.n_in);
  STL_CUDA(cudaMemsetAsync(tcount.p, 0, tcount.bytes, s));
  STL_CUDA(cudaMemsetAsync(tfill.p, 0, tfill.bytes, s));
  k_tcount<<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.cell.as<int32_t>(), counts.as<int>(), a.n_rows, op.S,
                                                   tcount.as<int>());
  STL_CUDA(cudaGetLastError());
  op.ST = std::max(1, device_max(tcount.as<int>(), a.n_in, s));
  op.tent.alloc(sizeof(uint32_t) * op.ST * a.n_in);
  k_tfill<<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.cell.as<int32_t>(), counts.as<int>(), a.n_rows, op.S, op.shift,
                                                  a.n_in, tfill.as<int>(), op.tent.as<uint32_t>());
  STL_CUDA(cudaGetLastError());
  k_tsort<<<nblocks(a.n_in, 256), 256, 0, s>>>(op.tent.as<uint32_t>(), tcount.as<int>(), a.n_in, op.ST);
  STL_CUDA(cudaGetLastError());
  STL_CUDA(cudaStreamSynchronize(s));
}

void build_conv(const ConvSpec& spec, const std::vector<double>& kernel, DType dtype, ConvOp& out, cudaStream_t s) {
  if (dtype == DType::F64) build_conv_t<double>(spec, kernel, out, s);
  else build_conv_t<float>(spec, kernel, out, s);
}

template <typename T>
static void build_dec_t(const DecSpec& sp, DecOp& op, cudaStream_t s) {
  DecArgs a;
  a.nside = sp.nside; a.order = order_of(sp.nside); a.corder = order_of(sp.nside / 2);
  a.ids = sp.d_ids; a.n_in = sp.d_ids ? sp.n_in : npix_of(sp.nside);
  a.out = sp.d_out; a.n_out = sp.d_out ? sp.n_out : npix_of(sp.nside / 2);
  double pix_deg = std::sqrt(4.0 * kPi / (double)npix_of(sp.nside)) * (180.0 / kPi);
  a.radius = (3.0 * pix_deg) * (kPi / 180.0);
  a.sigma = a.radius / 2.0;
  op.n_out = a.n_out; op.n_in = a.n_in;
  op.dtype = sizeof(T) == 8 ? DType::F64 : DType::F32;
  DevMem counts(sizeof(int) * std::max<i64>(a.n_out, 1)), flag(sizeof(int));
  STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  const int TB = 64;
  k_dec_rows<T><<<nblocks(a.n_out, TB), TB, 0, s>>>(a, counts.as<int>(), 0, nullptr, nullptr, flag.as<int>());
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) throw std::runtime_error("a decimation row has more candidates than the builder holds");
  op.W = std::max(1, device_max(counts.as<int>(), a.n_out, s));
  op.col.alloc(sizeof(int32_t) * op.W * a.n_out);
  op.w.alloc(sizeof(T) * op.W * a.n_out);
  k_dec_rows<T><<<nblocks(a.n_out, TB), TB, 0, s>>>(a, counts.as<int>(), op.W, op.col.as<int32_t>(), op.w.as<T>(),
                                                   flag.as<int>());
  STL_CUDA(cudaGetLastError());
  DevMem tcount(sizeof(int) * a.n_in), tfill(sizeof(int) * a.n_in);
  STL_CUDA(cudaMemsetAsync(tcount.p, 0, tcount.bytes, s));
  STL_CUDA(cudaMemsetAsync(tfill.p, 0, tfill.bytes, s));
  k_tcount<<<nblocks(a.n_out, 256), 256, 0, s>>>(op.col.as<int32_t>(), counts.as<int>(), a.n_out, op.W,
                                                  tcount.as<int>());
  STL_CUDA(cudaGetLastError());
  op.WT = std::max(1, device_max(tcount.as<int>(), a.n_in, s));
  op.tcol.alloc(sizeof(int32_t) * op.WT * a.n_in);
  op.tw.alloc(sizeof(T) * op.WT * a.n_in);
  k_dec_tfill<T><<<nblocks(a.n_out, 256), 256, 0, s>>>(op.col.as<int32_t>(), op.w.as<T>(), counts.as<int>(), a.n_out,
                                                       a.n_in, tfill.as<int>(), op.tcol.as<int32_t>(), op.tw.as<T>());
  STL_CUDA(cudaGetLastError());
  k_dec_tsort<T><<<nblocks(a.n_in, 256), 256, 0, s>>>(op.tcol.as<int32_t>(), op.tw.as<T>(), tcount.as<int>(), a.n_in,
                                                      op.WT);
  STL_CUDA(cudaGetLastError());
  STL_CUDA(cudaStreamSynchronize(s));
}

void build_dec(const DecSpec& spec, DType dtype, DecOp& out, cudaStream_t s) {
  if (dtype == DType::F64) build_dec_t<double>(spec, out, s);
  else build_dec_t<float>(spec, out, s);
}

}  // namespace stl
