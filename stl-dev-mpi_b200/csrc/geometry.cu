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
#include <type_traits>

#include "engine.cuh"
#include "healpix.cuh"

namespace stl {

namespace {

constexpr int kFoldCap = 128;  // distinct cells one row may read
constexpr int kDecCap = 256;   // candidates of one decimation row
constexpr uint32_t kSentinel = 0xFFFFFFFFu;

// position of v in the sorted grid[lo, hi) (whole sky: v itself), or -1
__device__ __forceinline__ i64 grid_find(const i64* grid, i64 lo, i64 hi, i64 v) {
  if (!grid) return (v >= 0 && v < hi) ? v : -1;
  const i64 end = hi;
  while (lo < hi) {
    i64 mid = (lo + hi) >> 1;
    if (grid[mid] < v) lo = mid + 1; else hi = mid;
  }
  return (lo < end && grid[lo] == v) ? lo : -1;
}

// index of the segment of seg (nseg + 1 ascending starts) holding position k
__device__ __forceinline__ int segment_index(const i64* seg, int nseg, i64 k) {
  int a = 0, b = nseg;  // seg[a] <= k < seg[b]
  while (b - a > 1) {
    const int m = (a + b) >> 1;
    if (seg[m] <= k) a = m; else b = m;
  }
  return a;
}

struct FoldArgs {
  i64 nside;
  int order, ksz, P, G, gauge, p_ref;
  double eps;
  const i64* grid;
  i64 n_in;
  const i64* seg;         // segments of grid (rows == grid), or nullptr
  int nseg;
  const i64* rows;
  i64 n_rows;             // rows built (the stored rows)
  int sym;                // stored row u is pixel (4 (u >> sym_o2)) << sym_o2 | local
  int sym_o2;
  const double* stencil;  // [P][3]
  const double* kernel;   // [G][2][P]
};

// One thread per output row: bind and fold.  Pass 1 (cell == nullptr)
// only counts the distinct cells; pass 2 writes the S slots.
template <typename T>
__global__ void k_fold(FoldArgs a, int* counts, int S, int32_t* cell, T* coef, int* overflow) {
  i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n_rows) return;
  i64 id;
  if (a.sym) {
    i64 mask = (i64(1) << a.sym_o2) - 1;
    id = ((4 * (k >> a.sym_o2)) << a.sym_o2) | (k & mask);
  } else {
    id = a.rows ? a.rows[k] : (a.grid ? a.grid[k] : k);
  }
  i64 g_lo = 0, g_hi = a.n_in;  // the cells this row may read
  if (a.seg) {
    const int sg = segment_index(a.seg, a.nseg, k);
    g_lo = a.seg[sg];
    g_hi = a.seg[sg + 1];
  }
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
        found[q] = grid_find(a.grid, g_lo, g_hi, ix[q]);
        if (a.eps > 0.0 && wx[q] <= a.eps) found[q] = -1;
      }
      if (found[0] < 0 && found[1] < 0 && found[2] < 0 && found[3] < 0) {  // empty tap: central tap
        ix = ref_pix;
        wx = ref_w;
        for (int q = 0; q < 4; ++q) {
          found[q] = grid_find(a.grid, g_lo, g_hi, ix[q]);
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

// transposed entries of the wavelet: stored row u reads cell c at slot s;
// c is rotation j of the stored cell v (full sky), or v = c, j = 0.
__device__ __forceinline__ void split_cell(i64 c, int sym, int sym_o2, i64& v, int& j) {
  if (sym) {
    i64 f = c >> sym_o2;
    v = ((f >> 2) << sym_o2) | (c & ((i64(1) << sym_o2) - 1));
    j = (int)(f & 3);
  } else {
    v = c;
    j = 0;
  }
}

__global__ void k_conv_tcount(const int32_t* cell, const int* counts, i64 n_rep, int sym, int sym_o2, int* tcount) {
  i64 u = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n_rep) return;
  for (int s = 0; s < counts[u]; ++s) {
    i64 v;
    int j;
    split_cell(cell[(i64)s * n_rep + u], sym, sym_o2, v, j);
    atomicAdd(&tcount[v], 1);
  }
}

__global__ void k_conv_tfill(const int32_t* cell, const int* counts, i64 n_rep, int sym, int sym_o2, int tshift,
                             int* tfill, uint32_t* tent) {
  i64 u = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n_rep) return;
  for (int s = 0; s < counts[u]; ++s) {
    i64 v;
    int j;
    split_cell(cell[(i64)s * n_rep + u], sym, sym_o2, v, j);
    int pos = atomicAdd(&tfill[v], 1);
    tent[(i64)pos * n_rep + v] = (uint32_t)(((uint64_t)u << tshift) | ((uint64_t)s << 2) | (uint64_t)j);
  }
}

// coefficients of the (sorted) transposed entries, zeros past the end
template <typename T>
__global__ void k_conv_coefT(const uint32_t* tent, const T* coef, i64 n_rep, int ST, int tshift, T* coefT) {
  i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_rep) return;
  const uint32_t smask = (1u << (tshift - 2)) - 1u;
  for (int e = 0; e < ST; ++e) {
    uint32_t ent = tent[(i64)e * n_rep + v];
    T* dst = coefT + ((i64)e * n_rep + v) * 8;
    if (ent == kSentinel) {
      for (int o = 0; o < 8; ++o) dst[o] = (T)0;
      continue;
    }
    i64 u = (i64)(ent >> tshift);
    int s = (int)((ent >> 2) & smask);
    const T* src = coef + ((i64)s * n_rep + u) * 8;
    for (int o = 0; o < 8; ++o) dst[o] = src[o];
  }
}

// Adjoint tiles: one block per tile of kAdjTile stored rows.  The cells the
// tile's rows read (all slots) are sorted in shared memory (bitonic), made
// unique, written to the tile's list, and every (slot, row) gets the index
// of its cell in that list.
__global__ void k_adj_tiles(const int32_t* cell, int S, i64 n_rep, int P2, int32_t* tile_cells, int32_t* tile_nc,
                            uint16_t* lcell, int* overflow) {
  extern __shared__ int32_t buf[];  // [P2] sorted cells, then [kAdjCells] unique, then [256] counts
  int32_t* uniq = buf + P2;
  int32_t* cnt = uniq + kAdjCells;
  const int tid = threadIdx.x;
  const i64 u0 = (i64)blockIdx.x * kAdjTile;
  const int n = S * kAdjTile;
  for (int i = tid; i < P2; i += blockDim.x) {
    int32_t v = 0x7fffffff;
    if (i < n) {
      const int s = i / kAdjTile, ul = i % kAdjTile;
      if (u0 + ul < n_rep) v = cell[(i64)s * n_rep + u0 + ul];
    }
    buf[i] = v;
  }
  __syncthreads();
  for (int k = 2; k <= P2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int32_t a = buf[i], c = buf[l];
          if (((i & k) == 0) ? (a > c) : (a < c)) { buf[i] = c; buf[l] = a; }
        }
      }
      __syncthreads();
    }
  const int per = P2 / blockDim.x;
  int mine = 0;
  for (int i = tid * per; i < (tid + 1) * per; ++i)
    if (buf[i] != 0x7fffffff && (i == 0 || buf[i - 1] != buf[i])) ++mine;
  cnt[tid] = mine;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) { const int c = cnt[t]; cnt[t] = acc; acc += c; }
    tile_nc[blockIdx.x] = acc;
    if (acc > kAdjCells) atomicExch(overflow, 1);
  }
  __syncthreads();
  int pos = cnt[tid];
  for (int i = tid * per; i < (tid + 1) * per; ++i)
    if (buf[i] != 0x7fffffff && (i == 0 || buf[i - 1] != buf[i])) {
      if (pos < kAdjCells) {
        uniq[pos] = buf[i];
        tile_cells[(i64)blockIdx.x * kAdjCells + pos] = buf[i];
      }
      ++pos;
    }
  __syncthreads();
  const int nc = min(tile_nc[blockIdx.x], kAdjCells);
  for (int i = tid; i < n; i += blockDim.x) {
    const int s = i / kAdjTile, ul = i % kAdjTile;
    if (u0 + ul >= n_rep) continue;
    const int32_t v = cell[(i64)s * n_rep + u0 + ul];
    int lo = 0, hi = nc;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (uniq[mid] < v) lo = mid + 1; else hi = mid;
    }
    lcell[(i64)s * n_rep + u0 + ul] = (uint16_t)lo;
  }
}

// Per tile and slot chunk, the entries (slot, row) of every tile cell in
// the order (slot, row): keys chunk << 22 | cell << 11 | slot % kAdjSC << 8
// | row, sorted (bitonic); the low 11 bits are the entry, and off[chunk][lc]
// the position of the first key of (chunk, lc).  Slots past a row's cell
// count repeat its first cell: they are left out.
__global__ void k_adj_csr(const int32_t* cell, const uint16_t* lcell, int S, i64 n_rep, int P2, int nch, int ncs,
                          const int32_t* tile_nc, uint16_t* tile_ent, uint16_t* tile_off) {
  extern __shared__ uint32_t key[];
  const int tid = threadIdx.x;
  const i64 u0 = (i64)blockIdx.x * kAdjTile;
  const int n = S * kAdjTile;
  for (int i = tid; i < P2; i += blockDim.x) {
    uint32_t v = 0xFFFFFFFFu;
    if (i < n) {
      const int sl = i / kAdjTile, ul = i % kAdjTile;
      const i64 u = u0 + ul;
      if (u < n_rep) {
        const i64 e = (i64)sl * n_rep + u;
        if (sl == 0 || cell[e] != cell[u])
          v = ((uint32_t)(sl / kAdjSC) << 22) | ((uint32_t)lcell[e] << 11) | ((uint32_t)(sl % kAdjSC) << 8) | (uint32_t)ul;
      }
    }
    key[i] = v;
  }
  __syncthreads();
  for (int k = 2; k <= P2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const uint32_t a = key[i], c = key[l];
          if (((i & k) == 0) ? (a > c) : (a < c)) { key[i] = c; key[l] = a; }
        }
      }
      __syncthreads();
    }
  uint16_t* ent = tile_ent + (i64)blockIdx.x * n;
  for (int i = tid; i < n; i += blockDim.x)
    if (key[i] != 0xFFFFFFFFu) ent[i] = (uint16_t)(key[i] & 0x7FFu);
  const int nc = tile_nc[blockIdx.x];
  uint16_t* off = tile_off + (i64)blockIdx.x * nch * ncs;
  for (int q = tid; q < nch * (nc + 1); q += blockDim.x) {
    const int ch = q / (nc + 1), lc = q % (nc + 1);
    const uint32_t t = ((uint32_t)ch << 22) | ((uint32_t)lc << 11);
    int lo = 0, hi = P2;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (key[mid] < t) lo = mid + 1; else hi = mid;
    }
    off[ch * ncs + lc] = (uint16_t)lo;
  }
}

// most slots used by a row of each adjoint tile
__global__ void k_tile_slots(const int* counts, i64 n_rep, i64 n_tiles, int32_t* out) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  int m = 1;
  for (i64 u = t * kAdjTile; u < min(n_rep, (t + 1) * kAdjTile); ++u) m = max(m, counts[u]);
  out[t] = m;
}

// sum over the slots of every stored row's coefficients, in FP64
template <typename T>
__global__ void k_rowsum(const T* coef, int S, i64 n_rep, T* out) {
  const i64 u = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n_rep) return;
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int s = 0; s < S; ++s)
    for (int j = 0; j < 8; ++j) a[j] += (double)coef[((i64)s * n_rep + u) * 8 + j];
  for (int j = 0; j < 8; ++j) out[u * 8 + j] = (T)a[j];
}

// Edge colouring of a tile's (row, tile cell) entries with D colours, D the
// largest degree of a row or of a cell in the tile: a bipartite graph needs
// no more (Konig's line colouring theorem).  The entries are coloured in
// (row, slot) order; when the colour a free at the row is taken at the cell,
// the path from the cell alternating a and b (a colour free at the cell) has
// its two colours swapped, which frees a at the cell and cannot reach the
// row (rows are entered on a-edges and a is free at the row).  Every colour
// class is then a matching -- no two rows of the tile read one cell in the
// same colour -- and the colouring is deterministic.  col[s][u] gets the
// colour of slot s of row u; tile_d the tile's D (above kColMax: *fail).
constexpr int kColMax = 64;

__global__ void k_color_tiles(const uint16_t* lcell, const int* counts, int S, i64 n_rep, const int32_t* tile_nc,
                              uint8_t* col, int32_t* tile_d, int* fail) {
  extern __shared__ __align__(16) unsigned char sm[];
  uint64_t* row_used = reinterpret_cast<uint64_t*>(sm);                      // [kAdjTile]
  uint64_t* cell_used = row_used + kAdjTile;                                 // [kAdjCells]
  int* cdeg = reinterpret_cast<int*>(cell_used + kAdjCells);                 // [kAdjCells]
  uint16_t* row_at = reinterpret_cast<uint16_t*>(cdeg + kAdjCells);          // [kAdjTile][kColMax]: cell
  uint16_t* path = row_at + kAdjTile * kColMax;                              // [kAdjTile + kAdjCells + 2]
  uint16_t* lc = path + (kAdjTile + kAdjCells + 2);                          // [S][kAdjTile]
  uint8_t* cell_at = reinterpret_cast<uint8_t*>(lc + (size_t)S * kAdjTile);  // [kAdjCells][kColMax]: row
  const int tile = blockIdx.x, lane = threadIdx.x;
  const i64 u0 = (i64)tile * kAdjTile;
  const int rows = (int)min((i64)kAdjTile, n_rep - u0);
  const int nc = min(tile_nc[tile], kAdjCells);
  for (int i = lane; i < kAdjCells; i += 32) { cell_used[i] = 0; cdeg[i] = 0; }
  for (int i = lane; i < kAdjTile; i += 32) row_used[i] = 0;
  for (int i = lane; i < S * kAdjTile; i += 32) {
    const int sl = i / kAdjTile, r = i % kAdjTile;
    lc[i] = r < rows ? lcell[(i64)sl * n_rep + u0 + r] : (uint16_t)0;
  }
  __syncwarp();
  int dmax = 0;
  for (int r = lane; r < rows; r += 32) {
    const int cnt = counts[u0 + r];
    dmax = max(dmax, cnt);
    for (int sl = 0; sl < cnt; ++sl) atomicAdd(&cdeg[lc[sl * kAdjTile + r]], 1);
  }
  __syncwarp();
  for (int c = lane; c < nc; c += 32) dmax = max(dmax, cdeg[c]);
  for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
  if (lane == 0) tile_d[tile] = dmax;
  if (dmax > kColMax) {
    if (lane == 0) atomicExch(fail, 1);
    return;
  }
  // (every walk and colour is checked against its bound: an inconsistent
  // state ends the colouring with *fail set instead of running on)
  int bad = 0;
  if (lane == 0) {
    for (int r = 0; r < rows && !bad; ++r) {
      const int cnt = counts[u0 + r];
      for (int sl = 0; sl < cnt && !bad; ++sl) {
        const int c = lc[sl * kAdjTile + r];
        const int a = __ffsll((long long)~row_used[r]) - 1;
        if (c >= nc || a < 0 || a >= dmax) { bad = 1; break; }
        if ((cell_used[c] >> a) & 1ull) {
          const int b = __ffsll((long long)~cell_used[c]) - 1;
          if (b < 0 || b >= dmax) { bad = 1; break; }
          // path[0] = c, then row, cell, ...; edge i colour a (i even) or b
          int len = 1, v = c, k = a;
          bool at_cell = true;
          path[0] = (uint16_t)c;
          while (true) {
            if (len > kAdjTile + kAdjCells) { bad = 1; break; }
            int w;
            if (at_cell) {
              if (!((cell_used[v] >> k) & 1ull)) break;
              w = cell_at[v * kColMax + k];
            } else {
              if (!((row_used[v] >> k) & 1ull)) break;
              w = row_at[v * kColMax + k];
            }
            path[len++] = (uint16_t)w;
            v = w;
            at_cell = !at_cell;
            k = k == a ? b : a;
          }
          if (bad) break;
          for (int i = 0; i + 1 < len; ++i) {
            const int kc = (i & 1) ? b : a;
            const int cv = (i & 1) ? path[i + 1] : path[i], rv = (i & 1) ? path[i] : path[i + 1];
            cell_used[cv] &= ~(1ull << kc);
            row_used[rv] &= ~(1ull << kc);
          }
          for (int i = 0; i + 1 < len; ++i) {
            const int kn = (i & 1) ? a : b;
            const int cv = (i & 1) ? path[i + 1] : path[i], rv = (i & 1) ? path[i] : path[i + 1];
            cell_used[cv] |= 1ull << kn;
            row_used[rv] |= 1ull << kn;
            cell_at[cv * kColMax + kn] = (uint8_t)rv;
            row_at[rv * kColMax + kn] = (uint16_t)cv;
          }
        }
        row_used[r] |= 1ull << a;
        cell_used[c] |= 1ull << a;
        row_at[r * kColMax + a] = (uint16_t)c;
        cell_at[c * kColMax + a] = (uint8_t)r;
      }
    }
    if (bad) atomicExch(fail, 1);
  }
  bad = __shfl_sync(0xffffffffu, bad, 0);
  if (bad) return;
  __syncwarp();
  // the colour of every entry: the row's cells are distinct
  for (int r = lane; r < rows; r += 32) {
    const int cnt = counts[u0 + r];
    uint64_t m = row_used[r];
    while (m) {
      const int k = __ffsll((long long)m) - 1;
      m &= m - 1;
      const int c = row_at[r * kColMax + k];
      for (int sl = 0; sl < cnt; ++sl)
        if (lc[sl * kAdjTile + r] == c) {
          col[(i64)sl * n_rep + u0 + r] = (uint8_t)k;
          break;
        }
    }
  }
}

size_t color_smem(int S) {
  return sizeof(uint64_t) * (kAdjTile + kAdjCells) + sizeof(int) * kAdjCells +
         sizeof(uint16_t) * ((size_t)kAdjTile * kColMax + kAdjTile + kAdjCells + 2 + (size_t)S * kAdjTile) +
         (size_t)kAdjCells * kColMax;
}

// Coloured layout: slot k of row u holds its entry of colour k, or padding
// (zero coefficients, the row's first cell, tile cell nc = none).
template <typename T>
__global__ void k_color_apply(const int32_t* cell, const T* coef, const uint16_t* lcell, const uint8_t* col,
                              const int* counts, int S, int S2, i64 n_rep, const int32_t* tile_nc, int32_t* cell2,
                              T* coef2, uint16_t* lcell2) {
  const i64 u = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n_rep) return;
  const uint16_t none = (uint16_t)tile_nc[u / kAdjTile];
  const int32_t c0 = cell[u];
  for (int k = 0; k < S2; ++k) {
    const i64 e = (i64)k * n_rep + u;
    cell2[e] = c0;
    lcell2[e] = none;
    for (int j = 0; j < 8; ++j) coef2[e * 8 + j] = (T)0;
  }
  const int cnt = counts[u];
  for (int sl = 0; sl < cnt; ++sl) {
    const i64 e = (i64)sl * n_rep + u, e2 = (i64)col[e] * n_rep + u;
    cell2[e2] = cell[e];
    lcell2[e2] = lcell[e];
    for (int j = 0; j < 8; ++j) coef2[e2 * 8 + j] = coef[e * 8 + j];
  }
}

// lcell [S][n_rep] -> tile-major [n_tiles][nch * 4][kAdjTile] (slots padded
// to a multiple of 4 with index 0: their coefficients are never read)
__global__ void k_lcell_tiles(const uint16_t* lcell, int S, i64 n_rep, int S4, i64 n_tiles, uint16_t* out) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tiles * S4 * kAdjTile) return;
  const i64 tile = i / ((i64)S4 * kAdjTile);
  const int rem = (int)(i % ((i64)S4 * kAdjTile));
  const int s = rem / kAdjTile, ul = rem % kAdjTile;
  const i64 u = tile * kAdjTile + ul;
  out[i] = (s < S && u < n_rep) ? lcell[(i64)s * n_rep + u] : (uint16_t)0;
}

// Tile cells -> stored input cells: cell c of a tile is rotation j of
// stored cell v (nk = 4: c in face 4m + j; nk = 1: v = c, j = 0).
__device__ __forceinline__ void tile_cell_owner(int32_t c, int nk, int o2, i64& v, int& j) {
  if (nk == 4) {
    const i64 f = (i64)c >> o2;
    j = (int)(f & 3);
    v = ((f >> 2) << o2) | ((i64)c & ((i64(1) << o2) - 1));
  } else {
    v = c;
    j = 0;
  }
}

__global__ void k_adj_ccount(const int32_t* tile_cells, const int32_t* tile_nc, i64 n_tiles, int nk, int o2,
                             int* ccount) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tiles * kAdjCells) return;
  const i64 tile = i / kAdjCells;
  const int lc = (int)(i % kAdjCells);
  if (lc >= tile_nc[tile]) return;
  i64 v; int j;
  tile_cell_owner(tile_cells[i], nk, o2, v, j);
  atomicAdd(ccount + v, 1);
}

__global__ void k_adj_cfill(const int32_t* tile_cells, const int32_t* tile_nc, i64 n_tiles, int nk, int o2,
                            const i64* coff, int* cursor, uint32_t* clist) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tiles * kAdjCells) return;
  const i64 tile = i / kAdjCells;
  const int lc = (int)(i % kAdjCells);
  if (lc >= tile_nc[tile]) return;
  i64 v; int j;
  tile_cell_owner(tile_cells[i], nk, o2, v, j);
  const int pos = atomicAdd(cursor + v, 1);
  clist[coff[v] + pos] = ((uint32_t)tile << 12) | ((uint32_t)lc << 2) | (uint32_t)j;
}

// fixed order of every stored cell's list (insertion sort; lists are short)
__global__ void k_adj_csort(const i64* coff, i64 n, uint32_t* clist) {
  const i64 v = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  uint32_t* l = clist + coff[v];
  const int m = (int)(coff[v + 1] - coff[v]);
  for (int a = 1; a < m; ++a) {
    const uint32_t x = l[a];
    int b = a - 1;
    while (b >= 0 && l[b] > x) { l[b + 1] = l[b]; --b; }
    l[b + 1] = x;
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

// ---- tensor-core layout -------------------------------------------------------
// One block (256 threads) per tile of kMmaRows stored rows, run twice: pass
// 0 measures (chunks of every row and tile, plane cells, warp-local cells),
// pass 1 writes the layout with the strides pass 0 fixed.  The tile's
// distinct cells are sorted (bitonic) and numbered 4 rank + class within
// their class (class = the cell's NESTED bits x0 + 2 y0, which the 4-face
// rotations keep); a row's cells keep their slot order within each class,
// the j-th of class q going to chunk j / 2 at position mma_pos(q, j % 2).
struct MmaArgs {
  const int32_t* cell;  // [S][n_rep]
  const int* counts;    // cells per row
  const float* coef;    // [S][n_rep][8]
  int S;
  i64 n_rep;
  int Sm, pcs;          // pass 1: slots and plane stride
  int32_t* tile_ch;     // [tiles] chunks
  int32_t* tile_pc;     // [tiles] plane cells used: 4 (largest class + 1)
  int32_t* tile_wl;     // [tiles] warp-local cells used: 4 (largest class + 1), most over the tile's warps
  uint8_t* rowch;       // [n_rep]
  float* m_coef;        // pass 1 outputs (ConvOp::m_*)
  int32_t* m_cells;
  uint16_t* m_lc;
  uint8_t* m_wlc;
  uint8_t* m_winv;
  int* overflow;
};

__host__ __device__ constexpr int mma_pos(int q, int j) { return j == 0 ? q : 4 + (q ^ 1); }

constexpr int kMmaMaxSlots = 128;  // slots of the layout (16 chunks)

__global__ void __launch_bounds__(256) k_mma_layout(MmaArgs a, int pass, int P2) {
  extern __shared__ int32_t mbuf[];
  int32_t* sorted = mbuf;                       // [P2]
  int32_t* uniq = sorted + P2;                  // [kMmaPlaneMax]
  int16_t* upl = reinterpret_cast<int16_t*>(uniq + kMmaPlaneMax);      // [kMmaPlaneMax] plane index
  uint8_t* gmap = reinterpret_cast<uint8_t*>(upl + kMmaPlaneMax);      // [groups][kMmaPlaneMax]
  __shared__ int cnt[256];
  __shared__ int s_nc, s_mc, s_ch, s_wl, s_bad;
  __shared__ int s_mcw[kMmaRows / kMmaWarpRows];
  constexpr int NG = kMmaRows / kMmaWarpRows;
  const int tid = threadIdx.x;
  const i64 tile = blockIdx.x, u0 = tile * kMmaRows;
  const int n = a.S * kMmaRows;
  if (tid == 0) { s_ch = 0; s_wl = 0; s_bad = 0; }
  for (int i = tid; i < P2; i += blockDim.x) {
    int32_t v = 0x7fffffff;
    if (i < n) {
      const int sl = i / kMmaRows, ul = i % kMmaRows;
      const i64 u = u0 + ul;
      if (u < a.n_rep && sl < a.counts[u]) v = a.cell[(i64)sl * a.n_rep + u];
    }
    sorted[i] = v;
  }
  __syncthreads();
  for (int k = 2; k <= P2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int32_t x = sorted[i], y = sorted[l];
          if (((i & k) == 0) ? (x > y) : (x < y)) { sorted[i] = y; sorted[l] = x; }
        }
      }
      __syncthreads();
    }
  const int per = P2 / blockDim.x;
  int mine = 0;
  for (int i = tid * per; i < (tid + 1) * per; ++i)
    if (sorted[i] != 0x7fffffff && (i == 0 || sorted[i - 1] != sorted[i])) ++mine;
  cnt[tid] = mine;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) { const int c = cnt[t]; cnt[t] = acc; acc += c; }
    s_nc = acc;
    if (acc > kMmaPlaneMax) s_bad = 1;
  }
  __syncthreads();
  if (s_bad) {
    if (tid == 0) atomicExch(a.overflow, 1);
    return;
  }
  int pos = cnt[tid];
  for (int i = tid * per; i < (tid + 1) * per; ++i)
    if (sorted[i] != 0x7fffffff && (i == 0 || sorted[i - 1] != sorted[i])) uniq[pos++] = sorted[i];
  __syncthreads();
  const int nc = s_nc;
  // plane index of every tile cell: 4 (rank in its class) + class
  if (tid < 4) {
    int r = 0;
    for (int i = 0; i < nc; ++i)
      if ((uniq[i] & 3) == tid) upl[i] = (int16_t)(4 * r++ + tid);
    cnt[tid] = r;
  }
  __syncthreads();
  if (tid == 0) {
    s_mc = max(max(cnt[0], cnt[1]), max(cnt[2], cnt[3]));
    if (4 * (s_mc + 1) > kMmaPlaneMax) s_bad = 1;
  }
  for (int i = tid; i < NG * kMmaPlaneMax; i += blockDim.x) gmap[i] = 255;
  __syncthreads();
  if (s_bad) {
    if (tid == 0) atomicExch(a.overflow, 1);
    return;
  }
  const int mc = s_mc;
  auto find = [&](int32_t v) {
    int lo = 0, hi = nc;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (uniq[mid] < v) lo = mid + 1; else hi = mid;
    }
    return (int)upl[lo];
  };
  // warp groups: the distinct plane cells of each group's rows, numbered
  // 4 rank + class in plane order
  if (tid < NG) {
    uint8_t* gm = gmap + tid * kMmaPlaneMax;
    for (int ul = tid * kMmaWarpRows; ul < (tid + 1) * kMmaWarpRows; ++ul) {
      const i64 u = u0 + ul;
      if (u >= a.n_rep) break;
      for (int sl = 0; sl < a.counts[u]; ++sl) gm[find(a.cell[(i64)sl * a.n_rep + u])] = 0;
    }
    int r[4] = {0, 0, 0, 0};
    for (int pl = 0; pl < 4 * mc; ++pl)
      if (gm[pl] == 0) gm[pl] = (uint8_t)(4 * r[pl & 3]++ + (pl & 3));
    const int mcw = max(max(r[0], r[1]), max(r[2], r[3]));
    s_mcw[tid] = mcw;
    if (4 * mcw + 3 > kMmaWarpMax) atomicExch(&s_bad, 1);
    atomicMax(&s_wl, 4 * (mcw + 1));
  }
  __syncthreads();
  if (s_bad) {
    if (tid == 0) atomicExch(a.overflow, 1);
    return;
  }
  // rows: chunks (pass 0) or the layout (pass 1)
  if (tid < kMmaRows) {
    const int ul = tid;
    const i64 u = u0 + ul;
    int nq[4] = {0, 0, 0, 0};
    const int n_u = u < a.n_rep ? a.counts[u] : 0;
    for (int sl = 0; sl < n_u; ++sl) ++nq[find(a.cell[(i64)sl * a.n_rep + u]) & 3];
    int ch = 0;
    for (int q = 0; q < 4; ++q) ch = max(ch, (nq[q] + 1) / 2);
    if (8 * ch > kMmaMaxSlots) atomicExch(&s_bad, 1);
    if (pass == 0) {
      if (u < a.n_rep) a.rowch[u] = (uint8_t)ch;
      atomicMax(&s_ch, ch);
    } else if (u < a.n_rep && 8 * ch <= kMmaMaxSlots) {
      int16_t src[kMmaMaxSlots];
      for (int ns = 0; ns < a.Sm; ++ns) src[ns] = -1;
      int jq[4] = {0, 0, 0, 0};
      for (int sl = 0; sl < n_u; ++sl) {
        const int q = find(a.cell[(i64)sl * a.n_rep + u]) & 3;
        const int j = jq[q]++;
        src[8 * (j >> 1) + mma_pos(q, j & 1)] = (int16_t)sl;
      }
      const int g = ul / kMmaWarpRows;
      const uint8_t* gm = gmap + g * kMmaPlaneMax;
      const int mcw = s_mcw[g];
      for (int ns = 0; ns < a.Sm; ++ns) {
        const int q = mma_class(ns & 7), sl = src[ns];
        float* dst = a.m_coef + ((i64)ns * a.n_rep + u) * 8;
        int pl, wl;
        if (sl >= 0) {
          const float* c = a.coef + ((i64)sl * a.n_rep + u) * 8;
          for (int o = 0; o < 8; ++o) dst[o] = c[o];
          pl = find(a.cell[(i64)sl * a.n_rep + u]);
          wl = gm[pl];
        } else {  // padding: zero coefficients on the class's spare cells
          for (int o = 0; o < 8; ++o) dst[o] = 0.0f;
          pl = 4 * mc + q;
          wl = 4 * mcw + q;
        }
        a.m_lc[(((i64)tile * (a.Sm / 8) + (ns >> 3)) * kMmaRows + ul) * 8 + (ns & 7)] = (uint16_t)pl;
        a.m_wlc[(((i64)tile * (a.Sm / 8) + (ns >> 3)) * kMmaRows + ul) * 8 + (ns & 7)] = (uint8_t)wl;
      }
    }
  }
  __syncthreads();
  if (s_bad) {
    if (tid == 0) atomicExch(a.overflow, 1);
    return;
  }
  if (pass == 0) {
    if (tid == 0) {
      a.tile_ch[tile] = s_ch;
      a.tile_pc[tile] = 4 * (mc + 1);
      a.tile_wl[tile] = s_wl;
    }
    return;
  }
  for (int pl = tid; pl < a.pcs; pl += blockDim.x) a.m_cells[(i64)tile * a.pcs + pl] = -1;
  __syncthreads();
  for (int i = tid; i < nc; i += blockDim.x) a.m_cells[(i64)tile * a.pcs + upl[i]] = uniq[i];
  for (int i = tid; i < NG * a.pcs; i += blockDim.x) {
    const int g = i / a.pcs, pl = i % a.pcs;
    a.m_winv[((i64)tile * NG + g) * a.pcs + pl] = pl < kMmaPlaneMax ? gmap[g * kMmaPlaneMax + pl] : (uint8_t)255;
  }
}

// tile plane cells -> stored input cells (holes, -1, have none)
__global__ void k_mma_ccount(const int32_t* cells, i64 n, int pcs, int o2, int* ccount) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cells[i] < 0) return;
  i64 v; int j;
  tile_cell_owner(cells[i], 4, o2, v, j);
  atomicAdd(ccount + v, 1);
  (void)pcs;
}

__global__ void k_mma_cfill(const int32_t* cells, i64 n, int pcs, int o2, const i64* coff, int* cursor,
                            uint32_t* clist) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cells[i] < 0) return;
  i64 v; int j;
  tile_cell_owner(cells[i], 4, o2, v, j);
  const i64 tile = i / pcs;
  const int pl = (int)(i % pcs);
  const int pos = atomicAdd(cursor + v, 1);
  clist[coff[v] + pos] = ((uint32_t)tile << 12) | ((uint32_t)pl << 2) | (uint32_t)j;
}

// ---- decimation ------------------------------------------------------------
struct DecArgs {
  i64 nside;      // fine
  int order, corder;
  const i64* ids;  // fine grid (nullptr: whole sky)
  i64 n_in;
  const i64* seg_in;   // segments of the fine grid and of the coarse rows, or nullptr
  const i64* seg_out;
  int nseg;
  const i64* out;  // coarse rows (nullptr: whole sky)
  i64 n_out;       // rows built (the stored rows)
  int sym;         // stored row u is coarse pixel (4 (u >> sym_co2)) << sym_co2 | local
  int sym_co2;
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
  i64 c;
  if (a.sym) c = ((4 * (r >> a.sym_co2)) << a.sym_co2) | (r & ((i64(1) << a.sym_co2) - 1));
  else c = a.out ? a.out[r] : r;
  i64 cn = a.nside / 2;
  i64 f_lo = 0, f_hi = a.n_in;  // the fine cells this row may read: its segment's
  if (a.seg_out) {
    const int sg = segment_index(a.seg_out, a.nseg, r);
    f_lo = a.seg_in[sg];
    f_hi = a.seg_in[sg + 1];
  }
  i64 cand[kDecCap];
  int n = 0;
  bool over = false;
  auto push = [&](i64 fine) {
    i64 q = grid_find(a.ids, f_lo, f_hi, fine);
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

// transpose of the stored decimation rows: for every stored fine cell v, the
// coarse rows (full-sky ids, or positions) reading it and their weights,
// sorted by coarse row (decimation.rs:70-91).  On the full sky a stored
// coarse row u reads rotation j of v when its column is rotation j of v;
// rotation (4 - j) mod 4 of u then reads v itself.
__device__ __forceinline__ i64 sym_pixel(i64 u, int k, int o2) {
  return ((4 * (u >> o2) + k) << o2) | (u & ((i64(1) << o2) - 1));
}

__global__ void k_dec_tcount(const int32_t* col, const int* counts, i64 n_rows, int sym, int fine_o2, int* tcount) {
  i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  for (int k = 0; k < counts[r]; ++k) {
    i64 v;
    int j;
    split_cell(col[(i64)k * n_rows + r], sym, fine_o2, v, j);
    atomicAdd(&tcount[v], 1);
  }
}

template <typename T>
__global__ void k_dec_tfill(const int32_t* col, const T* w, const int* counts, i64 n_rows, i64 n_cells, int sym,
                            int fine_o2, int coarse_o2, int* tfill, int32_t* tcol, T* tw) {
  i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  for (int k = 0; k < counts[r]; ++k) {
    i64 v;
    int j;
    split_cell(col[(i64)k * n_rows + r], sym, fine_o2, v, j);
    i64 coarse = sym ? sym_pixel(r, (4 - j) & 3, coarse_o2) : r;
    int pos = atomicAdd(&tfill[v], 1);
    tcol[(i64)pos * n_cells + v] = (int32_t)coarse;
    tw[(i64)pos * n_cells + v] = w[(i64)k * n_rows + r];
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

double device_mean(const int* d, i64 n, cudaStream_t s) {
  std::vector<int> h(n);
  STL_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  double t = 0.0;
  for (int v : h) t += v;
  return n > 0 ? t / (double)n : 0.0;
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

// The tensor-core layout of an FP32 full-sky operator (ConvOp::m_*) from its
// per-row slots; false (nothing kept) when a tile does not fit its limits.
static bool build_mma_layout(ConvOp& op, const DevMem& counts, bool adjoint, cudaStream_t s) {
  const i64 n_rep = op.n_rep;
  if (op.S > 64 || op.o2 < 2) return false;
  const i64 n_tiles = (n_rep + kMmaRows - 1) / kMmaRows;
  if ((uint64_t)n_tiles >= (1ull << 20)) return false;  // the combine lists hold 20-bit tiles
  int P2 = 256;  // at least one entry per thread of the sort's block
  while (P2 < op.S * kMmaRows) P2 <<= 1;
  const int NG = kMmaRows / kMmaWarpRows;
  const size_t smem = sizeof(int32_t) * ((size_t)P2 + kMmaPlaneMax) + sizeof(int16_t) * kMmaPlaneMax +
                      (size_t)NG * kMmaPlaneMax;
  allow_dynamic_smem(k_mma_layout);
  DevMem tch(sizeof(int32_t) * n_tiles), tpc(sizeof(int32_t) * n_tiles), twl(sizeof(int32_t) * n_tiles),
      rowch(std::max<i64>(n_rep, 1)), flag(sizeof(int));
  STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  MmaArgs a{};
  a.cell = op.cell.as<int32_t>();
  a.counts = counts.as<int>();
  a.coef = op.coef.as<float>();
  a.S = op.S;
  a.n_rep = n_rep;
  a.tile_ch = tch.as<int32_t>();
  a.tile_pc = tpc.as<int32_t>();
  a.tile_wl = twl.as<int32_t>();
  a.rowch = rowch.as<uint8_t>();
  a.overflow = flag.as<int>();
  k_mma_layout<<<(unsigned)n_tiles, 256, smem, s>>>(a, 0, P2);
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) return false;
  const int chunks = device_max(tch.as<int32_t>(), n_tiles, s);
  const int pc = device_max(tpc.as<int32_t>(), n_tiles, s);
  const int wl = device_max(twl.as<int32_t>(), n_tiles, s);
  auto stride = [](int v) { return ((v + 3) / 8) * 8 + 4; };  // the least value >= v that is 4 mod 8
  op.m_S = 8 * std::max(chunks, 1);
  op.m_pc = stride(pc);
  op.m_wl = stride(wl);
  if (op.m_S > kMmaMaxSlots || op.m_pc > kMmaPlaneMax) return false;
  op.m_tiles = n_tiles;
  op.m_coef.alloc(sizeof(float) * 8 * (size_t)op.m_S * n_rep);
  op.m_cells.alloc(sizeof(int32_t) * (size_t)n_tiles * op.m_pc);
  op.m_lc.alloc(sizeof(uint16_t) * (size_t)n_tiles * op.m_S * kMmaRows);
  op.m_wlc.alloc((size_t)n_tiles * op.m_S * kMmaRows);
  op.m_winv.alloc((size_t)n_tiles * NG * op.m_pc);
  STL_CUDA(cudaMemsetAsync(op.m_lc.p, 0, op.m_lc.bytes, s));
  STL_CUDA(cudaMemsetAsync(op.m_wlc.p, 0, op.m_wlc.bytes, s));
  a.Sm = op.m_S;
  a.pcs = op.m_pc;
  a.m_coef = op.m_coef.as<float>();
  a.m_cells = op.m_cells.as<int32_t>();
  a.m_lc = op.m_lc.as<uint16_t>();
  a.m_wlc = op.m_wlc.as<uint8_t>();
  a.m_winv = op.m_winv.as<uint8_t>();
  k_mma_layout<<<(unsigned)n_tiles, 256, smem, s>>>(a, 1, P2);
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) return false;
  op.m_rowch = std::move(rowch);
  op.m_tch = std::move(tch);
  op.mma = true;
  if (!adjoint) return true;
  // per stored input cell: the (tile, plane cell, rotation) entries of the
  // adjoint's tile partials, sorted
  const i64 n_cells = op.n_in / 4, nt = n_tiles * op.m_pc;
  DevMem cnt(sizeof(int) * n_cells);
  STL_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
  k_mma_ccount<<<nblocks(nt, 256), 256, 0, s>>>(op.m_cells.as<int32_t>(), nt, op.m_pc, op.o2, cnt.as<int>());
  STL_CUDA(cudaGetLastError());
  std::vector<int> hc(n_cells);
  STL_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, cnt.bytes, cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  std::vector<i64> ho(n_cells + 1, 0);
  for (i64 v = 0; v < n_cells; ++v) ho[v + 1] = ho[v] + hc[v];
  op.coff.alloc(sizeof(i64) * (n_cells + 1));
  op.clist.alloc(sizeof(uint32_t) * std::max<i64>(ho[n_cells], 1));
  STL_CUDA(cudaMemcpyAsync(op.coff.p, ho.data(), op.coff.bytes, cudaMemcpyHostToDevice, s));
  STL_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
  k_mma_cfill<<<nblocks(nt, 256), 256, 0, s>>>(op.m_cells.as<int32_t>(), nt, op.m_pc, op.o2, op.coff.as<i64>(),
                                               cnt.as<int>(), op.clist.as<uint32_t>());
  STL_CUDA(cudaGetLastError());
  k_adj_csort<<<nblocks(n_cells, 256), 256, 0, s>>>(op.coff.as<i64>(), n_cells, op.clist.as<uint32_t>());
  STL_CUDA(cudaGetLastError());
  STL_CUDA(cudaStreamSynchronize(s));
  op.ncs = op.m_pc;
  op.mma_adj = true;
  return true;
}

template <typename T>
static void build_conv_t(const ConvSpec& sp, const std::vector<double>& kernel, ConvOp& op, cudaStream_t s) {
  const int P = sp.ksz * sp.ksz;
  if (sp.G != 4) throw std::runtime_error("the engine's convolution is built for L = 4 orientations");
  std::vector<double> st = kernel_grid(sp.ksz, sp.nside);
  DevMem d_st(st.size() * 8), d_ker(kernel.size() * 8);
  STL_CUDA(cudaMemcpyAsync(d_st.p, st.data(), st.size() * 8, cudaMemcpyHostToDevice, s));
  STL_CUDA(cudaMemcpyAsync(d_ker.p, kernel.data(), kernel.size() * 8, cudaMemcpyHostToDevice, s));
  const bool sym = sp.symmetric && sp.d_grid == nullptr && sp.d_rows == nullptr;
  FoldArgs a;
  a.nside = sp.nside; a.order = order_of(sp.nside); a.ksz = sp.ksz; a.P = P; a.G = sp.G; a.gauge = sp.gauge;
  a.p_ref = (sp.ksz / 2) * (sp.ksz + 1); a.eps = sp.eps;
  a.grid = sp.d_grid; a.n_in = sp.d_grid ? sp.n_in : npix_of(sp.nside);
  if (sp.d_seg && (!sp.d_grid || sp.d_rows)) throw std::runtime_error("segments need a grid whose cells are the rows");
  a.seg = sp.d_seg; a.nseg = sp.nseg;
  a.rows = sp.d_rows;
  i64 n_rows = sp.d_rows ? sp.n_rows : a.n_in;
  a.n_rows = sym ? n_rows / 4 : n_rows;
  a.sym = sym ? 1 : 0;
  a.sym_o2 = 2 * a.order;
  a.stencil = d_st.as<double>(); a.kernel = d_ker.as<double>();
  op.n_rows = n_rows; op.n_in = a.n_in; op.n_rep = a.n_rows; op.G = sp.G;
  op.nk = sym ? 4 : 1;
  op.o2 = 2 * a.order;
  op.dtype = sizeof(T) == 8 ? DType::F64 : DType::F32;
  DevMem counts(sizeof(int) * std::max<i64>(a.n_rows, 1)), flag(sizeof(int));
  STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  const int TB = 64;
  k_fold<T><<<nblocks(a.n_rows, TB), TB, 0, s>>>(a, counts.as<int>(), 0, nullptr, nullptr, flag.as<int>());
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) throw std::runtime_error("a wavelet stencil reads more cells than the builder holds");
  op.S = std::max(1, device_max(counts.as<int>(), a.n_rows, s));
  op.mean_slots = device_mean(counts.as<int>(), a.n_rows, s);
  op.cell.alloc(sizeof(int32_t) * op.S * a.n_rows);
  op.coef.alloc(sizeof(T) * 2 * sp.G * op.S * a.n_rows);
  k_fold<T><<<nblocks(a.n_rows, TB), TB, 0, s>>>(a, counts.as<int>(), op.S, op.cell.as<int32_t>(), op.coef.as<T>(),
                                                flag.as<int>());
  STL_CUDA(cudaGetLastError());
  const i64 n_cells = sym ? a.n_in / 4 : a.n_in;  // stored cells == stored rows on the full sky
  if (sym && n_cells != a.n_rows) throw std::runtime_error("symmetric operator needs rows == cells");
  if (!sym && n_cells != a.n_rows) throw std::runtime_error("rows and grid must coincide");
  // row-centric adjoint tiles (full sky): the distinct cells of every tile
  // of kAdjTile stored rows, then the edge colouring of its entries
  op.adj_tiles = false;
  op.colored = false;
  op.mma = op.mma_adj = false;
  if (std::is_same<T, float>::value && sym && sp.tensor_cores > 0) {
    // FP32 full sky: the tensor-core layout when every tile fits it, for the
    // forward (the coloured layout below then serves the adjoint) or for both
    op.rowsum.alloc(sizeof(T) * 8 * a.n_rows);
    k_rowsum<T><<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.coef.as<T>(), op.S, a.n_rows, op.rowsum.as<T>());
    STL_CUDA(cudaGetLastError());
    if (build_mma_layout(op, counts, sp.tensor_cores == 2, s)) {
      if (op.mma_adj) {
        op.cell.release();
        op.coef.release();
        return;
      }
    } else {
      op.mma = op.mma_adj = false;
      op.rowsum.release();
      op.m_coef.release(); op.m_cells.release(); op.m_lc.release(); op.m_wlc.release(); op.m_winv.release();
      op.m_rowch.release(); op.m_tch.release();
    }
  }
  if (sym && op.S <= 128) {  // the tile sort holds 128 slots per row
    op.n_tiles = (a.n_rows + kAdjTile - 1) / kAdjTile;
    op.tile_slots.alloc(sizeof(int32_t) * op.n_tiles);
    k_tile_slots<<<nblocks(op.n_tiles, 256), 256, 0, s>>>(counts.as<int>(), a.n_rows, op.n_tiles,
                                                          op.tile_slots.as<int32_t>());
    STL_CUDA(cudaGetLastError());
    op.tile_cells.alloc(sizeof(int32_t) * kAdjCells * op.n_tiles);
    op.tile_ncells.alloc(sizeof(int32_t) * op.n_tiles);
    op.lcell.alloc(sizeof(uint16_t) * op.S * a.n_rows);
    int P2 = 1;
    while (P2 < op.S * kAdjTile) P2 <<= 1;
    const size_t smem = sizeof(int32_t) * ((size_t)P2 + kAdjCells + 256);
    if (smem > 48 * 1024)
      allow_dynamic_smem(k_adj_tiles);
    STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
    k_adj_tiles<<<(unsigned)op.n_tiles, 256, smem, s>>>(op.cell.as<int32_t>(), op.S, a.n_rows, P2,
                                                          op.tile_cells.as<int32_t>(), op.tile_ncells.as<int32_t>(),
                                                          op.lcell.as<uint16_t>(), flag.as<int>());
    STL_CUDA(cudaGetLastError());
    op.adj_tiles = !read_flag(flag, s);
    std::vector<int32_t> nc(op.n_tiles);
    STL_CUDA(cudaMemcpyAsync(nc.data(), op.tile_ncells.p, sizeof(int32_t) * op.n_tiles, cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    op.max_tile_cells = 0;
    for (int32_t v : nc) op.max_tile_cells = std::max(op.max_tile_cells, (int)v);
    if ((uint64_t)op.n_tiles >= (1ull << 20)) op.adj_tiles = false;
    if (op.adj_tiles && op.max_tile_cells < kAdjCells) {
      // every colour a matching: the coloured layout replaces the slots
      DevMem col((size_t)op.S * a.n_rows), tile_d(sizeof(int32_t) * op.n_tiles);
      const size_t csm = color_smem(op.S);
      allow_dynamic_smem(k_color_tiles);
      STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
      k_color_tiles<<<(unsigned)op.n_tiles, 32, csm, s>>>(op.lcell.as<uint16_t>(), counts.as<int>(), op.S, a.n_rows,
                                                          op.tile_ncells.as<int32_t>(), col.as<uint8_t>(),
                                                          tile_d.as<int32_t>(), flag.as<int>());
      STL_CUDA(cudaGetLastError());
      if (!read_flag(flag, s)) {
        const int S2 = std::max(1, device_max(tile_d.as<int32_t>(), op.n_tiles, s));
        DevMem cell2(sizeof(int32_t) * S2 * a.n_rows), coef2(sizeof(T) * 8 * S2 * a.n_rows),
            lcell2(sizeof(uint16_t) * S2 * a.n_rows);
        k_color_apply<T><<<nblocks(a.n_rows, 256), 256, 0, s>>>(
            op.cell.as<int32_t>(), op.coef.as<T>(), op.lcell.as<uint16_t>(), col.as<uint8_t>(), counts.as<int>(),
            op.S, S2, a.n_rows, op.tile_ncells.as<int32_t>(), cell2.as<int32_t>(), coef2.as<T>(),
            lcell2.as<uint16_t>());
        STL_CUDA(cudaGetLastError());
        STL_CUDA(cudaMemcpyAsync(op.tile_slots.p, tile_d.p, tile_d.bytes, cudaMemcpyDeviceToDevice, s));
        STL_CUDA(cudaStreamSynchronize(s));
        op.cell = std::move(cell2);
        op.coef = std::move(coef2);
        op.lcell = std::move(lcell2);
        op.S = S2;
        op.colored = true;
      }
    }
  }
  if (!op.rowsum.p) {  // the row sums (the tensor-core branch made them already)
    op.rowsum.alloc(sizeof(T) * 8 * a.n_rows);
    k_rowsum<T><<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.coef.as<T>(), op.S, a.n_rows, op.rowsum.as<T>());
    STL_CUDA(cudaGetLastError());
  }
  if (!op.colored) {
    // transposed gather table over the stored cells: entries (u, s, j)
    int sbits = 1;
    while ((1 << sbits) < op.S) ++sbits;
    op.tshift = sbits + 2;
    if ((uint64_t)std::max<i64>(a.n_rows - 1, 0) >= ((uint64_t)1 << (32 - op.tshift)) - 1)
      throw std::runtime_error("level too large for the 32-bit transposed table");
    DevMem tcount(sizeof(int) * n_cells), tfill(sizeof(int) * n_cells);
    STL_CUDA(cudaMemsetAsync(tcount.p, 0, tcount.bytes, s));
    STL_CUDA(cudaMemsetAsync(tfill.p, 0, tfill.bytes, s));
    k_conv_tcount<<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.cell.as<int32_t>(), counts.as<int>(), a.n_rows, a.sym,
                                                         a.sym_o2, tcount.as<int>());
    STL_CUDA(cudaGetLastError());
    op.ST = std::max(1, device_max(tcount.as<int>(), n_cells, s));
    op.tent.alloc(sizeof(uint32_t) * op.ST * n_cells);
    k_conv_tfill<<<nblocks(a.n_rows, 256), 256, 0, s>>>(op.cell.as<int32_t>(), counts.as<int>(), a.n_rows, a.sym,
                                                        a.sym_o2, op.tshift, tfill.as<int>(), op.tent.as<uint32_t>());
    STL_CUDA(cudaGetLastError());
    k_tsort<<<nblocks(n_cells, 256), 256, 0, s>>>(op.tent.as<uint32_t>(), tcount.as<int>(), n_cells, op.ST);
    STL_CUDA(cudaGetLastError());
    op.coefT.alloc(sizeof(T) * 8 * op.ST * n_cells);
    k_conv_coefT<T><<<nblocks(n_cells, 256), 256, 0, s>>>(op.tent.as<uint32_t>(), op.coef.as<T>(), n_cells, op.ST,
                                                          op.tshift, op.coefT.as<T>());
    STL_CUDA(cudaGetLastError());
  }
  if (!op.adj_tiles) return;
  op.nch = (op.S + kAdjSC - 1) / kAdjSC;
  op.ncs = op.max_tile_cells + 1;
  if (!op.colored) {
    // per tile and slot chunk: the entries of every tile cell
    op.tile_ent.alloc(sizeof(uint16_t) * (size_t)op.n_tiles * op.S * kAdjTile);
    op.tile_off.alloc(sizeof(uint16_t) * (size_t)op.n_tiles * op.nch * op.ncs);
    {
      int P2 = 1;
      while (P2 < op.S * kAdjTile) P2 <<= 1;
      const size_t smem = sizeof(uint32_t) * (size_t)P2;
      if (smem > 48 * 1024)
        allow_dynamic_smem(k_adj_csr);
      k_adj_csr<<<(unsigned)op.n_tiles, 256, smem, s>>>(op.cell.as<int32_t>(), op.lcell.as<uint16_t>(), op.S,
                                                          a.n_rows, P2, op.nch, op.ncs, op.tile_ncells.as<int32_t>(),
                                                          op.tile_ent.as<uint16_t>(), op.tile_off.as<uint16_t>());
      STL_CUDA(cudaGetLastError());
    }
  }
  {
    const int S4 = ((op.S + 3) / 4) * 4;
    op.lcell_t.alloc(sizeof(uint16_t) * (size_t)op.n_tiles * S4 * kAdjTile);
    const i64 n = op.n_tiles * S4 * kAdjTile;
    k_lcell_tiles<<<nblocks(n, 256), 256, 0, s>>>(op.lcell.as<uint16_t>(), op.S, a.n_rows, S4, op.n_tiles,
                                                  op.lcell_t.as<uint16_t>());
    STL_CUDA(cudaGetLastError());
    STL_CUDA(cudaStreamSynchronize(s));
    op.lcell.release();
  }
  // per stored input cell: the (tile, cell, rotation) entries holding its sums
  {
    const i64 n_in_rep = n_cells;
    const i64 nt = op.n_tiles * kAdjCells;
    DevMem cnt(sizeof(int) * n_in_rep);
    STL_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
    k_adj_ccount<<<nblocks(nt, 256), 256, 0, s>>>(op.tile_cells.as<int32_t>(), op.tile_ncells.as<int32_t>(),
                                                  op.n_tiles, op.nk, op.o2, cnt.as<int>());
    STL_CUDA(cudaGetLastError());
    std::vector<int> hc(n_in_rep);
    STL_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, cnt.bytes, cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    std::vector<i64> ho(n_in_rep + 1, 0);
    for (i64 v = 0; v < n_in_rep; ++v) ho[v + 1] = ho[v] + hc[v];
    op.coff.alloc(sizeof(i64) * (n_in_rep + 1));
    op.clist.alloc(sizeof(uint32_t) * std::max<i64>(ho[n_in_rep], 1));
    STL_CUDA(cudaMemcpyAsync(op.coff.p, ho.data(), op.coff.bytes, cudaMemcpyHostToDevice, s));
    STL_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
    k_adj_cfill<<<nblocks(nt, 256), 256, 0, s>>>(op.tile_cells.as<int32_t>(), op.tile_ncells.as<int32_t>(),
                                                 op.n_tiles, op.nk, op.o2, op.coff.as<i64>(), cnt.as<int>(),
                                                 op.clist.as<uint32_t>());
    STL_CUDA(cudaGetLastError());
    k_adj_csort<<<nblocks(n_in_rep, 256), 256, 0, s>>>(op.coff.as<i64>(), n_in_rep, op.clist.as<uint32_t>());
    STL_CUDA(cudaGetLastError());
    STL_CUDA(cudaStreamSynchronize(s));
  }
  STL_CUDA(cudaStreamSynchronize(s));
}

void build_conv(const ConvSpec& spec, const std::vector<double>& kernel, DType dtype, ConvOp& out, cudaStream_t s) {
  if (dtype == DType::F64) build_conv_t<double>(spec, kernel, out, s);
  else build_conv_t<float>(spec, kernel, out, s);
}

template <typename T>
static void build_dec_t(const DecSpec& sp, DecOp& op, cudaStream_t s) {
  const bool sym = sp.symmetric && sp.d_ids == nullptr && sp.d_out == nullptr && sp.nside >= 2;
  DecArgs a;
  a.nside = sp.nside; a.order = order_of(sp.nside); a.corder = order_of(sp.nside / 2);
  a.ids = sp.d_ids; a.n_in = sp.d_ids ? sp.n_in : npix_of(sp.nside);
  if ((sp.d_seg_in != nullptr) != (sp.d_seg_out != nullptr) || (sp.d_seg_in && (!sp.d_ids || !sp.d_out)))
    throw std::runtime_error("decimation segments need both grids");
  a.seg_in = sp.d_seg_in; a.seg_out = sp.d_seg_out; a.nseg = sp.nseg;
  a.out = sp.d_out;
  i64 n_out = sp.d_out ? sp.n_out : npix_of(sp.nside / 2);
  a.n_out = sym ? n_out / 4 : n_out;
  a.sym = sym ? 1 : 0;
  a.sym_co2 = 2 * a.corder;
  double pix_deg = std::sqrt(4.0 * kPi / (double)npix_of(sp.nside)) * (180.0 / kPi);
  a.radius = (3.0 * pix_deg) * (kPi / 180.0);
  a.sigma = a.radius / 2.0;
  op.n_out = n_out; op.n_in = a.n_in;
  op.nk = sym ? 4 : 1;
  op.o2 = 2 * a.order; op.co2 = 2 * a.corder;
  op.n_rep_out = a.n_out;
  op.n_rep_in = sym ? a.n_in / 4 : a.n_in;
  op.dtype = sizeof(T) == 8 ? DType::F64 : DType::F32;
  DevMem counts(sizeof(int) * std::max<i64>(a.n_out, 1)), flag(sizeof(int));
  STL_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  const int TB = 64;
  k_dec_rows<T><<<nblocks(a.n_out, TB), TB, 0, s>>>(a, counts.as<int>(), 0, nullptr, nullptr, flag.as<int>());
  STL_CUDA(cudaGetLastError());
  if (read_flag(flag, s)) throw std::runtime_error("a decimation row has more candidates than the builder holds");
  op.W = std::max(1, device_max(counts.as<int>(), a.n_out, s));
  op.mean_w = device_mean(counts.as<int>(), a.n_out, s);
  op.col.alloc(sizeof(int32_t) * op.W * a.n_out);
  op.w.alloc(sizeof(T) * op.W * a.n_out);
  k_dec_rows<T><<<nblocks(a.n_out, TB), TB, 0, s>>>(a, counts.as<int>(), op.W, op.col.as<int32_t>(), op.w.as<T>(),
                                                   flag.as<int>());
  STL_CUDA(cudaGetLastError());
  const i64 n_cells = op.n_rep_in;
  const int fine_o2 = op.o2, symi = sym ? 1 : 0;
  DevMem tcount(sizeof(int) * n_cells), tfill(sizeof(int) * n_cells);
  STL_CUDA(cudaMemsetAsync(tcount.p, 0, tcount.bytes, s));
  STL_CUDA(cudaMemsetAsync(tfill.p, 0, tfill.bytes, s));
  k_dec_tcount<<<nblocks(a.n_out, 256), 256, 0, s>>>(op.col.as<int32_t>(), counts.as<int>(), a.n_out, symi, fine_o2,
                                                      tcount.as<int>());
  STL_CUDA(cudaGetLastError());
  op.WT = std::max(1, device_max(tcount.as<int>(), n_cells, s));
  op.tcol.alloc(sizeof(int32_t) * op.WT * n_cells);
  op.tw.alloc(sizeof(T) * op.WT * n_cells);
  k_dec_tfill<T><<<nblocks(a.n_out, 256), 256, 0, s>>>(op.col.as<int32_t>(), op.w.as<T>(), counts.as<int>(), a.n_out,
                                                       n_cells, symi, fine_o2, op.co2, tfill.as<int>(),
                                                       op.tcol.as<int32_t>(), op.tw.as<T>());
  STL_CUDA(cudaGetLastError());
  k_dec_tsort<T><<<nblocks(n_cells, 256), 256, 0, s>>>(op.tcol.as<int32_t>(), op.tw.as<T>(), tcount.as<int>(),
                                                       n_cells, op.WT);
  STL_CUDA(cudaGetLastError());
  STL_CUDA(cudaStreamSynchronize(s));
}

void build_dec(const DecSpec& spec, DType dtype, DecOp& out, cudaStream_t s) {
  if (dtype == DType::F64) build_dec_t<double>(spec, out, s);
  else build_dec_t<float>(spec, out, s);
}

}  // namespace stl
