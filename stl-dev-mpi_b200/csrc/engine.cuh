// B200 ScatCov engine: device operators, kernels and the level sweeps.
//
// The engine evaluates mean, var, S1..S4 (L orientations, J scales,
// dg(j) = j) of HEALPix NESTED maps over the smooth-decimation pyramid, and
// the exact VJP, on one GPU.  It is the device counterpart of the
// reference's LocalEngine/GpuEngine (crates/stl-core/src/engine.rs,
// crates/stl-gpu/src/engine.rs); the sky split of the reference becomes
// full-sky level sweeps with no collective.
//
// Operators (built once per handle on the device, FP64 geometry):
//  * ConvOp: the oriented wavelet of a level, folded per output row into S
//    slots of (input cell, 2G coefficients) -- the bilinear binding of the
//    rotated 5x5 stencil and the kernel multiplied out, in the union of the
//    cells the G gauges read (about 44 per row at L = 4).  Slot-major
//    layout [S][rows] so a warp's loads of one slot are contiguous.  The
//    adjoint gathers per input cell over a transposed table of
//    (row, slot) entries, sorted, so no atomics touch the results.
//  * DecOp: the smooth decimation D of a level and its transpose as ELL
//    rows (about 28 weights per coarse pixel).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace stl {

typedef int64_t i64;

#define STL_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t err__ = (call);                                                                 \
    if (err__ != cudaSuccess)                                                                   \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(err__) + " at " + \
                               __FILE__ + ":" + std::to_string(__LINE__));                      \
  } while (0)

// Owning device allocation.
struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  DevMem() = default;
  explicit DevMem(size_t n) { alloc(n); }
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  DevMem(DevMem&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevMem& operator=(DevMem&& o) noexcept {
    if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevMem() { release(); }
  void alloc(size_t n);
  void release();
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Lets kernel f use up to the device's opt-in shared memory per CTA.  The
// attribute is process-wide and the launch's own size decides occupancy, so
// it is always set to the maximum: threads launching f with different sizes
// cannot undo each other's setting.
void allow_dynamic_smem_fn(const void* f);
template <typename F>
inline void allow_dynamic_smem(F* f) {
  allow_dynamic_smem_fn(reinterpret_cast<const void*>(f));
}

// Page-locked host memory (copies from it run asynchronously).
struct PinnedMem {
  void* p = nullptr;
  size_t bytes = 0;
  PinnedMem() = default;
  PinnedMem(const PinnedMem&) = delete;
  PinnedMem& operator=(const PinnedMem&) = delete;
  ~PinnedMem() { release(); }
  void alloc(size_t n);
  void release();
};

// Message of a kernel's timed-out copy wait (the error flag's value: 1 a
// wait ran out, 2 also the drain of the copies in flight); the results of
// the sweep are discarded either way.
inline std::string wait_timeout_message(int err, const char* where) {
  std::string m = std::string("a wait on a staged device copy timed out in ") + where;
  if (err >= 2) m += " while copies were still in flight (rebuild the engine before using it again)";
  return m;
}

// Device memory accounting (bytes held by live DevMem allocations).
size_t device_bytes_live();
size_t device_bytes_peak();
void device_bytes_reset_peak();

enum class DType { F64 = 0, F32 = 1 };
inline size_t dsize(DType t) { return t == DType::F64 ? 8 : 4; }

// Geometry of one wavelet operator: output rows reading an input grid.
struct ConvSpec {
  i64 nside = 0;
  // FP32 full sky: 0 the coloured layout only (CUDA cores), 1 the tensor-core
  // layout for the forward and the coloured one for the adjoint, 2 the
  // tensor-core layout for both
  int tensor_cores = 0;
  int ksz = 5, G = 4, gauge = 0;
  double eps = 0.0;
  const i64* d_grid = nullptr;  // sorted NESTED ids of the grid (device), nullptr: whole sky
  i64 n_in = 0;
  const i64* d_rows = nullptr;  // NESTED ids of the output rows (device), nullptr: rows == grid
  i64 n_rows = 0;
  const i64* d_seg = nullptr;   // segments of the grid: nseg + 1 starts (device), nullptr: one
  int nseg = 0;
  bool symmetric = true;        // full sky: store the rows of faces 0, 4, 8 only
};

// Full sky: HEALPix's 4-fold azimuthal symmetry (faces 4m + k, k = 0..3,
// are rotations by k pi / 2 of face 4m) makes the folded stencil of
// pixel (4m + k, x, y) the one of (4m, x, y) with every cell read rotated
// to face 4m + k, the gauges permuted (g <- (g + 2k) mod 4) and the
// imaginary part negated when the rotated gauge angle wraps by pi.  Only
// the rows of faces 0, 4 and 8 ("representative rows", nk = 4) are
// stored; kernels evaluate the 4 rotations from one coefficient load.
// Partial grids (disc patches) store every row (nk = 1).
struct ConvOp {
  i64 n_rows = 0, n_in = 0;  // output rows, input cells (full level or grid)
  i64 n_rep = 0;             // stored rows (n_rows / nk)
  int nk = 1;                // 4: full-sky rotations, 1: every row stored
  int o2 = 0;                // 2 log2(nside): pixel = face << o2 | local
  int S = 0;                 // slots per stored row
  int ST = 0;                // transposed entries per stored cell
  int tshift = 0;            // transposed entry = u << tshift | s << 2 | j
  DType dtype = DType::F32;
  DevMem cell;               // int32 [S][n_rep]: cell read (full-sky id, or grid position)
  DevMem coef;               // T [S][n_rep][8]: (gauge, re/im) coefficients
  DevMem tent;               // uint32 [ST][n_rep]: entries (u, s, j) reading rotation j of a stored cell
  DevMem coefT;              // T [ST][n_rep][8]: coef of each transposed entry
  DevMem rowsum;             // T [n_rep][8]: sum over the slots of coef (the response to a constant field)
  // Row-centric adjoint: stored rows in tiles of kAdjTile.  Per tile the
  // sorted distinct cells its rows read; per (tile, chunk of kAdjSC slots)
  // the (slot, row) entries of every tile cell in (slot, row) order; per
  // stored input cell the (tile, tile cell, rotation) entries that hold its
  // partial sums, sorted.  Every sum of the adjoint has a fixed order.
  i64 n_tiles = 0;
  int nch = 0;               // slot chunks: ceil(S / kAdjSC)
  int ncs = 0;               // stride of the tile cell lists: most cells of a tile + 1
  int max_tile_cells = 0;
  bool adj_tiles = false;    // tables built (every tile within kAdjCells cells)
  // Coloured layout: within a tile, slot k of every row holds its entry of
  // colour k of an edge colouring of the tile's (row, cell) entries, so no
  // two rows of a tile read one cell in the same slot; padding slots have
  // zero coefficients and tile cell ncells (none).  The adjoint then adds
  // every product straight into its cell's sums, slot by slot; the
  // transposed table and the entry lists are not built.
  bool colored = false;
  DevMem tile_cells;         // int32 [n_tiles][kAdjCells]
  DevMem tile_ncells;        // int32 [n_tiles]
  DevMem tile_slots;         // int32 [n_tiles]: slots the tile's rows use (later slots are zero)
  DevMem lcell;              // uint16 [S][n_rep]: tile cell of every (slot, row) (build only)
  DevMem lcell_t;            // uint16 [n_tiles][nch 4][kAdjTile]: the same, tile-major, slots padded to 4
  DevMem tile_ent;           // uint16 [n_tiles][S kAdjTile]: slot % kAdjSC << 8 | row
  DevMem tile_off;           // uint16 [n_tiles][nch][ncs]: first entry of (chunk, tile cell)
  DevMem coff;               // int64 [stored cells + 1]
  DevMem clist;              // uint32 tile << 12 | tile cell << 2 | rotation
  int G = 4;
  double mean_slots = 0.0;   // cells read per row, averaged over the rows
  // Tensor-core layout (FP32 full sky; replaces the coloured one).  Tiles of
  // kMmaRows stored rows; per tile a plane of input cells in which cell c
  // sits at 4 (its rank among the tile's cells of its class) + class, the
  // class being c's NESTED bits x0 + 2 y0 (the parity of its face
  // coordinates); slots in chunks of 8 whose position p holds a cell of
  // class kMmaClass[p] (zero coefficients where a row has none left), so the
  // 8 cells an mma step gathers fall in distinct shared-memory banks.  The
  // adjoint adds into per-warp sums over the distinct cells of the warp's
  // kMmaWarpRows rows (numbered the same way), combined per tile cell in
  // warp order.  Every sum has a fixed order.
  bool mma = false;          // the forward uses the tensor-core layout
  bool mma_adj = false;      // the adjoint too (else the coloured layout's)
  i64 m_tiles = 0;
  int m_S = 0;               // slots: 8 x the most chunks of a row
  int m_pc = 0;              // plane stride (cells; 4 mod 8)
  int m_wl = 0;              // stride of a warp's private sums (cells; 4 mod 8)
  DevMem m_coef;             // float [m_S][n_rep][8]
  DevMem m_cells;            // int32 [m_tiles][m_pc]: plane cell ids (-1: none)
  DevMem m_lc;               // uint16 [m_tiles][m_S / 8][kMmaRows][8]: plane cell of every (row, slot)
  DevMem m_wlc;              // uint8 [m_tiles][m_S / 8][kMmaRows][8]: warp-local cell of every (row, slot)
  DevMem m_winv;             // uint8 [m_tiles][kMmaRows / kMmaWarpRows][m_pc]: warp-local cell of each plane cell (255: none)
  DevMem m_rowch;            // uint8 [n_rep]: chunks of every row
  DevMem m_tch;              // int32 [m_tiles]: chunks of the tile (its rows' most)
  size_t bytes() const {
    return cell.bytes + coef.bytes + tent.bytes + coefT.bytes + rowsum.bytes + tile_cells.bytes + tile_ncells.bytes +
           tile_slots.bytes + lcell.bytes + lcell_t.bytes + tile_ent.bytes + tile_off.bytes + coff.bytes +
           clist.bytes + m_coef.bytes + m_cells.bytes + m_lc.bytes + m_wlc.bytes + m_winv.bytes + m_rowch.bytes +
           m_tch.bytes;
  }
};
constexpr int kMmaRows = 64;      // stored rows per tile of the tensor-core layout
constexpr int kMmaWarpRows = 8;   // rows per warp of the adjoint (one block of private sums)
constexpr int kMmaPlaneMax = 1024;  // plane cells a tile may index
constexpr int kMmaWarpMax = 252;    // warp-local cells (uint8 indices, 255: none)
// class of the cell at position p of a chunk: every class twice, positions
// 0-3 and 4-7 all four, positions 0, 2, 4, 6 and 1, 3, 5, 7 all four
__host__ __device__ constexpr int mma_class(int p) { return (0x23013210 >> (4 * p)) & 3; }
constexpr int kAdjTile = 128;    // stored rows per tile of the tiled forward and adjoint
constexpr int kAdjCells = 1024;  // cells a tile may read
constexpr int kAdjSC = 8;        // slots per chunk of the two-phase adjoint

// Scratch of the row-centric adjoint: the tile partial sums
// [n_tiles][4][ncs][R] (capacity bytes).
struct AdjScratch {
  void* part = nullptr;
  size_t capacity = 0;
};
size_t adjoint_part_bytes(const ConvOp& op, size_t elem, int R);
bool adjoint_tiles_usable(const ConvOp& op, size_t elem, int R, const AdjScratch* scr);

struct DecSpec {
  i64 nside = 0;           // fine level
  const i64* d_ids = nullptr;  // sorted fine grid (device), nullptr: whole sky
  i64 n_in = 0;
  const i64* d_out = nullptr;  // sorted coarse ids = parents of the grid (device), nullptr: whole sky
  i64 n_out = 0;
  // segments of both grids (nseg + 1 starts each, device; coarse segment k
  // holds the parents of fine segment k), nullptr: one
  const i64* d_seg_in = nullptr;
  const i64* d_seg_out = nullptr;
  int nseg = 0;
  bool symmetric = true;       // full sky: store the rows of faces 0, 4, 8 only
};

// Decimation rows, stored for the coarse pixels of faces 0, 4, 8 on the
// full sky (nk = 4: rows of the other faces are the rotated ones, as for
// ConvOp), and the transposed rows for the fine pixels of faces 0, 4, 8.
struct DecOp {
  i64 n_out = 0, n_in = 0;         // coarse rows, fine cells (full level or grid)
  i64 n_rep_out = 0, n_rep_in = 0; // stored coarse rows, stored fine cells
  int nk = 1, o2 = 0, co2 = 0;     // rotations; 2 log2 nside of the fine and coarse levels
  int W = 0, WT = 0;
  DType dtype = DType::F32;
  DevMem col, w;    // int32 / T [W][n_rep_out]: fine column (full-sky id or grid position)
  DevMem tcol, tw;  // int32 / T [WT][n_rep_in]: coarse row (full-sky id or position)
  double mean_w = 0.0;  // weights per coarse row, averaged
  size_t bytes() const { return col.bytes + w.bytes + tcol.bytes + tw.bytes; }
};

// Builders (geometry.cu).  The kernel weights are [G][2][P], f32-rounded.
void build_conv(const ConvSpec& spec, const std::vector<double>& kernel, DType dtype, ConvOp& out,
                cudaStream_t stream);
void build_dec(const DecSpec& spec, DType dtype, DecOp& out, cudaStream_t stream);

// Kernel launchers (kernels.cu).  Fields are pixel-major (a vector of
// rows per pixel); complex values interleave (re, im).
//  conv_forward: x [n_in][R] -> out [n_rows][R][4] complex; with mod, |out|
//    of row r, gauge g at mod[p mod_pix + r mod_row + mod_off + g].
//  conv_adjoint: gy [n_rows][R][4] complex -> gx [n_in][R] (or += gx).
//  dec_apply: y[c][ro][ri] = (D or D^T) x, row (ro, ri) of pixel c at
//    c pix + ro outer + ri.
//  With err (device int, set on a timed-out copy wait), operators with tile
//  tables use the tiled forward; otherwise the per-row gather.  rc (R FP64
//  constants, or null): the input rows are deviations from rc, whose
//  response rc x rowsum is added to the outputs.
//  rb: rows of the field a thread takes (the tile height of the launch); 0
//  picks the default, else one of conv_forward_choices.  Results do not
//  depend on it: every output row is computed alone, in the same order.
template <typename T>
void conv_forward(const ConvOp& op, const T* x, int R, T* out, T* mod, int mod_pix, int mod_row, int mod_off,
                  cudaStream_t s, int* err = nullptr, const double* rc = nullptr, int rb = 0);
std::vector<int> conv_forward_choices(const ConvOp& op, size_t elem, int R, bool err);
//  With scratch, operators in the coloured layout use the coloured adjoint
//  (bounded waits on its bulk copies set *err on timeout), other operators
//  with tile tables the two-phase adjoint; otherwise the transposed gather.
//  madd (coloured adjoint only): first add the modulus VJP to the input,
//  gy[p][r][l] += g[p g_pix + r g_row + l] z[p][r][l] / |z[p][r][l]| (0 at
//  z = 0), the rows r being the maps.
template <typename T>
struct ModulusAdd {
  const T* z = nullptr;
  const T* g = nullptr;
  int g_pix = 0, g_row = 0;
};
bool conv_adjoint_fuses_modulus(const ConvOp& op, size_t elem, int R, const AdjScratch* scr, int* err);
template <typename T>
void conv_adjoint(const ConvOp& op, const T* gy, int R, T* gx, bool accumulate, cudaStream_t s,
                  const AdjScratch* scr = nullptr, int* err = nullptr, const ModulusAdd<T>* madd = nullptr,
                  int rb = 0);
std::vector<int> conv_adjoint_choices(const ConvOp& op, size_t elem, int R, const AdjScratch* scr);
//    Input and output types may differ (FP32 and FP64 levels); the sums are
//    in the operator's type.
template <typename Tin, typename Tout>
void dec_apply(const DecOp& op, bool transpose, const Tin* x, int x_pix, int x_outer, Tout* y, int y_pix,
               int y_outer, int R_outer, int R_inner, bool accumulate, cudaStream_t s, int rb = 0);
std::vector<int> dec_choices(size_t elem_in, int R_inner);
// gz[p][b][l] += g z / |z|, z and gz [N][B][L] complex, g at p g_pix + b g_row + l
template <typename T>
void modulus_vjp_add(const T* z, const T* g, int g_pix, int g_row, T* gz, i64 N, int B, int L, cudaStream_t s);

// Coefficient products of one level (see kernels.cu for the slot layout).
struct ProductShape {
  int nd = 1;        // levels of the branches: n + 1
  int K = 0;         // operand vector length: (n + 1) L branches + z
  int L = 4;
  int B = 1;
  i64 N = 0;         // pixels of the level
  bool level0 = false;
  int blocks = 0;    // partial sums per map (pixel ranges)
  int slots = 0;     // doubles per (b, l3) partial
  int items = 0;     // Gram items per (b, l3)
  int item_chunks = 0;  // role chunks (grid z)
  int warps = 0;     // warps per CTA
  std::vector<int32_t> roles;      // [item_chunks][warps]: role | replica << 16 | replicas << 24, or -1
  const int32_t* d_roles = nullptr;  // the same on the device
  int px_chunk = 0;  // pixels per staged chunk
  i64 chunk = 0;     // pixels per range
  size_t smem = 0;   // staged chunks
  // Several regions (segments), each with its own sums: the CTAs take pixel
  // ranges inside one segment -- forward ranges blk (blocks + 1 starts),
  // reverse ranges rev_blk (rev_blocks + 1 starts) with their segments
  // rev_seg -- and the partials of segment k are the forward ranges
  // seg_blk[k] .. seg_blk[k + 1] - 1; its sums start k seg_stride after
  // those of segment 0.  Empty tables: one region, uniform ranges.
  int nseg = 1, rev_blocks = 0;
  size_t seg_stride = 0;
  std::vector<i64> blk, rev_blk;
  std::vector<int32_t> rev_seg, seg_blk;
  const i64* d_blk = nullptr;
  const i64* d_rev_blk = nullptr;
  const int32_t* d_rev_seg = nullptr;
  const int32_t* d_seg_blk = nullptr;
};
ProductShape product_shape(int n, int L, int B, i64 N, size_t elem);
// fills the range tables of sh for the segments seg (nseg + 1 starts) of its
// level; the device copies are the caller's
void segment_ranges(ProductShape& sh, const std::vector<i64>& seg);
// z [N][B][L], br [N][B][(n+1) L][L] complex, x0 [N][B] (level 0) ->
// sums [B][L][slots] (FP64), per segment with segments
// *err becomes nonzero when a wait on a staged copy timed out.  x0 holds
// the level-0 maps as deviations from x0c [B], x0r (or null) their rounding
// residuals: the map sums take x0c + x0 + x0r in FP64.
// mask (or null): 1 on the pixels the sums cover.  moments: also the
// second sums the coefficient variances need (otherwise zero).
template <typename T>
void products_forward(const ProductShape& sh, const T* z, const T* br, const T* x0, const T* x0r, const double* x0c,
                      const uint8_t* mask, double* partials, double* sums, int* err, cudaStream_t s, bool moments);
// M [B][L][K][K] complex, s1c [B][L] -> gz [N][B][L], gbr [N][B][(n+1) L][L]
// (with segments: M [nseg][B][L][K][K], s1c [nseg][B][L])
// accumulate: add to gz / gbr (on the mask's pixels) instead of writing them
template <typename T>
void products_reverse(const ProductShape& sh, const T* z, const T* br, const T* M, const T* s1c, const uint8_t* mask,
                      bool accumulate, T* gz, T* gbr, cudaStream_t s);
// gx[p][b] += coefs[b][0] + coefs[b][1] (xc[b] + x0[p][b]); with segments
// (seg: nseg + 1 starts, device) the coefficients of p's segment,
// coefs [nseg][B][2]
template <typename T>
void mean_var_grad(const T* x0, const double* xc, const uint8_t* mask, const double* coefs, int B, i64 N, T* gx,
                   cudaStream_t s, const i64* seg = nullptr, int nseg = 1);
// ---- coefficients <-> sums on the device (kernels.cu) -------------------------
// Where plan coefficient i reads a mask's sums: the row of map 0 of its
// level and l3 at base, that of map b at base + b stride; the slots of its
// real part, imaginary part (-1: exactly zero) and second moment.
struct PlanSlots {
  int32_t level, base, stride, re, im, second;
  int32_t conj;  // the coefficient is the conjugate of the sum (a cross term in channel order (1, 0))
};
// values [B][K][np] complex and var [B][K][np] (or null) from the sums of K
// masks (mask k at sums + k mask_stride); counts [K][levels]: the pixels
// mask k averages at every level.  value = sum / count, var = max(second /
// count - |value|^2, 0).
void assemble_values(const double* sums, size_t mask_stride, const PlanSlots* plan, int np, const double* counts,
                     int levels, int B, int K, double* values, double* var, cudaStream_t s);
// Sources of one entry of a level's cotangent matrices (or of an S1 scale,
// or of the mean / variance scales): up to two plan coefficients, each
// entering as g (mode 0), conj(g) (1) or 2 Re g (2), divided by the mask's
// pixel count, added in that order (plan order).
struct CotSources {
  int32_t i0, i1, m0, m1;
};
// Cotangent matrices M [K][B][L][Kd][Kd] complex and S1 scales s1 [K][B][L]
// of level n in the field type U, from the coefficient cotangents cot
// [B][K][np] complex: entry (b, l3, r, q) from src[(l3 Kd + r) Kd + q], the
// real S1 scale (b, l) from s1src[l].
// (s1_complex: s1 [K][B][L] complex, the cross S1 terms' cotangents)
template <typename U>
void build_cotangents(const double* cot, int np, int B, int K, const double* counts, int levels, int n, int Kd,
                      int L, const CotSources* src, const CotSources* s1src, U* M, U* s1, cudaStream_t s,
                      bool s1_complex = false);
// Cross terms of channel pairs (kernels.cu): maps 2 b + c; per level the
// sums [B][L][cross_slots(K)] of G = sum v_0 conj(v_1) (K x K), of the cross
// S1 and, with moments, their second sums; nblk pixel ranges (cross_blocks),
// partials [nblk][B][L][cross_slots(K)].
int cross_blocks(i64 N);
__host__ __device__ constexpr int cross_slots(int K) { return 3 * K * K + 3; }
template <typename T>
void cross_forward(int K, i64 N, int Bm, const T* z, const T* br, const uint8_t* mask, bool moments,
                   double* partials, int nblk, double* sums, cudaStream_t s);
// their VJP: M [B][L][K][K] complex (cotangents of G), s1 [B][L] complex
// (of the cross S1) -> gz, gbr of both channels (accumulate: add)
template <typename T>
void cross_reverse(int K, i64 N, int Bm, const T* z, const T* br, const T* M, const T* s1, const uint8_t* mask,
                   bool accumulate, T* gz, T* gbr, cudaStream_t s);
// Synthesis terms: cot_o = 2 w (v_o - t_o) and *loss = sum_o w |v_o - t_o|^2
// (w = weights[o mod np], or 1) over nv complex values, in a fixed order.
void objective_terms(const double* values, const double* target, const double* weights, i64 nv, int np,
                     double* cot, double* loss, cudaStream_t s);
// mv [K][B][2]: the scales of the mean (plan entry i_mean) and variance
// (i_var) cotangents of every map
void build_mean_var(const double* cot, int np, int B, int K, const double* counts, int levels, int i_mean, int i_var,
                    double* mv, cudaStream_t s);

// Per-row constants (kernels.cu): out[r] = mean over the N pixels of row r
// of a pixel-major [N][R] field (complex_moduli: the moduli of a complex
// field) or of a map-major [R][N] field; partials: kMeansBlocks x R doubles.
constexpr int kMeansBlocks = 2048;
template <typename T>
void row_means(const T* f, bool complex_moduli, bool pixel_major, i64 N, int R, double* partials, double* out,
               cudaStream_t s);
// mod[p mod_pix + b mod_row + mod_off + l] = |z[p][b][l]| - cz[b][l]
template <typename T>
void moduli_deviations(const T* z, i64 N, int B, int L, const double* cz, T* mod, int mod_pix, int mod_row,
                       int mod_off, cudaStream_t s);
// rc[(b, d, l)] = zc[d][b][l] for the branch rows of level n
void branch_constants(const double* zc, int n, int B, int L, double* rc, cudaStream_t s);
template <typename Tin, typename Tout>
void convert(const Tin* in, Tout* out, i64 n, cudaStream_t s);
// [B][N] map-major <-> [N][B] pixel-major (minus sub[b] / plus add[b] in
// FP64); res (or null): the rounding residual of each output, in Tout
template <typename Tin, typename Tout>
void to_pixel_major(const Tin* in, Tout* out, i64 N, int B, cudaStream_t s, const double* sub = nullptr,
                    Tout* res = nullptr);
// FP64 values as FP32 pairs (hi rounded, lo the rounded rest) and back
void split_f64(const double* x, float* hi, float* lo, i64 n, cudaStream_t s);
void join_f64(const float* hi, const float* lo, double* x, i64 n, cudaStream_t s);
template <typename Tin, typename Tout>
void to_map_major(const Tin* in, Tout* out, i64 N, int B, cudaStream_t s, const double* add = nullptr);

}  // namespace stl
