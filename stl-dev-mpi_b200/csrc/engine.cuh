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

// Device memory accounting (bytes held by live DevMem allocations).
size_t device_bytes_live();
size_t device_bytes_peak();
void device_bytes_reset_peak();

enum class DType { F64 = 0, F32 = 1 };
inline size_t dsize(DType t) { return t == DType::F64 ? 8 : 4; }

// Geometry of one wavelet operator: output rows reading an input grid.
struct ConvSpec {
  i64 nside = 0;
  int ksz = 5, G = 4, gauge = 0;
  double eps = 0.0;
  const i64* d_grid = nullptr;  // sorted NESTED ids of the grid (device), nullptr: whole sky
  i64 n_in = 0;
  const i64* d_rows = nullptr;  // NESTED ids of the output rows (device), nullptr: rows == grid
  i64 n_rows = 0;
};

struct ConvOp {
  i64 n_rows = 0, n_in = 0;
  int S = 0;        // slots per row
  int ST = 0;       // transposed entries per input cell
  int shift = 0;    // transposed entry = row << shift | slot
  DType dtype = DType::F32;
  DevMem cell;      // int32 [S][n_rows]
  DevMem coef;      // T [S][n_rows][8] (G = 4) or [S][n_rows][2G]
  DevMem tent;      // uint32 [ST][n_in], 0xFFFFFFFF past the end of a cell's list
  int G = 4;
  size_t bytes() const { return cell.bytes + coef.bytes + tent.bytes; }
};

struct DecSpec {
  i64 nside = 0;           // fine level
  const i64* d_ids = nullptr;  // sorted fine grid (device), nullptr: whole sky
  i64 n_in = 0;
  const i64* d_out = nullptr;  // sorted coarse ids = parents of the grid (device), nullptr: whole sky
  i64 n_out = 0;
};

struct DecOp {
  i64 n_out = 0, n_in = 0;
  int W = 0, WT = 0;
  DType dtype = DType::F32;
  DevMem col, w;    // int32 / T [W][n_out]
  DevMem tcol, tw;  // int32 / T [WT][n_in]
  size_t bytes() const { return col.bytes + w.bytes + tcol.bytes + tw.bytes; }
};

// Builders (geometry.cu).  The kernel weights are [G][2][P], f32-rounded.
void build_conv(const ConvSpec& spec, const std::vector<double>& kernel, DType dtype, ConvOp& out,
                cudaStream_t stream);
void build_dec(const DecSpec& spec, DType dtype, DecOp& out, cudaStream_t stream);

// Kernel launchers (kernels.cu).  Rows of every field are planes of
// `plane` elements; complex fields interleave (re, im).
template <typename T>
void conv_forward(const ConvOp& op, const T* x, int R, T* out, i64 out_row_stride, T* mod_out, i64 mod_row_stride,
                  cudaStream_t s);
template <typename T>
void conv_adjoint(const ConvOp& op, const T* gy, i64 gy_row_stride, int R, T* gx, bool accumulate, cudaStream_t s);
// y[ro][ri] = D x[ro][ri] with row (ro, ri) at base + ro * outer + ri * plane
template <typename T>
void dec_apply(const DecOp& op, bool transpose, const T* x, i64 x_outer, T* y, i64 y_outer, int R_outer,
               int R_inner, bool accumulate, cudaStream_t s);
template <typename T>
void modulus_vjp_add(const T* z, const T* g, i64 g_outer, T* gz, int B, i64 plane_elems, cudaStream_t s);

// Coefficient products of one level (see kernels.cu for the slot layout).
struct ProductShape {
  int K = 0;         // operand vector length: (n + 1) L branches + z
  int L = 4;
  int B = 1;
  i64 N = 0;         // pixels of the level
  bool level0 = false;
  int blocks = 0;    // partial sums per (b, l3)
  int slots = 0;     // doubles per partial
};
ProductShape product_shape(int n, int L, int B, i64 N);
template <typename T>
void products_forward(const ProductShape& sh, const T* z, const T* br, const T* x0, double* partials,
                      double* sums, cudaStream_t s);
template <typename T>
void products_reverse(const ProductShape& sh, const T* z, const T* br, const T* M, const T* s1c, T* gz, T* gbr,
                      cudaStream_t s);
template <typename T>
void mean_var_grad(const T* x0, const double* coefs, int B, i64 N, T* gx, cudaStream_t s);
template <typename Tin, typename Tout>
void convert(const Tin* in, Tout* out, i64 n, cudaStream_t s);

}  // namespace stl
