// CPU FP64 restatement of the reference's HEALPix geometry and operators.
//
// TEST INFRASTRUCTURE ONLY: this file is the oracle the CUDA engine is
// checked against.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg may load it; the engine never links it.
//
// Each function follows the floating-point operation order of the
// reference file it cites (paths inside jmdelouis/STL-Dev-MPI), so that the
// results agree with the reference's committed fixtures to a few ulps.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>
#include <array>
#include <algorithm>
#include <functional>

namespace orc {

using i64 = int64_t;
using cplx = std::complex<double>;

constexpr double PI = 3.141592653589793115997963468544185161590576171875;  // f64 pi
constexpr double RAD2DEG = 57.295779513082320876798154814105170332405472466564;
constexpr double DEG2RAD = 0.017453292519943295769236907684886127134428718885417;

// -- parallel helper ------------------------------------------------------
int num_threads();
void set_num_threads(int n);
// Runs f(begin, end, worker) over [0, n) split into contiguous chunks, one
// per worker, in parallel.  The split only depends on n and the worker count.
void parallel_chunks(i64 n, const std::function<void(i64, i64, int)>& f);

// -- HEALPix primitives (crates/stl-core/src/healpix.rs) -------------------
inline double rad2deg(double x) { return x * RAD2DEG; }
inline double deg2rad(double x) { return x * DEG2RAD; }
// torch.remainder / Python % (healpix.rs:33-39)
inline double remainder(double a, double b) {
  double m = std::fmod(a, b);
  if (m != 0.0 && ((b < 0.0) != (m < 0.0))) m += b;
  return m;
}
inline i64 floor_div(i64 a, i64 b) {  // Rust div_euclid for b > 0
  i64 q = a / b;
  if ((a % b) < 0) q -= 1;
  return q;
}
inline int order_of(i64 nside) { int o = 0; while ((i64(1) << o) < nside) ++o; return o; }
inline i64 npix(i64 nside) { return 12 * nside * nside; }

void nest2xyf(i64 pix, int order, i64& ix, i64& iy, i64& face);
i64 xyf2nest(i64 ix, i64 iy, i64 face, int order);
void xyf2ang(i64 ix, i64 iy, i64 face, i64 nside, double& theta, double& phi);
void pix2ang_nest(i64 pix, i64 nside, double& theta, double& phi);
void centre_lonlat(i64 pix, i64 nside, double& lon, double& lat);
i64 ring2nest(i64 pix, int order);
void get_interpol_ring(double theta, double phi, i64 nside, i64 pix[4], double w[4]);
void interp_weights_nested(const double v[3], int order, i64 pix[4], double w[4]);

// -- stencil + wavelet (stencil.rs, wavelet.rs) ----------------------------
using Mat3 = std::array<std::array<double, 3>, 3>;
enum class Gauge { Cosmo = 0, Phi = 1 };
std::vector<std::array<double, 3>> local_kernel_grid(int ksz, i64 nside);
std::vector<Mat3> rotation_matrices(double theta, double phi, int G, Gauge gauge);
std::vector<cplx> wavelet_kernel(int ksz, double sigma);
// [C_out = 2, P]: real parts then imaginary parts (wavelet.rs:142-145)
std::vector<double> wavelet_weights(int ksz);
// the kernel cast through f32 (conv.rs:167-172), [G][2][P]
std::vector<double> shared_kernel(const std::vector<double>& weights, int G, int P);

// -- face frames (dia.rs:24-101) -------------------------------------------
bool ext_pix(i64 face, i64 ex, i64 ey, i64 nside, int order, i64& out);
bool rel_offset(i64 row, i64 cell, i64 nside, int order, i64& dx, i64& dy);

// -- neighbourhoods (neighbours.rs) ----------------------------------------
// Sorted set of the cells within k rings of id (k <= nside): the content of
// cdshealpix 0.10.1 kth_neighbourhood, built from the extended face frame.
std::vector<i64> kth_neighbourhood_set(i64 id, i64 nside, int k);
std::vector<i64> parents(const std::vector<i64>& ids);
std::vector<i64> children(const std::vector<i64>& ids);
std::vector<i64> dilate(const std::vector<i64>& ids, i64 nside, int rings);
std::vector<i64> dilate_fine(const std::vector<i64>& ids, i64 nside, int rings);

// -- bound stencils (conv.rs:73-135) ---------------------------------------
// Layout: entry ((k * G + g) * P + p) * 4 + n for output row k, gauge g,
// tap p and bilinear neighbour n.  pos indexes the grid.
struct Bound {
  i64 K = 0, G = 0, P = 0;
  std::vector<int32_t> pos;
  std::vector<double> w;
  std::vector<uint8_t> complete;
};
// Bound stencils of `rows` (NESTED ids) on the sorted grid `grid`; grid
// nullptr (ngrid = npix) means the whole sky (position == id).
void bind_rows(const i64* grid, i64 ngrid, const i64* rows, i64 nrows, i64 nside, int ksz, int G,
               Gauge gauge, double eps, Bound& out, i64 row0 = 0);

// Convolution operator of one level: output rows, input grid, and the
// geometry held whole or rebuilt per chunk of rows at every application.
struct ConvOp {
  std::vector<i64> grid;  // empty: whole sky
  std::vector<i64> rows;  // empty: whole sky (rows == grid)
  i64 nside = 0, n_in = 0, n_rows = 0;
  int ksz = 5, G = 4;
  Gauge gauge = Gauge::Cosmo;
  double eps = 0.0;
  bool cached = false;
  Bound whole;
  void init(std::vector<i64> grid_, std::vector<i64> rows_, i64 nside_, int ksz_, int G_, Gauge gauge_,
            double eps_, size_t cache_budget_bytes);
  // y [R, G*2, n_rows] from x [R, n_in] (conv.rs:253-294); kernel [G][2][P]
  void forward(const std::vector<double>& ker, const double* x, i64 R, double* y,
               const std::vector<i64>* sel = nullptr) const;
  // gx [R, n_in] += adjoint of gy [R, G*2, |sel|] (conv.rs:199-241)
  void adjoint_add(const std::vector<double>& ker, const double* gy, i64 R, double* gx,
                   const std::vector<i64>* sel = nullptr) const;
 private:
  void chunk(i64 k0, i64 k1, const std::vector<i64>* sel, Bound& b) const;
};

// -- smooth decimation (decimation.rs) -------------------------------------
struct Csr {
  i64 n_rows = 0, n_cols = 0;
  std::vector<i64> indptr, indices;
  std::vector<double> values;
  Csr transpose() const;
  void apply(const double* x, double* y) const;  // y = A x, column order
};
// Decimation of the sorted fine grid `ids` at `nside` (whole sky when
// ids is nullptr) to its parents; returns the coarse ids.
std::vector<i64> smooth_decimation(const i64* ids, i64 n, i64 nside, Csr& out);

}  // namespace orc
