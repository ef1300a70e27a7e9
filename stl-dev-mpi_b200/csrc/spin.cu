// Spin-2 front end on the device: operators (built in FP64, one warp per
// stored row), their application and adjoint, the transported pyramid, the
// cross pairs and the eroded masks.  Counterpart of the reference's
// crates/stl-core/src/spin.rs with its bridge glue
// (crates/stl-bridge/src/lib.rs:139-240, 396-454, 474-640).
//
// Stored rows.  Only the rows of faces 0, 4 and 8 are built (index u in
// [0, 3 nside^2): face 4 (u >> 2 order) and the NESTED bits of u); the row
// of the pixel turned by k quarter turns about the pole reads the turned
// cells with the same weights.  Weights are entry-major ([entry][u]) so the
// threads of a warp, eight rows times four turns, read one line per entry.
// The transpose (adjoint) holds, for every column of faces 0, 4, 8, the
// (row, conj w) entries of all full-sky rows reading it, ascending by row.
//
// Arithmetic.  This file is compiled with --fmad=false and the weights are
// computed in the operation order of spin.rs (binary powering for x^n,
// sequential sums), so the only differences from a host build are CUDA's
// sin, cos, exp and atan2 against the host's libm, within a few ulps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.cuh"
#include "healpix.cuh"
#include "spin.hpp"

namespace stl {
namespace {

constexpr int kSpinCells = 96;   // most cells one stencil row may read
constexpr int kBuildWarps = 4;   // stored rows per build block
constexpr int kApplyThreads = 256;

inline unsigned blocks_of(i64 n, int t) { return (unsigned)((n + t - 1) / t); }
void check_launch() { STL_CUDA(cudaGetLastError()); }

__host__ __device__ inline int order_bits(i64 nside) {
  int o = 0;
  while ((i64(1) << o) < nside) ++o;
  return o;
}
// pixel of turn k of stored row u (faces 4 (u >> o2) + k)
__device__ __forceinline__ i64 turn_pixel(i64 u, int k, int o2) {
  return ((4 * (u >> o2) + k) << o2) | (u & ((i64(1) << o2) - 1));
}
// pixel c turned by k quarter turns (its face within the same ring of faces)
__device__ __forceinline__ i64 turn_cell(i64 c, int k, int o2) {
  const i64 f = c >> o2;
  return (((f & ~i64(3)) | ((f + k) & 3)) << o2) | (c & ((i64(1) << o2) - 1));
}
// stored row of a pixel of faces 0, 4, 8
__device__ __forceinline__ i64 stored_index(i64 c, int o2) {
  return ((c >> o2) >> 2 << o2) | (c & ((i64(1) << o2) - 1));
}

// x^b by binary powering (the lowering of Rust's powi for a run-time exponent)
__device__ double powi_d(double a, int b) {
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
__device__ void frame_d(i64 pix, i64 nside, double c[3], double et[3], double ep[3]) {
  double t, p;
  pix2ang_nest(pix, nside, t, p);
  const double st = sin(t), ct = cos(t), sp = sin(p), cp = cos(p);
  c[0] = st * cp; c[1] = st * sp; c[2] = ct;
  et[0] = ct * cp; et[1] = ct * sp; et[2] = -st;
  ep[0] = -sp; ep[1] = cp; ep[2] = 0.0;
}
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
// angle in the frame of m of the tangent vector v at a carried along the
// geodesic to the centre of m (spin.rs:55-74)
__device__ double transported_angle_d(const double a[3], const double v[3], i64 m, i64 nside) {
  double b[3], et[3], ep[3], axis[3], w[3];
  frame_d(m, nside, b, et, ep);
  cross3(a, b, axis);
  const double s = sqrt(dot3(axis, axis));
  const double c = dot3(a, b);
  if (s < 1e-15) {
    w[0] = v[0]; w[1] = v[1]; w[2] = v[2];
  } else {
    const double k[3] = {axis[0] / s, axis[1] / s, axis[2] / s};
    double kv[3];
    cross3(k, v, kv);
    const double kd = dot3(k, v);
    for (int i = 0; i < 3; ++i) w[i] = v[i] * c + kv[i] * s + k[i] * kd * (1.0 - c);
  }
  return atan2(dot3(w, ep), dot3(w, et));
}
// e^{-2 i psi} times (re, im)
__device__ __forceinline__ double2 turn_by(double re, double im, double psi) {
  const double cr = cos(-2.0 * psi), ci = sin(-2.0 * psi);
  return make_double2(re * cr - im * ci, re * ci + im * cr);
}

// monomial i of the order of spin.rs:214-231 (by total degree t, then a
// descending): x^a y^b
__device__ __forceinline__ void monomial(int i, int& a, int& b) {
  int t = 0;
  while ((t + 1) * (t + 2) / 2 <= i) ++t;
  const int j = i - t * (t + 1) / 2;
  a = t - j;
  b = j;
}

// shared memory of one build warp, in doubles: the Gram matrix (rounded to
// even), the complex solution, x, y and the weights of the cells, the cells
__host__ __device__ inline size_t build_warp_doubles(int kmax) {
  return (size_t)((kmax * kmax + 1) & ~1) + 2 * kmax + 4 * kSpinCells;
}

struct BuildArgs {
  i64 nside;
  int order, rings, width, kmax;  // kmax: monomials at degree 2 rings
  i64 rows;                       // stored rows 3 nside^2
  int* col;                       // [width][rows] cells (-1: none)
  double2* w;                     // [width][rows]
  int* err;                       // 1: too many cells, 2: singular at degree 2 (and the row in err[1])
};

// One warp per stored row: the cells, their gnomonic coordinates and Gaussian
// weights, the Gram matrix of the monomials, its Cholesky solve against the
// monomials' images, the least-norm weights and the transport rotation
// (spin.rs:276-338).
__global__ void k_spin_rows(BuildArgs a) {
  extern __shared__ double sm_spin[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const i64 u = (i64)blockIdx.x * kBuildWarps + warp;
  if (u >= a.rows) return;  // whole warps leave together
  const int K2 = (a.kmax * a.kmax + 1) & ~1;  // even: the complex solution after it stays 16-byte aligned
  double* base = sm_spin + (size_t)warp * build_warp_doubles(a.kmax);
  double* G = base;
  double2* l = reinterpret_cast<double2*>(G + K2);
  double* px = reinterpret_cast<double*>(l + a.kmax);
  double* py = px + kSpinCells;
  double* wt = py + kSpinCells;
  i64* cells = reinterpret_cast<i64*>(wt + kSpinCells);
  __shared__ int s_count[kBuildWarps], s_fail[kBuildWarps];

  const int o2 = 2 * a.order;
  const i64 p = turn_pixel(u, 0, o2);
  const i64 nside = a.nside;
  if (lane == 0) {
    int M = 0;
    bool over = false;
    if ((i64)a.rings < nside) {
      // the cells within `rings` rings: the (2 rings + 1)^2 box of the face
      // frame, ascending and unique (the set of cdshealpix kth_neighbourhood)
      i64 ix, iy, f;
      nest2xyf(p, a.order, ix, iy, f);
      for (int dy = -a.rings; dy <= a.rings; ++dy)
        for (int dx = -a.rings; dx <= a.rings; ++dx) {
          i64 q;
          if (!ext_pix(f, ix + dx, iy + dy, nside, a.order, q)) continue;
          int at = M;
          while (at > 0 && cells[at - 1] > q) --at;
          if (at > 0 && cells[at - 1] == q) continue;
          if (M == kSpinCells) { over = true; continue; }
          for (int m = M; m > at; --m) cells[m] = cells[m - 1];
          cells[at] = q;
          ++M;
        }
    } else {
      // a level smaller than the stencil: every pixel within (rings + 1) h
      // (at most 1.2 rad) of the centre
      double c[3], et[3], ep[3];
      frame_d(p, nside, c, et, ep);
      const double h = sqrt(4.0 * kPi / (double)npix_of(nside));
      const double cut = cos(fmin(((double)a.rings + 1.0) * h, 1.2));
      for (i64 m = 0; m < npix_of(nside); ++m) {
        double v[3], e1[3], e2[3];
        frame_d(m, nside, v, e1, e2);
        if (dot3(v, c) >= cut) {
          if (M == kSpinCells) { over = true; break; }
          cells[M++] = m;
        }
      }
    }
    if (over || M > a.width) atomicExch(a.err, 1);
    s_count[warp] = over ? 0 : min(M, a.width);
    s_fail[warp] = 0;
  }
  __syncwarp();
  const int M = s_count[warp];
  double c[3], et[3], ep[3];
  frame_d(p, nside, c, et, ep);
  const double h = sqrt(4.0 * kPi / (double)npix_of(nside));
  const double r2 = (double)(a.rings * a.rings);
  for (int m = lane; m < M; m += 32) {
    double v[3], e1[3], e2[3];
    frame_d(cells[m], nside, v, e1, e2);
    const double z = dot3(v, c);
    px[m] = dot3(v, et) / z / h;
    py[m] = dot3(v, ep) / z / h;
    wt[m] = exp(-(px[m] * px[m] + py[m] * py[m]) / r2);
  }
  __syncwarp();
  int degree = 2 * a.rings;
  bool solved = false;
  while (M > 0) {
    const int K = (degree + 1) * (degree + 2) / 2;
    // Gram matrix sum_m (A_im w_m) A_jm, lower triangle, mirrored
    for (int e = lane; e < K * (K + 1) / 2; e += 32) {
      int i = 0;
      while ((i + 1) * (i + 2) / 2 <= e) ++i;
      const int j = e - i * (i + 1) / 2;
      int ai, bi, aj, bj;
      monomial(i, ai, bi);
      monomial(j, aj, bj);
      double v = 0.0;
      for (int m = 0; m < M; ++m) {
        const double Ai = powi_d(px[m], ai) * powi_d(py[m], bi);
        const double Aj = powi_d(px[m], aj) * powi_d(py[m], bj);
        v += Ai * wt[m] * Aj;
      }
      G[i * K + j] = v;
      G[j * K + i] = v;
    }
    __syncwarp();
    // Cholesky, column by column: the pivot on lane 0, the column's rows
    // across the lanes (spin.rs:235-253)
    bool ok = true;
    for (int j = 0; j < K && ok; ++j) {
      if (lane == 0) {
        double d = G[j * K + j];
        for (int k = 0; k < j; ++k) d -= G[j * K + k] * G[j * K + k];
        if (d <= 1e-12 * fmax(fabs(G[j * K + j]), 1e-300)) {
          s_fail[warp] = 1;
        } else {
          G[j * K + j] = sqrt(d);
        }
      }
      __syncwarp();
      ok = s_fail[warp] == 0;
      if (ok)
        for (int i = j + 1 + lane; i < K; i += 32) {
          double v = G[i * K + j];
          for (int k = 0; k < j; ++k) v -= G[i * K + k] * G[j * K + k];
          G[i * K + j] = v / G[j * K + j];
        }
      __syncwarp();
    }
    if (ok) {
      if (lane == 0) {  // the two triangular solves (spin.rs:254-271)
        for (int i = 0; i < K; ++i) {
          int ai, bi;
          monomial(i, ai, bi);
          double re = 0.0, im = 0.0;
          if (ai == 2 && bi == 0) re = -2.0;
          else if (ai == 0 && bi == 2) re = 2.0;
          else if (ai == 1 && bi == 1) im = 2.0;
          l[i] = make_double2(re, im);
        }
        for (int i = 0; i < K; ++i) {
          double2 y = l[i];
          for (int k = 0; k < i; ++k) {
            y.x -= l[k].x * G[i * K + k];
            y.y -= l[k].y * G[i * K + k];
          }
          l[i] = make_double2(y.x / G[i * K + i], y.y / G[i * K + i]);
        }
        for (int i = K - 1; i >= 0; --i) {
          double2 y = l[i];
          for (int k = i + 1; k < K; ++k) {
            y.x -= l[k].x * G[k * K + i];
            y.y -= l[k].y * G[k * K + i];
          }
          l[i] = make_double2(y.x / G[i * K + i], y.y / G[i * K + i]);
        }
      }
      __syncwarp();
      // the weights of the cells, turned into the centre's frame
      for (int m = lane; m < M; m += 32) {
        double sre = 0.0, sim = 0.0;
        for (int i = 0; i < K; ++i) {
          int ai, bi;
          monomial(i, ai, bi);
          const double A = powi_d(px[m], ai) * powi_d(py[m], bi);
          sre += l[i].x * A;
          sim += l[i].y * A;
        }
        sre *= wt[m];
        sim *= wt[m];
        const double psi = transported_angle_d(c, et, cells[m], nside);
        a.col[(size_t)m * a.rows + u] = (int)cells[m];
        a.w[(size_t)m * a.rows + u] = turn_by(sre, sim, psi);
      }
      solved = true;
      break;
    }
    if (degree <= 2) break;
    degree = 2;
    if (lane == 0) s_fail[warp] = 0;
    __syncwarp();
  }
  for (int m = M + lane; m < a.width; m += 32) {
    a.col[(size_t)m * a.rows + u] = -1;
    a.w[(size_t)m * a.rows + u] = make_double2(0.0, 0.0);
  }
  if (!solved && lane == 0 && M > 0) {
    if (atomicCAS(a.err, 0, 2) == 0) a.err[1] = (int)p;
  }
}

// the transported mean of the four children of every stored coarse row u
// (spin.rs:193-210): 0.25 e^{-2 i psi}, psi the angle of the parent's
// e_theta carried to the child
__global__ void k_spin_down_rows(i64 nside_c, int order_c, i64 rows, int* col, double2* w) {
  const i64 u = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= rows) return;
  const i64 p = turn_pixel(u, 0, 2 * order_c);
  double c[3], et[3], ep[3];
  frame_d(p, nside_c, c, et, ep);
  for (int k = 0; k < 4; ++k) {
    const i64 child = 4 * p + k;
    const double psi = transported_angle_d(c, et, child, 2 * nside_c);
    const double cr = cos(-2.0 * psi), ci = sin(-2.0 * psi);
    col[(size_t)k * rows + u] = (int)child;
    w[(size_t)k * rows + u] = make_double2(0.25 * cr, 0.25 * ci);
  }
}

// entries of every turned row into the stored columns they read: counts
__global__ void k_spin_tcount(const int* __restrict__ col, i64 rows, int width, int o2,
                              unsigned long long* __restrict__ count) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 u = t >> 2;
  const int k = (int)(t & 3);
  if (u >= rows) return;
  for (int e = 0; e < width; ++e) {
    const int c0 = col[(size_t)e * rows + u];
    if (c0 < 0) break;
    const i64 c = turn_cell(c0, k, o2);
    if (((c >> o2) & 3) == 0) atomicAdd(count + stored_index(c, o2), 1ull);
  }
}
__global__ void k_spin_tfill(const int* __restrict__ col, const double2* __restrict__ w, i64 rows, int width,
                             int o2, unsigned long long* __restrict__ cursor, int* __restrict__ trow,
                             double2* __restrict__ tw) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 u = t >> 2;
  const int k = (int)(t & 3);
  if (u >= rows) return;
  const i64 r = turn_pixel(u, k, o2);
  for (int e = 0; e < width; ++e) {
    const int c0 = col[(size_t)e * rows + u];
    if (c0 < 0) break;
    const i64 c = turn_cell(c0, k, o2);
    if (((c >> o2) & 3) != 0) continue;
    const unsigned long long slot = atomicAdd(cursor + stored_index(c, o2), 1ull);
    const double2 v = w[(size_t)e * rows + u];
    trow[slot] = (int)r;
    tw[slot] = make_double2(v.x, -v.y);
  }
}
// every column's entries ascending by row (insertion sort: tens of entries)
__global__ void k_spin_tsort(const i64* __restrict__ tptr, i64 cols, int* __restrict__ trow,
                             double2* __restrict__ tw) {
  const i64 cu = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (cu >= cols) return;
  const i64 a = tptr[cu], b = tptr[cu + 1];
  for (i64 i = a + 1; i < b; ++i) {
    const int r = trow[i];
    const double2 v = tw[i];
    i64 j = i;
    while (j > a && trow[j - 1] > r) {
      trow[j] = trow[j - 1];
      tw[j] = tw[j - 1];
      --j;
    }
    trow[j] = r;
    tw[j] = v;
  }
}

// Field addressing: element p of component q (0: real part, 1: imaginary
// part) of map r at base + r map + q comp + p.
struct FieldRef {
  const double* base;
  i64 map, comp;
};
struct FieldOut {
  double* base;
  i64 map, comp;
};

// y = A x (rows stored per turn), maps [r0, r0 + RB) of R; accumulate: y +=
template <int RB>
__global__ void __launch_bounds__(kApplyThreads) k_spin_apply(const int* __restrict__ col,
                                                              const double2* __restrict__ w, i64 rows, int width,
                                                              int o2_out, int o2_in, FieldRef x, FieldOut y, int R,
                                                              bool accumulate) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 u = t >> 2;
  const int k = (int)(t & 3);
  if (u >= rows) return;
  const i64 p = turn_pixel(u, k, o2_out);
  for (int r0 = 0; r0 < R; r0 += RB) {
    double are[RB], aim[RB];
#pragma unroll
    for (int j = 0; j < RB; ++j) are[j] = aim[j] = 0.0;
    for (int e = 0; e < width; ++e) {
      const int c0 = col[(size_t)e * rows + u];
      if (c0 < 0) break;
      const i64 c = turn_cell(c0, k, o2_in);
      const double2 v = w[(size_t)e * rows + u];
#pragma unroll
      for (int j = 0; j < RB; ++j)
        if (r0 + j < R) {
          const double* xm = x.base + (i64)(r0 + j) * x.map + c;
          const double q = xm[0], uu = xm[x.comp];
          are[j] += v.x * q - v.y * uu;
          aim[j] += v.x * uu + v.y * q;
        }
    }
#pragma unroll
    for (int j = 0; j < RB; ++j)
      if (r0 + j < R) {
        double* ym = y.base + (i64)(r0 + j) * y.map + p;
        if (accumulate) {
          ym[0] += are[j];
          ym[y.comp] += aim[j];
        } else {
          ym[0] = are[j];
          ym[y.comp] = aim[j];
        }
      }
  }
}

// x = A^T g over the transposed entries of the stored columns
template <int RB>
__global__ void __launch_bounds__(kApplyThreads) k_spin_adjoint(const i64* __restrict__ tptr,
                                                                const int* __restrict__ trow,
                                                                const double2* __restrict__ tw, i64 cols, int o2_in,
                                                                int o2_out, FieldRef g, FieldOut x, int R,
                                                                bool accumulate) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 cu = t >> 2;
  const int k = (int)(t & 3);
  if (cu >= cols) return;
  const i64 c = turn_pixel(cu, k, o2_in);
  const i64 a = tptr[cu], b = tptr[cu + 1];
  for (int r0 = 0; r0 < R; r0 += RB) {
    double are[RB], aim[RB];
#pragma unroll
    for (int j = 0; j < RB; ++j) are[j] = aim[j] = 0.0;
    for (i64 e = a; e < b; ++e) {
      const i64 r = turn_cell(trow[e], k, o2_out);
      const double2 v = tw[e];
#pragma unroll
      for (int j = 0; j < RB; ++j)
        if (r0 + j < R) {
          const double* gm = g.base + (i64)(r0 + j) * g.map + r;
          const double q = gm[0], uu = gm[g.comp];
          are[j] += v.x * q - v.y * uu;
          aim[j] += v.x * uu + v.y * q;
        }
    }
#pragma unroll
    for (int j = 0; j < RB; ++j)
      if (r0 + j < R) {
        double* xm = x.base + (i64)(r0 + j) * x.map + c;
        if (accumulate) {
          xm[0] += are[j];
          xm[x.comp] += aim[j];
        } else {
          xm[0] = are[j];
          xm[x.comp] = aim[j];
        }
      }
  }
}

// x (fine) += D^T g (coarse): every fine pixel reads its parent only
__global__ void k_spin_down_adjoint(const double2* __restrict__ w, i64 rows_c, int o2_c, FieldRef g, FieldOut x,
                                    int R, i64 n_fine, bool accumulate) {
  const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_fine) return;
  const i64 P = c >> 2;
  const int j = (int)(c & 3);
  const i64 f = P >> o2_c;
  const i64 uP = ((f >> 2) << o2_c) | (P & ((i64(1) << o2_c) - 1));
  const double2 v = w[(size_t)j * rows_c + uP];  // conj(v) g
  for (int r = 0; r < R; ++r) {
    const double* gm = g.base + (i64)r * g.map + P;
    const double q = gm[0], uu = gm[g.comp];
    const double re = v.x * q + v.y * uu, im = v.x * uu - v.y * q;
    double* xm = x.base + (i64)r * x.map + c;
    if (accumulate) {
      xm[0] += re;
      xm[x.comp] += im;
    } else {
      xm[0] = re;
      xm[x.comp] = im;
    }
  }
}

// rows whose stencil reads valid data only (spin.rs:415-432); turned rows
__global__ void k_spin_valid(const int* __restrict__ col, i64 rows, int width, int o2,
                             const uint8_t* __restrict__ data, uint8_t* __restrict__ valid) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 u = t >> 2;
  const int k = (int)(t & 3);
  if (u >= rows) return;
  uint8_t ok = 1;
  for (int e = 0; e < width && ok; ++e) {
    const int c0 = col[(size_t)e * rows + u];
    if (c0 < 0) break;
    ok = data[turn_cell(c0, k, o2)];
  }
  valid[turn_pixel(u, k, o2)] = ok;
}

__global__ void k_nonfinite(const void* x, i64 n, bool f32, unsigned long long* bad) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = f32 ? (double)static_cast<const float*>(x)[i] : static_cast<const double*>(x)[i];
  if (!isfinite(v)) atomicAdd(bad, 1ull);
}
__global__ void k_to_f64(const void* x, i64 n, bool f32, double* y) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = f32 ? (double)static_cast<const float*>(x)[i] : static_cast<const double*>(x)[i];
}
__global__ void k_from_f64(const double* x, i64 n, bool f32, void* y) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (f32) static_cast<float*>(y)[i] = (float)x[i];
  else static_cast<double*>(y)[i] = x[i];
}
// cross with a scalar first field: T of pair i into channel 0 of both rows
// (maps [2B][2][n]: row 2 i + k, channel 0); its cotangent the sum of both
__global__ void k_copy_t(const double* t, i64 n, int B, double* maps) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (i64)B * n) return;
  const i64 b = i / n, p = i % n;
  maps[(2 * b) * 2 * n + p] = t[i];
  maps[(2 * b + 1) * 2 * n + p] = t[i];
}
__global__ void k_sum_t(const double* g, i64 n, int B, double* gt) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (i64)B * n) return;
  const i64 b = i / n, p = i % n;
  gt[i] = g[(2 * b) * 2 * n + p] + g[(2 * b + 1) * 2 * n + p];
}

// ---------------------------------------------------------------------------
// one operator: a level's stencil (rows and columns of that level) or the
// transported means (rows: coarse pixels, columns: the level below)
struct SpinOp {
  i64 nside_out = 0, nside_in = 0;
  int o2_out = 0, o2_in = 0, width = 0;
  i64 rows = 0, cols = 0;  // stored rows and stored columns (3 nside^2 each)
  DevMem col, w, tptr, trow, tw;
  size_t bytes() const { return col.bytes + w.bytes + tptr.bytes + trow.bytes + tw.bytes; }
};

int monomials_of(int degree) { return (degree + 1) * (degree + 2) / 2; }

void build_eth(SpinOp& op, i64 nside, int kernel, cudaStream_t s, DevMem& err) {
  const int rings = kernel / 2;
  const int order = order_bits(nside);
  op.nside_out = op.nside_in = nside;
  op.o2_out = op.o2_in = 2 * order;
  op.rows = op.cols = 3 * nside * nside;
  const i64 npix = 12 * nside * nside;
  op.width = (i64)rings < nside ? (2 * rings + 1) * (2 * rings + 1) : (int)std::min<i64>(npix, kSpinCells);
  op.col.alloc(sizeof(int) * op.width * op.rows);
  op.w.alloc(sizeof(double2) * op.width * op.rows);
  BuildArgs a;
  a.nside = nside;
  a.order = order;
  a.rings = rings;
  a.width = op.width;
  a.kmax = monomials_of(2 * rings);
  a.rows = op.rows;
  a.col = op.col.as<int>();
  a.w = op.w.as<double2>();
  a.err = err.as<int>();
  const size_t smem = sizeof(double) * kBuildWarps * build_warp_doubles(a.kmax);
  allow_dynamic_smem(k_spin_rows);
  k_spin_rows<<<blocks_of(op.rows, kBuildWarps), 32 * kBuildWarps, smem, s>>>(a);
  check_launch();
  int e[2] = {0, 0};
  STL_CUDA(cudaMemcpyAsync(e, err.p, sizeof(e), cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  if (e[0] == 1) throw std::runtime_error("spin stencil: more cells than a row holds");
  if (e[0] == 2)
    throw std::runtime_error("spin stencil: singular system at pixel " + std::to_string(e[1]) + " of nside " +
                             std::to_string(nside));
  // the transpose: counts, offsets (host scan of the stored columns), fill, sort
  DevMem cnt(sizeof(unsigned long long) * (op.cols + 1));
  STL_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
  k_spin_tcount<<<blocks_of(4 * op.rows, 256), 256, 0, s>>>(op.col.as<int>(), op.rows, op.width, op.o2_out,
                                                             cnt.as<unsigned long long>());
  check_launch();
  std::vector<unsigned long long> h((size_t)op.cols + 1);
  STL_CUDA(cudaMemcpyAsync(h.data(), cnt.p, sizeof(unsigned long long) * op.cols, cudaMemcpyDeviceToHost, s));
  STL_CUDA(cudaStreamSynchronize(s));
  std::vector<i64> ptr((size_t)op.cols + 1);
  ptr[0] = 0;
  for (i64 i = 0; i < op.cols; ++i) ptr[i + 1] = ptr[i] + (i64)h[i];
  const i64 nnz = ptr[op.cols];
  op.tptr.alloc(sizeof(i64) * (op.cols + 1));
  op.trow.alloc(sizeof(int) * std::max<i64>(nnz, 1));
  op.tw.alloc(sizeof(double2) * std::max<i64>(nnz, 1));
  STL_CUDA(cudaMemcpyAsync(op.tptr.p, ptr.data(), sizeof(i64) * (op.cols + 1), cudaMemcpyHostToDevice, s));
  STL_CUDA(cudaMemcpyAsync(cnt.p, ptr.data(), sizeof(i64) * op.cols, cudaMemcpyHostToDevice, s));
  k_spin_tfill<<<blocks_of(4 * op.rows, 256), 256, 0, s>>>(op.col.as<int>(), op.w.as<double2>(), op.rows, op.width,
                                                            op.o2_out, cnt.as<unsigned long long>(),
                                                            op.trow.as<int>(), op.tw.as<double2>());
  check_launch();
  k_spin_tsort<<<blocks_of(op.cols, 256), 256, 0, s>>>(op.tptr.as<i64>(), op.cols, op.trow.as<int>(),
                                                        op.tw.as<double2>());
  check_launch();
  STL_CUDA(cudaStreamSynchronize(s));
}

void build_down(SpinOp& op, i64 nside_fine, cudaStream_t s) {
  const i64 nc = nside_fine / 2;
  op.nside_out = nc;
  op.nside_in = nside_fine;
  op.o2_out = 2 * order_bits(nc);
  op.o2_in = 2 * order_bits(nside_fine);
  op.rows = 3 * nc * nc;
  op.cols = 3 * nside_fine * nside_fine;
  op.width = 4;
  op.col.alloc(sizeof(int) * 4 * op.rows);
  op.w.alloc(sizeof(double2) * 4 * op.rows);
  k_spin_down_rows<<<blocks_of(op.rows, 128), 128, 0, s>>>(nc, order_bits(nc), op.rows, op.col.as<int>(),
                                                            op.w.as<double2>());
  check_launch();
}

void apply(const SpinOp& op, FieldRef x, FieldOut y, int R, bool accumulate, cudaStream_t s) {
  if (R <= 0) return;
  k_spin_apply<4><<<blocks_of(4 * op.rows, kApplyThreads), kApplyThreads, 0, s>>>(
      op.col.as<int>(), op.w.as<double2>(), op.rows, op.width, op.o2_out, op.o2_in, x, y, R, accumulate);
  check_launch();
}
void adjoint(const SpinOp& op, bool is_down, FieldRef g, FieldOut x, int R, bool accumulate, cudaStream_t s) {
  if (R <= 0) return;
  if (is_down) {
    const i64 n_fine = 12 * op.nside_in * op.nside_in;
    k_spin_down_adjoint<<<blocks_of(n_fine, 256), 256, 0, s>>>(op.w.as<double2>(), op.rows, op.o2_out, g, x, R,
                                                                n_fine, accumulate);
  } else {
    k_spin_adjoint<4><<<blocks_of(4 * op.cols, kApplyThreads), kApplyThreads, 0, s>>>(
        op.tptr.as<i64>(), op.trow.as<int>(), op.tw.as<double2>(), op.cols, op.o2_in, op.o2_out, g, x, R,
        accumulate);
  }
  check_launch();
}

// ---------------------------------------------------------------------------
class SpinFrontImpl final : public SpinFront {
 public:
  SpinFrontImpl(const SpinConfig& c, cudaStream_t s) : s_(s) {
    cfg_ = c;
    if (c.kernel != 3 && c.kernel != 5 && c.kernel != 7 && c.kernel != 9)
      throw std::runtime_error("spin_kernel must be 3, 5, 7 or 9");
    if (c.cross && c.transported) throw std::runtime_error("spin 2: cross statistics need the scalar pyramid");
    if (c.spin_a != 0 && c.spin_a != 2) throw std::runtime_error("spin_a must be 0 or 2");
    const int nl = c.transported ? c.levels : 1;
    if ((c.nside >> (nl - 1)) < 1) throw std::runtime_error("too many levels for nside");
  }

  // the operators, on the device, at the first use (as the engine's)
  void prepare() override {
    if (built_) return;
    const int nl = cfg_.transported ? cfg_.levels : 1;
    err_.alloc(2 * sizeof(int));
    STL_CUDA(cudaMemsetAsync(err_.p, 0, err_.bytes, s_));
    eth_.resize(nl);
    for (int j = 0; j < nl; ++j) build_eth(eth_[j], cfg_.nside >> j, cfg_.kernel, s_, err_);
    down_.resize(nl - 1);
    for (int j = 0; j + 1 < nl; ++j) build_down(down_[j], cfg_.nside >> j, s_);
    bad_.alloc(sizeof(unsigned long long));
    STL_CUDA(cudaStreamSynchronize(s_));
    built_ = true;
  }

  size_t input_len() const override {
    const size_t n = npix(0), B = cfg_.batch;
    if (cfg_.cross) return B * ((cfg_.spin_a == 2 ? 2 : 1) + 2) * n;
    return B * 2 * n;
  }
  void set_stream(cudaStream_t s) override { s_ = s; }
  size_t bytes() const override {
    size_t b = 0;
    for (const auto& o : eth_) b += o.bytes();
    for (const auto& o : down_) b += o.bytes();
    return b;
  }

  void load_host(Engine& e, const double* x) override {
    prepare();
    const size_t n = input_len();
    in_.alloc_at_least(8 * n);
    // through the engine's pinned staging, the non-finite values counted on the way
    if (e.host_to_device(in_.p, x, 8 * n, true)) throw std::runtime_error("input map contains non-finite values");
    run_forward(e);
  }
  void load_device(Engine& e, const void* x, bool f32) override {
    prepare();
    const size_t n = input_len();
    in_.alloc_at_least(8 * n);
    check_finite(x, n, f32);
    k_to_f64<<<blocks_of((i64)n, 256), 256, 0, s_>>>(x, (i64)n, f32, in_.as<double>());
    check_launch();
    run_forward(e);
  }

  void reverse_host(Engine& e, const double* cot, double* out) override {
    run_reverse(e, cot);
    e.device_to_host(out, gin_.p, 8 * input_len());
  }
  void reverse_device(Engine& e, const double* cot, void* out, bool f32) override {
    run_reverse(e, cot);
    const i64 n = (i64)input_len();
    k_from_f64<<<blocks_of(n, 256), 256, 0, s_>>>(gin_.as<double>(), n, f32, out);
    check_launch();
    STL_CUDA(cudaStreamSynchronize(s_));
  }

  void fields(const double* x, int level, double* qu, double* chi) override {
    prepare();
    if (cfg_.cross) throw std::runtime_error("spin fields of auto handles only");
    if (level < 0 || level >= (int)eth_.size()) throw std::runtime_error("level out of range");
    const size_t n0 = input_len();
    DevMem xin(8 * n0);
    STL_CUDA(cudaMemcpyAsync(xin.p, x, 8 * n0, cudaMemcpyHostToDevice, s_));
    std::vector<DevMem> pol(level + 1);
    const int B = cfg_.batch;
    for (int j = 0; j <= level; ++j) {
      if (j == 0) continue;
      pol[j].alloc(8 * (size_t)B * 2 * npix(j));
      const double* src = j == 1 ? xin.as<double>() : pol[j - 1].as<double>();
      apply(down_[j - 1], FieldRef{src, 2 * npix(j - 1), npix(j - 1)},
            FieldOut{pol[j].as<double>(), 2 * npix(j), npix(j)}, B, false, s_);
    }
    const double* P = level == 0 ? xin.as<double>() : pol[level].as<double>();
    DevMem c(8 * (size_t)B * 2 * npix(level));
    apply(eth_[level], FieldRef{P, 2 * npix(level), npix(level)}, FieldOut{c.as<double>(), 2 * npix(level), npix(level)},
          B, false, s_);
    const size_t nl = (size_t)B * 2 * npix(level);
    STL_CUDA(cudaMemcpyAsync(qu, P, 8 * nl, cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaMemcpyAsync(chi, c.p, 8 * nl, cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaStreamSynchronize(s_));
  }

  std::vector<std::vector<std::vector<uint8_t>>> mask_levels(const double* w, size_t k) override {
    prepare();
    const int levels = cfg_.levels;
    std::vector<std::vector<std::vector<uint8_t>>> out(k);
    DevMem data(npix(0)), valid(npix(0));
    std::vector<uint8_t> h(npix(0));
    for (size_t q = 0; q < k; ++q) {
      for (i64 p = 0; p < npix(0); ++p) {
        const double v = w[q * npix(0) + p];
        if (!std::isfinite(v)) throw std::runtime_error("mask weights must be finite");
        h[p] = v != 0.0;
      }
      std::vector<std::vector<uint8_t>> lv(levels);
      std::vector<uint8_t> cur = h;  // the valid data of the level
      for (int j = 0; j < (int)eth_.size(); ++j) {
        if (j > 0) {  // a parent is valid data when its four children are
          std::vector<uint8_t> up(npix(j));
          for (i64 p = 0; p < npix(j); ++p) up[p] = cur[4 * p] & cur[4 * p + 1] & cur[4 * p + 2] & cur[4 * p + 3];
          cur.swap(up);
        }
        STL_CUDA(cudaMemcpyAsync(data.p, cur.data(), npix(j), cudaMemcpyHostToDevice, s_));
        const SpinOp& op = eth_[j];
        k_spin_valid<<<blocks_of(4 * op.rows, 256), 256, 0, s_>>>(op.col.as<int>(), op.rows, op.width, op.o2_out,
                                                                   data.as<uint8_t>(), valid.as<uint8_t>());
        check_launch();
        lv[j].resize(npix(j));
        STL_CUDA(cudaMemcpyAsync(lv[j].data(), valid.p, npix(j), cudaMemcpyDeviceToHost, s_));
        STL_CUDA(cudaStreamSynchronize(s_));
      }
      if (!cfg_.transported) scalar_pyramid(lv);
      keep_nonempty(lv);
      out[q] = std::move(lv);
    }
    return out;
  }

  void save_input(std::vector<double>& x) override {
    if (!loaded_) throw std::runtime_error("no spin-2 input staged");
    x.resize(input_len());
    STL_CUDA(cudaMemcpyAsync(x.data(), in_.p, 8 * x.size(), cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaStreamSynchronize(s_));
  }

  void export_rows(int level, int kind, std::vector<int64_t>& cells, std::vector<double>& w, int& width) override {
    prepare();
    const SpinOp* op = nullptr;
    if (kind == 0 && level >= 0 && level < (int)eth_.size()) op = &eth_[level];
    if (kind == 1 && level >= 0 && level < (int)down_.size()) op = &down_[level];
    if (!op) throw std::runtime_error("no such spin operator");
    width = op->width;
    std::vector<int> c((size_t)op->width * op->rows);
    std::vector<double> v(2 * (size_t)op->width * op->rows);
    STL_CUDA(cudaMemcpyAsync(c.data(), op->col.p, sizeof(int) * c.size(), cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaMemcpyAsync(v.data(), op->w.p, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaStreamSynchronize(s_));
    const i64 nrows = 12 * op->nside_out * op->nside_out;
    cells.assign((size_t)nrows * width, -1);
    w.assign(2 * (size_t)nrows * width, 0.0);
    const int o2o = op->o2_out, o2i = op->o2_in;
    auto turn = [](i64 x, int k, int o2) {
      const i64 f = x >> o2;
      return (((f & ~i64(3)) | ((f + k) & 3)) << o2) | (x & ((i64(1) << o2) - 1));
    };
    for (i64 u = 0; u < op->rows; ++u)
      for (int k = 0; k < 4; ++k) {
        const i64 p = ((4 * (u >> o2o) + k) << o2o) | (u & ((i64(1) << o2o) - 1));
        for (int e = 0; e < width; ++e) {
          const int c0 = c[(size_t)e * op->rows + u];
          if (c0 < 0) break;
          cells[(size_t)p * width + e] = turn(c0, k, o2i);
          w[2 * ((size_t)p * width + e)] = v[2 * ((size_t)e * op->rows + u)];
          w[2 * ((size_t)p * width + e) + 1] = v[2 * ((size_t)e * op->rows + u) + 1];
        }
      }
  }

 private:
  struct Buffer {
    DevMem m;
    void* p = nullptr;
    void alloc_at_least(size_t b) {
      if (m.bytes < b) m.alloc(b);
      p = m.p;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
  };

  i64 npix(int j) const { return 12 * (cfg_.nside >> j) * (cfg_.nside >> j); }

  void check_finite(const void* x, size_t n, bool f32) {
    STL_CUDA(cudaMemsetAsync(bad_.p, 0, sizeof(unsigned long long), s_));
    k_nonfinite<<<blocks_of((i64)n, 256), 256, 0, s_>>>(x, (i64)n, f32, bad_.as<unsigned long long>());
    check_launch();
    unsigned long long bad = 0;
    STL_CUDA(cudaMemcpyAsync(&bad, bad_.p, sizeof(bad), cudaMemcpyDeviceToHost, s_));
    STL_CUDA(cudaStreamSynchronize(s_));
    if (bad) throw std::runtime_error("input map contains non-finite values");
  }

  // the engine's maps from the staged input in_, then loaded
  void run_forward(Engine& e) {
    const int B = cfg_.batch;
    const i64 n = npix(0);
    if (cfg_.cross) {  // maps [2B][2][n]: row 2 i + k, channel 0 chi_a (or T), channel 1 chi_b
      maps_[0].alloc_at_least(8 * (size_t)2 * B * 2 * n);
      const int pa = cfg_.spin_a == 2 ? 2 : 1;
      const double* a = in_.as<double>();
      const double* b = a + (size_t)B * pa * n;
      double* m = maps_[0].as<double>();
      apply(eth_[0], FieldRef{b, 2 * n, n}, FieldOut{m + n, 4 * n, 2 * n}, B, false, s_);
      if (pa == 2) {
        apply(eth_[0], FieldRef{a, 2 * n, n}, FieldOut{m, 4 * n, 2 * n}, B, false, s_);
      } else {
        k_copy_t<<<blocks_of((i64)B * n, 256), 256, 0, s_>>>(a, n, B, m);
        check_launch();
      }
      e.load_device(m, false);
    } else if (!cfg_.transported) {  // chi of level 0 as maps [2B][n] (= [B][2][n])
      maps_[0].alloc_at_least(8 * (size_t)B * 2 * n);
      apply(eth_[0], FieldRef{in_.as<double>(), 2 * n, n}, FieldOut{maps_[0].as<double>(), 2 * n, n}, B, false, s_);
      e.load_device(maps_[0].as<double>(), false);
    } else {  // P_j and chi_j of every level
      const int L = (int)eth_.size();
      std::vector<const double*> lv(L);
      for (int j = 0; j < L; ++j) {
        const i64 nj = npix(j);
        if (j > 0) {
          pol_[j].alloc_at_least(8 * (size_t)B * 2 * nj);
          const double* src = j == 1 ? in_.as<double>() : pol_[j - 1].as<double>();
          apply(down_[j - 1], FieldRef{src, 2 * npix(j - 1), npix(j - 1)}, FieldOut{pol_[j].as<double>(), 2 * nj, nj},
                B, false, s_);
        }
        maps_[j].alloc_at_least(8 * (size_t)B * 2 * nj);
        const double* P = j == 0 ? in_.as<double>() : pol_[j].as<double>();
        apply(eth_[j], FieldRef{P, 2 * nj, nj}, FieldOut{maps_[j].as<double>(), 2 * nj, nj}, B, false, s_);
        lv[j] = maps_[j].as<double>();
      }
      e.load_device_levels(lv.data());
    }
    loaded_ = true;
  }

  // gin_ = the input cotangent of the engine's reverse sweep for cot
  void run_reverse(Engine& e, const double* cot) {
    const int B = cfg_.batch;
    const i64 n = npix(0);
    gin_.alloc_at_least(8 * input_len());
    if (cfg_.transported) {
      const int L = (int)eth_.size();
      std::vector<double*> lv(L);
      for (int j = 0; j < L; ++j) {
        gmaps_[j].alloc_at_least(8 * (size_t)B * 2 * npix(j));
        lv[j] = gmaps_[j].as<double>();
      }
      e.reverse_levels(cot, lv.data());
      // h_j = eth_j^T g_j + down_j^T h_{j+1}, from the top level down
      for (int j = L - 1; j >= 0; --j) {
        const i64 nj = npix(j);
        if (j > 0) gpol_[j].alloc_at_least(8 * (size_t)B * 2 * nj);
        double* hj = j == 0 ? gin_.as<double>() : gpol_[j].as<double>();
        adjoint(eth_[j], false, FieldRef{lv[j], 2 * nj, nj}, FieldOut{hj, 2 * nj, nj}, B, false, s_);
        if (j + 1 < L)
          adjoint(down_[j], true, FieldRef{gpol_[j + 1].as<double>(), 2 * npix(j + 1), npix(j + 1)},
                  FieldOut{hj, 2 * nj, nj}, B, true, s_);
      }
      return;
    }
    const size_t rows = cfg_.cross ? (size_t)2 * B * 2 : (size_t)2 * B;
    gmaps_[0].alloc_at_least(8 * rows * n);
    e.reverse_device(cot, gmaps_[0].as<double>(), false);
    const double* g = gmaps_[0].as<double>();
    if (!cfg_.cross) {
      adjoint(eth_[0], false, FieldRef{g, 2 * n, n}, FieldOut{gin_.as<double>(), 2 * n, n}, B, false, s_);
      return;
    }
    const int pa = cfg_.spin_a == 2 ? 2 : 1;
    double* ga = gin_.as<double>();
    double* gb = ga + (size_t)B * pa * n;
    adjoint(eth_[0], false, FieldRef{g + n, 4 * n, 2 * n}, FieldOut{gb, 2 * n, n}, B, false, s_);
    if (pa == 2) {
      adjoint(eth_[0], false, FieldRef{g, 4 * n, 2 * n}, FieldOut{ga, 2 * n, n}, B, false, s_);
    } else {
      k_sum_t<<<blocks_of((i64)B * n, 256), 256, 0, s_>>>(g, n, B, ga);
      check_launch();
    }
  }

  // scalar pyramid: a parent is valid unless a bad pixel of the level below
  // lies within the decimation's reach (lib.rs:428-441, local.rs:130-134)
  void scalar_pyramid(std::vector<std::vector<uint8_t>>& lv) const {
    for (int d = 0; d + 1 < (int)lv.size(); ++d) {
      const i64 nside = cfg_.nside >> d;
      const double pix_deg = std::sqrt(4.0 * kPi / (double)npix(d)) * (180.0 / kPi);
      const double radius = 3.0 * pix_deg;
      const int rings = (int)std::ceil(radius / pix_deg) + 1;
      const int order = order_bits(nside);
      std::vector<uint8_t> next(npix(d + 1), (i64)rings >= nside ? 0 : 1);  // a reach over the whole level
      const auto& fine = lv[d];
      for (i64 p = 0; p < npix(d) && (i64)rings < nside; ++p) {
        if (fine[p]) continue;
        i64 ix, iy, f;
        nest2xyf(p, order, ix, iy, f);
        for (int dy = -rings; dy <= rings; ++dy)
          for (int dx = -rings; dx <= rings; ++dx) {
            i64 q;
            if (ext_pix(f, ix + dx, iy + dy, nside, order, q)) next[q >> 2] = 0;
          }
      }
      lv[d + 1] = std::move(next);
    }
  }
  // a level the erosion emptied gets the parents of the level below
  // (lib.rs:447-454)
  static void keep_nonempty(std::vector<std::vector<uint8_t>>& lv) {
    for (size_t d = 1; d < lv.size(); ++d) {
      bool any = false;
      for (uint8_t v : lv[d]) any |= v != 0;
      if (any) continue;
      for (size_t p = 0; p < lv[d].size(); ++p)
        lv[d][p] = lv[d - 1][4 * p] | lv[d - 1][4 * p + 1] | lv[d - 1][4 * p + 2] | lv[d - 1][4 * p + 3];
    }
  }

  cudaStream_t s_;
  std::vector<SpinOp> eth_, down_;
  DevMem err_, bad_;
  Buffer in_, gin_;
  Buffer maps_[32], pol_[32], gmaps_[32], gpol_[32];
  bool loaded_ = false, built_ = false;
};

}  // namespace

std::unique_ptr<SpinFront> SpinFront::create(const SpinConfig& c, cudaStream_t s) {
  if (c.levels > 32) throw std::runtime_error("too many levels");
  return std::make_unique<SpinFrontImpl>(c, s);
}

}  // namespace stl
