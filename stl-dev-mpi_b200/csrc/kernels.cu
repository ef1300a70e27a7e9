// Compute kernels of the engine's level sweeps (sm_100a).
//
//  conv_forward  y[r, g, :] = sum_s coef[s, p, g] x[r, cell[s, p]]   (+ |y|)
//  conv_adjoint  gx[r, c]   = sum over the (p, s) reading c of coef[s, p] . gy[r, :, p]
//  dec_apply     y = D x or D^T x over ELL rows
//  products      the coefficient sums of one level (FP64) and their VJP
//
// Every reduction has a fixed order (no floating-point atomics): results
// are bit-reproducible run to run.
#include <cstdio>

#include "engine.cuh"

namespace stl {

namespace {

inline unsigned nblocks(i64 n, int t) { return (unsigned)((n + t - 1) / t); }

template <typename T> struct V2;
template <> struct V2<float> { typedef float2 type; };
template <> struct V2<double> { typedef double2 type; };

// 8 coefficients of one (slot, row): float4 x 2 or double2 x 4
__device__ __forceinline__ void load8(const float* p, float w[8]) {
  float4 a = __ldg(reinterpret_cast<const float4*>(p));
  float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w; w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}
__device__ __forceinline__ void load8(const double* p, double w[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double2 a = __ldg(reinterpret_cast<const double2*>(p) + k);
    w[2 * k] = a.x; w[2 * k + 1] = a.y;
  }
}

// One thread per (output row, RB input rows).  out row r, gauge g, pixel p
// at out + r * out_row_stride + (g * n_rows + p) * 2 (complex, interleaved).
template <typename T, int RB>
__global__ void __launch_bounds__(128) k_conv_fwd(const int32_t* __restrict__ cell, const T* __restrict__ coef, int S,
                                                  i64 n_rows, const T* __restrict__ x, i64 n_in, int R,
                                                  T* __restrict__ out, i64 out_row_stride, T* __restrict__ mod_out,
                                                  i64 mod_row_stride) {
  i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_rows) return;
  int r0 = blockIdx.y * RB;
  T acc[RB][8];
#pragma unroll
  for (int rb = 0; rb < RB; ++rb)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[rb][k] = (T)0;
  const T* xr[RB];
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) xr[rb] = x + (i64)min(r0 + rb, R - 1) * n_in;
  for (int s = 0; s < S; ++s) {
    i64 e = (i64)s * n_rows + p;
    int c = __ldg(cell + e);
    T w[8];
    load8(coef + e * 8, w);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      T xv = __ldg(xr[rb] + c);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[rb][k] = fma(w[k], xv, acc[rb][k]);
    }
  }
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    int r = r0 + rb;
    if (r >= R) break;
    typedef typename V2<T>::type T2;
    T2* o = reinterpret_cast<T2*>(out + (i64)r * out_row_stride);
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      T2 v;
      v.x = acc[rb][2 * g];
      v.y = acc[rb][2 * g + 1];
      o[(i64)g * n_rows + p] = v;
      if (mod_out) mod_out[(i64)r * mod_row_stride + (i64)g * n_rows + p] = hypot(v.x, v.y);
    }
  }
}

// One thread per (input cell, RB cotangent rows); gy row r, gauge g, row p
// at gy + r * gy_row_stride + (g * n_rows + p) * 2.
template <typename T, int RB>
__global__ void __launch_bounds__(128) k_conv_adj(const uint32_t* __restrict__ tent, int ST, int shift, i64 n_in,
                                                  const T* __restrict__ coef, i64 n_rows, const T* __restrict__ gy,
                                                  i64 gy_row_stride, int R, T* __restrict__ gx, int accumulate) {
  i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_in) return;
  int r0 = blockIdx.y * RB;
  const uint32_t mask = (1u << shift) - 1u;
  T acc[RB];
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) acc[rb] = (T)0;
  typedef typename V2<T>::type T2;
  const T2* gr[RB];
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) gr[rb] = reinterpret_cast<const T2*>(gy + (i64)min(r0 + rb, R - 1) * gy_row_stride);
  for (int q = 0; q < ST; ++q) {
    uint32_t v = __ldg(tent + (i64)q * n_in + c);
    if (v == 0xFFFFFFFFu) break;
    i64 row = (i64)(v >> shift);
    int s = (int)(v & mask);
    T w[8];
    load8(coef + ((i64)s * n_rows + row) * 8, w);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        T2 gv = gr[rb][(i64)g * n_rows + row];
        acc[rb] = fma(w[2 * g], gv.x, acc[rb]);
        acc[rb] = fma(w[2 * g + 1], gv.y, acc[rb]);
      }
    }
  }
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    int r = r0 + rb;
    if (r >= R) break;
    T* o = gx + (i64)r * n_in + c;
    *o = accumulate ? *o + acc[rb] : acc[rb];
  }
}

// y[ro][ri][c] (+)= sum_k w[k][c] x[ro][ri][col[k][c]]
template <typename T>
__global__ void k_ell(const int32_t* __restrict__ col, const T* __restrict__ w, int W, i64 n_out, i64 n_in,
                      const T* __restrict__ x, i64 x_outer, T* __restrict__ y, i64 y_outer, int accumulate) {
  i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_out) return;
  const T* xr = x + (i64)blockIdx.z * x_outer + (i64)blockIdx.y * n_in;
  T* yr = y + (i64)blockIdx.z * y_outer + (i64)blockIdx.y * n_out;
  T s = (T)0;
  for (int k = 0; k < W; ++k) {
    i64 e = (i64)k * n_out + c;
    s = fma(__ldg(w + e), __ldg(xr + __ldg(col + e)), s);
  }
  yr[c] = accumulate ? yr[c] + s : s;
}

// gz[b][e] += g[b][e] z/|z| (0 at z = 0), e over L * N complex values
template <typename T>
__global__ void k_modvjp(const T* __restrict__ z, const T* __restrict__ g, i64 g_outer, T* __restrict__ gz,
                         i64 plane) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= plane) return;
  i64 b = blockIdx.y;
  i64 zi = (b * plane + e) * 2;
  T zr = z[zi], zm = z[zi + 1];
  T mag = hypot(zr, zm);
  T gv = g[b * g_outer + e];
  T d = mag == (T)0 ? (T)1 : mag;
  gz[zi] += gv * zr / d;
  gz[zi + 1] += gv * zm / d;
}

// ---- coefficient products --------------------------------------------------
//
// Per level n, map b and orientation l3, the operand vector of a pixel is
// v = (branch[d][l1][l3] for d <= n, l1 < L; z[l3]), K = (n + 1) L + 1
// complex values.  Every S3/S4 coefficient of the level is an entry of the
// Hermitian Gram matrix sum_p v v^H (S3: (branch, z); S4: (branch,
// branch)), S2 its (z, z) entry.  A block owns (b, l3) and a set of
// 128-pixel sub-chunks; work items are (Gram entry i <= j, pixel subgroup).
// Sums are FP64 from the FP32 or FP64 operands.  Partial layout per block
// (doubles): [2 E] complex entries (i-major upper triangle), [E] second
// moments sum |v_i|^2 |v_j|^2, then sum |z|, sum |z|^4, and at level 0 (l3 =
// 0 blocks) sum x, sum x^2, sum x^4.
constexpr int kPC = 128;  // pixels per sub-chunk
constexpr int kPT = 256;  // threads of a products block

template <typename T>
__global__ void __launch_bounds__(kPT) k_products(int K, int L, i64 N, int nsub, const T* __restrict__ z,
                                                  const T* __restrict__ br, const T* __restrict__ x0, int Q,
                                                  double* __restrict__ partials, int slots) {
  extern __shared__ __align__(16) unsigned char smem[];
  typedef typename V2<T>::type T2;
  T2* v = reinterpret_cast<T2*>(smem);                                   // [K][kPC]
  double* u = reinterpret_cast<double*>(v + (size_t)K * kPC);           // [K][kPC] |v|^2
  double* red = u + (size_t)K * kPC;                                     // [kPT] scratch
  const int b = blockIdx.z, l3 = blockIdx.y, tid = threadIdx.x;
  const int E = K * (K + 1) / 2;
  const int items = E * Q;
  const int per = kPC / Q;
  const int nb = K - 1;  // branches
  const T2* zr = reinterpret_cast<const T2*>(z) + ((i64)b * L + l3) * N;
  const T2* brb = reinterpret_cast<const T2*>(br) + (i64)b * nb * L * N;
  constexpr int MAXI = 4;
  double acc[MAXI][3];
  int it_i[MAXI], it_j[MAXI], it_q[MAXI];
  int nit = 0;
  for (int it = tid; it < items && nit < MAXI; it += kPT, ++nit) {
    int e = it % E, q = it / E;
    int i = 0, rem = e;
    while (rem >= K - i) { rem -= K - i; ++i; }
    it_i[nit] = i; it_j[nit] = i + rem; it_q[nit] = q;
    acc[nit][0] = acc[nit][1] = acc[nit][2] = 0.0;
  }
  double s_abs = 0.0, s_z4 = 0.0, s_x = 0.0, s_x2 = 0.0, s_x4 = 0.0;
  const bool extra_x = x0 != nullptr && l3 == 0;
  for (int sc = blockIdx.x; sc < nsub; sc += gridDim.x) {
    i64 p0 = (i64)sc * kPC;
    __syncthreads();
    for (int idx = tid; idx < K * kPC; idx += kPT) {
      int i = idx / kPC, px = idx % kPC;
      i64 p = p0 + px;
      T2 a;
      a.x = (T)0; a.y = (T)0;
      if (p < N) a = (i == nb) ? zr[p] : brb[((i64)i * L + l3) * N + p];
      v[idx] = a;
      u[idx] = (double)a.x * (double)a.x + (double)a.y * (double)a.y;
    }
    __syncthreads();
    for (int k = 0; k < nit; ++k) {
      const T2* vi = v + it_i[k] * kPC + it_q[k] * per;
      const T2* vj = v + it_j[k] * kPC + it_q[k] * per;
      const double* ui = u + it_i[k] * kPC + it_q[k] * per;
      const double* uj = u + it_j[k] * kPC + it_q[k] * per;
      double ar = 0.0, ai = 0.0, am = 0.0;
      for (int px = 0; px < per; ++px) {
        double xr = vi[px].x, xi = vi[px].y, yr = vj[px].x, yi = vj[px].y;
        ar = fma(xr, yr, fma(xi, yi, ar));
        ai = fma(xi, yr, fma(-xr, yi, ai));
        am = fma(ui[px], uj[px], am);
      }
      acc[k][0] += ar; acc[k][1] += ai; acc[k][2] += am;
    }
    if (tid < kPC && p0 + tid < N) {
      T2 zz = v[nb * kPC + tid];
      double m = hypot((double)zz.x, (double)zz.y);
      double m2 = m * m;
      s_abs += m;
      s_z4 += m2 * m2;
      if (extra_x) {
        double xv = (double)x0[(i64)b * N + p0 + tid];
        double x2 = xv * xv;
        s_x += xv; s_x2 += x2; s_x4 += x2 * x2;
      }
    }
  }
  __syncthreads();
  double* out = partials + (((i64)b * L + l3) * gridDim.x + blockIdx.x) * slots;
  // Gram entries: subgroup partials through shared memory, summed in q order
  double* gs = reinterpret_cast<double*>(smem);  // reuse: [Q][E][3]
  for (int k = 0; k < nit; ++k) {
    int e = 0;
    for (int r = 0; r < it_i[k]; ++r) e += K - r;
    e += it_j[k] - it_i[k];
    double* d = gs + ((size_t)it_q[k] * E + e) * 3;
    d[0] = acc[k][0]; d[1] = acc[k][1]; d[2] = acc[k][2];
  }
  __syncthreads();
  for (int e = tid; e < E; e += kPT) {
    double r = 0.0, im = 0.0, m = 0.0;
    for (int q = 0; q < Q; ++q) {
      const double* d = gs + ((size_t)q * E + e) * 3;
      r += d[0]; im += d[1]; m += d[2];
    }
    out[2 * e] = r; out[2 * e + 1] = im; out[2 * E + e] = m;
  }
  // per-pixel extras: fixed tree over the block
  double ext[5] = {s_abs, s_z4, s_x, s_x2, s_x4};
  for (int k = 0; k < 5; ++k) {
    __syncthreads();
    red[tid] = ext[k];
    __syncthreads();
    for (int w = kPT / 2; w > 0; w >>= 1) {
      if (tid < w) red[tid] += red[tid + w];
      __syncthreads();
    }
    if (tid == 0) out[3 * E + k] = red[0];
  }
}

// sums[row][slot] = sum over blocks of partials[row][blk][slot] in block order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblk, int slots, double* __restrict__ sums) {
  i64 row = blockIdx.y;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
    double a = 0.0;
    const double* p = partials + row * (i64)nblk * slots + s;
    for (int k = 0; k < nblk; ++k) a += p[(i64)k * slots];
    sums[row * slots + s] = a;
  }
}

// gv = M v per pixel (M: K x K complex of the coefficient cotangents of one
// (b, l3)); gz additionally gets s1c z / |z| (auto S1).
template <typename T>
__global__ void __launch_bounds__(kPC) k_products_rev(int K, int L, i64 N, const T* __restrict__ z,
                                                      const T* __restrict__ br, const T* __restrict__ M,
                                                      const T* __restrict__ s1c, T* __restrict__ gz,
                                                      T* __restrict__ gbr) {
  extern __shared__ __align__(16) unsigned char smem[];
  typedef typename V2<T>::type T2;
  T2* m = reinterpret_cast<T2*>(smem);  // [K][K]
  T2* v = m + (size_t)K * K;            // [K][kPC]
  const int b = blockIdx.z, l3 = blockIdx.y, tid = threadIdx.x;
  const int nb = K - 1;
  const T2* Mb = reinterpret_cast<const T2*>(M) + ((i64)b * L + l3) * K * K;
  for (int i = tid; i < K * K; i += kPC) m[i] = Mb[i];
  i64 p0 = (i64)blockIdx.x * kPC;
  const T2* zr = reinterpret_cast<const T2*>(z) + ((i64)b * L + l3) * N;
  const T2* brb = reinterpret_cast<const T2*>(br) + (i64)b * nb * L * N;
  for (int idx = tid; idx < K * kPC; idx += kPC) {
    int i = idx / kPC, px = idx % kPC;
    i64 p = p0 + px;
    T2 a;
    a.x = (T)0; a.y = (T)0;
    if (p < N) a = (i == nb) ? zr[p] : brb[((i64)i * L + l3) * N + p];
    v[idx] = a;
  }
  __syncthreads();
  i64 p = p0 + tid;
  if (p >= N) return;
  T2* gzr = reinterpret_cast<T2*>(gz) + ((i64)b * L + l3) * N;
  T2* gbb = reinterpret_cast<T2*>(gbr) + (i64)b * nb * L * N;
  for (int i = 0; i < K; ++i) {
    T ar = (T)0, ai = (T)0;
    for (int j = 0; j < K; ++j) {
      T2 mm = m[i * K + j], vv = v[j * kPC + tid];
      ar = fma(mm.x, vv.x, fma(-mm.y, vv.y, ar));
      ai = fma(mm.x, vv.y, fma(mm.y, vv.x, ai));
    }
    T2 o;
    if (i < nb) {
      o.x = ar; o.y = ai;
      gbb[((i64)i * L + l3) * N + p] = o;
    } else {
      T2 zz = v[nb * kPC + tid];
      T mag = hypot(zz.x, zz.y);
      T c = s1c[(i64)b * L + l3] / (mag == (T)0 ? (T)1 : mag);
      o.x = ar + c * zz.x;
      o.y = ai + c * zz.y;
      gzr[p] = o;
    }
  }
}

template <typename T>
__global__ void k_mean_var_grad(const T* __restrict__ x0, const double* __restrict__ coefs, i64 N, T* __restrict__ gx) {
  i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  i64 b = blockIdx.y;
  double c0 = coefs[2 * b], c1 = coefs[2 * b + 1];
  gx[b * N + p] += (T)(c0 + c1 * (double)x0[b * N + p]);
}

template <typename Tin, typename Tout>
__global__ void k_convert(const Tin* __restrict__ in, Tout* __restrict__ out, i64 n) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (Tout)in[i];
}

}  // namespace

template <typename T>
void conv_forward(const ConvOp& op, const T* x, int R, T* out, i64 out_row_stride, T* mod_out, i64 mod_row_stride,
                  cudaStream_t s) {
  constexpr int RB = sizeof(T) == 4 ? 4 : 2;
  dim3 grid(nblocks(op.n_rows, 128), (R + RB - 1) / RB);
  k_conv_fwd<T, RB><<<grid, 128, 0, s>>>(op.cell.as<int32_t>(), op.coef.as<T>(), op.S, op.n_rows, x, op.n_in, R, out,
                                         out_row_stride, mod_out, mod_row_stride);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void conv_adjoint(const ConvOp& op, const T* gy, i64 gy_row_stride, int R, T* gx, bool accumulate, cudaStream_t s) {
  constexpr int RB = sizeof(T) == 4 ? 4 : 2;
  dim3 grid(nblocks(op.n_in, 128), (R + RB - 1) / RB);
  k_conv_adj<T, RB><<<grid, 128, 0, s>>>(op.tent.as<uint32_t>(), op.ST, op.shift, op.n_in, op.coef.as<T>(), op.n_rows,
                                         gy, gy_row_stride, R, gx, accumulate ? 1 : 0);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void dec_apply(const DecOp& op, bool transpose, const T* x, i64 x_outer, T* y, i64 y_outer, int R_outer, int R_inner,
               bool accumulate, cudaStream_t s) {
  if (R_outer <= 0 || R_inner <= 0) return;
  i64 n_out = transpose ? op.n_in : op.n_out;
  i64 n_in = transpose ? op.n_out : op.n_in;
  dim3 grid(nblocks(n_out, 256), R_inner, R_outer);
  if (transpose)
    k_ell<T><<<grid, 256, 0, s>>>(op.tcol.as<int32_t>(), op.tw.as<T>(), op.WT, n_out, n_in, x, x_outer, y, y_outer,
                                  accumulate ? 1 : 0);
  else
    k_ell<T><<<grid, 256, 0, s>>>(op.col.as<int32_t>(), op.w.as<T>(), op.W, n_out, n_in, x, x_outer, y, y_outer,
                                  accumulate ? 1 : 0);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void modulus_vjp_add(const T* z, const T* g, i64 g_outer, T* gz, int B, i64 plane, cudaStream_t s) {
  dim3 grid(nblocks(plane, 256), B);
  k_modvjp<T><<<grid, 256, 0, s>>>(z, g, g_outer, gz, plane);
  STL_CUDA(cudaGetLastError());
}

ProductShape product_shape(int n, int L, int B, i64 N) {
  ProductShape sh;
  sh.K = (n + 1) * L + 1;
  sh.L = L; sh.B = B; sh.N = N; sh.level0 = n == 0;
  int E = sh.K * (sh.K + 1) / 2;
  sh.slots = 3 * E + 5;
  i64 nsub = (N + kPC - 1) / kPC;
  sh.blocks = (int)std::min<i64>(nsub, 256);
  return sh;
}

template <typename T>
void products_forward(const ProductShape& sh, const T* z, const T* br, const T* x0, double* partials, double* sums,
                      cudaStream_t s) {
  const int K = sh.K, E = K * (K + 1) / 2;
  int Q = 1;
  while (Q < 16 && E * Q * 2 <= kPT) Q *= 2;
  if ((E * Q + kPT - 1) / kPT > 4) throw std::runtime_error("too many coefficient products per level");
  size_t sm_fields = (size_t)K * kPC * (2 * sizeof(T) + sizeof(double));
  size_t sm_gram = (size_t)Q * E * 3 * sizeof(double);
  size_t smem = std::max(sm_fields, sm_gram) + kPT * sizeof(double);
  if (smem > 48 * 1024)
    STL_CUDA(cudaFuncSetAttribute(k_products<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  i64 nsub = (sh.N + kPC - 1) / kPC;
  dim3 grid(sh.blocks, sh.L, sh.B);
  k_products<T><<<grid, kPT, smem, s>>>(K, sh.L, sh.N, (int)nsub, z, br, sh.level0 ? x0 : nullptr, Q, partials,
                                        sh.slots);
  STL_CUDA(cudaGetLastError());
  dim3 rg((sh.slots + 255) / 256, sh.B * sh.L);
  k_reduce_partials<<<rg, 256, 0, s>>>(partials, sh.blocks, sh.slots, sums);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void products_reverse(const ProductShape& sh, const T* z, const T* br, const T* M, const T* s1c, T* gz, T* gbr,
                      cudaStream_t s) {
  const int K = sh.K;
  size_t smem = (size_t)K * K * 2 * sizeof(T) + (size_t)K * kPC * 2 * sizeof(T);
  if (smem > 48 * 1024)
    STL_CUDA(cudaFuncSetAttribute(k_products_rev<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(nblocks(sh.N, kPC), sh.L, sh.B);
  k_products_rev<T><<<grid, kPC, smem, s>>>(K, sh.L, sh.N, z, br, M, s1c, gz, gbr);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void mean_var_grad(const T* x0, const double* coefs, int B, i64 N, T* gx, cudaStream_t s) {
  dim3 grid(nblocks(N, 256), B);
  k_mean_var_grad<T><<<grid, 256, 0, s>>>(x0, coefs, N, gx);
  STL_CUDA(cudaGetLastError());
}

template <typename Tin, typename Tout>
void convert(const Tin* in, Tout* out, i64 n, cudaStream_t s) {
  if (n <= 0) return;
  k_convert<Tin, Tout><<<nblocks(n, 256), 256, 0, s>>>(in, out, n);
  STL_CUDA(cudaGetLastError());
}

#define INST(T)                                                                                                   \
  template void conv_forward<T>(const ConvOp&, const T*, int, T*, i64, T*, i64, cudaStream_t);                    \
  template void conv_adjoint<T>(const ConvOp&, const T*, i64, int, T*, bool, cudaStream_t);                       \
  template void dec_apply<T>(const DecOp&, bool, const T*, i64, T*, i64, int, int, bool, cudaStream_t);           \
  template void modulus_vjp_add<T>(const T*, const T*, i64, T*, int, i64, cudaStream_t);                          \
  template void products_forward<T>(const ProductShape&, const T*, const T*, const T*, double*, double*,          \
                                    cudaStream_t);                                                                \
  template void products_reverse<T>(const ProductShape&, const T*, const T*, const T*, const T*, T*, T*,          \
                                    cudaStream_t);                                                                \
  template void mean_var_grad<T>(const T*, const double*, int, i64, T*, cudaStream_t);
INST(float)
INST(double)
template void convert<double, float>(const double*, float*, i64, cudaStream_t);
template void convert<float, double>(const float*, double*, i64, cudaStream_t);
template void convert<double, double>(const double*, double*, i64, cudaStream_t);
template void convert<float, float>(const float*, float*, i64, cudaStream_t);

}  // namespace stl
