// Compute kernels of the engine's level sweeps (sm_100a).
//
// Fields are pixel-major: a level's field holds, per pixel, a contiguous
// vector of rows (maps [N][B]; moduli [N][B][n+1][L]; complex wavelet
// outputs [N][R][4 gauges] interleaved (re, im)), so the gathers of the
// stencils read whole row vectors of a cell.
//
//  conv_forward  out[p][r][g] = sum_s coef[s][p][g] x[cell(p, s)][r]   (+ |out|)
//  conv_adjoint  gx[c][r]     = sum over the (p, s) reading c of coef[s][p] . gy[p][r]
//  dec_apply     y = D x or D^T x over ELL rows
//  products      the coefficient sums of one level (FP64) and their VJP
//
// On the full sky the operators are stored for faces 0, 4, 8 and every
// thread evaluates the 4 rotated pixels (ConvOp in engine.cuh).  Every
// reduction has a fixed order (no floating-point atomics): results are
// bit-reproducible run to run.
#include <algorithm>
#include <numeric>
#include <cstdio>

#include "engine.cuh"

namespace stl {

namespace {

inline unsigned nblocks(i64 n, int t) { return (unsigned)((n + t - 1) / t); }

template <typename T> struct V2;
template <> struct V2<float> { typedef float2 type; };
template <> struct V2<double> { typedef double2 type; };

// |z| of every kernel (forward and VJP take moduli through the same
// function).  FP32: sqrt(x^2 + y^2) with one FMA, within about an ulp of
// hypotf and without its overflow scaling (fields and moduli are far from
// overflow); it took the FP32 row means of |z| from 2.27 to 2.02-2.06 ms a step at
// nside 1024, J 9, B 4.  FP64 keeps hypot: the FMA form measured no faster there.
__device__ __forceinline__ float zabs(float x, float y) { return sqrtf(fmaf(x, x, y * y)); }
__device__ __forceinline__ double zabs(double x, double y) { return hypot(x, y); }

constexpr uint32_t kSentinel = 0xFFFFFFFFu;

// pixel of rotation k of stored index u (full sky: faces 4 (u >> o2) + k)
__device__ __forceinline__ i64 rot_pixel(i64 u, int k, int o2) {
  return ((4 * (u >> o2) + k) << o2) | (u & ((i64(1) << o2) - 1));
}
// cell c rotated by k within its ring of faces
__device__ __forceinline__ i64 rot_cell(i64 c, int k, int o2) {
  i64 f = c >> o2;
  return (((f & ~i64(3)) | ((f + k) & 3)) << o2) | (c & ((i64(1) << o2) - 1));
}

// ---- bulk asynchronous copies ------------------------------------------------
// Every wait on an mbarrier is bounded (kWaitLimit polls); a kernel that
// gives up records the failure in an error flag the host reads: kErrWait
// when a wait ran out and the CTA then saw its copies in flight land,
// kErrDrain when that drain ran out too (a copy may still have been writing
// the CTA's shared memory when it exited).  Either way the launch's results
// are discarded by the host.
constexpr int kWaitLimit = 1 << 20;
constexpr int kErrWait = 1, kErrDrain = 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// one arrival (a consumer releasing a stage)
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// BYTES (4, 8 or 16) global -> shared, zero fill when !live, not waited
template <int BYTES>
__device__ __forceinline__ void cp_async_r(void* dst, const void* src, bool live) {
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(live ? 16 : 0)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES),
                 "r"(live ? BYTES : 0)
                 : "memory");
}
// 16-byte global -> shared copy of src_bytes (16, or 0: zero fill), not waited
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 8 values of one (slot, row): float4 x 2 or double2 x 4
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
// the same from shared memory (plain loads: __ldg reads global memory only)
__device__ __forceinline__ void load8_shared(const float* p, float w[8]) {
  const float4 a = reinterpret_cast<const float4*>(p)[0];
  const float4 b = reinterpret_cast<const float4*>(p)[1];
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w; w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}
__device__ __forceinline__ void load8_shared(const double* p, double w[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 a = reinterpret_cast<const double2*>(p)[k];
    w[2 * k] = a.x; w[2 * k + 1] = a.y;
  }
}
__device__ __forceinline__ void store8(float* p, const float w[8]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(w[0], w[1], w[2], w[3]);
  reinterpret_cast<float4*>(p)[1] = make_float4(w[4], w[5], w[6], w[7]);
}
__device__ __forceinline__ void store8(double* p, const double w[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) reinterpret_cast<double2*>(p)[k] = make_double2(w[2 * k], w[2 * k + 1]);
}
__device__ __forceinline__ void store4(float* p, const float w[4]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(w[0], w[1], w[2], w[3]);
}
__device__ __forceinline__ void store4(double* p, const double w[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(w[0], w[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(w[2], w[3]);
}

// RB consecutive values of a row vector (RB in 1, 2, 4)
template <int RB>
__device__ __forceinline__ void loadR(const float* p, float v[RB]) {
  if (RB % 4 == 0) {
#pragma unroll
    for (int k = 0; k < RB / 4; ++k) {
      float4 a = __ldg(reinterpret_cast<const float4*>(p) + k);
      v[4 * k] = a.x; v[4 * k + 1] = a.y; v[4 * k + 2] = a.z; v[4 * k + 3] = a.w;
    }
  } else if (RB == 2) {
    float2 a = __ldg(reinterpret_cast<const float2*>(p));
    v[0] = a.x; v[1] = a.y;
  } else {
    v[0] = __ldg(p);
  }
}
template <int RB>
__device__ __forceinline__ void loadR(const double* p, double v[RB]) {
  if (RB >= 2) {
#pragma unroll
    for (int k = 0; k < RB / 2; ++k) {
      double2 a = __ldg(reinterpret_cast<const double2*>(p) + k);
      v[2 * k] = a.x; v[2 * k + 1] = a.y;
    }
  } else {
    v[0] = __ldg(p);
  }
}

// RB consecutive values in shared memory at an address aligned to RB values
// (one vector access where RB values make 8 or 16 bytes), read or added to
template <int RB, typename T>
__device__ __forceinline__ void loadR_shared(const T* p, T v[RB]) {
  if (sizeof(T) == 4 && RB == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  } else if (RB == 2) {
    typedef typename V2<T>::type V;
    const V a = *reinterpret_cast<const V*>(p);
    v[0] = a.x; v[1] = a.y;
  } else {
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) v[rb] = p[rb];
  }
}
template <int RB, typename T>
__device__ __forceinline__ void addR_shared(T* p, const T a[RB]) {
  if (sizeof(T) == 4 && RB == 4) {
    float4 v = *reinterpret_cast<float4*>(p);
    v.x += a[0]; v.y += a[1]; v.z += a[2]; v.w += a[3];
    *reinterpret_cast<float4*>(p) = v;
  } else if (RB == 2) {
    typedef typename V2<T>::type V;
    V v = *reinterpret_cast<V*>(p);
    v.x += a[0]; v.y += a[1];
    *reinterpret_cast<V*>(p) = v;
  } else {
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) p[rb] += a[rb];
  }
}

// The per-slot products of the tiled wavelets.  FP32 pairs go through the
// paired FMA of sm_100 (__ffma2_rn: each component rounds as fmaf), half the
// instructions of the scalar form.
// acc[rb][j] += w[j] xv[rb]: the same roundings as scalar fmas, pair by pair
template <int RB>
__device__ __forceinline__ void fma_rows(float (&acc)[RB][8], const float (&w)[8], const float (&xv)[RB]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    const float2 x2 = make_float2(xv[rb], xv[rb]);
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const float2 r = __ffma2_rn(make_float2(w[j], w[j + 1]), x2, make_float2(acc[rb][j], acc[rb][j + 1]));
      acc[rb][j] = r.x;
      acc[rb][j + 1] = r.y;
    }
  }
}
template <int RB>
__device__ __forceinline__ void fma_rows(double (&acc)[RB][8], const double (&w)[8], const double (&xv)[RB]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[rb][j] = fma(w[j], xv[rb], acc[rb][j]);
}
// a[rb] = sum_q w[q] g[rb][q]; FP32: the even and the odd terms in two
// chains, then added (a fixed order)
template <int RB>
__device__ __forceinline__ void dot8_rows(const float (&w)[8], const float (&g)[RB][8], float (&a)[RB]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    float2 p = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; q += 2) p = __ffma2_rn(make_float2(w[q], w[q + 1]), make_float2(g[rb][q], g[rb][q + 1]), p);
    a[rb] = p.x + p.y;
  }
}
template <int RB>
__device__ __forceinline__ void dot8_rows(const double (&w)[8], const double (&g)[RB][8], double (&a)[RB]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    a[rb] = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) a[rb] = fma(w[q], g[rb][q], a[rb]);
  }
}

// gauge map of rotation k: output gauge g of pixel (4m + k) takes the
// stored gauge (g + 2k) mod 4, conjugated when ((2k - g + 3) >> 2) is odd
__host__ __device__ constexpr int rot_src(int k, int g) { return (g + 2 * k) & 3; }
__host__ __device__ constexpr int rot_conj(int k, int g) { return ((2 * k - g + 3) >> 2) & 1; }

// ---- forward ----------------------------------------------------------------
// One thread per (stored row u, chunk of RB input rows); NK rotations per
// thread.  threadIdx.x runs over the chunks of a row vector, threadIdx.y over
// stored rows, so a warp reads whole row vectors of the cells it gathers.
template <typename T, int NK, int RB>
__global__ void __launch_bounds__(128) k_conv_fwd(const int32_t* __restrict__ cell, const T* __restrict__ coef, int S,
                                                  i64 n_rep, int o2, const T* __restrict__ x, int R,
                                                  T* __restrict__ out, T* __restrict__ mod, int mod_pix, int mod_row,
                                                  int mod_off, const T* __restrict__ rowsum,
                                                  const double* __restrict__ rc) {
  const i64 u = (i64)blockIdx.x * blockDim.y + threadIdx.y;
  const int chunk = blockIdx.y * blockDim.x + threadIdx.x;
  if (u >= n_rep || chunk * RB >= R) return;
  const int r0 = chunk * RB;
  T acc[NK][RB][8];
#pragma unroll
  for (int k = 0; k < NK; ++k)
#pragma unroll
    for (int rb = 0; rb < RB; ++rb)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[k][rb][j] = (T)0;
  // Two-stage software pipeline: the gathers of slot s + 1 and the cell of
  // slot s + 2 are in flight while slot s is accumulated.
  T xv[NK][RB], xn[NK][RB], w[8], wn[8];
  i64 cn = 0;
  auto gather = [&](i64 c, T (&dst)[NK][RB]) {
#pragma unroll
    for (int k = 0; k < NK; ++k) loadR<RB>(x + (NK == 1 ? c : rot_cell(c, k, o2)) * R + r0, dst[k]);
  };
  if (S > 0) {
    const i64 c0 = __ldg(cell + u);
    gather(c0, xv);
    load8(coef + u * 8, w);
    if (S > 1) cn = __ldg(cell + n_rep + u);
  }
  for (int s = 0; s < S; ++s) {
    if (s + 1 < S) {
      gather(cn, xn);
      load8(coef + ((i64)(s + 1) * n_rep + u) * 8, wn);
      if (s + 2 < S) cn = __ldg(cell + (i64)(s + 2) * n_rep + u);
    }
#pragma unroll
    for (int k = 0; k < NK; ++k) fma_rows<RB>(acc[k], w, xv[k]);
#pragma unroll
    for (int k = 0; k < NK; ++k)
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) xv[k][rb] = xn[k][rb];
#pragma unroll
    for (int j = 0; j < 8; ++j) w[j] = wn[j];
  }
  if (rc) {  // the rows' constants times the row sums of the coefficients
    T rs[8];
    load8(rowsum + u * 8, rs);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      const double c = rc[r0 + rb];
#pragma unroll
      for (int k = 0; k < NK; ++k)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[k][rb][j] += (T)(c * (double)rs[j]);
    }
  }
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const i64 p = NK == 1 ? u : rot_pixel(u, k, o2);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      const int r = r0 + rb;
      T o[8];
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const int src = NK == 1 ? g : rot_src(k, g);
        const bool cj = NK == 1 ? false : rot_conj(k, g);
        o[2 * g] = acc[k][rb][2 * src];
        o[2 * g + 1] = cj ? -acc[k][rb][2 * src + 1] : acc[k][rb][2 * src + 1];
      }
      store8(out + (p * R + r) * 8, o);
      if (mod) {
        T* m = mod + p * mod_pix + (i64)r * mod_row + mod_off;
#pragma unroll
        for (int g = 0; g < 4; ++g) m[g] = zabs(o[2 * g], o[2 * g + 1]);
      }
    }
  }
}

// Tiled forward: a CTA takes a tile of kAdjTile stored rows and RB input
// rows; thread (row, rotation k), k fastest, so the 4 rotations of a row
// share each coefficient read.  The CTA gathers the tile's cells (4
// rotations x RB values) into shared memory once; the coefficients and
// tile-cell indices of the tile stream through shared memory in chunks of
// SC slots, two stages deep, by bulk asynchronous copies.
constexpr int kFwdThreads = 4 * kAdjTile;
// cells of a gather plane: at least nc + 1, plane bytes = 32 mod 128 when
// reachable (within 32 extra cells)
template <typename T, int RB>
__host__ __device__ inline int fwd_plane_cells(int nc) {
  const int cb = RB * (int)sizeof(T);
  int pc = nc + 1;
  for (int e = 0; e < 32 && (pc * cb) % 128 != 32; ++e) ++pc;
  return (pc * cb) % 128 == 32 ? pc : nc + 1;
}

template <typename T>
__host__ __device__ constexpr int fwd_sc() { return sizeof(T) == 4 ? 8 : 4; }
// bulk-copy stages of the coefficient stream
template <typename T>
__host__ __device__ constexpr int fwd_stages() { return 2; }

template <typename T, int RB>
__global__ void __launch_bounds__(kFwdThreads, 2) k_conv_fwd_tiles(
    const uint16_t* __restrict__ lcell_t, const T* __restrict__ coef, int S, i64 n_rep, int o2,
    const int32_t* __restrict__ tile_cells, const int32_t* __restrict__ tile_nc, const T* __restrict__ x, int R,
    T* __restrict__ out, T* __restrict__ mod, int mod_pix, int mod_row, int mod_off, int* __restrict__ err,
    const T* __restrict__ rowsum, const double* __restrict__ rc, const int32_t* __restrict__ tile_slots) {
  constexpr int SC = fwd_sc<T>(), NST = fwd_stages<T>();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // bar: a stage's copies have landed; empty: every warp has read the stage
  __shared__ __align__(8) uint64_t bar[NST], empty[NST];
  __shared__ int fail;
  // stage: coef [SC][kAdjTile][8] T, then indices [SC][kAdjTile] uint16
  constexpr size_t kStageCoef = (size_t)SC * kAdjTile * 8 * sizeof(T);
  constexpr size_t kStage = kStageCoef + (size_t)SC * kAdjTile * sizeof(uint16_t);
  T* sx = reinterpret_cast<T*>(smem_raw + NST * kStage);  // [4][pc][RB]: cell nc (padding) is zero
  const int ngroups = R / RB;  // CTAs of a tile: consecutive, so its coefficients stay in L2
  const int tile = blockIdx.x / ngroups, tid = threadIdx.x;
  const int k = tid & 3, row = tid >> 2;
  const int r0 = (blockIdx.x % ngroups) * RB;
  const int nc = tile_nc[tile];
  const i64 u0 = (i64)tile * kAdjTile;
  const int rows = (int)min((i64)kAdjTile, n_rep - u0);
  const int S4 = ((S + 3) / 4) * 4;  // slots per tile in the tile-major index table
  S = tile_slots[tile];              // the tile's rows use no later slot
  const int nch = (S + SC - 1) / SC;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NST; ++q) {
      mbar_init(&bar[q], 1);
      mbar_init(&empty[q], kFwdThreads / 32);
    }
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int c) {
    const int st = c % NST;
    unsigned char* base = smem_raw + st * kStage;
    const int s0 = c * SC, sn = min(SC, S - s0);
    const int sn4 = min(SC, S4 - s0);  // index rows are padded to 4 slots
    const unsigned cb = (unsigned)(rows * 8 * sizeof(T));
    const unsigned lb = (unsigned)(sn4 * kAdjTile * sizeof(uint16_t));
    mbar_expect_tx(&bar[st], sn * cb + lb);
    for (int sl = 0; sl < sn; ++sl)
      bulk_g2s(base + (size_t)sl * kAdjTile * 8 * sizeof(T), coef + ((i64)(s0 + sl) * n_rep + u0) * 8, cb, &bar[st]);
    bulk_g2s(base + kStageCoef, lcell_t + ((i64)tile * S4 + s0) * kAdjTile, lb, &bar[st]);
  };
  if (tid == 0)
    for (int c = 0; c < min(nch, NST); ++c) issue(c);
  const int32_t* tc = tile_cells + (i64)tile * kAdjCells;
  // planes of pc >= nc + 1 cells, pc chosen so that consecutive planes start
  // 32 bytes apart modulo 128: the 4 rotations of a row, which read the same
  // cell index in the 4 planes, then read different banks
  const int pc = fwd_plane_cells<T, RB>(nc);
  for (int i = tid; i < 4 * pc; i += kFwdThreads) {
    const int kk = i / pc, lc = i - kk * pc;
    const bool live = lc < nc;
    const T* src = x + (live ? rot_cell(tc[lc], kk, o2) * R + r0 : 0);
    cp_async_r<RB * sizeof(T)>(sx + (size_t)i * RB, src, live);  // cells >= nc: zero
  }
  cp_async_wait_all();
  T acc[RB][8];
#pragma unroll
  for (int rb = 0; rb < RB; ++rb)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[rb][j] = (T)0;
  const T* sxk = sx + (size_t)k * pc * RB;
  __syncthreads();  // the cell gather, before any thread reads it
  // The chunks: every warp waits for a stage's copies on its own, reads it,
  // then releases it (one arrival per warp on `empty`); thread 0 refills a
  // stage once every warp has released it.  No CTA-wide barrier in the loop:
  // warps drift apart by up to a stage.
  const int lane = tid & 31;
  bool ok = true;
  int issued = min(nch, NST);  // chunks issued (thread 0's count)
  for (int c = 0; c < nch; ++c) {
    const int st = c % NST;
    const unsigned par = (unsigned)(c / NST) & 1;
    if (!mbar_wait(&bar[st], par)) {
      ok = false;
      break;
    }
    const unsigned char* base = smem_raw + st * kStage;
    const T* cs = reinterpret_cast<const T*>(base);
    const uint16_t* ls = reinterpret_cast<const uint16_t*>(base + kStageCoef);
    const int sn = min(SC, S - c * SC);
    if (row < rows) {
#pragma unroll
      for (int sl = 0; sl < SC; ++sl) {
        if (sl < sn) {
          T w[8];
          load8_shared(cs + ((size_t)sl * kAdjTile + row) * 8, w);
          T xv[RB];
          loadR_shared<RB>(sxk + (size_t)ls[sl * kAdjTile + row] * RB, xv);
          fma_rows<RB>(acc, w, xv);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[st]);
    if (tid == 0 && c + NST < nch) {
      if (!mbar_wait(&empty[st], par)) {
        ok = false;
        break;
      }
      issue(c + NST);
      issued = c + NST + 1;
    }
  }
  if (!ok) fail = 1;
  __syncthreads();
  if (fail) {  // thread 0 waits (bounded) for the copies it may have in flight
    if (tid == 0) {
      bool drained = true;
      for (int q = max(0, issued - NST); q < issued; ++q) drained &= mbar_wait(&bar[q % NST], (q / NST) & 1);
      atomicMax(err, drained ? kErrWait : kErrDrain);
    }
    return;
  }
  if (row >= rows) return;
  const i64 p = rot_pixel(u0 + row, k, o2);
  const bool odd = k & 1;
  if (rc) {  // the rows' constants times the row sums of the coefficients
    T rs[8];
    load8(rowsum + (u0 + row) * 8, rs);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      const double c = rc[r0 + rb];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[rb][j] += (T)(c * (double)rs[j]);
    }
  }
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    const int r = r0 + rb;
    T o[8];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      // stored gauge of output gauge g under rotation k: g, or g ^ 2 for odd k
      const T re = odd ? acc[rb][2 * (g ^ 2)] : acc[rb][2 * g];
      const T im = odd ? acc[rb][2 * (g ^ 2) + 1] : acc[rb][2 * g + 1];
      o[2 * g] = re;
      o[2 * g + 1] = rot_conj(k, g) ? -im : im;
    }
    store8(out + (p * R + r) * 8, o);
    if (mod) {
      T* m = mod + p * mod_pix + (i64)r * mod_row + mod_off;
#pragma unroll
      for (int g = 0; g < 4; ++g) m[g] = zabs(o[2 * g], o[2 * g + 1]);
    }
  }
}

// ---- adjoint ----------------------------------------------------------------
// dot of stored coefficients w (rotation k applied) with a cotangent g8
template <typename T, int K>
__device__ __forceinline__ T rot_dot(const T w[8], const T g8[8]) {
  T a = (T)0;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const int src = rot_src(K, g);
    a = fma(w[2 * src], g8[2 * g], a);
    a = rot_conj(K, g) ? fma(-w[2 * src + 1], g8[2 * g + 1], a) : fma(w[2 * src + 1], g8[2 * g + 1], a);
  }
  return a;
}

// One thread per (stored cell v, RB cotangent rows): for each transposed
// entry (u, j) -- stored row u reads rotation j of v -- rotation k of row
// u reads rotation (k + j) mod 4 of v.
template <typename T, int NK, int RB>
__global__ void __launch_bounds__(128) k_conv_adj(const uint32_t* __restrict__ tent, const T* __restrict__ coefT,
                                                  int ST, int tshift, i64 n_rep, int o2, const T* __restrict__ gy,
                                                  int R, T* __restrict__ gx, int accumulate) {
  const i64 v = (i64)blockIdx.x * blockDim.y + threadIdx.y;
  const int chunk = blockIdx.y * blockDim.x + threadIdx.x;
  if (v >= n_rep || chunk * RB >= R) return;
  const int r0 = chunk * RB;
  T acc[NK][RB];
#pragma unroll
  for (int k = 0; k < NK; ++k)
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) acc[k][rb] = (T)0;
  if (NK == 1) {
    // Grid operators: a two-stage software pipeline, as in k_conv_fwd: the
    // coefficients and cotangent rows of entry q + 1 and the entry index of
    // q + 2 are in flight while entry q is added (entries in order).
    T w[8], g[RB][8], wn[8], gn[RB][8];
    uint32_t ent = ST > 0 ? __ldg(tent + v) : kSentinel;
    if (ent != kSentinel) {
      load8(coefT + v * 8, w);
      const i64 u = (i64)(ent >> tshift);
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) load8(gy + (u * R + r0 + rb) * 8, g[rb]);
    }
    uint32_t ent1 = (ST > 1 && ent != kSentinel) ? __ldg(tent + n_rep + v) : kSentinel;
    for (int q = 0; q < ST && ent != kSentinel; ++q) {
      uint32_t ent2 = kSentinel;
      if (ent1 != kSentinel) {
        load8(coefT + ((i64)(q + 1) * n_rep + v) * 8, wn);
        const i64 u = (i64)(ent1 >> tshift);
#pragma unroll
        for (int rb = 0; rb < RB; ++rb) load8(gy + (u * R + r0 + rb) * 8, gn[rb]);
        if (q + 2 < ST) ent2 = __ldg(tent + (i64)(q + 2) * n_rep + v);
      }
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) acc[0][rb] += rot_dot<T, 0>(w, g[rb]);
      ent = ent1;
      ent1 = ent2;
#pragma unroll
      for (int j = 0; j < 8; ++j) w[j] = wn[j];
#pragma unroll
      for (int rb = 0; rb < RB; ++rb)
#pragma unroll
        for (int j = 0; j < 8; ++j) g[rb][j] = gn[rb][j];
    }
  } else {
  for (int q = 0; q < ST; ++q) {
    const i64 e = (i64)q * n_rep + v;
    const uint32_t ent = __ldg(tent + e);
    if (ent == kSentinel) break;
    const i64 u = (i64)(ent >> tshift);
    const int j = (int)(ent & 3u);
    T w[8];
    load8(coefT + e * 8, w);
    T d[NK][RB];
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const i64 p = NK == 1 ? u : rot_pixel(u, k, o2);
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) {
        T g8[8];
        load8(gy + (p * R + r0 + rb) * 8, g8);
        d[k][rb] = k == 0 ? rot_dot<T, 0>(w, g8)
                          : (k == 1 ? rot_dot<T, 1>(w, g8) : (k == 2 ? rot_dot<T, 2>(w, g8) : rot_dot<T, 3>(w, g8)));
      }
    }
    if (NK == 1) {
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) acc[0][rb] += d[0][rb];
    } else {
      // rotation k of u reads rotation (k + j) of v: rotate d by j
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) {
        T t0 = d[0][rb], t1 = d[NK > 1 ? 1 : 0][rb], t2 = d[NK > 2 ? 2 : 0][rb], t3 = d[NK > 3 ? 3 : 0][rb];
        if (j & 1) { T t = t3; t3 = t2; t2 = t1; t1 = t0; t0 = t; }
        if (j & 2) { T a = t0, b = t1; t0 = t2; t1 = t3; t2 = a; t3 = b; }
        acc[0][rb] += t0;
        acc[NK > 1 ? 1 : 0][rb] += t1;
        acc[NK > 2 ? 2 : 0][rb] += t2;
        acc[NK > 3 ? 3 : 0][rb] += t3;
      }
    }
  }
  }
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const i64 c = NK == 1 ? v : rot_pixel(v, k, o2);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      T* o = gx + c * R + r0 + rb;
      *o = accumulate ? *o + acc[k][rb] : acc[k][rb];
    }
  }
}

// ---- row-centric adjoint (two phases) -----------------------------------------
// The transposed gather above re-reads every cotangent vector once per entry
// that reads its row (about 44 times, 32 bytes per rotation and row).  Here
// a CTA takes a tile of kAdjTile stored rows and RB cotangent rows; each
// thread keeps its row's 4 rotated cotangent vectors in registers and, per
// chunk of kAdjSC slots, writes the products of its slots to shared memory
// (phase 1); then every tile cell adds the products of its entries in
// (slot, row) order (phase 2).  The tile's sums go to a partial buffer, and
// k_adj_combine adds the partials of every cell in (tile, cell) order: all
// sums have a fixed order, so results are bit-reproducible.
// Thread = stored row, holding its 4 rotated cotangent vectors (the
// rotation's gauge permutation and conjugation folded in, so every product
// is a plain 8-term dot with the stored coefficients).  Product planes
// [rb][k] are kAdjPlane values apart.
constexpr int kAdjPlane = kAdjSC * kAdjTile;

template <typename T, int RB>
__global__ void __launch_bounds__(kAdjTile, 2) k_conv_adj_tiles(
    const T* __restrict__ coef, int S, i64 n_rep, int o2, int nch, int ncs, const int32_t* __restrict__ tile_nc,
    const uint16_t* __restrict__ tile_ent, const uint16_t* __restrict__ tile_off, const T* __restrict__ gy, int R,
    T* __restrict__ part, const int32_t* __restrict__ tile_slots) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* P = reinterpret_cast<T*>(smem_raw);                 // [RB][4][kAdjPlane]
  T* acc = P + 4 * RB * kAdjPlane;                       // [RB][4][ncs]
  uint16_t* ent = reinterpret_cast<uint16_t*>(acc + 4 * RB * ncs);  // [kAdjSC kAdjTile]
  uint16_t* off = ent + kAdjSC * kAdjTile;               // [ncs + 1]
  const int ngroups = R / RB;
  const int tile = blockIdx.x / ngroups, tid = threadIdx.x;
  const int r0 = (blockIdx.x % ngroups) * RB;
  const int nc = tile_nc[tile];
  const i64 u = (i64)tile * kAdjTile + tid;
  const bool valid = u < n_rep;
  T g[4][RB][8];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      T t[8];
      if (valid) load8(gy + (rot_pixel(u, k, o2) * R + r0 + rb) * 8, t);
      else
#pragma unroll
        for (int q = 0; q < 8; ++q) t[q] = (T)0;
#pragma unroll
      for (int gg = 0; gg < 4; ++gg) {
        const int q = rot_src(k, gg);
        g[k][rb][2 * q] = t[2 * gg];
        g[k][rb][2 * q + 1] = rot_conj(k, gg) ? -t[2 * gg + 1] : t[2 * gg + 1];
      }
    }
  for (int i = tid; i < 4 * RB * ncs; i += kAdjTile) acc[i] = (T)0;
  const uint16_t* toff = tile_off + (i64)tile * nch * ncs;
  const uint16_t* tent = tile_ent + (i64)tile * S * kAdjTile;
  const T* cu = coef + u * 8;
  const int St = tile_slots[tile];  // the tile's rows use no later slot (their entries end there too)
  const int ncht = (St + kAdjSC - 1) / kAdjSC;
  const i64 cstride = n_rep * 8;
  T wn[8];
  if (valid) load8(cu, wn);
  for (int ch = 0; ch < ncht; ++ch) {
    const int s0 = ch * kAdjSC;
    const int sn = min(kAdjSC, St - s0);
    if (valid) {
      for (int sl = 0; sl < sn; ++sl) {
        T w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) w[q] = wn[q];
        if (s0 + sl + 1 < St) load8(cu + (i64)(s0 + sl + 1) * cstride, wn);
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int rb = 0; rb < RB; ++rb) {
            T a = (T)0;
#pragma unroll
            for (int q = 0; q < 8; ++q) a = fma(w[q], g[k][rb][q], a);
            P[(rb * 4 + k) * kAdjPlane + sl * kAdjTile + tid] = a;
          }
      }
    }
    const int e0 = toff[ch * ncs], e1 = toff[ch * ncs + nc];
    for (int i = tid; i < e1 - e0; i += kAdjTile) ent[i] = tent[e0 + i];
    for (int i = tid; i <= nc; i += kAdjTile) off[i] = (uint16_t)(toff[ch * ncs + i] - e0);
    __syncthreads();
    for (int lc = tid; lc < nc; lc += kAdjTile) {
      const int a0 = off[lc], a1 = off[lc + 1];
      if (a0 == a1) continue;
      T a[4 * RB];
#pragma unroll
      for (int q = 0; q < 4 * RB; ++q) a[q] = acc[q * ncs + lc];
      for (int e = a0; e < a1; ++e) {
        const int en = ent[e];
        const T* p = P + (en >> 8) * kAdjTile + (en & 255);
#pragma unroll
        for (int q = 0; q < 4 * RB; ++q) a[q] += p[q * kAdjPlane];
      }
#pragma unroll
      for (int q = 0; q < 4 * RB; ++q) acc[q * ncs + lc] = a[q];
    }
    __syncthreads();
  }
  // partials [tile][k][ncs][R]
  for (int i = tid; i < 4 * RB * nc; i += kAdjTile) {
    const int q = i / nc, lc = i - q * nc;
    const int rb = q >> 2, kk = q & 3;
    part[(((i64)tile * 4 + kk) * ncs + lc) * R + r0 + rb] = acc[q * ncs + lc];
  }
}

// Coloured adjoint (operators in the coloured layout): a CTA takes a tile
// of kAdjTile stored rows and RB cotangent rows; thread (row, rotation k), k
// fastest, keeps the row's cotangents under rotation k in registers.  No two
// rows of a tile read one cell in the same slot, so per slot every thread
// adds its RB products into its cell's sums in shared memory ([cell][k][rb])
// with no two threads on one address, and a barrier separates the slots.
// The coefficients and tile cells of SC slots arrive by bulk asynchronous
// copies, two stages deep.  Every cell sums its products in slot order, so
// the results are bit-reproducible.
constexpr int kAdjCThreads = 4 * kAdjTile;

template <typename T>
__host__ __device__ constexpr int adjc_sc() { return sizeof(T) == 4 ? 8 : 4; }

template <typename T, int RB>
__global__ void __launch_bounds__(kAdjCThreads, 2) k_conv_adj_colored(
    const uint16_t* __restrict__ lcell_t, const T* __restrict__ coef, int S, i64 n_rep, int o2, int ncs,
    const int32_t* __restrict__ tile_nc, const T* __restrict__ gy, int R, T* __restrict__ part,
    const int32_t* __restrict__ tile_slots, int* __restrict__ err, ModulusAdd<T> madd) {
  constexpr int SC = adjc_sc<T>();
  constexpr size_t kStageCoef = (size_t)SC * kAdjTile * 8 * sizeof(T);
  constexpr size_t kStage = kStageCoef + (size_t)SC * kAdjTile * sizeof(uint16_t);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int fail;
  T* acc = reinterpret_cast<T*>(smem_raw + 2 * kStage);  // [nc + 1][4][RB]
  const int ngroups = R / RB;  // CTAs of a tile: consecutive, so its coefficients stay in L2
  const int tile = blockIdx.x / ngroups, tid = threadIdx.x;
  const int k = tid & 3, row = tid >> 2;
  const int r0 = (blockIdx.x % ngroups) * RB;
  const int nc = tile_nc[tile];
  const i64 u0 = (i64)tile * kAdjTile;
  const int rows = (int)min((i64)kAdjTile, n_rep - u0);
  const int S4 = ((S + 3) / 4) * 4;  // slots per tile in the tile-major cell table
  const int St = tile_slots[tile];
  const int nch = (St + SC - 1) / SC;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int c) {
    const int st = c & 1;
    unsigned char* base = smem_raw + st * kStage;
    const int s0 = c * SC, sn = min(SC, St - s0);
    const int sn4 = min(SC, S4 - s0);  // cell rows are padded to 4 slots
    const unsigned cb = (unsigned)(rows * 8 * sizeof(T));
    const unsigned lb = (unsigned)(sn4 * kAdjTile * sizeof(uint16_t));
    mbar_expect_tx(&bar[st], sn * cb + lb);
    for (int sl = 0; sl < sn; ++sl)
      bulk_g2s(base + (size_t)sl * kAdjTile * 8 * sizeof(T), coef + ((i64)(s0 + sl) * n_rep + u0) * 8, cb, &bar[st]);
    bulk_g2s(base + kStageCoef, lcell_t + ((i64)tile * S4 + s0) * kAdjTile, lb, &bar[st]);
  };
  if (tid == 0) {
    if (nch > 0) issue(0);
    if (nch > 1) issue(1);
  }
  for (int i = tid; i < (nc + 1) * 4 * RB; i += kAdjCThreads) acc[i] = (T)0;
  // the row's cotangents under rotation k (gauge permutation and
  // conjugation folded in): every product is a plain 8-term dot; the
  // permutation is selected without indexing registers by the runtime k
  T g[RB][8];
  const bool valid = row < rows, odd = k & 1;
  const i64 pk = valid ? rot_pixel(u0 + row, k, o2) : 0;
#pragma unroll
  for (int rb = 0; rb < RB; ++rb) {
    T t[8];
    if (valid) {
      load8(gy + (pk * R + r0 + rb) * 8, t);
      if (madd.z) {  // the modulus VJP of row r0 + rb (map b): t += g z / |z|
        T zz[8];
        load8(madd.z + (pk * R + r0 + rb) * 8, zz);
        const T* gm = madd.g + pk * madd.g_pix + (i64)(r0 + rb) * madd.g_row;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const T mag = zabs(zz[2 * l], zz[2 * l + 1]);
          const T dd = mag == (T)0 ? (T)1 : mag;
          const T gv = gm[l];
          t[2 * l] += gv * zz[2 * l] / dd;
          t[2 * l + 1] += gv * zz[2 * l + 1] / dd;
        }
      }
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q) t[q] = (T)0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int gg = odd ? (q ^ 2) : q;
      const T re = odd ? t[2 * (q ^ 2)] : t[2 * q];
      const T im = odd ? t[2 * (q ^ 2) + 1] : t[2 * q + 1];
      g[rb][2 * q] = re;
      g[rb][2 * q + 1] = rot_conj(k, gg) ? -im : im;
    }
  }
  int c = 0;
  for (; c < nch; ++c) {
    const int st = c & 1;
    if (!mbar_wait(&bar[st], (c >> 1) & 1)) fail = 1;
    __syncthreads();  // the stage (and, first, the zeroed sums) everywhere
    if (fail) break;
    const unsigned char* base = smem_raw + st * kStage;
    const T* cs = reinterpret_cast<const T*>(base);
    const uint16_t* ls = reinterpret_cast<const uint16_t*>(base + kStageCoef);
    const int sn = min(SC, St - c * SC);
    for (int sl = 0; sl < sn; ++sl) {
      const int lc = ls[sl * kAdjTile + row];
      if (valid && lc < nc) {
        T w[8];
        load8_shared(cs + ((size_t)sl * kAdjTile + row) * 8, w);
        T a[RB];
        dot8_rows<RB>(w, g, a);
        addR_shared<RB>(acc + ((size_t)lc * 4 + k) * RB, a);
      }
      __syncthreads();  // the slot's sums are in: the next slot may read them
    }
    if (tid == 0 && c + 2 < nch) issue(c + 2);
  }
  if (fail) {
    bool drained = true;
    for (int q = c; q < min(nch, c + 2); ++q) drained &= mbar_wait(&bar[q & 1], (q >> 1) & 1);
    if (tid == 0) atomicMax(err, drained ? kErrWait : kErrDrain);
    return;
  }
  // partials [tile][k][ncs][R]
  for (int i = tid; i < nc * 4; i += kAdjCThreads) {
    const int lc = i >> 2, kk = i & 3;
    T* o = part + (((i64)tile * 4 + kk) * ncs + lc) * R + r0;
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) o[rb] = acc[(size_t)i * RB + rb];
  }
}

// gx[rotation k' of stored cell v][r] (+)= sum over the entries (tile, lc, j)
// of v, in order, of part[tile][(k' - j) mod 4][lc][r]
template <typename T, int NK, int RB>
__global__ void __launch_bounds__(128) k_adj_combine(const i64* __restrict__ coff, const uint32_t* __restrict__ clist,
                                                     i64 n_cells, int o2, int ncs, const T* __restrict__ part, int R,
                                                     T* __restrict__ gx, int accumulate) {
  const i64 v = (i64)blockIdx.x * blockDim.y + threadIdx.y;
  const int chunk = blockIdx.y * blockDim.x + threadIdx.x;
  if (v >= n_cells || chunk * RB >= R) return;
  const int r0 = chunk * RB;
  T a[NK][RB];
#pragma unroll
  for (int k = 0; k < NK; ++k)
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) a[k][rb] = (T)0;
  const i64 e1 = coff[v + 1];
  for (i64 e = coff[v]; e < e1; ++e) {
    const uint32_t en = __ldg(clist + e);
    const i64 tile = en >> 12;
    const int lc = (en >> 2) & 1023, j = en & 3;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const T* p = part + ((tile * 4 + ((k - j) & 3)) * ncs + lc) * R + r0;
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) a[k][rb] += p[rb];
    }
  }
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const i64 c = NK == 1 ? v : rot_pixel(v, k, o2);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      T* o = gx + c * R + r0 + rb;
      *o = accumulate ? *o + a[k][rb] : a[k][rb];
    }
  }
}

// ---- tensor-core wavelets (FP32 fields, ConvOp::mma) ---------------------------
// Per stored row u the wavelet is a small product: for the 16 (rotation k,
// field row r) pairs of an M tile, out[(k, r)][o] = sum_s X[k][cell(u, s)][r]
// C_u[s][o] (o = the 4 gauges' re, im), so one mma.sync m16n8k8 covers one
// row and a chunk of 8 slots.  FP32 accuracy from TF32 operands by the
// 3xTF32 split: a = a_hi + a_lo (a_hi = tf32(a), a_lo = tf32(a - a_hi)),
// a b ~ a_lo b_hi + a_hi b_lo + a_hi b_hi, the three products of a chunk
// accumulated from zero (small ones first) and the chunk's result added in
// FP32 registers -- the tensor core's own accumulation truncates, which
// would bias sums carried across chunks.
// Fragments (lane = 4 g + t): A a0 (g, t), a1 (g + 8, t), a2 (g, t + 4),
// a3 (g + 8, t + 4); B b0 (t, g), b1 (t + 4, g); D d0 (g, 2 t), d1 (g,
// 2 t + 1), d2 (g + 8, 2 t), d3 (g + 8, 2 t + 1).  M row g is (k = g >> 1,
// field row r(h = 0)) and g + 8 (k, r(h = 1)) with r = (g & 1) 2 MT + 2 mt
// + h in M tile mt, so a lane's rows of one cell are contiguous.
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// one chunk (K = 8) in 3xTF32, from zero
__device__ __forceinline__ void mma3(float d[4], const uint32_t ah[4], const uint32_t al[4], const uint32_t bh[2],
                                     const uint32_t bl[2]) {
  d[0] = d[1] = d[2] = d[3] = 0.0f;
  mma_tf32(d, al, bh);
  mma_tf32(d, ah, bl);
  mma_tf32(d, ah, bh);
}

constexpr int kMmaFwdWarpRows = 8;     // rows per warp of the forward
constexpr int kMmaFwdWarps = kMmaRows / kMmaFwdWarpRows;
constexpr int kMmaFwdThreads = 32 * kMmaFwdWarps;
constexpr int kMmaAdjWarps = kMmaRows / kMmaWarpRows;
constexpr int kMmaAdjThreads = 32 * kMmaAdjWarps;
// floats per staged slot (kMmaRows rows of 8 coefficients, then padding):
// slot stride 8 (forward) or 4 (adjoint) banks mod 32, so the B fragments'
// 32 words fall in distinct banks
constexpr int kMmaFwdSlot = kMmaRows * 8 + 8;
constexpr int kMmaAdjSlot = kMmaRows * 8 + 4;
constexpr size_t kMmaFwdStage = 8 * kMmaFwdSlot * sizeof(float) + 8 * kMmaRows * sizeof(uint16_t);
constexpr size_t kMmaAdjStage = 8 * kMmaAdjSlot * sizeof(float) + 8 * kMmaRows;

// Forward: one CTA per (tile, group of 4 MT field rows), warp w the rows
// 8 w .. 8 w + 7 of the tile.  The tile's plane [4 k][pcs][4 MT] of input
// rows (cell -1: zero) is gathered once by asynchronous copies and split
// once into its TF32 high and low parts (two planes: every element serves
// about 44 rows, so no product splits its A operand); per chunk of 8 slots
// the coefficients and plane cells of every row arrive by bulk copies (NS
// stages); every row's accumulators live in registers across the chunks.
template <int MT, int NS>
__global__ void __launch_bounds__(kMmaFwdThreads, 2) k_conv_fwd_mma(
    const uint16_t* __restrict__ m_lc, const float* __restrict__ coef, int Sm, i64 n_rep, int o2,
    const int32_t* __restrict__ cells, int pcs, const int32_t* __restrict__ tch, const float* __restrict__ x, int R,
    float* __restrict__ out, float* __restrict__ mod, int mod_pix, int mod_row, int mod_off, int* __restrict__ err,
    const float* __restrict__ rowsum, const double* __restrict__ rc) {
  constexpr int RM = 4 * MT;
  constexpr size_t kCoefBytes = 8 * kMmaFwdSlot * sizeof(float);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[NS];
  __shared__ int fail;
  float* ph = reinterpret_cast<float*>(smem_raw + NS * kMmaFwdStage);  // high parts [4][pcs][RM]
  float* pl_ = ph + (size_t)4 * pcs * RM;                                 // low parts
  const int ngroups = (R + RM - 1) / RM;
  const i64 tile = blockIdx.x / ngroups;
  const int r0 = (int)(blockIdx.x % ngroups) * RM;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int k = g >> 1, rq = g & 1;
  const i64 u0 = tile * kMmaRows;
  const int rows = (int)min((i64)kMmaRows, n_rep - u0);
  const int nch = tch[tile];
  if (tid == 0) {
    for (int b = 0; b < NS; ++b) mbar_init(&bar[b], 1);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int c) {
    const int st = c % NS;
    unsigned char* base = smem_raw + st * kMmaFwdStage;
    const unsigned cb = (unsigned)(rows * 8 * sizeof(float));
    const unsigned lb = (unsigned)(8 * kMmaRows * sizeof(uint16_t));
    mbar_expect_tx(&bar[st], 8 * cb + lb);
    for (int sl = 0; sl < 8; ++sl)
      bulk_g2s(base + (size_t)sl * kMmaFwdSlot * sizeof(float), coef + ((i64)(8 * c + sl) * n_rep + u0) * 8, cb,
               &bar[st]);
    bulk_g2s(base + kCoefBytes, m_lc + ((i64)tile * (Sm / 8) + c) * kMmaRows * 8, lb, &bar[st]);
  };
  if (tid == 0)
    for (int c = 0; c < min(nch, NS); ++c) issue(c);
  // the plane: per tile cell and rotation, the CTA's RM input rows, by
  // asynchronous 16-byte copies (all in flight at once; a hole or a missing
  // cell copies zero bytes, which fills zeros); rows past R (R % 4 != 0)
  // by plain loads.  Each thread then splits the elements it copied.
  const int32_t* tc = cells + tile * pcs;
  const bool whole = R % 4 == 0;
  for (int q = tid; q < pcs; q += kMmaFwdThreads) {
    const int32_t cl = tc[q];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      float* dst = ph + ((size_t)kk * pcs + q) * RM;
      const float* xp = x + (cl >= 0 ? rot_cell(cl, kk, o2) * R + r0 : 0);
      if (whole) {
#pragma unroll
        for (int j = 0; j < MT; ++j) cp_async16(dst + 4 * j, xp + 4 * j, cl >= 0 ? 16 : 0);
      } else {
#pragma unroll
        for (int j = 0; j < RM; ++j) dst[j] = (cl >= 0 && r0 + j < R) ? __ldg(xp + j) : 0.0f;
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();  // every thread's copies have landed
  // split, in consecutive 16-byte units (conflict-free)
  for (int q = tid; q < pcs * RM; q += kMmaFwdThreads) {
    float4* h = reinterpret_cast<float4*>(ph) + q;
    float4 v = *h, w;
    uint32_t hi, lo;
    split_tf32(v.x, hi, lo); v.x = __uint_as_float(hi); w.x = __uint_as_float(lo);
    split_tf32(v.y, hi, lo); v.y = __uint_as_float(hi); w.y = __uint_as_float(lo);
    split_tf32(v.z, hi, lo); v.z = __uint_as_float(hi); w.z = __uint_as_float(lo);
    split_tf32(v.w, hi, lo); v.w = __uint_as_float(hi); w.w = __uint_as_float(lo);
    *h = v;
    reinterpret_cast<float4*>(pl_)[q] = w;
  }
  float acc[kMmaFwdWarpRows][MT][4];
#pragma unroll
  for (int i = 0; i < kMmaFwdWarpRows; ++i)
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][mt][q] = 0.0f;
  const size_t koff = (size_t)k * pcs * RM + rq * 2 * MT;
  const float* hk = ph + koff;
  const float* lk = pl_ + koff;
  int c = 0;
  for (; c < nch; ++c) {
    const int st = c % NS;
    if (!mbar_wait(&bar[st], (c / NS) & 1)) fail = 1;
    __syncthreads();  // also orders the split planes before the first chunk
    if (fail) break;
    const unsigned char* base = smem_raw + st * kMmaFwdStage;
    const float* cs = reinterpret_cast<const float*>(base);
    const uint16_t* ls = reinterpret_cast<const uint16_t*>(base + kCoefBytes);
    // no branch per row, so the rows' independent mma chains interleave: a
    // row past its own chunks multiplies zero coefficients (its padding),
    // a row past the tile's end (the last tile) reads clamped plane cells
    // and is never stored
#pragma unroll
    for (int i = 0; i < kMmaFwdWarpRows; ++i) {
      const int ul = warp * kMmaFwdWarpRows + i;
      const int lc0 = min((int)ls[ul * 8 + t], pcs - 1), lc1 = min((int)ls[ul * 8 + t + 4], pcs - 1);
      uint32_t bh[2], bl[2];
      split_tf32(cs[t * kMmaFwdSlot + ul * 8 + g], bh[0], bl[0]);
      split_tf32(cs[(t + 4) * kMmaFwdSlot + ul * 8 + g], bh[1], bl[1]);
      uint32_t ha[2 * MT], hb[2 * MT], la[2 * MT], lb[2 * MT];
      if (MT == 2) {
        const uint4 p = *reinterpret_cast<const uint4*>(hk + (size_t)lc0 * RM);
        const uint4 q = *reinterpret_cast<const uint4*>(hk + (size_t)lc1 * RM);
        const uint4 u = *reinterpret_cast<const uint4*>(lk + (size_t)lc0 * RM);
        const uint4 v = *reinterpret_cast<const uint4*>(lk + (size_t)lc1 * RM);
        ha[0] = p.x; ha[1] = p.y; ha[2] = p.z; ha[3] = p.w;
        hb[0] = q.x; hb[1] = q.y; hb[2] = q.z; hb[3] = q.w;
        la[0] = u.x; la[1] = u.y; la[2] = u.z; la[3] = u.w;
        lb[0] = v.x; lb[1] = v.y; lb[2] = v.z; lb[3] = v.w;
      } else {
        const uint2 p = *reinterpret_cast<const uint2*>(hk + (size_t)lc0 * RM);
        const uint2 q = *reinterpret_cast<const uint2*>(hk + (size_t)lc1 * RM);
        const uint2 u = *reinterpret_cast<const uint2*>(lk + (size_t)lc0 * RM);
        const uint2 v = *reinterpret_cast<const uint2*>(lk + (size_t)lc1 * RM);
        ha[0] = p.x; ha[1] = p.y;
        hb[0] = q.x; hb[1] = q.y;
        la[0] = u.x; la[1] = u.y;
        lb[0] = v.x; lb[1] = v.y;
      }
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const uint32_t ah[4] = {ha[2 * mt], ha[2 * mt + 1], hb[2 * mt], hb[2 * mt + 1]};
        const uint32_t al[4] = {la[2 * mt], la[2 * mt + 1], lb[2 * mt], lb[2 * mt + 1]};
        float d[4];
        mma3(d, ah, al, bh, bl);
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][mt][q] += d[q];
      }
    }
    __syncthreads();  // the stage is read: refill it
    if (tid == 0 && c + NS < nch) issue(c + NS);
  }
  if (fail) {
    bool drained = true;
    for (int q = c; q < min(nch, c + NS); ++q) drained &= mbar_wait(&bar[q % NS], (q / NS) & 1);
    if (tid == 0) atomicMax(err, drained ? kErrWait : kErrDrain);
    return;
  }
  const bool odd = k & 1;
  const int go = odd ? (t ^ 2) : t;  // output gauge of stored gauge t under rotation k
  const bool cj = rot_conj(k, go);
#pragma unroll
  for (int i = 0; i < kMmaFwdWarpRows; ++i) {
    const int ul = warp * kMmaFwdWarpRows + i;
    if (ul >= rows) continue;
    const i64 u = u0 + ul;
    const i64 p = rot_pixel(u, k, o2);
    float rs0 = 0.0f, rs1 = 0.0f;
    if (rc) {
      rs0 = rowsum[u * 8 + 2 * t];
      rs1 = rowsum[u * 8 + 2 * t + 1];
    }
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + rq * 2 * MT + 2 * mt + h;
        if (r >= R) continue;
        float re = acc[i][mt][2 * h], im = acc[i][mt][2 * h + 1];
        if (rc) {  // the row's constant times the row sums of the coefficients
          const double cr = rc[r];
          re += (float)(cr * (double)rs0);
          im += (float)(cr * (double)rs1);
        }
        if (cj) im = -im;
        *reinterpret_cast<float2*>(out + (p * R + r) * 8 + 2 * go) = make_float2(re, im);
        if (mod) mod[p * mod_pix + (i64)r * mod_row + mod_off + go] = zabs(re, im);
      }
  }
}

// Adjoint: one CTA per (tile, 4 cotangent rows), warp w the rows 8 w ..
// 8 w + 7 of the tile.  Warp w adds the products of its rows into private
// sums [4 k][wls][4 r] over the distinct cells of its rows (warp-local
// numbering), so no other warp touches them and no barrier separates the
// slots; per chunk and row one mma gives the 16 x 8 products (rotation and
// row) x (slot) of the row's cotangents with its coefficients.  The
// coefficients and warp-local cells stream through NS bulk-copy stages.
// Then every tile cell's partial is the sum over the warps, in warp order,
// written to part[tile][k][pcs][R].  madd: the modulus VJP added to the
// cotangents first, as k_conv_adj_colored.
template <int NS>
__global__ void __launch_bounds__(kMmaAdjThreads, 2) k_conv_adj_mma(
    const uint8_t* __restrict__ m_wlc, const float* __restrict__ coef, int Sm, i64 n_rep, int o2,
    const int32_t* __restrict__ tch, const uint8_t* __restrict__ m_winv, int pcs, int wls,
    const float* __restrict__ gy, int R, float* __restrict__ part, int* __restrict__ err, ModulusAdd<float> madd) {
  constexpr size_t kCoefBytes = 8 * kMmaAdjSlot * sizeof(float);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[NS];
  __shared__ int fail;
  float* sums = reinterpret_cast<float*>(smem_raw + NS * kMmaAdjStage);  // [warps][4][wls][4]
  const int ngroups = (R + 3) / 4;  // rows past R (the last group of R % 4 != 0) are zero
  const i64 tile = blockIdx.x / ngroups;
  const int r0 = (int)(blockIdx.x % ngroups) * 4;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int k = g >> 1, rp = g & 1;
  const i64 u0 = tile * kMmaRows;
  const int rows = (int)min((i64)kMmaRows, n_rep - u0);
  const int nch = tch[tile];
  if (tid == 0) {
    for (int b = 0; b < NS; ++b) mbar_init(&bar[b], 1);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int c) {
    const int st = c % NS;
    unsigned char* base = smem_raw + st * kMmaAdjStage;
    const unsigned cb = (unsigned)(rows * 8 * sizeof(float));
    const unsigned wb = (unsigned)(8 * kMmaRows);
    mbar_expect_tx(&bar[st], 8 * cb + wb);
    for (int sl = 0; sl < 8; ++sl)
      bulk_g2s(base + (size_t)sl * kMmaAdjSlot * sizeof(float), coef + ((i64)(8 * c + sl) * n_rep + u0) * 8, cb,
               &bar[st]);
    bulk_g2s(base + kCoefBytes, m_wlc + ((i64)tile * (Sm / 8) + c) * kMmaRows * 8, wb, &bar[st]);
  };
  if (tid == 0)
    for (int c = 0; c < min(nch, NS); ++c) issue(c);
  float* mine = sums + (size_t)warp * 16 * wls;
  for (int i = lane; i < 16 * wls; i += 32) mine[i] = 0.0f;
  // the rows' cotangents under rotation k (gauge permutation, conjugation
  // and the modulus VJP folded in) as split A fragments; rows past the
  // tile's end are zero
  const bool odd = k & 1;
  auto cot = [&](i64 p, int rr, int o) {
    if (r0 + rr >= R) return 0.0f;
    const int q = o >> 1, pt = o & 1;
    const int gg = odd ? (q ^ 2) : q;
    const i64 e = (p * R + r0 + rr) * 8;
    float v = gy[e + 2 * gg + pt];
    if (madd.z) {
      const float zr = madd.z[e + 2 * gg], zi = madd.z[e + 2 * gg + 1];
      const float mag = zabs(zr, zi);
      const float dd = mag == 0.0f ? 1.0f : mag;
      const float gv = madd.g[p * madd.g_pix + (i64)(r0 + rr) * madd.g_row + gg];
      v += gv * (pt ? zi : zr) / dd;
    }
    return (pt && rot_conj(k, gg)) ? -v : v;
  };
  uint32_t ah[kMmaWarpRows][4], al[kMmaWarpRows][4];
#pragma unroll
  for (int i = 0; i < kMmaWarpRows; ++i) {
    const int ul = warp * kMmaWarpRows + i;
    float a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (ul < rows) {
      const i64 p = rot_pixel(u0 + ul, k, o2);
      a[0] = cot(p, 2 * rp, t);
      a[1] = cot(p, 2 * rp + 1, t);
      a[2] = cot(p, 2 * rp, t + 4);
      a[3] = cot(p, 2 * rp + 1, t + 4);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) split_tf32(a[q], ah[i][q], al[i][q]);
  }
  float* mk = mine + (size_t)k * wls * 4 + 2 * rp;
  int c = 0;
  for (; c < nch; ++c) {
    const int st = c % NS;
    if (!mbar_wait(&bar[st], (c / NS) & 1)) fail = 1;
    __syncthreads();  // also orders the zeroed sums before the first chunk
    if (fail) break;
    const unsigned char* base = smem_raw + st * kMmaAdjStage;
    const float* cs = reinterpret_cast<const float*>(base);
    const uint8_t* ws = base + kCoefBytes;
    // per row: the products (independent of the other rows, so the chains
    // interleave; a row past its own chunks multiplies zero coefficients),
    // then the additions in row order: a later row may add to the same
    // cells, and the warp's shared-memory accesses are issued in program
    // order (no lane diverges here; the compiler keeps the order of
    // accesses that may alias)
#pragma unroll
    for (int i = 0; i < kMmaWarpRows; ++i) {
      const int ul = warp * kMmaWarpRows + i;
      uint32_t bh[2], bl[2];
      split_tf32(cs[g * kMmaAdjSlot + ul * 8 + t], bh[0], bl[0]);
      split_tf32(cs[g * kMmaAdjSlot + ul * 8 + t + 4], bh[1], bl[1]);
      float d[4];
      mma3(d, ah[i], al[i], bh, bl);
      if (ul < rows) {  // past the tile's end: the stage holds no data for the row
        const uint16_t wp = *reinterpret_cast<const uint16_t*>(ws + ul * 8 + 2 * t);
        float2* s0 = reinterpret_cast<float2*>(mk + (size_t)(wp & 0xff) * 4);
        float2* s1 = reinterpret_cast<float2*>(mk + (size_t)(wp >> 8) * 4);
        float2 v0 = *s0, v1 = *s1;
        v0.x += d[0]; v0.y += d[2];
        v1.x += d[1]; v1.y += d[3];
        *s0 = v0;
        *s1 = v1;
      }
    }
    __syncthreads();  // the stage is read: refill it
    if (tid == 0 && c + NS < nch) issue(c + NS);
  }
  if (fail) {
    bool drained = true;
    for (int q = c; q < min(nch, c + NS); ++q) drained &= mbar_wait(&bar[q % NS], (q / NS) & 1);
    if (tid == 0) atomicMax(err, drained ? kErrWait : kErrDrain);
    return;
  }
  __syncthreads();  // every warp's sums are complete (also when the tile has no chunk)
  // tile partials: per plane cell, for every (k, r), the warps' sums in warp order
  const uint8_t* winv = m_winv + tile * kMmaAdjWarps * pcs;
  for (int pl = tid; pl < pcs; pl += kMmaAdjThreads) {
    float4 v[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) v[kk] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int w = 0; w < kMmaAdjWarps; ++w) {
      const int wl = winv[w * pcs + pl];
      if (wl == 255) continue;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const float4 a = *reinterpret_cast<const float4*>(sums + (((size_t)w * 4 + kk) * wls + wl) * 4);
        v[kk].x += a.x; v[kk].y += a.y; v[kk].z += a.z; v[kk].w += a.w;
      }
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      float* o = part + ((tile * 4 + kk) * pcs + pl) * R + r0;
      if (R % 4 == 0) {
        *reinterpret_cast<float4*>(o) = v[kk];
      } else {
        const float e[4] = {v[kk].x, v[kk].y, v[kk].z, v[kk].w};
        for (int r = 0; r < 4 && r0 + r < R; ++r) o[r] = e[r];
      }
    }
  }
}

// ---- decimation ---------------------------------------------------------------
// y[c][ro][ri] (+)= sum_e w[e][c] x[col[e][c]][ro][ri]; one thread per (stored
// row u, chunk of RB rows of the R_outer x R_inner rows), NK rotations per
// thread; threadIdx.x runs over the chunks of a pixel's rows.
// Input, output and weight types may differ (a decimation between an FP32
// and an FP64 level): the sums are in the weights' type.
template <typename Tin, typename Tout, typename Tw, int NK, int RB>
__global__ void k_ell(const int32_t* __restrict__ col, const Tw* __restrict__ w, int W, i64 n_rep, int o2_out,
                      int o2_in, const Tin* __restrict__ x, int x_pix, int x_outer, Tout* __restrict__ y, int y_pix,
                      int y_outer, int R_outer, int R_inner, int accumulate) {
  const i64 u = (i64)blockIdx.x * blockDim.y + threadIdx.y;
  const int chunk = blockIdx.y * blockDim.x + threadIdx.x;
  const int per = R_inner / RB;
  if (u >= n_rep || chunk >= R_outer * per) return;
  const int ro = chunk / per, ri = (chunk % per) * RB;
  Tw acc[NK][RB];
#pragma unroll
  for (int k = 0; k < NK; ++k)
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) acc[k][rb] = (Tw)0;
#pragma unroll 4
  for (int e = 0; e < W; ++e) {  // unrolled: the loads of several entries in flight
    const i64 idx = (i64)e * n_rep + u;
    const Tw we = __ldg(w + idx);
    const i64 c = __ldg(col + idx);
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      const i64 ck = NK == 1 ? c : rot_cell(c, k, o2_in);
      Tin xv[RB];
      loadR<RB>(x + ck * x_pix + (i64)ro * x_outer + ri, xv);
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) acc[k][rb] = fma(we, (Tw)xv[rb], acc[k][rb]);
    }
  }
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const i64 p = NK == 1 ? u : rot_pixel(u, k, o2_out);
    Tout* yr = y + p * y_pix + (i64)ro * y_outer + ri;
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) yr[rb] = accumulate ? (Tout)((Tw)yr[rb] + acc[k][rb]) : (Tout)acc[k][rb];
  }
}

// gz[p][b][l] += g[p][b][l] z/|z| (0 at z = 0); g at g + p g_pix + b g_row + l
template <typename T>
__global__ void k_modvjp(const T* __restrict__ z, const T* __restrict__ g, int g_pix, int g_row, T* __restrict__ gz,
                         i64 N, int B, int L) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;  // over N * B * L
  if (i >= N * B * L) return;
  const i64 p = i / (B * L);
  const int b = (int)((i / L) % B), l = (int)(i % L);
  const T zr = z[2 * i], zm = z[2 * i + 1];
  const T mag = zabs(zr, zm);
  const T gv = g[p * g_pix + (i64)b * g_row + l];
  const T dd = mag == (T)0 ? (T)1 : mag;
  gz[2 * i] += gv * zr / dd;
  gz[2 * i + 1] += gv * zm / dd;
}

// ---- coefficient products --------------------------------------------------------
//
// Per level n, map b and orientation l3, the operand vector of a pixel is
// v = (branch[d][l1][l3] for d <= n, l1 < L; z[l3]).  Every S3/S4
// coefficient of the level is an entry of the Hermitian Gram matrix
// sum_p v v^H: S4 in the 4 x 4 blocks (d1, d2), d1 <= d2, of the branches,
// S3 in the blocks (d, z), S2 its (z, z) entry.  Items per l3: the (d1, d2)
// blocks, the (d, z) blocks and one item for the per-pixel sums (|z|,
// |z|^2, |z|^4 and, at level 0, x, x^2, x^4).  Partial layout per (block,
// b, l3), in doubles:
//   BB block t (d1 <= d2, d1-major): [t 48 .. +32) 16 complex (l1, l2)
//                                    [t 48 + 32 .. +16) 16 sums |a|^2 |b|^2
//   Bz block d: [nBB 48 + 12 d .. +8) 4 complex (l1, z), then 4 second sums
//   z item:     [nBB 48 + 12 (n + 1) .. +6) |z|, |z|^2, |z|^4, x, x^2, x^4
//
// A CTA takes a contiguous pixel range of all maps.  Chunks of PC pixels
// (branch rows and z of every map: contiguous bytes) stream into shared
// memory by bulk asynchronous copies (cp.async.bulk, completion on an
// mbarrier), kProdStages deep.  Every warp has one role -- a (map, item)
// pair -- and a replica index: replica r of P takes every P-th iteration
// of its role over a chunk.  Lanes of a role:
//   BB block (d1, d2): (l3, l1, half h); entries (l1, 2h), (l1, 2h + 1);
//                      one pixel per iteration
//   Bz block d:        (l3, l1, x); entry (l1, z) of pixel 2 it + x
//   per-pixel item:    (l3, q); pixel 8 it + q
// so a warp never diverges on the item kind and its shared-memory reads hit
// distinct banks.  Roles and replica counts come from a table balanced by
// cost (product_shape); the CTA's replicas and lanes are summed in a fixed
// order, then the CTAs in k_reduce_partials.  In FP32 mode the products and
// the sums over one chunk are FP32 (at most a few dozen pixels per lane),
// added into FP64 sums after every chunk; FP64 mode sums in FP64.  Every wait
// on a copy is bounded: on timeout the CTA records the failure in *err.
constexpr int kProdMaxWarps = 32;
constexpr int kProdStages = 3;
constexpr int kProdStageBytes = 72 * 1024;

// MOM: also the second sums (|a|^2 |b|^2, |z|^4, x^4) that only the
// variances of the coefficients need; without them their slots stay zero.
template <typename T, bool MOM>
__global__ void __launch_bounds__(kProdMaxWarps * 32, 1) k_products(
    int nd, i64 N, int B, const T* __restrict__ z, const T* __restrict__ br, const T* __restrict__ x0, int slots,
    const int32_t* __restrict__ roles, int W, int PC, i64 chunk, double* __restrict__ partials,
    int* __restrict__ err, const double* __restrict__ x0c, const uint8_t* __restrict__ mask,
    const i64* __restrict__ blk, const T* __restrict__ x0r) {
  typedef typename V2<T>::type T2;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[kProdStages];
  __shared__ int fail;
  constexpr int L = 4;
  const int K1 = nd * L;
  const int nBB = nd * (nd + 1) / 2, I = nBB + nd + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t rc = roles[(i64)blockIdx.z * W + warp];
  const bool active = rc >= 0;
  const int role = active ? (rc & 0xFFFF) : 0, rep = (rc >> 16) & 0xFF, nrep = active ? (rc >> 24) & 0xFF : 1;
  const int b = role / I, item = role % I;
  int kind = 2, d1 = 0, d2 = 0;
  if (item < nBB) {
    kind = 0;
    int r = item;
    while (r >= nd - d1) { r -= nd - d1; ++d1; }
    d2 = d1 + r;
  } else if (item < nBB + nd) {
    kind = 1;
    d1 = item - nBB;
  }
  const int l3 = lane & 3, l1 = (lane >> 2) & 3, hx = lane >> 4, q8 = lane >> 2;
  // stage s: branch rows [PC][B][K1][L], z [PC][B][L], then at level 0 the
  // maps [PC][B], copied from the 16-byte boundary at or below the chunk's
  // first map value (x_off(pc) bytes before it)
  const size_t br_px = (size_t)B * K1 * L, z_px = (size_t)B * L;  // T2 per pixel
  const size_t x_bytes = x0 ? (((size_t)PC * B * sizeof(T) + 15) & ~(size_t)15) + 16 : 0;
  const size_t stage_bytes = (size_t)PC * (br_px + z_px) * sizeof(T2) + x_bytes;
  unsigned char* stage0 = smem;
  // the pixel range: uniform, or from the range table (segments)
  const i64 P0 = blk ? blk[blockIdx.x] : (i64)blockIdx.x * chunk;
  const i64 P1 = blk ? blk[blockIdx.x + 1] : min(N, P0 + chunk);
  auto x_off = [&](i64 pc) { return (unsigned)(((size_t)pc * B * sizeof(T)) & 15u); };
  const int nchunks = P1 > P0 ? (int)((P1 - P0 + PC - 1) / PC) : 0;
  const T2* brv = reinterpret_cast<const T2*>(br);
  const T2* zv = reinterpret_cast<const T2*>(z);
  if (threadIdx.x == 0) {
    for (int st = 0; st < kProdStages; ++st) mbar_init(&bar[st], 1);
    fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // the map copy rounds up to 16 bytes: its buffer is padded
  auto round16 = [](unsigned n) { return (n + 15u) & ~15u; };
  auto issue = [&](int c) {
    const int st = c % kProdStages;
    const i64 pc = P0 + (i64)c * PC;
    const int np = (int)min((i64)PC, P1 - pc);
    unsigned char* base = stage0 + st * stage_bytes;
    T2* sb = reinterpret_cast<T2*>(base);
    T2* sz = sb + (size_t)PC * br_px;
    unsigned char* sx = reinterpret_cast<unsigned char*>(sz + (size_t)PC * z_px);
    const unsigned nb = (unsigned)(np * br_px * sizeof(T2)), nz = (unsigned)(np * z_px * sizeof(T2));
    const unsigned xo = x_off(pc);
    const unsigned nx = x0 ? round16((unsigned)(np * B * sizeof(T)) + xo) : 0u;
    mbar_expect_tx(&bar[st], nb + nz + nx);
    bulk_g2s(sb, brv + pc * br_px, nb, &bar[st]);
    bulk_g2s(sz, zv + pc * z_px, nz, &bar[st]);
    if (x0) bulk_g2s(sx, reinterpret_cast<const unsigned char*>(x0 + pc * B) - xo, nx, &bar[st]);
  };
  if (threadIdx.x == 0)
    for (int c = 0; c < min(nchunks, kProdStages); ++c) issue(c);
  constexpr bool kSplit = sizeof(T) == 4;  // FP32: chunk sums in FP32, then FP64
  double acc[6];
  T f[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) { acc[i] = 0.0; f[i] = (T)0; }
  int c = 0;
  for (; c < nchunks; ++c) {
    const int st = c % kProdStages;
    if (!mbar_wait(&bar[st], (c / kProdStages) & 1)) fail = 1;
    __syncthreads();
    if (fail) break;
    const i64 pc = P0 + (i64)c * PC;
    const int np = (int)min((i64)PC, P1 - pc);
    const T2* sb = reinterpret_cast<const T2*>(stage0 + st * stage_bytes);
    const T2* sz = sb + (size_t)PC * br_px;
    const T* sx = reinterpret_cast<const T*>(reinterpret_cast<const unsigned char*>(sz + (size_t)PC * z_px) +
                                             x_off(pc));
    if (active) {
      if (kind == 0) {
        const int ra = (d1 * 4 + l1) * L + l3, rb = (d2 * 4 + 2 * hx) * L + l3;
        for (int j = rep; j < np; j += nrep) {
          if (mask && !mask[pc + j]) continue;
          const T2* rowp = sb + ((size_t)j * B + b) * K1 * L;
          const T2 a = rowp[ra], y0 = rowp[rb], y1 = rowp[rb + L];
          const T am = fma(a.x, a.x, a.y * a.y);
          f[0] = fma(a.x, y0.x, fma(a.y, y0.y, f[0]));
          f[1] = fma(a.y, y0.x, fma(-a.x, y0.y, f[1]));
          f[2] = fma(a.x, y1.x, fma(a.y, y1.y, f[2]));
          f[3] = fma(a.y, y1.x, fma(-a.x, y1.y, f[3]));
          if (MOM) {
            f[4] = fma(am, fma(y0.x, y0.x, y0.y * y0.y), f[4]);
            f[5] = fma(am, fma(y1.x, y1.x, y1.y * y1.y), f[5]);
          }
        }
      } else if (kind == 1) {
        const int ra = (d1 * 4 + l1) * L + l3;
        const int ni = (np + 1) >> 1;
        for (int it = rep; it < ni; it += nrep) {
          const int j = 2 * it + hx;
          if (j < np && (!mask || mask[pc + j])) {
            const T2 x = sb[((size_t)j * B + b) * K1 * L + ra];
            const T2 zz = sz[((size_t)j * B + b) * L + l3];
            f[0] = fma(x.x, zz.x, fma(x.y, zz.y, f[0]));
            f[1] = fma(x.y, zz.x, fma(-x.x, zz.y, f[1]));
            if (MOM) f[2] = fma(fma(x.x, x.x, x.y * x.y), fma(zz.x, zz.x, zz.y * zz.y), f[2]);
          }
        }
      } else {
        const int ni = (np + 7) >> 3;
        for (int it = rep; it < ni; it += nrep) {
          const int j = 8 * it + q8;
          if (j < np && (!mask || mask[pc + j])) {
            const T2 zz = sz[((size_t)j * B + b) * L + l3];
            const T m = zabs(zz.x, zz.y);
            const T m2 = m * m;
            f[0] += m;
            f[1] += m2;
            if (MOM) f[2] = fma(m2, m2, f[2]);
            if (x0 && l3 == 0) {
              const double xv = x0c[b] + (double)sx[(size_t)j * B + b] +
                                (x0r ? (double)x0r[(pc + j) * B + b] : 0.0);
              const double x2 = xv * xv;
              acc[3] += xv;
              acc[4] += x2;
              if (MOM) acc[5] += x2 * x2;
            }
          }
        }
      }
    }
    if (kSplit) {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        acc[i] += (double)f[i];
        f[i] = (T)0;
      }
    }
    __syncthreads();  // the stage is read: refill it
    if (threadIdx.x == 0 && c + kProdStages < nchunks) issue(c + kProdStages);
  }
  if (fail) {
    // wait (bounded) for the copies still in flight into this CTA's stages
    bool drained = true;
    for (int k = c; k < min(nchunks, c + kProdStages); ++k)
      drained &= mbar_wait(&bar[k % kProdStages], (k / kProdStages) & 1);
    if (threadIdx.x == 0) atomicMax(err, drained ? kErrWait : kErrDrain);
  }
  if (!kSplit) {
#pragma unroll
    for (int i = 0; i < 6; ++i) acc[i] += (double)f[i];
  }
  // replicas of a role are consecutive warps, replica 0 first: sum them in
  // order (through the stage memory, free now), then the lanes
  __syncthreads();
  double* red = reinterpret_cast<double*>(smem);
#pragma unroll
  for (int i = 0; i < 6; ++i) red[(warp * 32 + lane) * 6 + i] = acc[i];
  __syncthreads();
  if (!active || rep != 0) return;
  double v[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double a = 0.0;
    for (int r = 0; r < nrep; ++r) a += red[((warp + r) * 32 + lane) * 6 + i];
    v[i] = a;
  }
  double* out = partials + (((i64)blockIdx.x * B + b) * L + l3) * slots;
  if (kind == 0) {
    const int e0 = l1 * 4 + 2 * hx, e1 = e0 + 1;
    double* o = out + item * 48;
    o[2 * e0] = v[0];
    o[2 * e0 + 1] = v[1];
    o[2 * e1] = v[2];
    o[2 * e1 + 1] = v[3];
    o[32 + e0] = v[4];
    o[32 + e1] = v[5];
  } else if (kind == 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], 16);
    if (hx == 0) {
      double* o = out + nBB * 48 + (item - nBB) * 12;
      o[2 * l1] = v[0];
      o[2 * l1 + 1] = v[1];
      o[8 + l1] = v[2];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      v[i] += __shfl_down_sync(0xffffffffu, v[i], 16);
      v[i] += __shfl_down_sync(0xffffffffu, v[i], 8);
      v[i] += __shfl_down_sync(0xffffffffu, v[i], 4);
    }
    if (q8 == 0) {
      double* o = out + nBB * 48 + nd * 12;
#pragma unroll
      for (int i = 0; i < 6; ++i) o[i] = (i < 3 || l3 == 0) ? v[i] : 0.0;
    }
  }
}

// Products without variances at the levels with ND = 1 or 2 branch blocks
// (levels 0 and 1): one thread per (pixel, map b, l3) holds the pixel's
// operand vector (branches a_(d, l), d < ND, l < 4, and z) and adds every
// Gram entry the coefficients read: the diagonal blocks (d, d) through
// |a|^2 and a_l1 conj(a_l2) for l1 < l2 (l1 > l2 are conjugates), the blocks
// (d1 < d2) in full, a_(d, l) conj(z), |z|, |z|^2 and, at level 0 (l3 = 0),
// the map value and its square in FP64.  Lanes: (l3, b) fastest, then the
// pixel, so the P = 32 / 4B pixels of a warp read whole operand rows.  No
// staging and no barrier in the loop: the operand rows are read once through
// L1.  Every kP0Flush pixels a thread's sums in T are added over the warp's
// pixel lanes (a fixed xor tree) and into the warp's FP64 sums in shared
// memory; at the end the warps' sums are added in warp order into the
// partials of the general products kernel's layout.
constexpr int kP0Flush = 16;

template <int ND>
__host__ __device__ constexpr int p0_sums() {  // diag blocks, full blocks, (d, z) blocks, |z|, |z|^2
  return ND * 16 + ND * (ND - 1) / 2 * 32 + ND * 8 + 2;
}
template <typename T, int ND>
__host__ __device__ constexpr int p0_threads() {
  return sizeof(T) == 4 ? (ND == 1 ? 768 : 1024 / ND) : 512 / ND;
}

// warps of a CTA: the FP64 sums of the warps fit in 200 KB
template <typename T, int ND>
inline int p0_warps(int B) {
  const int per_warp = 4 * B * p0_sums<ND>() * 8 + B * 2 * 8;
  const int w = (200 * 1024) / per_warp, most = p0_threads<T, ND>() / 32;
  return w < most ? w : most;
}

// source of partial slot s (layout of k_products, ND blocks) in the thread
// sums: index i, -1 (zero), -2 - i (minus sum i), 100 / 101 (map value / square)
template <int ND>
__device__ __forceinline__ int p0_source(int s) {
  constexpr int nBB = ND * (ND + 1) / 2, NF = p0_sums<ND>();
  if (s < nBB * 48) {
    int t = s / 48, d1 = 0;
    const int w = s % 48;
    while (t >= ND - d1) { t -= ND - d1; ++d1; }
    const int d2 = d1 + t;
    if (w >= 32) return -1;
    const int e = w >> 1, im = w & 1, l1 = e >> 2, l2 = e & 3;
    if (d1 == d2) {
      const int base = d1 * 16;
      if (l1 == l2) return im ? -1 : base + l1;
      const int a = l1 < l2 ? l1 : l2, c = l1 < l2 ? l2 : l1;
      const int k = a * (7 - a) / 2 + (c - a - 1);
      if (!im) return base + 4 + 2 * k;
      return l1 < l2 ? base + 5 + 2 * k : -2 - (base + 5 + 2 * k);
    }
    int pair = 0;  // index of (d1, d2) among the pairs d1 < d2, lexicographic
    for (int x = 0; x < d1; ++x) pair += ND - 1 - x;
    pair += d2 - d1 - 1;
    return ND * 16 + pair * 32 + 2 * e + im;
  }
  s -= nBB * 48;
  if (s < 12 * ND) {
    const int d = s / 12, w = s % 12;
    return w < 8 ? ND * 16 + ND * (ND - 1) / 2 * 32 + d * 8 + w : -1;
  }
  s -= 12 * ND;
  if (s == 0) return NF - 2;
  if (s == 1) return NF - 1;
  if (s == 3) return 100;
  if (s == 4) return 101;
  return -1;
}

template <typename T, int ND>
__global__ void __launch_bounds__(p0_threads<T, ND>(), 1) k_products0(
    i64 N, int B, const T* __restrict__ z, const T* __restrict__ br, const T* __restrict__ x0,
    const double* __restrict__ x0c, const uint8_t* __restrict__ mask, i64 chunk, int slots,
    double* __restrict__ partials, const i64* __restrict__ blk, const T* __restrict__ x0r) {
  typedef typename V2<T>::type T2;
  constexpr int NF = p0_sums<ND>(), OFF = ND * 16 + ND * (ND - 1) / 2 * 32, ZB = OFF;  // (d, z) blocks start
  extern __shared__ __align__(16) double p0s[];  // [warps][4B][NF], then map sums [warps][B][2]
  const int rows = 4 * B, P = 32 / rows;
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = lane % rows, pw = lane / rows, b = r >> 2, l3 = r & 3;
  double* acc = p0s + ((size_t)warp * rows + r) * NF;
  double* xacc = p0s + (size_t)nw * rows * NF;
  for (int i = lane; i < rows * NF; i += 32) p0s[(size_t)warp * rows * NF + i] = 0.0;
  T f[NF];
#pragma unroll
  for (int i = 0; i < NF; ++i) f[i] = (T)0;
  double xs = 0.0, xs2 = 0.0;
  const T2* brv = reinterpret_cast<const T2*>(br);
  const T2* zv = reinterpret_cast<const T2*>(z);
  __syncwarp();
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < NF; ++i) {
      T v = f[i];
      for (int o = rows; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (pw == 0) acc[i] += (double)v;
      f[i] = (T)0;
    }
  };
  const i64 p0 = blk ? blk[blockIdx.x] : (i64)blockIdx.x * chunk;
  const i64 p1 = blk ? blk[blockIdx.x + 1] : min(N, p0 + chunk);
  int cnt = 0;
  // the operands of the thread's next pixel are loaded while this pixel's
  // products run (two pixels' loads in flight a thread)
  const i64 step = (i64)nw * P;
  T2 an[ND][4], zn;
  bool live_n = false;
  auto fetch = [&](i64 p, T2 (&a)[ND][4], T2& zz) -> bool {
    if (!(p < p1 && (!mask || mask[p]))) return false;
    const i64 q = (p * B + b) * (ND * 16) + l3;  // Br [N][B][ND L][L]
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
      for (int l = 0; l < 4; ++l) a[d][l] = __ldg(brv + q + (d * 4 + l) * 4);
    zz = __ldg(zv + (p * B + b) * 4 + l3);
    return true;
  };
  if (ND == 1) live_n = fetch(p0 + (i64)warp * P + pw, an, zn);  // ND > 1: no registers to spare
  for (i64 base = p0 + (i64)warp * P; base < p1; base += step) {
    const i64 p = base + pw;
    T2 a[ND][4], zz;
    bool live;
    if (ND == 1) {
      live = live_n;
#pragma unroll
      for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int l = 0; l < 4; ++l) a[d][l] = an[d][l];
      zz = zn;
      live_n = fetch(p + step, an, zn);
    } else {
      live = fetch(p, a, zz);
    }
    if (live) {
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        T* fd = f + d * 16;
#pragma unroll
        for (int l = 0; l < 4; ++l) fd[l] = fma(a[d][l].x, a[d][l].x, fma(a[d][l].y, a[d][l].y, fd[l]));
        int k = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = i + 1; j < 4; ++j, ++k) {
            fd[4 + 2 * k] = fma(a[d][i].x, a[d][j].x, fma(a[d][i].y, a[d][j].y, fd[4 + 2 * k]));
            fd[5 + 2 * k] = fma(a[d][i].y, a[d][j].x, fma(-a[d][i].x, a[d][j].y, fd[5 + 2 * k]));
          }
      }
      int pair = 0;
#pragma unroll
      for (int d1 = 0; d1 < ND; ++d1)
#pragma unroll
        for (int d2 = d1 + 1; d2 < ND; ++d2, ++pair) {
          T* fp = f + ND * 16 + pair * 32;
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int e = i * 4 + j;
              fp[2 * e] = fma(a[d1][i].x, a[d2][j].x, fma(a[d1][i].y, a[d2][j].y, fp[2 * e]));
              fp[2 * e + 1] = fma(a[d1][i].y, a[d2][j].x, fma(-a[d1][i].x, a[d2][j].y, fp[2 * e + 1]));
            }
        }
#pragma unroll
      for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          T* fz = f + ZB + d * 8;
          fz[2 * l] = fma(a[d][l].x, zz.x, fma(a[d][l].y, zz.y, fz[2 * l]));
          fz[2 * l + 1] = fma(a[d][l].y, zz.x, fma(-a[d][l].x, zz.y, fz[2 * l + 1]));
        }
      const T m = zabs(zz.x, zz.y);
      f[NF - 2] += m;
      f[NF - 1] = fma(m, m, f[NF - 1]);
      if (x0 && l3 == 0) {
        const double xv = x0c[b] + (double)x0[p * B + b] + (x0r ? (double)x0r[p * B + b] : 0.0);
        xs += xv;
        xs2 += xv * xv;
      }
    }
    if (++cnt == kP0Flush) {
      flush();
      cnt = 0;
    }
  }
  flush();
  for (int o = rows; o < 32; o <<= 1) {
    xs += __shfl_xor_sync(0xffffffffu, xs, o);
    xs2 += __shfl_xor_sync(0xffffffffu, xs2, o);
  }
  if (pw == 0 && l3 == 0) {
    xacc[((size_t)warp * B + b) * 2] = xs;
    xacc[((size_t)warp * B + b) * 2 + 1] = xs2;
  }
  __syncthreads();
  // partial row (blk, b, l3): every slot from its source, warps in order
  for (int o = threadIdx.x; o < rows * slots; o += blockDim.x) {
    const int rr = o / slots, sl = o - rr * slots, bb = rr >> 2, ll = rr & 3;
    const int src = p0_source<ND>(sl);
    double v = 0.0;
    if (src >= 100) {
      if (x0 && ll == 0)
        for (int w = 0; w < nw; ++w) v += xacc[((size_t)w * B + bb) * 2 + (src - 100)];
    } else if (src != -1) {
      const int i = src >= 0 ? src : -2 - src;
      for (int w = 0; w < nw; ++w) v += p0s[((size_t)w * rows + rr) * NF + i];
      if (src < -1) v = -v;
    }
    partials[((i64)blockIdx.x * rows + rr) * slots + sl] = v;
  }
}

template <typename T, int ND>
void products0_launch(const ProductShape& sh, const T* z, const T* br, const T* x0, const T* x0r, const double* x0c,
                      const uint8_t* mask, double* partials, cudaStream_t s) {
  const int nw = p0_warps<T, ND>(sh.B);
  const size_t smem = (size_t)nw * (4 * sh.B * p0_sums<ND>() + sh.B * 2) * sizeof(double);
  allow_dynamic_smem(k_products0<T, ND>);
  const i64 chunk = (sh.N + sh.blocks - 1) / sh.blocks;
  k_products0<T, ND><<<sh.blocks, 32 * nw, smem, s>>>(sh.N, sh.B, z, br, sh.level0 ? x0 : nullptr, x0c, mask, chunk,
                                                      sh.slots, partials, sh.d_blk, sh.level0 ? x0r : nullptr);
  STL_CUDA(cudaGetLastError());
}

// sums[row][slot] = sum over blocks of partials[blk][row][slot] in block order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblk, int rows, int slots,
                                  double* __restrict__ sums) {
  const i64 total = (i64)rows * slots;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (i64)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int k = 0; k < nblk; ++k) a += partials[(i64)k * total + i];
    sums[i] = a;
  }
}

// segments: sums[k stride + i] = sum over the ranges seg_blk[k] ..
// seg_blk[k + 1] - 1 of partials[blk][i] in range order
__global__ void k_reduce_segments(const double* __restrict__ partials, const int32_t* __restrict__ seg_blk, int nseg,
                                  int rows, int slots, double* __restrict__ sums, size_t stride) {
  const i64 total = (i64)rows * slots;
  for (int k = blockIdx.y; k < nseg; k += gridDim.y) {
    const int b0 = seg_blk[k], b1 = seg_blk[k + 1];
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (i64)gridDim.x * blockDim.x) {
      double a = 0.0;
      for (int j = b0; j < b1; ++j) a += partials[(i64)j * total + i];
      sums[(size_t)k * stride + i] = a;
    }
  }
}

// gv = M v per pixel and l3 (M: K x K complex of the coefficient cotangents
// of one (b, l3), in shared memory); gz additionally gets s1c z / |z| (auto
// S1).  Thread (pixel, l3), l3 fastest, holds v in registers; CTAs stride
// over 64-pixel tiles of one map.
constexpr int kRevThreads = 256;

template <typename T, int K>
__global__ void __launch_bounds__(kRevThreads) k_products_rev(i64 N, int B, int bs, const T* __restrict__ z,
                                                              const T* __restrict__ br, const T* __restrict__ M,
                                                              const T* __restrict__ s1c,
                                                              const uint8_t* __restrict__ mask, int accumulate,
                                                              T* __restrict__ gz, T* __restrict__ gbr,
                                                              const i64* __restrict__ blk,
                                                              const int32_t* __restrict__ bseg) {
  extern __shared__ __align__(16) unsigned char smem[];
  typedef typename V2<T>::type T2;
  constexpr int L = 4, K1 = K - 1;
  T2* m = reinterpret_cast<T2*>(smem);  // [bs][L][K][K]
  // a CTA takes maps b0 .. b0 + bs - 1: thread (pixel, map, l3), l3 fastest,
  // so the maps of a pixel (contiguous rows) are read and written together
  // with a range table: the CTA's pixel range, inside segment sg
  const int b0 = blockIdx.y * bs, t = threadIdx.x, sg = blk ? bseg[blockIdx.x] : 0;
  const T2* Mb = reinterpret_cast<const T2*>(M) + ((i64)sg * B + b0) * L * K * K;
  for (int i = t; i < bs * L * K * K; i += kRevThreads) m[i] = Mb[i];
  __syncthreads();
  const int l3 = t & 3, bl = (t >> 2) % bs, px = (t >> 2) / bs, b = b0 + bl;
  const int TPX = kRevThreads / (4 * bs);
  if (px >= TPX) return;
  const T2* ml = m + (bl * L + l3) * K * K;
  const T c1 = s1c[((i64)sg * B + b) * L + l3];
  const T2* brv = reinterpret_cast<const T2*>(br);
  const T2* zv = reinterpret_cast<const T2*>(z);
  T2* gbrv = reinterpret_cast<T2*>(gbr);
  T2* gzv = reinterpret_cast<T2*>(gz);
  // PPT adjacent pixels per thread: every cotangent matrix entry read from
  // shared memory serves PPT pixels
  constexpr int PPT = K <= 21 ? 2 : 1;
  const i64 lo = blk ? blk[blockIdx.x] : 0, hi = blk ? blk[blockIdx.x + 1] : N;
  const i64 g0 = blk ? (i64)px : (i64)blockIdx.x * TPX + px, gstep = blk ? (i64)TPX : (i64)gridDim.x * TPX;
  for (i64 g = g0; lo + g * PPT < hi; g += gstep) {
    T2 v[PPT][K];
    bool on[PPT];
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const i64 p = lo + g * PPT + q;
      const i64 row = (p * B + b) * K1;
      on[q] = p < hi && (!mask || mask[p]);
      if (p < hi && !on[q] && !accumulate) {  // outside the averaged pixels: no cotangent
        T2 zero;
        zero.x = (T)0; zero.y = (T)0;
        for (int i = 0; i < K1; ++i) gbrv[(row + i) * L + l3] = zero;
        gzv[(p * B + b) * L + l3] = zero;
      }
#pragma unroll
      for (int i = 0; i < K1; ++i) {
        if (on[q]) v[q][i] = brv[(row + i) * L + l3];
        else { v[q][i].x = (T)0; v[q][i].y = (T)0; }
      }
      if (on[q]) v[q][K1] = zv[(p * B + b) * L + l3];
      else { v[q][K1].x = (T)0; v[q][K1].y = (T)0; }
    }
#pragma unroll 1
    for (int i = 0; i < K; ++i) {
      T ar[PPT], ai[PPT];
#pragma unroll
      for (int q = 0; q < PPT; ++q) { ar[q] = (T)0; ai[q] = (T)0; }
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const T2 mm = ml[i * K + j];
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          ar[q] = fma(mm.x, v[q][j].x, fma(-mm.y, v[q][j].y, ar[q]));
          ai[q] = fma(mm.x, v[q][j].y, fma(mm.y, v[q][j].x, ai[q]));
        }
      }
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        if (!on[q]) continue;
        const i64 p = lo + g * PPT + q;
        T2 o;
        T2* dst;
        if (i == K1) {
          const T mag = zabs(v[q][K1].x, v[q][K1].y);
          const T c = c1 / (mag == (T)0 ? (T)1 : mag);
          o.x = ar[q] + c * v[q][K1].x;
          o.y = ai[q] + c * v[q][K1].y;
          dst = gzv + (p * B + b) * L + l3;
        } else {
          o.x = ar[q];
          o.y = ai[q];
          dst = gbrv + ((p * B + b) * K1 + i) * L + l3;
        }
        if (accumulate) {
          const T2 prev = *dst;
          o.x += prev.x;
          o.y += prev.y;
        }
        *dst = o;
      }
    }
  }
}

template <typename T, typename I>
__global__ void k_mean_var_grad(const T* __restrict__ x0, const double* __restrict__ xc,
                                const uint8_t* __restrict__ mask, const double* __restrict__ coefs, i64 N, int B,
                                T* __restrict__ gx, const i64* __restrict__ seg, int nseg) {
  const I i = (I)blockIdx.x * blockDim.x + threadIdx.x;
  if ((i64)i >= N * B) return;
  const I p = i / (I)B;
  if (mask && !mask[p]) return;
  const int b = (int)(i - p * (I)B);
  if (seg) {  // the coefficients of p's segment
    int a = 0, e = nseg;
    while (e - a > 1) {
      const int m = (a + e) >> 1;
      if (seg[m] <= (i64)p) a = m; else e = m;
    }
    coefs += (size_t)a * 2 * B;
  }
  const double x = (xc ? xc[b] : 0.0) + (double)x0[i];
  gx[i] += (T)(coefs[2 * b] + coefs[2 * b + 1] * x);
}

// ---- per-row constants of the fields -------------------------------------------
// Fields that the wavelet reads (maps, moduli) are stored as deviations from a
// per-row FP64 constant (its mean over the level's pixels): the wavelet is
// zero-mean, so a field of a large mean and small fluctuations would lose
// the fluctuations to the rounding of the mean in FP32.  The constant's
// contribution, constant x (row sums of the coefficients), is added in the
// wavelet's epilogue; the decimation rows sum to one and carry a constant
// unchanged.

// pixel-major field [N][R] (complex: the moduli): CTA = a pixel range,
// thread t adds the row t % R of its pixels; partials [CTA][R]
// |f[j]| of the complex value j of an interleaved array, one vector load
template <typename T>
__device__ __forceinline__ T cabs2(const T* f, i64 j) {
  const typename V2<T>::type v = reinterpret_cast<const typename V2<T>::type*>(f)[j];
  return zabs(v.x, v.y);
}

template <typename T, bool CPLX>
__global__ void k_means_pm(const T* __restrict__ f, i64 N, int R, i64 chunk, double* __restrict__ partials) {
  __shared__ double red[256];
  const int TR = (blockDim.x / R) * R;
  const int t = threadIdx.x;
  double a = 0.0;
  if (t < TR) {
    const i64 p0 = (i64)blockIdx.x * chunk, p1 = min(N, p0 + chunk);
    const i64 e1 = p1 * R;
    // four independent sums (more loads in flight), added in a fixed order
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    i64 i = p0 * R + t;
    for (; i + 3 * (i64)TR < e1; i += 4 * (i64)TR) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const i64 j = i + k * (i64)TR;
        q[k] += CPLX ? (double)cabs2(f, j) : (double)f[j];
      }
    }
    for (; i < e1; i += TR) q[0] += CPLX ? (double)cabs2(f, i) : (double)f[i];
    a = (q[0] + q[1]) + (q[2] + q[3]);
  }
  red[t] = a;
  __syncthreads();
  if (t < R) {
    double s = 0.0;
    for (int j = t; j < TR; j += R) s += red[j];
    partials[(i64)blockIdx.x * R + t] = s;
  }
}

// map-major rows [R][N]: grid (pixel ranges, R)
template <typename T>
__global__ void k_means_mm(const T* __restrict__ f, i64 N, i64 chunk, double* __restrict__ partials) {
  __shared__ double red[256];
  const int r = blockIdx.y, t = threadIdx.x;
  const i64 p0 = (i64)blockIdx.x * chunk, p1 = min(N, p0 + chunk);
  double q[4] = {0.0, 0.0, 0.0, 0.0};
  const T* fr = f + (i64)r * N;
  i64 p = p0 + t;
  for (; p + 3 * (i64)blockDim.x < p1; p += 4 * (i64)blockDim.x) {
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] += (double)fr[p + k * (i64)blockDim.x];
  }
  for (; p < p1; p += blockDim.x) q[0] += (double)fr[p];
  const double a = (q[0] + q[1]) + (q[2] + q[3]);
  red[t] = a;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (t < h) red[t] += red[t + h];
    __syncthreads();
  }
  if (t == 0) partials[(i64)blockIdx.x * gridDim.y + r] = red[0];
}

// one CTA per row: strided partial sums per thread, then a tree, all in a
// fixed order
__global__ void k_means_final(const double* __restrict__ partials, int nblk, int R, i64 N, double* __restrict__ out) {
  __shared__ double red[256];
  const int r = blockIdx.x, t = threadIdx.x;
  double a = 0.0;
  for (int k = t; k < nblk; k += blockDim.x) a += partials[(i64)k * R + r];
  red[t] = a;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (t < h) red[t] += red[t + h];
    __syncthreads();
  }
  if (t == 0) out[r] = red[0] / (double)N;
}

// moduli deviations: mod[p mod_pix + b mod_row + mod_off + l] = |z[p][b][l]| - cz[b][l]
// (I: the index type, 32-bit when N B L fits: a 64-bit division by a runtime
// value costs far more than the element's work)
template <typename T, typename I>
__global__ void k_mod_dev(const T* __restrict__ z, i64 N, int B, int L, const double* __restrict__ cz,
                          T* __restrict__ mod, int mod_pix, int mod_row, int mod_off) {
  // thread (pixel, map): the L = 4 orientations, contiguous in z and in mod
  typedef typename V2<T>::type T2;
  const I i = (I)blockIdx.x * blockDim.x + threadIdx.x;
  if ((i64)i >= N * B) return;
  const i64 p = (i64)(i / (I)B);
  const int b = (int)(i - (I)p * (I)B);
  const T2* zv = reinterpret_cast<const T2*>(z) + (i64)i * 4;
  T2 v[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) v[l] = zv[l];
  // |z| in the field type (z carries that type's rounding already); the
  // constant is subtracted in FP64 before the one rounding to T
  T o[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) o[l] = (T)((double)zabs(v[l].x, v[l].y) - cz[b * 4 + l]);
  store4(mod + p * mod_pix + (i64)b * mod_row + mod_off, o);
}

// constants of the branch rows (b, d, l) of level n from the moduli constants [level][B][L]
__global__ void k_branch_consts(const double* __restrict__ zc, int n, int B, int L, double* __restrict__ rc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int R = B * (n + 1) * L;
  if (i >= R) return;
  const int b = i / ((n + 1) * L), d = (i / L) % (n + 1), l = i % L;
  rc[i] = zc[((i64)d * B + b) * L + l];
}

template <typename Tin, typename Tout>
__global__ void k_convert(const Tin* __restrict__ in, Tout* __restrict__ out, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (Tout)in[i];
}

// [B][N] <-> [N][B] transposes of the level-0 maps at the boundary
// res (optional): the rounding residual of out, (x - sub) - out rounded to Tout
template <typename Tin, typename Tout, typename I>
__global__ void k_to_pixel_major(const Tin* __restrict__ in, Tout* __restrict__ out, i64 N, int B,
                                 const double* __restrict__ sub, Tout* __restrict__ res) {
  const I i = (I)blockIdx.x * blockDim.x + threadIdx.x;  // over N * B, output order
  if ((i64)i >= N * B) return;
  const I p = i / (I)B;
  const int b = (int)(i - p * (I)B);
  const Tin v = in[(i64)b * N + p];
  const double d = sub ? (double)v - sub[b] : (double)v;
  const Tout o = (Tout)d;
  out[i] = o;
  if (res) res[i] = (Tout)(d - (double)o);
}
// FP64 values as FP32 pairs: hi = x rounded, lo = (x - hi) rounded
__global__ void k_split_f64(const double* __restrict__ x, float* __restrict__ hi, float* __restrict__ lo, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float h = (float)x[i];
  hi[i] = h;
  lo[i] = (float)(x[i] - (double)h);
}
__global__ void k_join_f64(const float* __restrict__ hi, const float* __restrict__ lo, double* __restrict__ x, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = (double)hi[i] + (double)lo[i];
}
template <typename Tin, typename Tout, typename I>
__global__ void k_to_map_major(const Tin* __restrict__ in, Tout* __restrict__ out, i64 N, int B,
                               const double* __restrict__ add) {
  const I i = (I)blockIdx.x * blockDim.x + threadIdx.x;  // over B * N, output order
  if ((i64)i >= N * B) return;
  const int b = (int)(i / (I)N);
  const i64 p = (i64)(i - (I)b * (I)N);
  const Tin v = in[p * B + b];
  out[i] = add ? (Tout)((double)v + add[b]) : (Tout)v;
}

// CTA of 128 threads: blockDim.x = chunks of a row vector handled together
// (all of them up to 32), blockDim.y = stored rows.
inline dim3 cta_shape(int chunks) {
  int c = 1;
  while (c < chunks && c < 32) c *= 2;
  return dim3(c, 128 / c);
}

template <typename T, int NK, int RB>
void conv_forward_rb(const ConvOp& op, const T* x, int R, T* out, T* mod, int mod_pix, int mod_row, int mod_off,
                     const double* rc, cudaStream_t s) {
  const int chunks = R / RB;
  dim3 b = cta_shape(chunks);
  dim3 grid(nblocks(op.n_rep, b.y), (chunks + b.x - 1) / b.x);
  k_conv_fwd<T, NK, RB><<<grid, b, 0, s>>>(op.cell.as<int32_t>(), op.coef.as<T>(), op.S, op.n_rep, op.o2, x, R, out,
                                           mod, mod_pix, mod_row, mod_off, op.rowsum.as<T>(), rc);
}

template <typename T, int NK>
void conv_forward_nk(const ConvOp& op, const T* x, int R, T* out, T* mod, int mod_pix, int mod_row, int mod_off,
                     const double* rc, cudaStream_t s) {
  if (NK == 1 && R % 4 == 0) conv_forward_rb<T, NK, 4>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
  else if (R % 2 == 0) conv_forward_rb<T, NK, 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
  else conv_forward_rb<T, NK, 1>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
}

template <typename T, int NK, int RB>
void conv_adjoint_rb(const ConvOp& op, const T* gy, int R, T* gx, bool accumulate, cudaStream_t s) {
  const int chunks = R / RB;
  dim3 b = cta_shape(chunks);
  dim3 grid(nblocks(op.n_rep, b.y), (chunks + b.x - 1) / b.x);
  k_conv_adj<T, NK, RB><<<grid, b, 0, s>>>(op.tent.as<uint32_t>(), op.coefT.as<T>(), op.ST, op.tshift, op.n_rep,
                                           op.o2, gy, R, gx, accumulate ? 1 : 0);
}

template <typename T, int RB>
size_t adj_tiles_smem(const ConvOp& op) {
  return sizeof(T) * (4 * RB * (size_t)kAdjPlane + 4 * RB * (size_t)op.ncs) +
         sizeof(uint16_t) * (kAdjSC * kAdjTile + (size_t)op.ncs + 1);
}

// partials of every tile cell -> gx, k_adj_combine
template <typename T, int RB>
void adj_combine_rb(const ConvOp& op, int R, T* gx, bool accumulate, const AdjScratch& scr, cudaStream_t s) {
  const T* part = static_cast<const T*>(scr.part);
  const i64 n_cells = op.n_in / op.nk;
  const int chunks = R / RB;
  dim3 b = cta_shape(chunks);
  dim3 g2(nblocks(n_cells, b.y), (chunks + b.x - 1) / b.x);
  if (op.nk == 4)
    k_adj_combine<T, 4, RB><<<g2, b, 0, s>>>(op.coff.as<i64>(), op.clist.as<uint32_t>(), n_cells, op.o2, op.ncs, part,
                                             R, gx, accumulate ? 1 : 0);
  else
    k_adj_combine<T, 1, RB><<<g2, b, 0, s>>>(op.coff.as<i64>(), op.clist.as<uint32_t>(), n_cells, op.o2, op.ncs, part,
                                             R, gx, accumulate ? 1 : 0);
}

template <typename T, int RB>
size_t adjc_smem(const ConvOp& op) {
  return 2 * (size_t)adjc_sc<T>() * kAdjTile * (8 * sizeof(T) + sizeof(uint16_t)) +
         sizeof(T) * (size_t)op.ncs * 4 * RB;
}

template <typename T, int RB>
void conv_adjoint_tiles_rb(const ConvOp& op, const T* gy, int R, T* gx, bool accumulate, const AdjScratch& scr,
                           cudaStream_t s, int* err, const ModulusAdd<T>* madd) {
  if (op.colored) {
    if (!err) throw std::runtime_error("the coloured adjoint needs an error flag");
    const size_t smem = adjc_smem<T, RB>(op);
    allow_dynamic_smem(k_conv_adj_colored<T, RB>);
    dim3 grid((unsigned)(op.n_tiles * (R / RB)));
    k_conv_adj_colored<T, RB><<<grid, kAdjCThreads, smem, s>>>(
        op.lcell_t.as<uint16_t>(), op.coef.as<T>(), op.S, op.n_rep, op.o2, op.ncs, op.tile_ncells.as<int32_t>(), gy,
        R, static_cast<T*>(scr.part), op.tile_slots.as<int32_t>(), err, madd ? *madd : ModulusAdd<T>());
  } else {
    const size_t smem = adj_tiles_smem<T, RB>(op);
    if (smem > 48 * 1024)
      allow_dynamic_smem(k_conv_adj_tiles<T, RB>);
    dim3 grid((unsigned)(op.n_tiles * (R / RB)));
    k_conv_adj_tiles<T, RB><<<grid, kAdjTile, smem, s>>>(op.coef.as<T>(), op.S, op.n_rep, op.o2, op.nch, op.ncs,
                                                         op.tile_ncells.as<int32_t>(), op.tile_ent.as<uint16_t>(),
                                                         op.tile_off.as<uint16_t>(), gy, R,
                                                         static_cast<T*>(scr.part), op.tile_slots.as<int32_t>());
  }
  adj_combine_rb<T, RB>(op, R, gx, accumulate, scr, s);
}

template <typename T, int NK>
void conv_adjoint_nk(const ConvOp& op, const T* gy, int R, T* gx, bool accumulate, cudaStream_t s) {
  if (R % 2 == 0) conv_adjoint_rb<T, NK, 2>(op, gy, R, gx, accumulate, s);
  else conv_adjoint_rb<T, NK, 1>(op, gy, R, gx, accumulate, s);
}

template <typename Tin, typename Tout, typename Tw, int NK, int RB>
void ell_rb(const int32_t* col, const Tw* w, int W, i64 n_rep, int o2_out, int o2_in, const Tin* x, int x_pix,
            int x_outer, Tout* y, int y_pix, int y_outer, int R_outer, int R_inner, bool acc, cudaStream_t s) {
  const int chunks = R_outer * (R_inner / RB);
  dim3 b = cta_shape(chunks);
  dim3 grid(nblocks(n_rep, b.y), (chunks + b.x - 1) / b.x);
  k_ell<Tin, Tout, Tw, NK, RB><<<grid, b, 0, s>>>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix,
                                                 y_outer, R_outer, R_inner, acc ? 1 : 0);
}

template <typename Tin, typename Tout, typename Tw, int NK>
void ell_nk(const int32_t* col, const Tw* w, int W, i64 n_rep, int o2_out, int o2_in, const Tin* x, int x_pix,
            int x_outer, Tout* y, int y_pix, int y_outer, int R_outer, int R_inner, bool acc, cudaStream_t s,
            int rb) {
  if (rb == 1)
    ell_rb<Tin, Tout, Tw, NK, 1>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer,
                                 R_inner, acc, s);
  else if (rb == 2)
    ell_rb<Tin, Tout, Tw, NK, 2>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer,
                                 R_inner, acc, s);
  else if (rb == 4 || (R_inner % 4 == 0 && sizeof(Tin) == 4))
    ell_rb<Tin, Tout, Tw, NK, 4>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer,
                                 R_inner, acc, s);
  else if (R_inner % 2 == 0)
    ell_rb<Tin, Tout, Tw, NK, 2>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer,
                                 R_inner, acc, s);
  else
    ell_rb<Tin, Tout, Tw, NK, 1>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer,
                                 R_inner, acc, s);
}

template <typename Tin, typename Tout, typename Tw>
void dec_apply_w(const DecOp& op, bool transpose, const Tin* x, int x_pix, int x_outer, Tout* y, int y_pix,
                 int y_outer, int R_outer, int R_inner, bool accumulate, cudaStream_t s, int rb) {
  const int32_t* col = transpose ? op.tcol.as<int32_t>() : op.col.as<int32_t>();
  const Tw* w = transpose ? op.tw.as<Tw>() : op.w.as<Tw>();
  const int W = transpose ? op.WT : op.W;
  const i64 n_rep = transpose ? op.n_rep_in : op.n_rep_out;
  const int o2_out = transpose ? op.o2 : op.co2, o2_in = transpose ? op.co2 : op.o2;
  if (op.nk == 4)
    ell_nk<Tin, Tout, Tw, 4>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer, R_inner,
                             accumulate, s, rb);
  else
    ell_nk<Tin, Tout, Tw, 1>(col, w, W, n_rep, o2_out, o2_in, x, x_pix, x_outer, y, y_pix, y_outer, R_outer, R_inner,
                             accumulate, s, rb);
}

// stages of the tensor-core launches: as many (up to 4) as leave two CTAs per SM
inline size_t fwd_mma_planes(const ConvOp& op, int MT) { return 2 * sizeof(float) * 4 * op.m_pc * 4 * MT; }
inline int fwd_mma_stages(const ConvOp& op, int MT) {
  for (int ns = 4; ns > 2; --ns)
    if (ns * kMmaFwdStage + fwd_mma_planes(op, MT) <= 112 * 1024) return ns;
  return 2;
}
inline size_t fwd_mma_smem(const ConvOp& op, int MT) {
  return fwd_mma_stages(op, MT) * kMmaFwdStage + fwd_mma_planes(op, MT);
}
inline size_t adj_mma_sums(const ConvOp& op) { return sizeof(float) * kMmaAdjWarps * 16 * op.m_wl; }
inline int adj_mma_stages(const ConvOp& op) {
  for (int ns = 4; ns > 2; --ns)
    if (ns * kMmaAdjStage + adj_mma_sums(op) <= 112 * 1024) return ns;
  return 2;
}
inline size_t adj_mma_smem(const ConvOp& op) { return adj_mma_stages(op) * kMmaAdjStage + adj_mma_sums(op); }

template <int MT, int NS>
void conv_forward_mma_ns(const ConvOp& op, const float* x, int R, float* out, float* mod, int mod_pix, int mod_row,
                         int mod_off, int* err, const double* rc, cudaStream_t s) {
  allow_dynamic_smem(k_conv_fwd_mma<MT, NS>);
  dim3 grid((unsigned)(op.m_tiles * ((R + 4 * MT - 1) / (4 * MT))));
  k_conv_fwd_mma<MT, NS><<<grid, kMmaFwdThreads, fwd_mma_smem(op, MT), s>>>(
      op.m_lc.as<uint16_t>(), op.m_coef.as<float>(), op.m_S, op.n_rep, op.o2, op.m_cells.as<int32_t>(), op.m_pc,
      op.m_tch.as<int32_t>(), x, R, out, mod, mod_pix, mod_row, mod_off, err, op.rowsum.as<float>(), rc);
}

template <int MT>
void conv_forward_mma_mt(const ConvOp& op, const float* x, int R, float* out, float* mod, int mod_pix, int mod_row,
                         int mod_off, int* err, const double* rc, cudaStream_t s) {
  const int ns = fwd_mma_stages(op, MT);
  if (ns == 4) conv_forward_mma_ns<MT, 4>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err, rc, s);
  else if (ns == 3) conv_forward_mma_ns<MT, 3>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err, rc, s);
  else conv_forward_mma_ns<MT, 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err, rc, s);
}

template <int NS>
void conv_adjoint_mma_ns(const ConvOp& op, const float* gy, int R, const AdjScratch& scr, cudaStream_t s, int* err,
                         const ModulusAdd<float>* madd) {
  allow_dynamic_smem(k_conv_adj_mma<NS>);
  dim3 grid((unsigned)(op.m_tiles * ((R + 3) / 4)));
  k_conv_adj_mma<NS><<<grid, kMmaAdjThreads, adj_mma_smem(op), s>>>(
      op.m_wlc.as<uint8_t>(), op.m_coef.as<float>(), op.m_S, op.n_rep, op.o2, op.m_tch.as<int32_t>(),
      op.m_winv.as<uint8_t>(), op.m_pc, op.m_wl, gy, R, static_cast<float*>(scr.part), err,
      madd ? *madd : ModulusAdd<float>());
}

void conv_adjoint_mma(const ConvOp& op, const float* gy, int R, float* gx, bool accumulate, const AdjScratch& scr,
                      cudaStream_t s, int* err, const ModulusAdd<float>* madd) {
  const int ns = adj_mma_stages(op);
  if (ns == 4) conv_adjoint_mma_ns<4>(op, gy, R, scr, s, err, madd);
  else if (ns == 3) conv_adjoint_mma_ns<3>(op, gy, R, scr, s, err, madd);
  else conv_adjoint_mma_ns<2>(op, gy, R, scr, s, err, madd);
  if (R % 4 == 0) adj_combine_rb<float, 4>(op, R, gx, accumulate, scr, s);
  else if (R % 2 == 0) adj_combine_rb<float, 2>(op, R, gx, accumulate, scr, s);
  else adj_combine_rb<float, 1>(op, R, gx, accumulate, scr, s);
}

// cotangent rows per CTA: FP32 up to 4 (coloured) or 2; FP64 1 (the
// coloured kernel's 1024 threads hold 64 registers each)
inline int adj_rb(const ConvOp& op, size_t elem, int R) {
  if (elem != 4) return 1;
  if (op.colored && R % 4 == 0) return 4;
  return R % 2 == 0 ? 2 : 1;
}

}  // namespace

template <typename T, int RB>
size_t fwd_tiles_smem(const ConvOp& op) {
  const size_t stage = (size_t)fwd_sc<T>() * kAdjTile * (8 * sizeof(T) + sizeof(uint16_t));
  return fwd_stages<T>() * stage + sizeof(T) * 4 * (size_t)(op.max_tile_cells + 1 + 32) * RB;
}

template <typename T, int RB>
void conv_forward_tiles_rb(const ConvOp& op, const T* x, int R, T* out, T* mod, int mod_pix, int mod_row,
                           int mod_off, int* err, const double* rc, cudaStream_t s) {
  const size_t smem = fwd_tiles_smem<T, RB>(op);
  if (smem > 48 * 1024)
    allow_dynamic_smem(k_conv_fwd_tiles<T, RB>);
  dim3 grid((unsigned)(op.n_tiles * (R / RB)));
  k_conv_fwd_tiles<T, RB><<<grid, kFwdThreads, smem, s>>>(op.lcell_t.as<uint16_t>(), op.coef.as<T>(), op.S,
                                                          op.n_rep, op.o2, op.tile_cells.as<int32_t>(),
                                                          op.tile_ncells.as<int32_t>(), x, R, out, mod, mod_pix,
                                                          mod_row, mod_off, err, op.rowsum.as<T>(), rc,
                                                          op.tile_slots.as<int32_t>());
}

bool forward_tiles(const ConvOp& op, size_t elem, bool err);

template <typename T>
void conv_forward(const ConvOp& op, const T* x, int R, T* out, T* mod, int mod_pix, int mod_row, int mod_off,
                  cudaStream_t s, int* err, const double* rc, int rb) {
  if (rc && !op.rowsum.p) throw std::runtime_error("wavelet operator without row sums");
  if (op.mma) {
    if (sizeof(T) != 4 || !err) throw std::runtime_error("the tensor-core wavelet takes FP32 rows and an error flag");
    const int MT = R % 8 == 0 ? 2 : 1;
    if (rb && rb != 4 * MT) throw std::runtime_error("invalid wavelet tile height");
    const float* xf = reinterpret_cast<const float*>(x);
    float* of = reinterpret_cast<float*>(out);
    float* mf = reinterpret_cast<float*>(mod);
    if (MT == 2) conv_forward_mma_mt<2>(op, xf, R, of, mf, mod_pix, mod_row, mod_off, err, rc, s);
    else conv_forward_mma_mt<1>(op, xf, R, of, mf, mod_pix, mod_row, mod_off, err, rc, s);
    STL_CUDA(cudaGetLastError());
    return;
  }
  const std::vector<int> ok = conv_forward_choices(op, sizeof(T), R, err != nullptr);
  if (ok.empty() || (rb && std::find(ok.begin(), ok.end(), rb) == ok.end()))
    throw std::runtime_error("invalid wavelet tile height");
  if (!rb) rb = ok.back();  // default: the tallest tile
  if (forward_tiles(op, sizeof(T), err != nullptr)) {
    if (rb == 4) conv_forward_tiles_rb<T, sizeof(T) == 4 ? 4 : 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err,
                                                                  rc, s);
    else if (rb == 2) conv_forward_tiles_rb<T, 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err, rc, s);
    else conv_forward_tiles_rb<T, 1>(op, x, R, out, mod, mod_pix, mod_row, mod_off, err, rc, s);
  } else if (op.nk == 4) {
    if (rb == 2) conv_forward_rb<T, 4, 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
    else conv_forward_rb<T, 4, 1>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
  } else {
    if (rb == 4) conv_forward_rb<T, 1, 4>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
    else if (rb == 2) conv_forward_rb<T, 1, 2>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
    else conv_forward_rb<T, 1, 1>(op, x, R, out, mod, mod_pix, mod_row, mod_off, rc, s);
  }
  STL_CUDA(cudaGetLastError());
}

// the tiled forward serves full-sky operators with tile tables when its
// shared memory fits at the smallest tile height
bool forward_tiles(const ConvOp& op, size_t elem, bool err) {
  if (!err || op.nk != 4 || !op.adj_tiles || !op.lcell_t.p) return false;
  return (elem == 4 ? fwd_tiles_smem<float, 1>(op) : fwd_tiles_smem<double, 1>(op)) <= 220 * 1024;
}

// valid tile heights (rows of the field per thread) of a wavelet launch
std::vector<int> conv_forward_choices(const ConvOp& op, size_t elem, int R, bool err) {
  std::vector<int> v;
  if (op.mma) {  // one shape: M tiles of 16 (rotation, row) pairs, two per CTA when the rows allow
    if (elem == 4 && err) v.push_back(R % 8 == 0 ? 8 : 4);
    return v;
  }
  const bool tiles = forward_tiles(op, elem, err);
  for (int rb : {1, 2, 4}) {
    if (R % rb) continue;
    if (tiles) {
      if (rb == 4 && elem != 4) continue;
      const size_t sm = elem == 4 ? (rb == 4 ? fwd_tiles_smem<float, 4>(op) : rb == 2 ? fwd_tiles_smem<float, 2>(op)
                                                                                        : fwd_tiles_smem<float, 1>(op))
                                  : (rb == 2 ? fwd_tiles_smem<double, 2>(op) : fwd_tiles_smem<double, 1>(op));
      if (sm > 220 * 1024) continue;
    } else if (op.nk == 4 && rb == 4) {
      continue;
    }
    v.push_back(rb);
  }
  return v;
}

size_t adjoint_part_bytes(const ConvOp& op, size_t elem, int R) {
  if (op.mma_adj) return elem * (size_t)op.m_tiles * 4 * op.m_pc * R;
  if (!op.adj_tiles) return 0;
  return elem * (size_t)op.n_tiles * 4 * op.ncs * R;
}

bool adjoint_tiles_usable(const ConvOp& op, size_t elem, int R, const AdjScratch* scr) {
  if (op.mma_adj)
    return scr && elem == 4 && adjoint_part_bytes(op, elem, R) <= scr->capacity && adj_mma_smem(op) <= 227 * 1024;
  if (!scr || !op.adj_tiles || op.nk != 4) return false;
  if (adjoint_part_bytes(op, elem, R) > scr->capacity) return false;
  if (op.colored) return (elem == 4 ? adjc_smem<float, 4>(op) : adjc_smem<double, 1>(op)) <= 227 * 1024;
  const size_t smem = elem == 4 ? (adj_rb(op, elem, R) == 2 ? adj_tiles_smem<float, 2>(op) : adj_tiles_smem<float, 1>(op))
                                : adj_tiles_smem<double, 1>(op);
  return smem <= 200 * 1024;
}

bool conv_adjoint_fuses_modulus(const ConvOp& op, size_t elem, int R, const AdjScratch* scr, int* err) {
  return (op.colored || op.mma_adj) && err && adjoint_tiles_usable(op, elem, R, scr);
}

template <typename T>
void conv_adjoint(const ConvOp& op, const T* gy, int R, T* gx, bool accumulate, cudaStream_t s,
                  const AdjScratch* scr, int* err, const ModulusAdd<T>* madd, int rb) {
  if (madd && !conv_adjoint_fuses_modulus(op, sizeof(T), R, scr, err))
    throw std::runtime_error("this adjoint cannot add the modulus VJP");
  if (rb) {
    const std::vector<int> ok = conv_adjoint_choices(op, sizeof(T), R, scr);
    if (std::find(ok.begin(), ok.end(), rb) == ok.end()) throw std::runtime_error("invalid adjoint tile height");
  }
  if (op.mma_adj) {
    if (!adjoint_tiles_usable(op, sizeof(T), R, scr) || !err)
      throw std::runtime_error("the tensor-core adjoint needs FP32 rows, an error flag and tile scratch");
    conv_adjoint_mma(op, reinterpret_cast<const float*>(gy), R, reinterpret_cast<float*>(gx), accumulate, *scr, s,
                     err, reinterpret_cast<const ModulusAdd<float>*>(madd));
    STL_CUDA(cudaGetLastError());
    return;
  }
  if (adjoint_tiles_usable(op, sizeof(T), R, scr)) {
    if (!rb) rb = adj_rb(op, sizeof(T), R);
    if (rb == 4) conv_adjoint_tiles_rb<T, sizeof(T) == 4 ? 4 : 1>(op, gy, R, gx, accumulate, *scr, s, err, madd);
    else if (rb == 2) conv_adjoint_tiles_rb<T, sizeof(T) == 4 ? 2 : 1>(op, gy, R, gx, accumulate, *scr, s, err, madd);
    else conv_adjoint_tiles_rb<T, 1>(op, gy, R, gx, accumulate, *scr, s, err, madd);
  } else if (op.colored) {
    throw std::runtime_error("the coloured adjoint needs scratch for its tile partials");
  } else {
    if (!rb) rb = R % 2 == 0 ? 2 : 1;  // 4 rows per thread: more registers, fewer warps (measured slower)
    if (op.nk == 4) {
      if (rb == 2) conv_adjoint_rb<T, 4, 2>(op, gy, R, gx, accumulate, s);
      else conv_adjoint_rb<T, 4, 1>(op, gy, R, gx, accumulate, s);
    } else {
      if (rb == 4) conv_adjoint_rb<T, 1, sizeof(T) == 4 ? 4 : 2>(op, gy, R, gx, accumulate, s);
      else if (rb == 2) conv_adjoint_rb<T, 1, 2>(op, gy, R, gx, accumulate, s);
      else conv_adjoint_rb<T, 1, 1>(op, gy, R, gx, accumulate, s);
    }
  }
  STL_CUDA(cudaGetLastError());
}

// valid tile heights of an adjoint launch
std::vector<int> conv_adjoint_choices(const ConvOp& op, size_t elem, int R, const AdjScratch* scr) {
  std::vector<int> v;
  if (op.mma_adj) {
    if (adjoint_tiles_usable(op, elem, R, scr)) v.push_back(4);
    return v;
  }
  const bool tiles = adjoint_tiles_usable(op, elem, R, scr);
  for (int rb : {1, 2, 4}) {
    if (R % rb) continue;
    if (tiles) {
      if (elem != 4 && rb > 1) continue;
      if (!op.colored && rb == 4) continue;
      if (op.colored && elem == 4 &&
          (rb == 4 ? adjc_smem<float, 4>(op) : rb == 2 ? adjc_smem<float, 2>(op) : adjc_smem<float, 1>(op)) >
              227 * 1024)
        continue;
    } else if (rb == 4 && (op.nk == 4 || elem != 4)) {
      continue;
    }
    v.push_back(rb);
  }
  return v;
}

template <typename Tin, typename Tout>
void dec_apply(const DecOp& op, bool transpose, const Tin* x, int x_pix, int x_outer, Tout* y, int y_pix, int y_outer,
               int R_outer, int R_inner, bool accumulate, cudaStream_t s, int rb) {
  if (R_outer <= 0 || R_inner <= 0) return;
  if (rb) {
    const std::vector<int> ok = dec_choices(sizeof(Tin), R_inner);
    if (std::find(ok.begin(), ok.end(), rb) == ok.end()) throw std::runtime_error("invalid decimation tile height");
  }
  if (op.dtype == DType::F64)
    dec_apply_w<Tin, Tout, double>(op, transpose, x, x_pix, x_outer, y, y_pix, y_outer, R_outer, R_inner, accumulate,
                                   s, rb);
  else
    dec_apply_w<Tin, Tout, float>(op, transpose, x, x_pix, x_outer, y, y_pix, y_outer, R_outer, R_inner, accumulate,
                                  s, rb);
  STL_CUDA(cudaGetLastError());
}

// valid tile heights of a decimation launch
std::vector<int> dec_choices(size_t elem_in, int R_inner) {
  std::vector<int> v;
  for (int rb : {1, 2, 4})
    if (R_inner % rb == 0 && (rb < 4 || elem_in == 4)) v.push_back(rb);
  return v;
}

template <typename T>
void modulus_vjp_add(const T* z, const T* g, int g_pix, int g_row, T* gz, i64 N, int B, int L, cudaStream_t s) {
  const i64 n = N * B * L;
  k_modvjp<T><<<nblocks(n, 256), 256, 0, s>>>(z, g, g_pix, g_row, gz, N, B, L);
  STL_CUDA(cudaGetLastError());
}

ProductShape product_shape(int n, int L, int B, i64 N, size_t elem) {
  if (L != 4) throw std::runtime_error("the products are built for L = 4");
  if (B > 255) throw std::runtime_error("batch too large for the products kernel");
  ProductShape sh;
  sh.nd = n + 1;
  sh.K = sh.nd * L + 1;
  sh.L = L; sh.B = B; sh.N = N; sh.level0 = n == 0;
  const int nBB = sh.nd * (sh.nd + 1) / 2;
  sh.slots = nBB * 48 + sh.nd * 12 + 6;
  const int I = nBB + sh.nd + 1, R = B * I;
  sh.items = I;
  // roles (map, item) with a per-pixel cost: BB blocks 8, Bz blocks 3, the
  // per-pixel item 2; spread over chunks of at most kProdMaxWarps roles
  // (round robin by decreasing cost), replicated within a chunk in
  // proportion to cost
  auto cost = [&](int r) { const int it = r % I; return it < nBB ? 8 : (it < nBB + sh.nd ? 3 : 2); };
  std::vector<int> order(R);
  for (int r = 0; r < R; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b2) { return cost(a) > cost(b2); });
  sh.item_chunks = (R + kProdMaxWarps - 1) / kProdMaxWarps;
  std::vector<std::vector<int>> chunk_roles(sh.item_chunks);
  for (int k = 0; k < R; ++k) chunk_roles[k % sh.item_chunks].push_back(order[k]);
  std::vector<std::vector<int>> reps(sh.item_chunks);
  int W = 1;
  for (int zc = 0; zc < sh.item_chunks; ++zc) {
    auto& cr = chunk_roles[zc];
    std::sort(cr.begin(), cr.end());
    double total = 0.0;
    for (int r : cr) total += cost(r);
    auto& P = reps[zc];
    int sum = 0;
    for (int r : cr) {
      P.push_back(std::max(1, (int)std::lround(cost(r) * kProdMaxWarps / total)));
      sum += P.back();
    }
    while (sum > kProdMaxWarps) {
      int m = -1;
      for (int k = 0; k < (int)P.size(); ++k)
        if (P[k] > 1 && (m < 0 || P[k] > P[m])) m = k;
      --P[m];
      --sum;
    }
    W = std::max(W, sum);
  }
  sh.warps = W;
  sh.roles.assign((size_t)sh.item_chunks * W, -1);
  for (int zc = 0; zc < sh.item_chunks; ++zc) {
    int w = 0;
    for (size_t k = 0; k < chunk_roles[zc].size(); ++k)
      for (int rp = 0; rp < reps[zc][k]; ++rp)
        sh.roles[(size_t)zc * W + w++] = chunk_roles[zc][k] | (rp << 16) | (reps[zc][k] << 24);
  }
  // per pixel: operands and, at level 0, the maps; there the uniform chunks
  // and ranges are whole 16-byte units of the maps [N][B], and a stage
  // holds 16 bytes more (ranges of a range table start anywhere)
  const size_t op_bytes = (size_t)B * sh.K * L * 2 * elem, x_px = sh.level0 ? (size_t)B * elem : 0;
  const size_t px_bytes = op_bytes + x_px;
  const int align = sh.level0 ? 16 / (int)std::gcd((size_t)16, (size_t)B * elem) : 1;
  sh.px_chunk = (int)((kProdStageBytes - (sh.level0 ? 32 : 0)) / px_bytes) / align * align;
  if (sh.px_chunk < 1) throw std::runtime_error("a pixel's operands exceed a products stage");
  // one CTA per SM over (pixel ranges, role chunks); ranges of at least 4
  // pixel chunks
  const i64 want = std::max<i64>(1, (i64)148 / sh.item_chunks);
  const i64 most = std::max<i64>(1, N / (4 * (i64)sh.px_chunk));
  sh.blocks = (int)std::max<i64>(1, std::min(want, most));
  sh.chunk = ((N + sh.blocks - 1) / sh.blocks + align - 1) / align * align;
  const size_t stage = (size_t)sh.px_chunk * op_bytes + (sh.level0 ? ((sh.px_chunk * x_px + 15) & ~(size_t)15) + 16 : 0);
  sh.smem = std::max((size_t)kProdStages * stage, (size_t)W * 32 * 6 * sizeof(double));
  return sh;
}

// Forward ranges of about N / 296 pixels (2 per SM) and reverse ranges of
// at most 2048 pixels, split evenly inside every segment.
void segment_ranges(ProductShape& sh, const std::vector<i64>& seg) {
  if (seg.size() < 2 || seg.front() != 0 || seg.back() != sh.N) throw std::runtime_error("bad segment table");
  sh.nseg = (int)seg.size() - 1;
  const i64 fwd = std::max<i64>(1024, (sh.N + 295) / 296), rev = 2048;
  sh.blk.clear(); sh.rev_blk.clear(); sh.rev_seg.clear(); sh.seg_blk.clear();
  for (int k = 0; k < sh.nseg; ++k) {
    const i64 n = seg[k + 1] - seg[k];
    if (n <= 0) throw std::runtime_error("empty segment");
    const i64 nf = (n + fwd - 1) / fwd, nr = (n + rev - 1) / rev;
    sh.seg_blk.push_back((int32_t)sh.blk.size());
    for (i64 j = 0; j < nf; ++j) sh.blk.push_back(seg[k] + n * j / nf);
    for (i64 j = 0; j < nr; ++j) {
      sh.rev_blk.push_back(seg[k] + n * j / nr);
      sh.rev_seg.push_back(k);
    }
  }
  sh.blk.push_back(sh.N);
  sh.rev_blk.push_back(sh.N);
  sh.seg_blk.push_back((int32_t)sh.blk.size() - 1);
  if (sh.blk.size() - 1 > (size_t)INT32_MAX || sh.rev_blk.size() - 1 > (size_t)INT32_MAX)
    throw std::runtime_error("too many product ranges");
  sh.blocks = (int)sh.blk.size() - 1;
  sh.rev_blocks = (int)sh.rev_blk.size() - 1;
}

namespace {
// partials [blocks][B L][slots] -> sums [B L][slots] (per segment with a
// range table)
void reduce_partials(const ProductShape& sh, const double* partials, double* sums, cudaStream_t s) {
  const i64 total = (i64)sh.B * sh.L * sh.slots;
  const unsigned gx = (unsigned)std::min<i64>((total + 255) / 256, 1024);
  if (sh.d_seg_blk) {
    dim3 grid(gx, (unsigned)std::min(sh.nseg, 65535));
    k_reduce_segments<<<grid, 256, 0, s>>>(partials, sh.d_seg_blk, sh.nseg, sh.B * sh.L, sh.slots, sums,
                                           sh.seg_stride);
  } else {
    k_reduce_partials<<<gx, 256, 0, s>>>(partials, sh.blocks, sh.B * sh.L, sh.slots, sums);
  }
  STL_CUDA(cudaGetLastError());
}

template <typename T, int K>
void products_reverse_k(const ProductShape& sh, const T* z, const T* br, const T* M, const T* s1c,
                        const uint8_t* mask, bool accumulate, T* gz, T* gbr, cudaStream_t s) {
  // all maps in one CTA while their cotangent matrices fit in 48 KB
  const size_t per_map = (size_t)4 * K * K * 2 * sizeof(T);
  const int bs = (sh.B * per_map <= 48 * 1024 && 4 * sh.B <= kRevThreads) ? sh.B : 1;
  const size_t smem = bs * per_map;
  if (smem > 48 * 1024)
    allow_dynamic_smem(k_products_rev<T, K>);
  const int tpx = kRevThreads / (4 * bs) * (K <= 21 ? 2 : 1);  // pixels per CTA pass
  const i64 tiles = (sh.N + tpx - 1) / tpx;
  const unsigned gx = sh.d_rev_blk ? (unsigned)sh.rev_blocks
                                   : (unsigned)std::max<i64>(1, std::min<i64>(tiles, (i64)148 * 8 * bs / sh.B));
  dim3 grid(gx, sh.B / bs);
  k_products_rev<T, K><<<grid, kRevThreads, smem, s>>>(sh.N, sh.B, bs, z, br, M, s1c, mask, accumulate ? 1 : 0,
                                                       gz, gbr, sh.d_rev_blk, sh.d_rev_seg);
}
}  // namespace

template <typename T>
void products_forward(const ProductShape& sh, const T* z, const T* br, const T* x0, const T* x0r, const double* x0c,
                      const uint8_t* mask, double* partials, double* sums, int* err, cudaStream_t s, bool moments) {
  if (sh.level0 && !x0c) throw std::runtime_error("level-0 products need the map constants");
  const int L = sh.L, nd = sh.nd;
  if (!sh.d_roles) throw std::runtime_error("products role table not on the device");
  // levels 0 and 1 without variances: the register-resident kernel
  if (!moments && (sh.nd == 1 || sh.nd == 2) && 32 % (4 * sh.B) == 0 && (!sh.level0 || x0)) {
    if (sh.nd == 1) products0_launch<T, 1>(sh, z, br, x0, x0r, x0c, mask, partials, s);
    else products0_launch<T, 2>(sh, z, br, x0, x0r, x0c, mask, partials, s);
    reduce_partials(sh, partials, sums, s);
    return;
  }
  auto kern = moments ? k_products<T, true> : k_products<T, false>;
  if (sh.smem > 48 * 1024)
    allow_dynamic_smem(kern);
  dim3 grid(sh.blocks, 1, sh.item_chunks);
  kern<<<grid, 32 * sh.warps, sh.smem, s>>>(nd, sh.N, sh.B, z, br, sh.level0 ? x0 : nullptr, sh.slots, sh.d_roles,
                                             sh.warps, sh.px_chunk, sh.chunk, partials, err, x0c, mask, sh.d_blk,
                                             sh.level0 ? x0r : nullptr);
  STL_CUDA(cudaGetLastError());
  reduce_partials(sh, partials, sums, s);
}

template <typename T>
void products_reverse(const ProductShape& sh, const T* z, const T* br, const T* M, const T* s1c,
                      const uint8_t* mask, bool accumulate, T* gz, T* gbr, cudaStream_t s) {
  switch (sh.nd) {
    case 1: products_reverse_k<T, 5>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 2: products_reverse_k<T, 9>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 3: products_reverse_k<T, 13>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 4: products_reverse_k<T, 17>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 5: products_reverse_k<T, 21>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 6: products_reverse_k<T, 25>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 7: products_reverse_k<T, 29>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 8: products_reverse_k<T, 33>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 9: products_reverse_k<T, 37>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    case 10: products_reverse_k<T, 41>(sh, z, br, M, s1c, mask, accumulate, gz, gbr, s); break;
    default: throw std::runtime_error("more levels than the products are built for (10)");
  }
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void mean_var_grad(const T* x0, const double* xc, const uint8_t* mask, const double* coefs, int B, i64 N, T* gx,
                   cudaStream_t s, const i64* seg, int nseg) {
  if (N * B < ((i64)1 << 31))
    k_mean_var_grad<T, uint32_t><<<nblocks(N * B, 256), 256, 0, s>>>(x0, xc, mask, coefs, N, B, gx, seg, nseg);
  else k_mean_var_grad<T, i64><<<nblocks(N * B, 256), 256, 0, s>>>(x0, xc, mask, coefs, N, B, gx, seg, nseg);
  STL_CUDA(cudaGetLastError());
}

// ---- coefficients <-> sums ------------------------------------------------
// The arithmetic below is that of a plain sequential FP64 loop: products and
// sums rounded one by one (no fused multiply-add), so the results do not
// depend on the device.
__global__ void k_assemble(const double* __restrict__ sums, size_t mstride, const PlanSlots* __restrict__ plan,
                           int np, const double* __restrict__ counts, int levels, int B, int K,
                           double* __restrict__ values, double* __restrict__ var) {
  const i64 total = (i64)B * K * np;
  for (i64 o = (i64)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += (i64)gridDim.x * blockDim.x) {
    const int i = (int)(o % np);
    const i64 bk = o / np;
    const int k = (int)(bk % K), b = (int)(bk / K);
    const PlanSlots p = plan[i];
    const double* row = sums + (size_t)k * mstride + p.base + (i64)b * p.stride;
    const double N = counts[(size_t)k * levels + p.level];
    const double vr = row[p.re] / N, vi = p.im >= 0 ? (p.conj ? -row[p.im] : row[p.im]) / N : 0.0;
    values[2 * o] = vr;
    values[2 * o + 1] = vi;
    if (var) {
      const double m2 = __dadd_rn(__dmul_rn(vr, vr), __dmul_rn(vi, vi));
      var[o] = fmax(__dsub_rn(row[p.second] / N, m2), 0.0);
    }
  }
}

__device__ __forceinline__ void add_source(const double* g, int mode, double N, double& ar, double& ai) {
  if (mode == 2) {
    ar = __dadd_rn(ar, __dmul_rn(2.0, g[0]) / N);
  } else {
    ar = __dadd_rn(ar, g[0] / N);
    ai = __dadd_rn(ai, (mode ? -g[1] : g[1]) / N);
  }
}

template <typename U>
__global__ void k_build_cot(const double* __restrict__ cot, int np, int B, int K, const double* __restrict__ counts,
                            int levels, int n, int Kd, int L, const CotSources* __restrict__ src,
                            const CotSources* __restrict__ s1src, U* __restrict__ M, U* __restrict__ s1,
                            int s1_complex) {
  const int E = L * Kd * Kd, per = E + L;  // matrix entries, then the S1 scales, of one (k, b)
  const i64 total = (i64)K * B * per;
  for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (i64)gridDim.x * blockDim.x) {
    const int e = (int)(t % per);
    const i64 kb = t / per;  // k B + b
    const int k = (int)(kb / B), b = (int)(kb % B);
    const CotSources c = e < E ? src[e] : s1src[e - E];
    const double N = counts[(size_t)k * levels + n];
    const double* g = cot + 2 * ((i64)b * K + k) * np;
    double ar = 0.0, ai = 0.0;
    if (c.i0 >= 0) add_source(g + 2 * (i64)c.i0, c.m0, N, ar, ai);
    if (c.i1 >= 0) add_source(g + 2 * (i64)c.i1, c.m1, N, ar, ai);
    if (e < E) {
      U* m = M + 2 * (kb * E + e);
      m[0] = (U)ar;
      m[1] = (U)ai;
    } else if (s1_complex) {
      s1[2 * (kb * L + (e - E))] = (U)ar;
      s1[2 * (kb * L + (e - E)) + 1] = (U)ai;
    } else {
      s1[kb * L + (e - E)] = (U)ar;
    }
  }
}

__global__ void k_build_mean_var(const double* __restrict__ cot, int np, int B, int K,
                                 const double* __restrict__ counts, int levels, int i_mean, int i_var,
                                 double* __restrict__ mv) {
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (i64)K * B) return;
  const int k = (int)(t / B), b = (int)(t % B);
  const double N = counts[(size_t)k * levels];
  const double* g = cot + 2 * ((i64)b * K + k) * np;
  double a = 0.0, v = 0.0;
  if (i_mean >= 0) a = __dadd_rn(a, g[2 * (i64)i_mean] / N);
  if (i_var >= 0) v = __dadd_rn(v, __dmul_rn(2.0, g[2 * (i64)i_var]) / N);
  mv[2 * t] = a;
  mv[2 * t + 1] = v;
}

constexpr int kObjThreads = 1024;
__global__ void __launch_bounds__(kObjThreads) k_objective(const double* __restrict__ v, const double* __restrict__ t,
                                                           const double* __restrict__ w, i64 nv, int np,
                                                           double* __restrict__ cot, double* __restrict__ loss) {
  __shared__ double red[kObjThreads];
  const i64 chunk = (nv + kObjThreads - 1) / kObjThreads;
  const i64 lo = (i64)threadIdx.x * chunk, hi = min(nv, lo + chunk);
  double acc = 0.0;
  for (i64 o = lo; o < hi; ++o) {
    const double ww = w ? w[o % np] : 1.0;
    const double rr = __dsub_rn(v[2 * o], t[2 * o]), ri = __dsub_rn(v[2 * o + 1], t[2 * o + 1]);
    acc = __dadd_rn(acc, __dmul_rn(ww, __dadd_rn(__dmul_rn(rr, rr), __dmul_rn(ri, ri))));
    cot[2 * o] = __dmul_rn(__dmul_rn(2.0, ww), rr);
    cot[2 * o + 1] = __dmul_rn(__dmul_rn(2.0, ww), ri);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kObjThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0];
}

void objective_terms(const double* values, const double* target, const double* weights, i64 nv, int np,
                     double* cot, double* loss, cudaStream_t s) {
  k_objective<<<1, kObjThreads, 0, s>>>(values, target, weights, nv, np, cot, loss);
  STL_CUDA(cudaGetLastError());
}

void assemble_values(const double* sums, size_t mask_stride, const PlanSlots* plan, int np, const double* counts,
                     int levels, int B, int K, double* values, double* var, cudaStream_t s) {
  const i64 total = (i64)B * K * np;
  k_assemble<<<(unsigned)std::max<i64>(1, std::min<i64>(nblocks(total, 256), 148 * 16)), 256, 0, s>>>(
      sums, mask_stride, plan, np, counts, levels, B, K, values, var);
  STL_CUDA(cudaGetLastError());
}

template <typename U>
void build_cotangents(const double* cot, int np, int B, int K, const double* counts, int levels, int n, int Kd,
                      int L, const CotSources* src, const CotSources* s1src, U* M, U* s1, cudaStream_t s,
                      bool s1_complex) {
  const i64 total = (i64)K * B * (L * Kd * Kd + L);
  k_build_cot<U><<<(unsigned)std::max<i64>(1, std::min<i64>(nblocks(total, 256), 148 * 16)), 256, 0, s>>>(
      cot, np, B, K, counts, levels, n, Kd, L, src, s1src, M, s1, s1_complex ? 1 : 0);
  STL_CUDA(cudaGetLastError());
}

void build_mean_var(const double* cot, int np, int B, int K, const double* counts, int levels, int i_mean, int i_var,
                    double* mv, cudaStream_t s) {
  k_build_mean_var<<<nblocks((i64)K * B, 256), 256, 0, s>>>(cot, np, B, K, counts, levels, i_mean, i_var, mv);
  STL_CUDA(cudaGetLastError());
}

// ---- cross terms of two channels ------------------------------------------
// Maps come in channel pairs (map 2 b + c).  Per pixel, batch entry b and
// gauge l3 the operand vector of channel c is v_c = (branches (d, l1) of
// Br[p][2 b + c][.][l3], then z[p][2 b + c][l3]), K values.  The cross sums
// of a level are, per (b, l3), the K x K block G[r][q] = sum_p v_0[r]
// conj(v_1[q]) (every S2, S3 and S4 cross term is an entry of G or the
// conjugate of one), the sum of rn(z_0) conj(rn(z_1)), rn(z) = z / sqrt(|z| +
// 1e-8) (the cross S1, engine.rs:29-33, 1201-1206), and with moments the sums
// of the squared moduli of those terms.  Layout per (b, l3), xslots = 3 K^2 +
// 3 doubles: G (re, im) at 2 (r K + q), the S1 term at 2 K^2, the second
// sums of G at 2 K^2 + 2 + r K + q and of the S1 term at 3 K^2 + 2.
constexpr int kCrossThreads = 256;
// pixels staged at a time: as many as 48 KB hold (both channels, K + 1 values,
// FP64, with moduli 24 bytes a value), 16 to 256
inline int cross_chunk(int K, bool moduli = false) {
  return std::max(16, std::min(256, (48 * 1024) / (2 * (K + 1) * (moduli ? 24 : 16))));
}
constexpr int kCrossMaxEnt = 8;  // entries per thread (K^2 + 1 <= 8 x 256)
constexpr int kStageLoads = 4;   // operand loads a staging thread keeps in flight


__device__ __forceinline__ double2 cmul_conj(double2 a, double2 b) {  // a conj(b), products rounded one by one
  return make_double2(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y)));
}
// rn(z) = z / sqrt(|z| + 1e-8) as z times one reciprocal square root (a few
// ulp from the quotient; the operands are far from overflow, so |z| needs no
// hypot scaling)
__device__ __forceinline__ double2 root_normalise(double2 z) {
  const double inv = rsqrt(sqrt(fma(z.x, z.x, z.y * z.y)) + 1e-8);
  return make_double2(z.x * inv, z.y * inv);
}

// d rn(z)^H-side cotangent: g / sqrt(r + eps) - (Re(conj(g) z) / 2 / (r +
// eps)^1.5) z / |z| (|z| taken as 1 at z = 0), engine.rs:35-46
// with inv = (|z| + eps)^-1/2: (r + eps)^-1.5 = inv^3, and z / |z| takes one reciprocal
__device__ __forceinline__ double2 root_modulus_vjp(double2 z, double2 g) {
  const double r = sqrt(fma(z.x, z.x, z.y * z.y));
  const double radial = fma(g.x, z.x, g.y * z.y);
  const double inv = rsqrt(r + 1e-8);
  const double c = 0.5 * radial * (inv * inv * inv) * (1.0 / (r == 0.0 ? 1.0 : r));
  return make_double2(fma(g.x, inv, -c * z.x), fma(g.y, inv, -c * z.y));
}

// stage the chunk's operand vectors of both channels as FP64, K + 1 values a
// channel: sv[j][c][i], i < K the operands, i = K the channel's S1 factor,
// computed here once per pixel and channel in a pass of its own (one (j, c) a
// thread, the same instructions for both channels) instead of in the thread
// that owns the S1 term: rn(z_c) for the sums, and for the VJP (REV) the
// rn-VJP of the S1 term with cotangent sc, rn-VJP(z_c, sc_c rn(z_{1-c})), sc_0
// = sc and sc_1 = conj(sc).  Pixels outside the mask stage zeros.  With nv,
// the squared moduli of the staged values go to nv[j][c][i] as well.
template <typename T, bool REV>
__device__ __forceinline__ void cross_stage(double2* sv, double* nv, i64 p0, int np, int K, int Bm, int b, int l3,
                                            const T* __restrict__ z, const T* __restrict__ br,
                                            const uint8_t* __restrict__ mask, double2 sc) {
  typedef typename V2<T>::type T2;
  const T2* zv = reinterpret_cast<const T2*>(z);
  const T2* bv = reinterpret_cast<const T2*>(br);
  const int K1 = K - 1, KS = K + 1, L = 4, n = np * 2 * K;
  // kStageLoads independent loads in flight a thread (the pixel's mask byte
  // among them, applied after the loads return: every load is in range)
  for (int t0 = threadIdx.x; t0 < n; t0 += kStageLoads * (int)blockDim.x) {
    T2 w[kStageLoads];
    int at[kStageLoads];
    uint8_t on[kStageLoads];
#pragma unroll
    for (int u = 0; u < kStageLoads; ++u) {
      const int t = t0 + u * (int)blockDim.x;
      at[u] = -1;
      if (t < n) {
        const int j = t / (2 * K), rem = t - j * 2 * K, c = rem / K, i = rem - c * K;
        const i64 p = p0 + j;
        const i64 m = 2 * b + c;
        w[u] = i < K1 ? bv[((p * Bm + m) * K1 + i) * L + l3] : zv[(p * Bm + m) * L + l3];
        on[u] = mask ? mask[p] : 1;
        at[u] = j * 2 * KS + c * KS + i;
      }
    }
#pragma unroll
    for (int u = 0; u < kStageLoads; ++u) {
      if (at[u] < 0) continue;
      const double2 v = on[u] ? make_double2((double)w[u].x, (double)w[u].y) : make_double2(0.0, 0.0);
      sv[at[u]] = v;
      if (nv) nv[at[u]] = fma(v.x, v.x, v.y * v.y);
    }
  }
  for (int t = threadIdx.x; t < np * 2; t += blockDim.x) {
    const int j = t >> 1, c = t & 1;
    const i64 p = p0 + j;
    double2 v = make_double2(0.0, 0.0);
    if (!mask || mask[p]) {
      const T2 w = zv[(p * Bm + 2 * b + c) * L + l3];
      const double2 zs = make_double2((double)w.x, (double)w.y);
      if (!REV) {
        v = root_normalise(zs);
      } else {
        const T2 wo = zv[(p * Bm + 2 * b + 1 - c) * L + l3];
        const double2 r = root_normalise(make_double2((double)wo.x, (double)wo.y));
        const double sy = c ? -sc.y : sc.y;
        v = root_modulus_vjp(zs, make_double2(__dsub_rn(__dmul_rn(sc.x, r.x), __dmul_rn(sy, r.y)),
                                              __dadd_rn(__dmul_rn(sc.x, r.y), __dmul_rn(sy, r.x))));
      }
    }
    sv[(size_t)j * 2 * KS + c * KS + K] = v;
    if (nv) nv[(size_t)j * 2 * KS + c * KS + K] = fma(v.x, v.x, v.y * v.y);
  }
}

// grid: pixel ranges x (B L), (b, l3) fastest so that the four gauges of a
// range, which share the operands' 32-byte sectors, run together; partials
// [range][b][l3][xslots]
// NENT: entries a thread holds (the power of two at or above ceil((K^2 + 1) /
// 256)), so that a thread's sums take 3 NENT register pairs, not 3 kCrossMaxEnt.
// The products go through FMAs, and the second sums use |a conj(b)|^2 = |a|^2
// |b|^2 with the staged squared moduli.
template <typename T, bool MOM, int NENT>
__global__ void __launch_bounds__(kCrossThreads) k_cross_fwd(i64 N, int K, int Bm, const T* __restrict__ z,
                                                             const T* __restrict__ br,
                                                             const uint8_t* __restrict__ mask, i64 chunk, int PC,
                                                             double* __restrict__ partials) {
  extern __shared__ __align__(16) double2 sv[];  // [PC][2][K + 1], (MOM) moduli [PC][2][K + 1]; then the lane sums
  const int B = Bm / 2, bl = (int)(blockIdx.x % (unsigned)(B * 4)), b = bl / 4, l3 = bl % 4;
  const i64 range = blockIdx.x / (unsigned)(B * 4);
  const int E = K * K + 1, NE = min(E, kCrossThreads), Q = kCrossThreads / NE;
  const int t = threadIdx.x, q = t / NE, e0 = t - q * NE;
  const int nent = (E - e0 + NE - 1) / NE;  // entries of this thread: e0, e0 + NE, ...
  const bool lane = q < Q;
  const int KS = K + 1;
  double* nv = MOM ? reinterpret_cast<double*>(sv + (size_t)PC * 2 * KS) : nullptr;
  double acc[NENT][3];
  int ri[NENT], qi[NENT];  // the entry's operands: (r, q) of G, (K, K) for the S1 term
#pragma unroll
  for (int s = 0; s < NENT; ++s) {
    acc[s][0] = acc[s][1] = acc[s][2] = 0.0;
    const int e = e0 + s * NE;
    ri[s] = e < K * K ? e / K : K;
    qi[s] = e < K * K ? e - (e / K) * K : K;
  }
  const i64 P0 = range * chunk, P1 = min(N, P0 + chunk);
  for (i64 pc = P0; pc < P1; pc += PC) {
    const int np = (int)min((i64)PC, P1 - pc);
    __syncthreads();
    cross_stage<T, false>(sv, nv, pc, np, K, Bm, b, l3, z, br, mask, make_double2(0.0, 0.0));
    __syncthreads();
    if (!lane) continue;
    for (int j = q; j < np; j += Q) {
      const double2* v0 = sv + (size_t)j * 2 * KS;
      const double2* v1 = v0 + KS;
#pragma unroll
      for (int s = 0; s < NENT; ++s) {  // static indices: the sums stay in registers
        if (s >= nent) continue;
        const double2 a = v0[ri[s]], c = v1[qi[s]];
        acc[s][0] = fma(a.y, c.y, fma(a.x, c.x, acc[s][0]));
        acc[s][1] = fma(-a.x, c.y, fma(a.y, c.x, acc[s][1]));
        if (MOM) {
          const double* n0 = nv + (size_t)j * 2 * KS;
          acc[s][2] = fma(n0[ri[s]], n0[KS + qi[s]], acc[s][2]);
        }
      }
    }
  }
  // lanes of an entry added in lane order (through the staging memory)
  __syncthreads();
  double* red = reinterpret_cast<double*>(sv);  // [Q][NE][NENT][3]
  if (lane) {
#pragma unroll
    for (int s = 0; s < NENT; ++s)
      if (s < nent)
#pragma unroll
        for (int k = 0; k < 3; ++k) red[(((size_t)q * NE + e0) * NENT + s) * 3 + k] = acc[s][k];
  }
  __syncthreads();
  if (q != 0) return;
  double* out = partials + ((range * B + b) * 4 + l3) * cross_slots(K);
  for (int s = 0; s < nent; ++s) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int r = 0; r < Q; ++r)
      for (int k = 0; k < 3; ++k) v[k] = __dadd_rn(v[k], red[(((size_t)r * NE + e0) * NENT + s) * 3 + k]);
    const int e = e0 + s * NE;
    const int at = e < K * K ? 2 * e : 2 * K * K;
    out[at] = v[0];
    out[at + 1] = v[1];
    out[e < K * K ? 2 * K * K + 2 + e : 3 * K * K + 2] = v[2];
  }
}

// grid: pixel ranges x (B L), (b, l3) fastest; thread (entry i, pixel lane): the cotangents of
// entry i of both channels, gv_0 = M v_1 and gv_1 = M^H v_0 (M [K][K]: the
// cotangents of G), plus through rn the cross S1's (cotangent s):
// rn-VJP(z_0, s rn(z_1)) and rn-VJP(z_1, conj(s) rn(z_0)).  Pixels outside the
// mask get zero (accumulate: nothing).
template <typename T>
__global__ void __launch_bounds__(kCrossThreads) k_cross_rev(i64 N, int K, int Bm, const T* __restrict__ z,
                                                             const T* __restrict__ br, const T* __restrict__ M,
                                                             const T* __restrict__ s1, const uint8_t* __restrict__ mask,
                                                             int accumulate, i64 chunk, int PC, T* __restrict__ gz,
                                                             T* __restrict__ gbr) {
  typedef typename V2<T>::type T2;
  extern __shared__ __align__(16) double2 sm[];  // M [K][K], then [PC][2][K + 1]
  const int B = Bm / 2, bl = (int)(blockIdx.x % (unsigned)(B * 4)), b = bl / 4, l3 = bl % 4, L = 4, K1 = K - 1;
  const i64 range = blockIdx.x / (unsigned)(B * 4);
  const int KS = K + 1;
  double2* mk = sm;
  double2* sv = sm + K * K;
  const T2* Mb = reinterpret_cast<const T2*>(M) + ((i64)b * L + l3) * K * K;
  for (int i = threadIdx.x; i < K * K; i += blockDim.x) mk[i] = make_double2((double)Mb[i].x, (double)Mb[i].y);
  const T2 s1v = reinterpret_cast<const T2*>(s1)[(i64)b * L + l3];
  const double2 sc = make_double2((double)s1v.x, (double)s1v.y);
  const int Q = kCrossThreads / K, q = threadIdx.x / K, i = threadIdx.x - q * K;
  const bool lane = q < Q;
  T2* gzv = reinterpret_cast<T2*>(gz);
  T2* gbv = reinterpret_cast<T2*>(gbr);
  const i64 P0 = range * chunk, P1 = min(N, P0 + chunk);
  for (i64 pc = P0; pc < P1; pc += PC) {
    const int np = (int)min((i64)PC, P1 - pc);
    __syncthreads();
    cross_stage<T, true>(sv, nullptr, pc, np, K, Bm, b, l3, z, br, mask, sc);
    __syncthreads();
    if (!lane) continue;
    // two pixels a step (j and j + Q; the second repeats the first past the
    // chunk's end and is not written), so each entry of M loaded serves both;
    // pixels outside the mask staged zeros, so their cotangents come out zero
    for (int j = q; j < np; j += 2 * Q) {
      const int jb = j + Q < np ? j + Q : j;
      const double2* v0[2] = {sv + (size_t)j * 2 * KS, sv + (size_t)jb * 2 * KS};
      double2 g[2][2];
#pragma unroll
      for (int u = 0; u < 2; ++u) g[u][0] = g[u][1] = make_double2(0.0, 0.0);
      for (int k = 0; k < K; ++k) {
        const double2 a = mk[i * K + k], c = mk[k * K + i];
#pragma unroll
        for (int u = 0; u < 2; ++u) {  // g_0 += M[i][k] v_1[k]; g_1 += conj(M[k][i]) v_0[k]
          const double2 w0 = v0[u][k], w1 = v0[u][KS + k];
          g[u][0].x = fma(a.x, w1.x, fma(-a.y, w1.y, g[u][0].x));
          g[u][0].y = fma(a.x, w1.y, fma(a.y, w1.x, g[u][0].y));
          g[u][1].x = fma(c.x, w0.x, fma(c.y, w0.y, g[u][1].x));
          g[u][1].y = fma(c.x, w0.y, fma(-c.y, w0.x, g[u][1].y));
        }
      }
      for (int u = 0; u < 2; ++u) {
        if (u == 1 && jb == j) break;
        const int jj = u ? jb : j;
        const i64 p = pc + jj;
        if (accumulate && mask && !mask[p]) continue;
        if (i == K1) {  // the cross S1 through rn, staged
          g[u][0].x += v0[u][K].x; g[u][0].y += v0[u][K].y;
          g[u][1].x += v0[u][KS + K].x; g[u][1].y += v0[u][KS + K].y;
        }
        for (int c = 0; c < 2; ++c) {
          const double2 gv = g[u][c];
          const i64 m = 2 * b + c;
          T2* dst = i < K1 ? gbv + ((p * Bm + m) * K1 + i) * L + l3 : gzv + (p * Bm + m) * L + l3;
          T2 o;
          o.x = (T)gv.x;
          o.y = (T)gv.y;
          if (accumulate) {
            const T2 prev = *dst;
            o.x += prev.x;
            o.y += prev.y;
          }
          *dst = o;
        }
      }
    }
  }
}

// ---- the forward with the four gauges in one CTA (levels with K <= kCross4MaxK) ---
// The operands of a (pixel, map, operand) are the 4 gauges' complex values in
// one run (32 bytes in FP32): a CTA that takes all four gauges of a pixel range
// loads whole sectors, where one CTA a gauge used a quarter of each (the
// products of the nside 1024 bench: 17.5 -> 14.3 ms; the same form of the VJP
// was slower, 22.4 -> 27.2 ms, and is not used).  Staged values
// sv[j][g][c][i] (i < K the operands, i = K the S1 factor), FP64.
// levels 0-2 (K = 5, 9, 13): the deeper levels have too few pixel ranges to
// fill the GPU with a quarter of the CTAs (measured slower at K = 17, 21)
constexpr int kCross4MaxK = 13;

template <typename T>
__device__ __forceinline__ void load_gauges(const typename V2<T>::type* src, double2 v[4]) {
  if (sizeof(T) == 4) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(src)), c = __ldg(reinterpret_cast<const float4*>(src) + 1);
    v[0] = make_double2(a.x, a.y); v[1] = make_double2(a.z, a.w);
    v[2] = make_double2(c.x, c.y); v[3] = make_double2(c.z, c.w);
  } else {
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const double2 a = __ldg(reinterpret_cast<const double2*>(src) + g);
      v[g] = a;
    }
  }
}

template <typename T>
__device__ __forceinline__ void cross_stage4(double2* sv, double* nv, i64 p0, int np, int K, int Bm, int b,
                                             const T* __restrict__ z, const T* __restrict__ br,
                                             const uint8_t* __restrict__ mask) {
  typedef typename V2<T>::type T2;
  const T2* zv = reinterpret_cast<const T2*>(z);
  const T2* bv = reinterpret_cast<const T2*>(br);
  const int K1 = K - 1, KS = K + 1, L = 4, n = np * 2 * K;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {  // one (pixel, channel, operand) a thread
    const int j = t / (2 * K), rem = t - j * 2 * K, c = rem / K, i = rem - c * K;
    const i64 p = p0 + j, m = 2 * b + c;
    double2 v[4];
    load_gauges<T>(i < K1 ? bv + ((p * Bm + m) * K1 + i) * L : zv + (p * Bm + m) * L, v);
    const bool on = !mask || mask[p];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const double2 w = on ? v[g] : make_double2(0.0, 0.0);
      const int at = ((j * 4 + g) * 2 + c) * KS + i;
      sv[at] = w;
      if (nv) nv[at] = fma(w.x, w.x, w.y * w.y);
    }
  }
  for (int t = threadIdx.x; t < np * 8; t += blockDim.x) {  // rn(z) of (pixel, gauge, channel): the S1 factor
    const int j = t >> 3, g = (t >> 1) & 3, c = t & 1;
    const i64 p = p0 + j;
    double2 v = make_double2(0.0, 0.0);
    if (!mask || mask[p]) {
      const T2 w = zv[(p * Bm + 2 * b + c) * L + g];
      v = root_normalise(make_double2((double)w.x, (double)w.y));
    }
    const int at = ((j * 4 + g) * 2 + c) * KS + K;
    sv[at] = v;
    if (nv) nv[at] = fma(v.x, v.x, v.y * v.y);
  }
}

// forward: grid pixel ranges x B; thread (entry e of the 4 (K^2 + 1) of the
// four gauges, pixel lane q); partials [range][b][l3][xslots] as k_cross_fwd
template <typename T, bool MOM, int NENT>
__global__ void __launch_bounds__(kCrossThreads) k_cross_fwd4(i64 N, int K, int Bm, const T* __restrict__ z,
                                                              const T* __restrict__ br,
                                                              const uint8_t* __restrict__ mask, i64 chunk, int PC,
                                                              double* __restrict__ partials) {
  extern __shared__ __align__(16) double2 sv[];  // [PC][4][2][K + 1], (MOM) moduli; then the lane sums
  const int B = Bm / 2, b = (int)(blockIdx.x % (unsigned)B);
  const i64 range = blockIdx.x / (unsigned)B;
  const int E = K * K + 1, E4 = 4 * E, NE = min(E4, kCrossThreads), Q = kCrossThreads / NE;
  const int t = threadIdx.x, q = t / NE, e0 = t - q * NE;
  const int nent = (E4 - e0 + NE - 1) / NE;
  const bool lane = q < Q;
  const int KS = K + 1, G = 2 * KS, PS = 4 * G;  // values per (pixel, gauge) and per pixel
  double* nv = MOM ? reinterpret_cast<double*>(sv + (size_t)PC * PS) : nullptr;
  double acc[NENT][3];
  int o0[NENT], o1[NENT];  // the entry's operands within a pixel's values
#pragma unroll
  for (int s = 0; s < NENT; ++s) {
    acc[s][0] = acc[s][1] = acc[s][2] = 0.0;
    const int e = e0 + s * NE, g = e / E, el = e - g * E;
    o0[s] = g * G + (el < K * K ? el / K : K);
    o1[s] = g * G + KS + (el < K * K ? el - (el / K) * K : K);
  }
  const i64 P0 = range * chunk, P1 = min(N, P0 + chunk);
  for (i64 pc = P0; pc < P1; pc += PC) {
    const int np = (int)min((i64)PC, P1 - pc);
    __syncthreads();
    cross_stage4<T>(sv, nv, pc, np, K, Bm, b, z, br, mask);
    __syncthreads();
    if (!lane) continue;
    for (int j = q; j < np; j += Q) {
      const double2* v = sv + (size_t)j * PS;
#pragma unroll
      for (int s = 0; s < NENT; ++s) {
        if (s >= nent) continue;
        const double2 a = v[o0[s]], c = v[o1[s]];
        acc[s][0] = fma(a.y, c.y, fma(a.x, c.x, acc[s][0]));
        acc[s][1] = fma(-a.x, c.y, fma(a.y, c.x, acc[s][1]));
        if (MOM) {
          const double* n0 = nv + (size_t)j * PS;
          acc[s][2] = fma(n0[o0[s]], n0[o1[s]], acc[s][2]);
        }
      }
    }
  }
  __syncthreads();
  double* red = reinterpret_cast<double*>(sv);  // [Q][NE][NENT][3]
  if (lane) {
#pragma unroll
    for (int s = 0; s < NENT; ++s)
      if (s < nent)
#pragma unroll
        for (int k = 0; k < 3; ++k) red[(((size_t)q * NE + e0) * NENT + s) * 3 + k] = acc[s][k];
  }
  __syncthreads();
  if (q != 0) return;
  for (int s = 0; s < nent; ++s) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int r = 0; r < Q; ++r)
      for (int k = 0; k < 3; ++k) v[k] = __dadd_rn(v[k], red[(((size_t)r * NE + e0) * NENT + s) * 3 + k]);
    const int e = e0 + s * NE, g = e / E, el = e - g * E;
    double* out = partials + ((range * B + b) * 4 + g) * cross_slots(K);
    const int at = el < K * K ? 2 * el : 2 * K * K;
    out[at] = v[0];
    out[at + 1] = v[1];
    out[el < K * K ? 2 * K * K + 2 + el : 3 * K * K + 2] = v[2];
  }
}

template <typename T, bool MOM, int NENT>
void launch_cross_fwd(unsigned grid, size_t smem, cudaStream_t s, i64 N, int K, int Bm, const T* z, const T* br,
                      const uint8_t* mask, i64 chunk, int PC, double* partials) {
  if (smem > 48 * 1024) allow_dynamic_smem(k_cross_fwd<T, MOM, NENT>);
  k_cross_fwd<T, MOM, NENT><<<grid, kCrossThreads, smem, s>>>(N, K, Bm, z, br, mask, chunk, PC, partials);
}

template <typename T, bool MOM>
void launch_cross_fwd(int nent, unsigned grid, size_t smem, cudaStream_t s, i64 N, int K, int Bm, const T* z,
                      const T* br, const uint8_t* mask, i64 chunk, int PC, double* partials) {
  if (nent <= 1) launch_cross_fwd<T, MOM, 1>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else if (nent <= 2) launch_cross_fwd<T, MOM, 2>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else if (nent <= 4) launch_cross_fwd<T, MOM, 4>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else launch_cross_fwd<T, MOM, kCrossMaxEnt>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
}

template <typename T, bool MOM, int NENT>
void launch_cross_fwd4(unsigned grid, size_t smem, cudaStream_t s, i64 N, int K, int Bm, const T* z, const T* br,
                       const uint8_t* mask, i64 chunk, int PC, double* partials) {
  if (smem > 48 * 1024) allow_dynamic_smem(k_cross_fwd4<T, MOM, NENT>);
  k_cross_fwd4<T, MOM, NENT><<<grid, kCrossThreads, smem, s>>>(N, K, Bm, z, br, mask, chunk, PC, partials);
}
template <typename T, bool MOM>
void launch_cross_fwd4(int nent, unsigned grid, size_t smem, cudaStream_t s, i64 N, int K, int Bm, const T* z,
                       const T* br, const uint8_t* mask, i64 chunk, int PC, double* partials) {
  if (nent <= 1) launch_cross_fwd4<T, MOM, 1>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else if (nent <= 2) launch_cross_fwd4<T, MOM, 2>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else if (nent <= 4) launch_cross_fwd4<T, MOM, 4>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else launch_cross_fwd4<T, MOM, kCrossMaxEnt>(grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
}

template <typename T>
void cross_forward(int K, i64 N, int Bm, const T* z, const T* br, const uint8_t* mask, bool moments,
                   double* partials, int nblk, double* sums, cudaStream_t s) {
  if (K <= kCross4MaxK) {  // the four gauges a CTA
    const int E4 = 4 * (K * K + 1), NE = std::min(E4, kCrossThreads), Q = kCrossThreads / NE;
    const int nent = (E4 + NE - 1) / NE;
    const int per = 4 * 2 * (K + 1) * (moments ? 24 : 16);
    const int PC = std::max(8, std::min(256, (48 * 1024) / per));
    const size_t smem = std::max((size_t)PC * per, sizeof(double) * (size_t)Q * NE * kCrossMaxEnt * 3);
    const i64 chunk = (N + nblk - 1) / nblk;
    const unsigned grid = (unsigned)nblk * (unsigned)(Bm / 2);
    if (moments)
      launch_cross_fwd4<T, true>(nent, grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
    else
      launch_cross_fwd4<T, false>(nent, grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
    STL_CUDA(cudaGetLastError());
    const i64 rows = (i64)Bm / 2 * 4, total = rows * cross_slots(K);
    k_reduce_partials<<<(unsigned)std::min<i64>((total + 255) / 256, 1024), 256, 0, s>>>(partials, nblk, (int)rows,
                                                                                          cross_slots(K), sums);
    STL_CUDA(cudaGetLastError());
    return;
  }
  const int E = K * K + 1, NE = std::min(E, kCrossThreads), Q = kCrossThreads / NE;
  const int nent = (E + NE - 1) / NE;
  if (nent > kCrossMaxEnt) throw std::runtime_error("too many cross terms per level");
  const int NENT = nent <= 1 ? 1 : nent <= 2 ? 2 : nent <= 4 ? 4 : kCrossMaxEnt;
  const int PC = cross_chunk(K, moments);
  const size_t stage = (sizeof(double2) + (moments ? sizeof(double) : 0)) * (size_t)PC * 2 * (K + 1);
  const size_t smem = std::max(stage, sizeof(double) * (size_t)Q * NE * NENT * 3);
  const i64 chunk = (N + nblk - 1) / nblk;
  const unsigned grid = (unsigned)nblk * (unsigned)(Bm / 2 * 4);
  if (moments)
    launch_cross_fwd<T, true>(nent, grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  else
    launch_cross_fwd<T, false>(nent, grid, smem, s, N, K, Bm, z, br, mask, chunk, PC, partials);
  STL_CUDA(cudaGetLastError());
  const i64 rows = (i64)Bm / 2 * 4, total = rows * cross_slots(K);
  k_reduce_partials<<<(unsigned)std::min<i64>((total + 255) / 256, 1024), 256, 0, s>>>(partials, nblk, (int)rows,
                                                                                        cross_slots(K), sums);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void cross_reverse(int K, i64 N, int Bm, const T* z, const T* br, const T* M, const T* s1, const uint8_t* mask,
                   bool accumulate, T* gz, T* gbr, cudaStream_t s) {
  if (K > kCrossThreads) throw std::runtime_error("too many operands for the cross VJP");
  const int PC = cross_chunk(K);
  const size_t smem = sizeof(double2) * ((size_t)K * K + (size_t)PC * 2 * (K + 1));
  if (smem > 48 * 1024) allow_dynamic_smem(k_cross_rev<T>);
  const i64 per = 4 * (i64)PC;  // pixels per CTA
  const i64 nblk = std::max<i64>(1, (N + per - 1) / per);
  if (nblk * (Bm / 2 * 4) > INT32_MAX) throw std::runtime_error("too many pixels for the cross VJP");
  const unsigned grid = (unsigned)(nblk * (Bm / 2 * 4));
  k_cross_rev<T><<<grid, kCrossThreads, smem, s>>>(N, K, Bm, z, br, M, s1, mask, accumulate ? 1 : 0, per, PC, gz,
                                                   gbr);
  STL_CUDA(cudaGetLastError());
}

int cross_blocks(i64 N) { return (int)std::max<i64>(1, std::min<i64>(296, (N + 1023) / 1024)); }

int means_blocks(i64 N) { return (int)std::max<i64>(1, std::min<i64>(kMeansBlocks, (N + 1023) / 1024)); }

template <typename T>
void row_means(const T* f, bool complex_moduli, bool pixel_major, i64 N, int R, double* partials, double* out,
               cudaStream_t s) {
  if (R <= 0 || R > 256) throw std::runtime_error("row means: 1 to 256 rows");
  const int nblk = means_blocks(N);
  const i64 chunk = (N + nblk - 1) / nblk;
  if (pixel_major) {
    const int threads = (256 / R) * R;
    if (complex_moduli) k_means_pm<T, true><<<nblk, threads, 0, s>>>(f, N, R, chunk, partials);
    else k_means_pm<T, false><<<nblk, threads, 0, s>>>(f, N, R, chunk, partials);
  } else {
    if (complex_moduli) throw std::runtime_error("row means: complex map-major fields are not used");
    k_means_mm<T><<<dim3(nblk, R), 256, 0, s>>>(f, N, chunk, partials);
  }
  STL_CUDA(cudaGetLastError());
  k_means_final<<<R, 256, 0, s>>>(partials, nblk, R, N, out);
  STL_CUDA(cudaGetLastError());
}

template <typename T>
void moduli_deviations(const T* z, i64 N, int B, int L, const double* cz, T* mod, int mod_pix, int mod_row,
                       int mod_off, cudaStream_t s) {
  if (L != 4 || mod_pix % 4 || mod_row % 4 || mod_off % 4) throw std::runtime_error("moduli layout not in 4-row units");
  if (N * B < ((i64)1 << 31))
    k_mod_dev<T, uint32_t><<<nblocks(N * B, 256), 256, 0, s>>>(z, N, B, L, cz, mod, mod_pix, mod_row, mod_off);
  else
    k_mod_dev<T, i64><<<nblocks(N * B, 256), 256, 0, s>>>(z, N, B, L, cz, mod, mod_pix, mod_row, mod_off);
  STL_CUDA(cudaGetLastError());
}

void branch_constants(const double* zc, int n, int B, int L, double* rc, cudaStream_t s) {
  const int R = B * (n + 1) * L;
  k_branch_consts<<<nblocks(R, 256), 256, 0, s>>>(zc, n, B, L, rc);
  STL_CUDA(cudaGetLastError());
}

template <typename Tin, typename Tout>
void convert(const Tin* in, Tout* out, i64 n, cudaStream_t s) {
  if (n <= 0) return;
  k_convert<Tin, Tout><<<nblocks(n, 256), 256, 0, s>>>(in, out, n);
  STL_CUDA(cudaGetLastError());
}

template <typename Tin, typename Tout>
void to_pixel_major(const Tin* in, Tout* out, i64 N, int B, cudaStream_t s, const double* sub, Tout* res) {
  if (N * B < ((i64)1 << 31))
    k_to_pixel_major<Tin, Tout, uint32_t><<<nblocks(N * B, 256), 256, 0, s>>>(in, out, N, B, sub, res);
  else k_to_pixel_major<Tin, Tout, i64><<<nblocks(N * B, 256), 256, 0, s>>>(in, out, N, B, sub, res);
  STL_CUDA(cudaGetLastError());
}

void split_f64(const double* x, float* hi, float* lo, i64 n, cudaStream_t s) {
  if (n <= 0) return;
  k_split_f64<<<nblocks(n, 256), 256, 0, s>>>(x, hi, lo, n);
  STL_CUDA(cudaGetLastError());
}

void join_f64(const float* hi, const float* lo, double* x, i64 n, cudaStream_t s) {
  if (n <= 0) return;
  k_join_f64<<<nblocks(n, 256), 256, 0, s>>>(hi, lo, x, n);
  STL_CUDA(cudaGetLastError());
}

template <typename Tin, typename Tout>
void to_map_major(const Tin* in, Tout* out, i64 N, int B, cudaStream_t s, const double* add) {
  if (N * B < ((i64)1 << 31)) k_to_map_major<Tin, Tout, uint32_t><<<nblocks(N * B, 256), 256, 0, s>>>(in, out, N, B, add);
  else k_to_map_major<Tin, Tout, i64><<<nblocks(N * B, 256), 256, 0, s>>>(in, out, N, B, add);
  STL_CUDA(cudaGetLastError());
}

#define INST(T)                                                                                                   \
  template void conv_forward<T>(const ConvOp&, const T*, int, T*, T*, int, int, int, cudaStream_t, int*,          \
                                const double*, int);                                                              \
  template void conv_adjoint<T>(const ConvOp&, const T*, int, T*, bool, cudaStream_t, const AdjScratch*, int*,        \
                                const ModulusAdd<T>*, int);                                                           \
  template void modulus_vjp_add<T>(const T*, const T*, int, int, T*, i64, int, int, cudaStream_t);                \
  template void products_forward<T>(const ProductShape&, const T*, const T*, const T*, const T*, const double*,  \
                                    const uint8_t*, double*, double*, int*, cudaStream_t, bool);                                                                \
  template void products_reverse<T>(const ProductShape&, const T*, const T*, const T*, const T*, const uint8_t*, \
                                    bool, T*, T*, cudaStream_t);                                                                \
  template void mean_var_grad<T>(const T*, const double*, const uint8_t*, const double*, int, i64, T*,           \
                                 cudaStream_t, const i64*, int);                                                  \
  template void row_means<T>(const T*, bool, bool, i64, int, double*, double*, cudaStream_t);                     \
  template void build_cotangents<T>(const double*, int, int, int, const double*, int, int, int, int,             \
                                    const CotSources*, const CotSources*, T*, T*, cudaStream_t, bool);           \
  template void cross_forward<T>(int, i64, int, const T*, const T*, const uint8_t*, bool, double*, int, double*,  \
                                 cudaStream_t);                                                                   \
  template void cross_reverse<T>(int, i64, int, const T*, const T*, const T*, const T*, const uint8_t*, bool, T*, \
                                 T*, cudaStream_t);                                                               \
  template void moduli_deviations<T>(const T*, i64, int, int, const double*, T*, int, int, int, cudaStream_t);
INST(float)
INST(double)
template void dec_apply<float, float>(const DecOp&, bool, const float*, int, int, float*, int, int, int, int, bool,
                                     cudaStream_t, int);
template void dec_apply<double, double>(const DecOp&, bool, const double*, int, int, double*, int, int, int, int,
                                       bool, cudaStream_t, int);
template void dec_apply<float, double>(const DecOp&, bool, const float*, int, int, double*, int, int, int, int, bool,
                                      cudaStream_t, int);
template void dec_apply<double, float>(const DecOp&, bool, const double*, int, int, float*, int, int, int, int, bool,
                                      cudaStream_t, int);
template void convert<double, float>(const double*, float*, i64, cudaStream_t);
template void convert<float, double>(const float*, double*, i64, cudaStream_t);
template void convert<double, double>(const double*, double*, i64, cudaStream_t);
template void convert<float, float>(const float*, float*, i64, cudaStream_t);
template void to_pixel_major<double, float>(const double*, float*, i64, int, cudaStream_t, const double*, float*);
template void to_pixel_major<double, double>(const double*, double*, i64, int, cudaStream_t, const double*, double*);
template void to_pixel_major<float, float>(const float*, float*, i64, int, cudaStream_t, const double*, float*);
template void to_pixel_major<float, double>(const float*, double*, i64, int, cudaStream_t, const double*, double*);
template void to_map_major<float, double>(const float*, double*, i64, int, cudaStream_t, const double*);
template void to_map_major<double, double>(const double*, double*, i64, int, cudaStream_t, const double*);
template void to_map_major<float, float>(const float*, float*, i64, int, cudaStream_t, const double*);
template void to_map_major<double, float>(const double*, float*, i64, int, cudaStream_t, const double*);

}  // namespace stl
