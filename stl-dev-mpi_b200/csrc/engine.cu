// Level sweeps of the B200 ScatCov engine (forward and exact VJP).
//
// Forward, levels ascending (crates/stl-core/src/engine.rs:485-602 in
// full-sky form): z_n = psi * maps[n] with |z_n| into the stored-moduli
// field Mod[n] (slot n); the stored moduli of the finer levels pushed one
// decimation down, Mod[n][d] = D Mod[n-1][d] (m[d][n] = D^(n-d) |z_d|); the
// second wavelets Br[n] = psi * Mod[n] (all (d, l1) rows in one launch);
// then the FP64 coefficient sums of the level.
//
// Reverse, levels descending (engine.rs:610-724, 1117-1174): the
// cotangents of the stored moduli of level n start as D^T of those of
// level n + 1 (a Horner form of the reference's per-block decimation
// chains); the coefficient cotangents give (gz, gBr) per pixel; the
// adjoint of the second wavelet adds into gMod[n]; its own slot n goes
// through the modulus VJP into gz; the wavelet adjoint of gz plus D^T of
// the next level's map cotangent is the map cotangent of level n
// (map_cotangent, engine.rs:757-779).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>

#include "engine.cuh"
#include "scatcov.hpp"

namespace stl {

// ---- device memory accounting ----------------------------------------------
static std::mutex g_mem_mu;
static size_t g_live = 0, g_peak = 0;
void DevMem::alloc(size_t n) {
  release();
  if (n == 0) return;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    throw std::runtime_error("device allocation of " + std::to_string(n) + " bytes failed: " + cudaGetErrorString(e));
  }
  bytes = n;
  std::lock_guard<std::mutex> g(g_mem_mu);
  g_live += n;
  g_peak = std::max(g_peak, g_live);
}
void DevMem::release() {
  if (p) {
    cudaFree(p);
    std::lock_guard<std::mutex> g(g_mem_mu);
    g_live -= bytes;
  }
  p = nullptr;
  bytes = 0;
}
size_t device_bytes_live() { std::lock_guard<std::mutex> g(g_mem_mu); return g_live; }
size_t device_bytes_peak() { std::lock_guard<std::mutex> g(g_mem_mu); return g_peak; }
void device_bytes_reset_peak() { std::lock_guard<std::mutex> g(g_mem_mu); g_peak = g_live; }

// ---- plan (crates/stl-core/src/plan.rs:80-158, one channel) ---------------
const char* family_name(int f) {
  static const char* n[] = {"mean", "var", "S1", "S2", "S3", "S4"};
  return (f >= 0 && f < 6) ? n[f] : "?";
}

std::vector<Coef> build_plan(int J, int L) {
  std::vector<Coef> plan;
  auto mk = [](int fam, int nat) { return Coef{fam, nat, 0, 0, -1, -1, -1, -1, -1, -1}; };
  plan.push_back(mk(MEAN, 0));
  plan.push_back(mk(VAR, 0));
  for (int j3 = 0; j3 < J; ++j3) {
    for (int fam : {S1, S2})
      for (int l = 0; l < L; ++l) {
        Coef c = mk(fam, j3);
        c.j1 = j3; c.l1 = l;
        plan.push_back(c);
      }
    for (int j2 = 0; j2 <= j3; ++j2) {
      for (int l2 = 0; l2 < L; ++l2)
        for (int l3 = 0; l3 < L; ++l3) {
          Coef c = mk(S3, j3);
          c.j1 = j2; c.j3 = j3; c.l1 = l2; c.l3 = l3;
          plan.push_back(c);
        }
      for (int j1 = 0; j1 <= j2; ++j1)
        for (int l1 = 0; l1 < L; ++l1)
          for (int l2 = 0; l2 < L; ++l2)
            for (int l3 = 0; l3 < L; ++l3) {
              Coef c = mk(S4, j3);
              c.j1 = j1; c.j2 = j2; c.j3 = j3; c.l1 = l1; c.l2 = l2; c.l3 = l3;
              plan.push_back(c);
            }
    }
  }
  // already in native-level order (dg(j) = j, the stable sort of plan.rs:156)
  return plan;
}

// f32-rounded wavelet kernel [G][2][P] (wavelet.rs:11-35, conv.rs:167-172)
static std::vector<double> wavelet_kernel(int ksz, int G) {
  int P = ksz * ksz;
  std::vector<double> re, im;
  for (int i = 0; i < ksz; ++i)
    for (int j = 0; j < ksz; ++j) {
      double x = (double)j - ((double)ksz - 1.0) / 2.0, y = (double)i - ((double)ksz - 1.0) / 2.0;
      double mother = std::exp(-(x * x + y * y) / (2.0 * 1.0 * 1.0));
      double angle = 0.5 * 3.141592653589793115997963468544185161590576171875 * x;
      re.push_back(std::cos(angle) * mother);
      im.push_back(std::sin(angle) * mother);
    }
  double sr = 0.0, si = 0.0;
  for (int t = 0; t < P; ++t) { sr += re[t]; si += im[t]; }
  double mr = sr / P, mi = si / P;
  double l1 = 0.0;
  for (int t = 0; t < P; ++t) {
    re[t] -= mr; im[t] -= mi;
    l1 += std::hypot(re[t], im[t]);
  }
  std::vector<double> out;
  for (int g = 0; g < G; ++g) {
    for (int t = 0; t < P; ++t) out.push_back((double)(float)(re[t] / l1));
    for (int t = 0; t < P; ++t) out.push_back((double)(float)(im[t] / l1));
  }
  return out;
}

Engine::Engine(const Options& o) : opt_(o) {
  if (o.nside < 1 || (o.nside & (o.nside - 1)) != 0) throw std::runtime_error("nside must be a power of two");
  int order = 0;
  while ((i64(1) << order) < o.nside) ++order;
  if (o.J < 1 || o.J > order + 1) throw std::runtime_error("invalid number of scales");
  if (o.B < 1) throw std::runtime_error("batch must be positive");
  if (o.L != 4) throw std::runtime_error("the B200 engine is built for orientations = 4");
  if (o.ksz != 5 && o.ksz != 3) throw std::runtime_error("kernel must be 3 or 5");
  plan_ = build_plan(o.J, o.L);
  levels_ = o.J;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Launch accounting of the sweeps: counts and algorithmic bytes / flops
// always, device time from CUDA events on the launching stream when on.
class Profiler {
 public:
  enum Cat { CONV_FWD, CONV_ADJ, DEC, PROD_FWD, PROD_REV, ELEM, NCAT };
  bool on = false;
  KernelStat stat[NCAT];
  Profiler() {
    const char* names[NCAT] = {"conv_forward", "conv_adjoint", "decimation", "products_forward", "products_reverse",
                               "elementwise"};
    for (int c = 0; c < NCAT; ++c) stat[c].name = names[c];
  }
  ~Profiler() {
    for (auto& r : pending_) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : pool_) cudaEventDestroy(e);
  }
  template <typename F>
  void launch(Cat c, int kernels, double bytes, double flops, cudaStream_t s, F&& f) {
    stat[c].launches += kernels;
    stat[c].bytes += bytes;
    stat[c].flops += flops;
    if (!on) { f(); return; }
    cudaEvent_t a = get(), b = get();
    STL_CUDA(cudaEventRecord(a, s));
    f();
    STL_CUDA(cudaEventRecord(b, s));
    pending_.push_back({c, a, b});
  }
  // after the stream has been synchronised
  void collect() {
    for (auto& r : pending_) {
      float ms = 0.f;
      STL_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
      stat[r.c].ms += ms;
      pool_.push_back(r.a);
      pool_.push_back(r.b);
    }
    pending_.clear();
  }
  void reset() {
    collect();
    for (auto& s : stat) { s.launches = 0; s.ms = s.bytes = s.flops = 0.0; }
  }

 private:
  struct Rec { Cat c; cudaEvent_t a, b; };
  std::vector<Rec> pending_;
  std::vector<cudaEvent_t> pool_;
  cudaEvent_t get() {
    if (!pool_.empty()) { cudaEvent_t e = pool_.back(); pool_.pop_back(); return e; }
    cudaEvent_t e;
    STL_CUDA(cudaEventCreate(&e));
    return e;
  }
};

template <typename T>
class EngineImpl final : public Engine {
 public:
  explicit EngineImpl(const Options& o) : Engine(o) {
    int K0 = 0;
    (void)K0;
    // plan -> slot map of the product sums
    map_.resize(plan_.size());
    for (size_t i = 0; i < plan_.size(); ++i) map_[i] = locate(plan_[i]);
  }

  void prepare() override {
    if (ready_) return;
    auto t0 = std::chrono::steady_clock::now();
    STL_CUDA(cudaSetDevice(opt_.device));
    const int L = opt_.L, B = opt_.B;
    DType dt = sizeof(T) == 8 ? DType::F64 : DType::F32;
    std::vector<double> ker = wavelet_kernel(opt_.ksz, L);
    conv_.resize(levels_);
    dec_.resize(levels_ > 1 ? levels_ - 1 : 0);
    for (int n = 0; n < levels_; ++n) {
      ConvSpec cs;
      cs.nside = opt_.nside >> n; cs.ksz = opt_.ksz; cs.G = L; cs.gauge = 0;
      build_conv(cs, ker, dt, conv_[n], stream_);
      operator_bytes_ += conv_[n].bytes();
    }
    for (int d = 0; d + 1 < levels_; ++d) {
      DecSpec ds;
      ds.nside = opt_.nside >> d;
      build_dec(ds, dt, dec_[d], stream_);
      operator_bytes_ += dec_[d].bytes();
    }
    // fields
    X_.resize(levels_); Z_.resize(levels_); Mod_.resize(levels_); Br_.resize(levels_);
    gMod_.resize(levels_); gX_.resize(levels_);
    shapes_.resize(levels_);
    size_t max_part = 0, max_gz = 0, max_gbr = 0;
    for (int n = 0; n < levels_; ++n) {
      i64 N = npix(n);
      X_[n].alloc(sizeof(T) * B * N);
      Z_[n].alloc(sizeof(T) * 2 * B * L * N);
      Mod_[n].alloc(sizeof(T) * B * (n + 1) * L * N);
      Br_[n].alloc(sizeof(T) * 2 * B * (n + 1) * L * L * N);
      gMod_[n].alloc(sizeof(T) * B * (n + 1) * L * N);
      gX_[n].alloc(sizeof(T) * B * N);
      shapes_[n] = product_shape(n, L, B, N, sizeof(T));
      max_part = std::max(max_part, (size_t)B * L * shapes_[n].blocks * shapes_[n].slots);
      max_gz = std::max(max_gz, (size_t)2 * B * L * N);
      max_gbr = std::max(max_gbr, (size_t)2 * B * (n + 1) * L * L * N);
      field_bytes_ += X_[n].bytes + Z_[n].bytes + Mod_[n].bytes + Br_[n].bytes + gMod_[n].bytes + gX_[n].bytes;
    }
    partials_.alloc(sizeof(double) * max_part);
    {
      size_t nr = 0;
      for (int n = 0; n < levels_; ++n) nr += shapes_[n].roles.size();
      roles_.alloc(sizeof(int32_t) * nr);
      size_t off = 0;
      for (int n = 0; n < levels_; ++n) {
        const auto& r = shapes_[n].roles;
        STL_CUDA(cudaMemcpyAsync(roles_.as<int32_t>() + off, r.data(), sizeof(int32_t) * r.size(),
                                 cudaMemcpyHostToDevice, stream_));
        shapes_[n].d_roles = roles_.as<int32_t>() + off;
        off += r.size();
      }
      STL_CUDA(cudaStreamSynchronize(stream_));
    }
    size_t total_sums = 0;
    sum_off_.resize(levels_);
    for (int n = 0; n < levels_; ++n) {
      sum_off_[n] = total_sums;
      total_sums += (size_t)B * L * shapes_[n].slots;
    }
    sums_.alloc(sizeof(double) * total_sums);
    h_sums_.resize(total_sums);
    gZ_.alloc(sizeof(T) * max_gz);
    gBr_.alloc(sizeof(T) * max_gbr);
    size_t max_m = 0;
    for (int n = 0; n < levels_; ++n) max_m = std::max(max_m, (size_t)2 * B * L * shapes_[n].K * shapes_[n].K);
    M_.alloc(sizeof(T) * max_m);
    s1c_.alloc(sizeof(T) * B * L);
    mv_.alloc(sizeof(double) * 2 * B);
    err_.alloc(sizeof(int));
    STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_));
    in_f64_.alloc(sizeof(double) * B * npix(0));
    field_bytes_ += partials_.bytes + sums_.bytes + gZ_.bytes + gBr_.bytes + M_.bytes + in_f64_.bytes;
    // partial sums of the row-centric adjoint
    {
      size_t cap = 0;
      for (int n = 0; n < levels_; ++n)
        cap = std::max(cap, adjoint_part_bytes(conv_[n], sizeof(T), B * (n + 1) * L));
      if (cap) adj_part_.alloc(cap);
      adj_.part = adj_part_.p;
      adj_.capacity = cap;
      field_bytes_ += adj_part_.bytes;
    }
    STL_CUDA(cudaStreamSynchronize(stream_));
    ready_ = true;
    timers.build_s += ms_since(t0) / 1000.0;
  }

  void load_host(const double* x) override {
    prepare();
    size_t n = (size_t)opt_.B * npix(0);
    STL_CUDA(cudaMemcpyAsync(in_f64_.p, x, n * 8, cudaMemcpyHostToDevice, stream_));
    prof_.launch(Profiler::ELEM, 1, n * (8.0 + sizeof(T)), 0.0, stream_,
                 [&] { to_pixel_major<double, T>(in_f64_.as<double>(), X_[0].as<T>(), npix(0), opt_.B, stream_); });
    loaded_ = true;
    levels_given_ = false;
  }

  void load_levels(const double* x) override {
    prepare();
    size_t off = 0;
    for (int d = 0; d < levels_; ++d) {
      const size_t n = (size_t)opt_.B * npix(d);
      STL_CUDA(cudaMemcpyAsync(in_f64_.p, x + off, n * 8, cudaMemcpyHostToDevice, stream_));
      to_pixel_major<double, T>(in_f64_.as<double>(), X_[d].as<T>(), npix(d), opt_.B, stream_);
      STL_CUDA(cudaStreamSynchronize(stream_));  // the staging buffer is reused for the next level
      off += n;
    }
    loaded_ = true;
    levels_given_ = true;
  }

  void load_device(const void* x, bool f32) override {
    prepare();
    i64 n = (i64)opt_.B * npix(0);
    prof_.launch(Profiler::ELEM, 1, n * ((f32 ? 4.0 : 8.0) + sizeof(T)), 0.0, stream_, [&] {
      if (f32) to_pixel_major<float, T>(static_cast<const float*>(x), X_[0].as<T>(), npix(0), opt_.B, stream_);
      else to_pixel_major<double, T>(static_cast<const double*>(x), X_[0].as<T>(), npix(0), opt_.B, stream_);
    });
    loaded_ = true;
    levels_given_ = false;
  }

  void save_input(std::vector<double>& x) override {
    i64 n = (i64)opt_.B * npix(0);
    to_map_major<T, double>(X_[0].as<T>(), in_f64_.as<double>(), npix(0), opt_.B, stream_);
    x.resize(n);
    STL_CUDA(cudaMemcpyAsync(x.data(), in_f64_.p, n * 8, cudaMemcpyDeviceToHost, stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  void forward(bool moments, double* values, double* var) override {
    if (!loaded_) throw std::runtime_error("forward before the maps were loaded");
    auto t0 = std::chrono::steady_clock::now();
    const int L = opt_.L, B = opt_.B;
    cudaStream_t s = stream_;
    for (int d = 0; d + 1 < levels_ && !levels_given_; ++d)
      prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[d], B, false), dec_flops(dec_[d], B, false), s, [&] {
        dec_apply<T>(dec_[d], false, X_[d].as<T>(), B, 0, X_[d + 1].as<T>(), B, 0, 1, B, false, s);
      });
    for (int n = 0; n < levels_; ++n) {
      i64 N = npix(n);
      T* mod = Mod_[n].as<T>();
      const ConvOp& op = conv_[n];
      prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, B, true, true), conv_flops(op, B), s, [&] {
        conv_forward<T>(op, X_[n].as<T>(), B, Z_[n].as<T>(), mod, B * (n + 1) * L, (n + 1) * L, n * L, s,
                        err_.as<int>());
      });
      if (n > 0)
        prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n - 1], B * n * L, false), dec_flops(dec_[n - 1], B * n * L, false),
                     s, [&] {
                       dec_apply<T>(dec_[n - 1], false, Mod_[n - 1].as<T>(), B * n * L, n * L, mod, B * (n + 1) * L,
                                    (n + 1) * L, B, n * L, false, s);
                     });
      const int R = B * (n + 1) * L;
      prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, R, true, false), conv_flops(op, R), s, [&] {
        conv_forward<T>(op, mod, R, Br_[n].as<T>(), nullptr, 0, 0, 0, s, err_.as<int>());
      });
      const ProductShape& sh = shapes_[n];
      double E = sh.K * (sh.K + 1) / 2.0;
      prof_.launch(Profiler::PROD_FWD, 2, (double)B * L * N * sh.K * 2 * sizeof(T), (double)B * L * N * E * 10.0, s,
                   [&] {
                     products_forward<T>(sh, Z_[n].as<T>(), Br_[n].as<T>(), X_[0].as<T>(), partials_.as<double>(),
                                         sums_.as<double>() + sum_off_[n], err_.as<int>(), s);
                   });
    }
    STL_CUDA(cudaMemcpyAsync(h_sums_.data(), sums_.p, h_sums_.size() * 8, cudaMemcpyDeviceToHost, s));
    int err = 0;
    STL_CUDA(cudaMemcpyAsync(&err, err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    prof_.collect();
    if (err) {
      STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), s));
      throw std::runtime_error("a wait on a staged device copy timed out in the forward sweep");
    }
    assemble(values, moments ? var : nullptr);
    forward_done_ = true;
    timers.forward_ms += ms_since(t0);
    timers.forwards += 1;
  }

  void reverse_host(const double* cot, double* out) override {
    reverse_impl(cot);
    i64 n = (i64)opt_.B * npix(0);
    prof_.launch(Profiler::ELEM, 1, n * (8.0 + sizeof(T)), 0.0, stream_,
                 [&] { to_map_major<T, double>(gX_[0].as<T>(), in_f64_.as<double>(), npix(0), opt_.B, stream_); });
    STL_CUDA(cudaMemcpyAsync(out, in_f64_.p, n * 8, cudaMemcpyDeviceToHost, stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  void reverse_device(const double* cot, void* out, bool f32) override {
    reverse_impl(cot);
    i64 n = (i64)opt_.B * npix(0);
    prof_.launch(Profiler::ELEM, 1, n * ((f32 ? 4.0 : 8.0) + sizeof(T)), 0.0, stream_, [&] {
      if (f32) to_map_major<T, float>(gX_[0].as<T>(), static_cast<float*>(out), npix(0), opt_.B, stream_);
      else to_map_major<T, double>(gX_[0].as<T>(), static_cast<double*>(out), npix(0), opt_.B, stream_);
    });
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  std::vector<KernelStat> kernel_stats() const override {
    return std::vector<KernelStat>(prof_.stat, prof_.stat + Profiler::NCAT);
  }
  void reset_kernel_stats() override { prof_.reset(); }
  void set_profiling(bool on) override { prof_.on = on; }
  std::vector<double> mean_slots() const override {
    std::vector<double> v;
    for (const auto& c : conv_) v.push_back(c.mean_slots);
    return v;
  }

 private:
  // Algorithmic traffic of one wavelet launch over R rows: the used
  // coefficients of the stored rows (2L values and a 4-byte cell index per
  // cell read; a quarter of the rows on the full sky), the input rows read
  // once, the complex outputs written once (plus |z|, or the
  // read-modify-write of an accumulated adjoint).
  double conv_bytes(const ConvOp& op, int R, bool fwd, bool extra) const {
    const double s = sizeof(T), N = (double)op.n_rows, D = op.mean_slots;
    double coef = (double)op.n_rep * D * (8.0 * s + 4.0);
    double field = fwd ? R * N * s + R * N * 8.0 * s : R * N * 8.0 * s + R * N * s;
    if (extra) field += fwd ? R * N * 4.0 * s : R * N * s;
    return coef + field;
  }
  double conv_flops(const ConvOp& op, int R) const { return 2.0 * 8.0 * R * (double)op.n_rows * op.mean_slots; }
  double dec_bytes(const DecOp& op, int R, bool transpose) const {
    const double s = sizeof(T);
    double nnz = op.mean_w * (double)op.n_out;
    return nnz * (s + 4.0) + R * (double)(op.n_in + op.n_out) * s;
    (void)transpose;
  }
  double dec_flops(const DecOp& op, int R, bool) const { return 2.0 * R * op.mean_w * (double)op.n_out; }

  // where a plan coefficient's sums live: level, l3 row, and the slots of
  // its real part, imaginary part (-1: exactly zero) and second moment
  struct Loc {
    int level, l3, re, im, second;
  };

  // Sums of the products kernel per (b, l3) (kernels.cu): 4 x 4 Gram blocks
  // (d1 <= d2) of the branches, 4 x 1 blocks (d, z), then the per-pixel sums.
  Loc locate(const Coef& c) const {
    const int L = opt_.L;
    const int n = c.native, nd = n + 1;
    const int nBB = nd * (nd + 1) / 2, zb = nBB * 48 + nd * 12;
    auto tblock = [&](int d1, int d2) { return d1 * nd - d1 * (d1 - 1) / 2 + (d2 - d1); };
    Loc l{n, 0, 0, 0, 0};
    switch (c.family) {
      case MEAN: l.re = zb + 3; l.second = zb + 4; l.im = -1; break;
      case VAR: l.re = zb + 4; l.second = zb + 5; l.im = -1; break;
      case S1: l.l3 = c.l1; l.re = zb; l.second = zb + 1; l.im = -1; break;
      case S2: l.l3 = c.l1; l.re = zb + 1; l.second = zb + 2; l.im = -1; break;
      case S3: {
        const int base = nBB * 48 + 12 * c.j1;
        l.l3 = c.l3; l.re = base + 2 * c.l1; l.im = l.re + 1; l.second = base + 8 + c.l1;
        break;
      }
      case S4: {
        const int t = tblock(c.j1, c.j2), e = c.l1 * 4 + c.l2;
        l.l3 = c.l3; l.re = t * 48 + 2 * e; l.im = l.re + 1; l.second = t * 48 + 32 + e;
        if (c.j1 == c.j2 && c.l1 == c.l2) l.im = -1;  // v conj(v): an exactly real term
        break;
      }
    }
    (void)L;
    return l;
  }

  void assemble(double* values, double* var) const {
    const int L = opt_.L, B = opt_.B;
    const i64 np = (i64)plan_.size();
    for (int b = 0; b < B; ++b)
      for (i64 i = 0; i < np; ++i) {
        const Loc& l = map_[i];
        const ProductShape& sh = shapes_[l.level];
        const double* row = h_sums_.data() + sum_off_[l.level] + ((size_t)b * L + l.l3) * sh.slots;
        const double N = (double)npix(l.level);
        const double re = row[l.re], im = l.im >= 0 ? row[l.im] : 0.0, second = row[l.second];
        const double vr = re / N, vi = im / N;
        values[2 * (b * np + i)] = vr;
        values[2 * (b * np + i) + 1] = vi;
        if (var) var[b * np + i] = std::max(second / N - (vr * vr + vi * vi), 0.0);
      }
  }

  void reverse_impl(const double* cot) {
    if (!forward_done_) throw std::runtime_error("vjp before forward");
    auto t0 = std::chrono::steady_clock::now();
    const int L = opt_.L, B = opt_.B;
    const i64 np = (i64)plan_.size();
    cudaStream_t s = stream_;
    // host: per-level cotangent matrices, auto-S1 scales, mean/var scales
    std::vector<std::vector<std::complex<double>>> M(levels_);
    std::vector<std::vector<double>> s1(levels_, std::vector<double>((size_t)B * L, 0.0));
    std::vector<double> mv((size_t)2 * B, 0.0);
    for (int n = 0; n < levels_; ++n) M[n].assign((size_t)B * L * shapes_[n].K * shapes_[n].K, 0.0);
    for (int b = 0; b < B; ++b)
      for (i64 i = 0; i < np; ++i) {
        std::complex<double> g(cot[2 * (b * np + i)], cot[2 * (b * np + i) + 1]);
        if (g == std::complex<double>(0.0, 0.0)) continue;
        const Coef& c = plan_[i];
        int n = c.native, K = shapes_[n].K, z = K - 1;
        double N = (double)npix(n);
        auto at = [&](int l3, int r, int q) -> std::complex<double>& {
          return M[n][(((size_t)b * L + l3) * K + r) * K + q];
        };
        switch (c.family) {
          case MEAN: mv[2 * b] += g.real() / N; break;
          case VAR: mv[2 * b + 1] += 2.0 * g.real() / N; break;
          case S1: s1[n][(size_t)b * L + c.l1] += g.real() / N; break;
          case S2: at(c.l1, z, z) += 2.0 * g.real() / N; break;
          case S3: {
            int r = c.j1 * L + c.l1;
            at(c.l3, r, z) += g / N;
            at(c.l3, z, r) += std::conj(g) / N;
            break;
          }
          case S4: {
            int r = c.j1 * L + c.l1, q = c.j2 * L + c.l2;
            at(c.l3, r, q) += g / N;
            at(c.l3, q, r) += std::conj(g) / N;
            break;
          }
        }
      }
    for (int n = levels_ - 1; n >= 0; --n) {
      i64 N = npix(n);
      const ProductShape& sh = shapes_[n];
      const ConvOp& op = conv_[n];
      T* gmod = gMod_[n].as<T>();
      if (n + 1 < levels_)
        prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n], B * (n + 1) * L, true), dec_flops(dec_[n], B * (n + 1) * L, true),
                     s, [&] {
                       dec_apply<T>(dec_[n], true, gMod_[n + 1].as<T>(), B * (n + 2) * L, (n + 2) * L, gmod,
                                    B * (n + 1) * L, (n + 1) * L, B, (n + 1) * L, false, s);
                     });
      else
        STL_CUDA(cudaMemsetAsync(gmod, 0, gMod_[n].bytes, s));
      // cotangent matrices in the field precision
      h_M_.resize(2 * M[n].size());
      for (size_t q = 0; q < M[n].size(); ++q) { h_M_[2 * q] = (T)M[n][q].real(); h_M_[2 * q + 1] = (T)M[n][q].imag(); }
      h_s1_.resize(s1[n].size());
      for (size_t q = 0; q < s1[n].size(); ++q) h_s1_[q] = (T)s1[n][q];
      STL_CUDA(cudaMemcpyAsync(M_.p, h_M_.data(), h_M_.size() * sizeof(T), cudaMemcpyHostToDevice, s));
      STL_CUDA(cudaMemcpyAsync(s1c_.p, h_s1_.data(), h_s1_.size() * sizeof(T), cudaMemcpyHostToDevice, s));
      const double sz = sizeof(T);
      prof_.launch(Profiler::PROD_REV, 1, (double)B * L * N * sh.K * 4 * sz, (double)B * L * N * sh.K * sh.K * 8.0, s,
                   [&] {
                     products_reverse<T>(sh, Z_[n].as<T>(), Br_[n].as<T>(), M_.as<T>(), s1c_.as<T>(), gZ_.as<T>(),
                                         gBr_.as<T>(), s);
                   });
      const int R = B * (n + 1) * L;
      prof_.launch(Profiler::CONV_ADJ, adjoint_tiles_usable(op, sizeof(T), R, adj_ptr()) ? 2 : 1,
                   conv_bytes(op, R, false, true), conv_flops(op, R), s,
                   [&] { conv_adjoint<T>(op, gBr_.as<T>(), R, gmod, true, s, adj_ptr()); });
      prof_.launch(Profiler::ELEM, 1, (double)B * L * N * 5 * sz, (double)B * L * N * 6.0, s, [&] {
        modulus_vjp_add<T>(Z_[n].as<T>(), gmod + n * L, B * (n + 1) * L, (n + 1) * L, gZ_.as<T>(), N, B, L, s);
      });
      prof_.launch(Profiler::CONV_ADJ, adjoint_tiles_usable(op, sizeof(T), B, adj_ptr()) ? 2 : 1,
                   conv_bytes(op, B, false, false), conv_flops(op, B), s,
                   [&] { conv_adjoint<T>(op, gZ_.as<T>(), B, gX_[n].as<T>(), false, s, adj_ptr()); });
      if (n + 1 < levels_)
        prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n], B, true) + (double)B * N * sz, dec_flops(dec_[n], B, true), s,
                     [&] { dec_apply<T>(dec_[n], true, gX_[n + 1].as<T>(), B, 0, gX_[n].as<T>(), B, 0, 1, B, true, s); });
      // the host staging buffers are reused next level: wait for the copies
      STL_CUDA(cudaStreamSynchronize(s));
    }
    STL_CUDA(cudaMemcpyAsync(mv_.p, mv.data(), mv.size() * 8, cudaMemcpyHostToDevice, s));
    prof_.launch(Profiler::ELEM, 1, (double)B * npix(0) * 3 * sizeof(T), (double)B * npix(0) * 2.0, s,
                 [&] { mean_var_grad<T>(X_[0].as<T>(), mv_.as<double>(), B, npix(0), gX_[0].as<T>(), s); });
    STL_CUDA(cudaStreamSynchronize(s));
    prof_.collect();
    timers.reverse_ms += ms_since(t0);
    timers.reverses += 1;
  }

  Profiler prof_;
  bool ready_ = false, loaded_ = false, forward_done_ = false;
  bool levels_given_ = false;  // X_[d] for d > 0 were loaded, not decimated
  std::vector<ConvOp> conv_;
  std::vector<DecOp> dec_;
  std::vector<DevMem> X_, Z_, Mod_, Br_, gMod_, gX_;
  std::vector<ProductShape> shapes_;
  std::vector<size_t> sum_off_;
  DevMem partials_, sums_, gZ_, gBr_, M_, s1c_, mv_, in_f64_, err_, roles_;
  DevMem adj_part_;
  AdjScratch adj_;
  const AdjScratch* adj_ptr() const { return adj_.part ? &adj_ : nullptr; }
  std::vector<double> h_sums_;
  std::vector<T> h_M_, h_s1_;
  std::vector<Loc> map_;
};

std::unique_ptr<Engine> Engine::create(const Options& o) {
  if (o.fp32) return std::unique_ptr<Engine>(new EngineImpl<float>(o));
  return std::unique_ptr<Engine>(new EngineImpl<double>(o));
}

}  // namespace stl
