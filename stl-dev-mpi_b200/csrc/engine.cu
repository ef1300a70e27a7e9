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
#include <type_traits>
#include <chrono>
#include <condition_variable>
#include <thread>
#include <cmath>
#include <complex>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <string>

#include "engine.cuh"
#include "hostcopy.hpp"
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
// once per (kernel, device), under a lock: a thread that returns has seen the
// attribute set
void allow_dynamic_smem_fn(const void* f) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  STL_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (done.count({f, dev})) return;
  int most = 0;
  cudaFuncAttributes fa;
  STL_CUDA(cudaDeviceGetAttribute(&most, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  STL_CUDA(cudaFuncGetAttributes(&fa, f));  // the kernel's static shared memory counts against the limit
  STL_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, most - (int)fa.sharedSizeBytes));
  done.insert({f, dev});
}
void PinnedMem::alloc(size_t n) {
  release();
  if (n == 0) return;
  cudaError_t e = cudaMallocHost(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    throw std::runtime_error("pinned host allocation of " + std::to_string(n) + " bytes failed: " +
                             cudaGetErrorString(e));
  }
  bytes = n;
}
void PinnedMem::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  bytes = 0;
}
size_t device_bytes_live() { std::lock_guard<std::mutex> g(g_mem_mu); return g_live; }
size_t device_bytes_peak() { std::lock_guard<std::mutex> g(g_mem_mu); return g_peak; }
void device_bytes_reset_peak() { std::lock_guard<std::mutex> g(g_mem_mu); g_peak = g_live; }

// ---- host <-> device copies of large host buffers ---------------------------
// Caller buffers are pageable: the driver would move them through its own
// small staging at the rate of one host thread.  Instead host threads copy
// chunks into two pinned buffers while the DMA engine moves the chunk before
// (and the reverse for device-to-host), so the transfer runs at the PCIe rate.
namespace {

// a fixed pool of host threads that split one memcpy between them
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool* pool = new CopyPool();  // threads live until the process exits
    return *pool;
  }
  // dst[0, n) = src[0, n), split over the threads; returns when done.  With
  // check (n a multiple of 8): the number of non-finite doubles copied.
  // With widen: src holds n bytes of floats, dst receives them as doubles.
  size_t copy(void* dst, const void* src, size_t n, bool check = false, bool widen = false) {
    if (n < (size_t(1) << 20) || workers_.empty())
      return copy_part(static_cast<char*>(dst), static_cast<const char*>(src), n, check, widen);
    std::unique_lock<std::mutex> lk(call_mu_);  // one copy at a time
    const size_t parts = workers_.size() + 1;
    const size_t part = ((n + parts - 1) / parts + 63) & ~(size_t)63;
    {
      std::lock_guard<std::mutex> g(mu_);
      dst_ = static_cast<char*>(dst);
      src_ = static_cast<const char*>(src);
      n_ = n;
      part_ = part;
      check_ = check;
      widen_ = widen;
      bad_ = 0;
      pending_ = (int)workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    const size_t b0 = run(0);
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [&] { return pending_ == 0; });
    return bad_ + b0;
  }
  static size_t copy_part(char* dst, const char* src, size_t n, bool check, bool widen = false) {
    if (widen) {  // floats to doubles (exact)
      host_widen(reinterpret_cast<double*>(dst), reinterpret_cast<const float*>(src), n / 4);
      return 0;
    }
    return host_copy(dst, src, n, check);
  }

 private:
  CopyPool() {
    const unsigned h = std::thread::hardware_concurrency();
    const int t = (int)std::min<unsigned>(16, h > 1 ? h : 1) - 1;
    for (int i = 0; i < t; ++i) workers_.emplace_back([this, i] { loop(i + 1); });
    for (auto& w : workers_) w.detach();
  }
  size_t run(size_t k) {
    const size_t lo = std::min(n_, k * part_), hi = std::min(n_, lo + part_);
    return hi > lo ? copy_part(dst_ + (widen_ ? 2 * lo : lo), src_ + lo, hi - lo, check_, widen_) : 0;
  }
  void loop(size_t k) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
      }
      const size_t b = run(k);
      std::lock_guard<std::mutex> g(mu_);
      bad_ += b;
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, call_mu_;
  std::condition_variable cv_, done_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t n_ = 0, part_ = 0, bad_ = 0;
  bool check_ = false, widen_ = false;
  int pending_ = 0;
  uint64_t gen_ = 0;
};

// two pinned chunks and their copy events
class HostStage {
 public:
  ~HostStage() {
    for (cudaEvent_t& e : ev_)
      if (e) cudaEventDestroy(e);
  }
  // device dst <- host src (n bytes), queued on s; src is read before the
  // return.  With check (src holds doubles): the number of non-finite values.
  size_t to_device(void* dst, const void* src, size_t n, cudaStream_t s, bool check = false) {
    if (n < kDirect) {
      size_t bad = 0;
      if (check) {
        const double* v = static_cast<const double*>(src);
        for (size_t i = 0; i < n / 8; ++i) bad += !std::isfinite(v[i]);
      }
      STL_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s));
      return bad;
    }
    ensure();
    size_t bad = 0;
    for (size_t off = 0, c = 0; off < n; off += kChunk, ++c) {
      const size_t len = std::min(kChunk, n - off), b = c & 1;
      STL_CUDA(cudaEventSynchronize(ev_[b]));  // the last DMA out of this buffer has finished
      bad += CopyPool::get().copy(buf_[b].p, static_cast<const char*>(src) + off, len, check);
      STL_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, buf_[b].p, len, cudaMemcpyHostToDevice, s));
      STL_CUDA(cudaEventRecord(ev_[b], s));
    }
    return bad;
  }
  // host dst <- device src (n bytes) after the work queued on s; synchronises
  void to_host(void* dst, const void* src, size_t n, cudaStream_t s) {
    if (n < kDirect) {
      STL_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s));
      STL_CUDA(cudaStreamSynchronize(s));
      return;
    }
    ensure();
    const size_t nc = (n + kChunk - 1) / kChunk;
    auto drain = [&](size_t c) {  // chunk c: from its pinned buffer to dst
      const size_t off = c * kChunk, len = std::min(kChunk, n - off);
      STL_CUDA(cudaEventSynchronize(ev_[c & 1]));
      CopyPool::get().copy(static_cast<char*>(dst) + off, buf_[c & 1].p, len);
    };
    for (size_t c = 0; c < nc; ++c) {
      const size_t off = c * kChunk, len = std::min(kChunk, n - off);
      STL_CUDA(cudaMemcpyAsync(buf_[c & 1].p, static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, s));
      STL_CUDA(cudaEventRecord(ev_[c & 1], s));
      if (c > 0) drain(c - 1);
    }
    drain(nc - 1);
  }
  // host doubles dst <- device floats src (n floats), widened on the host: half
  // the bytes cross PCIe; synchronises
  void to_host_widen(double* dst, const float* src, size_t n, cudaStream_t s) {
    const size_t bytes = n * sizeof(float);
    if (bytes < kDirect) {
      std::vector<float> tmp(n);
      STL_CUDA(cudaMemcpyAsync(tmp.data(), src, bytes, cudaMemcpyDeviceToHost, s));
      STL_CUDA(cudaStreamSynchronize(s));
      for (size_t i = 0; i < n; ++i) dst[i] = (double)tmp[i];
      return;
    }
    ensure();
    const size_t nc = (bytes + kChunk - 1) / kChunk;
    auto drain = [&](size_t c) {
      const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
      STL_CUDA(cudaEventSynchronize(ev_[c & 1]));
      CopyPool::get().copy(reinterpret_cast<char*>(dst) + 2 * off, buf_[c & 1].p, len, false, true);
    };
    for (size_t c = 0; c < nc; ++c) {
      const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
      STL_CUDA(cudaMemcpyAsync(buf_[c & 1].p, reinterpret_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost,
                               s));
      STL_CUDA(cudaEventRecord(ev_[c & 1], s));
      if (c > 0) drain(c - 1);
    }
    drain(nc - 1);
  }

 private:
  static constexpr size_t kChunk = size_t(32) << 20, kDirect = size_t(4) << 20;
  void ensure() {
    if (buf_[0].p) return;
    for (int b = 0; b < 2; ++b) {
      buf_[b].alloc(kChunk);
      STL_CUDA(cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming));
      STL_CUDA(cudaEventRecord(ev_[b], 0));  // completed: the buffers start free
    }
  }
  PinnedMem buf_[2];
  cudaEvent_t ev_[2] = {nullptr, nullptr};
};

}  // namespace

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

std::vector<Coef> build_plan_cross(int J, int L) {
  std::vector<Coef> plan;
  auto mk = [](int fam, int nat, int c1, int c2) { return Coef{fam, nat, c1, c2, -1, -1, -1, -1, -1, -1}; };
  for (int j3 = 0; j3 < J; ++j3) {
    for (int fam : {S1, S2})
      for (int l = 0; l < L; ++l) {
        Coef c = mk(fam, j3, 0, 1);
        c.j1 = j3; c.l1 = l;
        plan.push_back(c);
      }
    for (int ca = 0; ca < 2; ++ca) {  // channel orders (0, 1), then (1, 0)
      const int cb = 1 - ca;
      for (int j2 = 0; j2 <= j3; ++j2) {
        for (int l2 = 0; l2 < L; ++l2)
          for (int l3 = 0; l3 < L; ++l3) {
            Coef c = mk(S3, j3, ca, cb);
            c.j1 = j2; c.j3 = j3; c.l1 = l2; c.l3 = l3;
            plan.push_back(c);
          }
        for (int j1 = 0; j1 <= j2; ++j1)
          for (int l1 = 0; l1 < L; ++l1)
            for (int l2 = 0; l2 < L; ++l2)
              for (int l3 = 0; l3 < L; ++l3) {
                Coef c = mk(S4, j3, ca, cb);
                c.j1 = j1; c.j2 = j2; c.j3 = j3; c.l1 = l1; c.l2 = l2; c.l3 = l3;
                plan.push_back(c);
              }
      }
    }
  }
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

Engine::Engine(const Options& o, const Support* sup) : opt_(o) {
  if (o.nside < 1 || (o.nside & (o.nside - 1)) != 0) throw std::runtime_error("nside must be a power of two");
  int order = 0;
  while ((i64(1) << order) < o.nside) ++order;
  if (o.J < 1 || o.J > order + 1) throw std::runtime_error("invalid number of scales");
  if (o.B < 1) throw std::runtime_error("batch must be positive");
  if (o.L != 4) throw std::runtime_error("the B200 engine is built for orientations = 4");
  if (o.ksz != 5 && o.ksz != 3) throw std::runtime_error("kernel must be 3 or 5");
  plan_ = o.cross ? build_plan_cross(o.J, o.L) : build_plan(o.J, o.L);
  vb_ = o.B;
  if (o.cross) {
    if (sup) throw std::runtime_error("cross statistics are not built for disc patches");
    opt_.B = 2 * o.B;  // the fields' maps: channel c of batch entry b is map 2 b + c
  }
  levels_ = o.J;
  for (int d = 0; d < levels_; ++d) {
    const i64 n = 12 * (o.nside >> d) * (o.nside >> d);
    npix_.push_back(n);
    ncore_.push_back(n);
  }
  if (sup) {
    if ((int)sup->ids.size() != levels_ || (int)sup->core.size() != levels_)
      throw std::runtime_error("support levels mismatch");
    if (o.B != 1) throw std::runtime_error("a patch engine holds one patch per segment");
    if (!sup->seg.empty() && (int)sup->seg.size() != levels_) throw std::runtime_error("segment levels mismatch");
    for (int d = 0; d < levels_; ++d) {
      const auto& ids = sup->ids[d];
      if (ids.empty()) throw std::runtime_error("empty support level");
      std::vector<i64> seg = sup->seg.empty() ? std::vector<i64>{0, (i64)ids.size()} : sup->seg[d];
      if (seg.size() < 2 || seg.front() != 0 || seg.back() != (i64)ids.size() ||
          (d > 0 && seg.size() != (sup->seg.empty() ? 2 : sup->seg[0].size())))
        throw std::runtime_error("segment offsets must run from 0 to the support size, equal in number per level");
      const auto& core = sup->core[d];
      size_t c = 0;
      for (size_t k = 0; k + 1 < seg.size(); ++k) {
        if (seg[k + 1] <= seg[k]) throw std::runtime_error("empty support segment");
        for (i64 i = seg[k]; i < seg[k + 1]; ++i)
          if (ids[i] < 0 || ids[i] >= npix_[d] || (i > seg[k] && ids[i] <= ids[i - 1]))
            throw std::runtime_error("support ids must be sorted, unique and in range");
        const size_t c0 = c;
        while (c < core.size() && core[c] < seg[k + 1]) {
          if (core[c] < seg[k] || (c > c0 && core[c] <= core[c - 1]))
            throw std::runtime_error("core positions must be ascending and in range");
          ++c;
        }
        if (c == c0) throw std::runtime_error("empty core level");
      }
      if (c != core.size()) throw std::runtime_error("core position out of range");
      npix_[d] = (i64)ids.size();
      ncore_[d] = (i64)core.size();
    }
    support_ = *sup;
  }
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
    stat[c].calls += 1;
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
    for (auto& s : stat) { s.launches = s.calls = 0; s.ms = s.bytes = s.flops = 0.0; }
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

// Coarse levels of an FP32 engine (nside at most kFp64Nside) run in FP64:
// there the wavelet answers small fluctuations of smooth fields (the map
// pyramid, the decimated moduli), and FP32 rounding of those fields and of
// the wavelet sums would pass the 1e-6 criterion on S1-S3; those levels hold
// well under 1 % of the work.
constexpr int kFp64Nside = 32;
constexpr double kBindEps = 1e-9;  // binding threshold of grid-mode wavelets (disc.rs BIND_EPS)

template <typename U> struct Tag { typedef U type; };

template <typename T>
class EngineImpl final : public Engine {
 public:
  ~EngineImpl() override {
    gfwd_.reset();
    grev_.reset();
    if (capture_stream_) cudaStreamDestroy(capture_stream_);
  }
  explicit EngineImpl(const Options& o, const Support* sup = nullptr) : Engine(o, sup) {
    int K0 = 0;
    (void)K0;
    // plan -> slot map of the product sums
    map_.resize(plan_.size());
    for (size_t i = 0; i < plan_.size(); ++i) map_[i] = locate(plan_[i]);
  }

  // Averages over k masks (level-0 indicators [k][npix(0)], nonzero: in
  // the mask; level n + 1 keeps a parent when one of its children is in the
  // mask, mask.rs:42-66), or over every pixel (k = 0).
  void set_masks(const double* w, size_t k) override {
    if (grid_mode()) throw std::runtime_error("a patch engine averages its core: no masks");
    std::vector<std::vector<std::vector<uint8_t>>> levels(k);
    const i64 n0 = npix(0);
    for (size_t q = 0; q < k; ++q) {
      auto& lv = levels[q];
      lv.resize(levels_);
      lv[0].resize(n0);
      for (i64 p = 0; p < n0; ++p) {
        const double v = w[q * n0 + p];
        if (!std::isfinite(v)) throw std::runtime_error("mask weights must be finite");
        lv[0][p] = v != 0.0;
      }
      for (int d = 1; d < levels_; ++d) {
        lv[d].assign(npix(d), 0);
        for (i64 p = 0; p < npix(d); ++p)
          lv[d][p] = lv[d - 1][4 * p] | lv[d - 1][4 * p + 1] | lv[d - 1][4 * p + 2] | lv[d - 1][4 * p + 3];
      }
    }
    upload_masks(levels);
  }
  void set_mask_levels(const std::vector<std::vector<std::vector<uint8_t>>>& levels) override {
    if (grid_mode()) throw std::runtime_error("a patch engine averages its core: no masks");
    for (const auto& lv : levels) {
      if ((int)lv.size() != levels_) throw std::runtime_error("masks of every level expected");
      for (int d = 0; d < levels_; ++d)
        if ((i64)lv[d].size() != npix(d)) throw std::runtime_error("mask size mismatch");
    }
    upload_masks(levels);
  }
  int nmasks() const override { return kmask_.empty() || grid_mode() ? 0 : K_; }
  i64 mask_count(int k, int n) const override { return count(k, n); }

  // masks [k][level][pixel] (empty: every pixel) to the device; the sums
  // hold one set per mask
  void upload_masks(const std::vector<std::vector<std::vector<uint8_t>>>& levels) {
    std::vector<std::vector<DevMem>> km(levels.size());
    std::vector<std::vector<i64>> kc(levels.size());
    for (size_t q = 0; q < levels.size(); ++q) {
      km[q].resize(levels_);
      kc[q].resize(levels_);
      for (int d = 0; d < levels_; ++d) {
        const auto& m = levels[q][d];
        i64 c = 0;
        for (uint8_t v : m) c += v;
        if (c == 0) throw std::runtime_error("empty mask");
        kc[q][d] = c;
        km[q][d].alloc(m.size());
        STL_CUDA(cudaMemcpyAsync(km[q][d].p, m.data(), m.size(), cudaMemcpyHostToDevice, stream_));
      }
      STL_CUDA(cudaStreamSynchronize(stream_));
    }
    kmask_ = std::move(km);
    kcount_ = std::move(kc);
    K_ = std::max<int>(1, (int)levels.size());
    if (ready_) size_mask_buffers();
    forward_done_ = false;
  }

  // field precision of level n
  bool hi(int n) const { return sizeof(T) == 8 || (opt_.nside >> n) <= kFp64Nside; }
  size_t esz(int n) const { return hi(n) ? 8 : sizeof(T); }
  // f(Tag<U>()) with U the field type of level n
  template <typename F>
  void typed(int n, F&& f) {
    if (hi(n)) f(Tag<double>());
    else f(Tag<float>());
  }

  void prepare() override {
    if (ready_) return;
    auto t0 = std::chrono::steady_clock::now();
    STL_CUDA(cudaSetDevice(opt_.device));
    const int L = opt_.L, B = opt_.B;
    auto dtype_of = [&](int n) { return hi(n) ? DType::F64 : DType::F32; };
    std::vector<double> ker = wavelet_kernel(opt_.ksz, L);
    conv_.resize(levels_);
    dec_.resize(levels_ > 1 ? levels_ - 1 : 0);
    if (grid_mode()) {
      // supports (and their segments) and core masks on the device
      ids_dev_.resize(levels_);
      seg_dev_.resize(segmented() ? levels_ : 0);
      std::vector<std::vector<uint8_t>> core(levels_);
      for (int d = 0; d < levels_; ++d) {
        const auto& ids = support_.ids[d];
        ids_dev_[d].alloc(sizeof(i64) * ids.size());
        STL_CUDA(cudaMemcpyAsync(ids_dev_[d].p, ids.data(), sizeof(i64) * ids.size(), cudaMemcpyHostToDevice,
                                 stream_));
        if (segmented()) {
          const auto& sg = support_.seg[d];
          seg_dev_[d].alloc(sizeof(i64) * sg.size());
          STL_CUDA(cudaMemcpyAsync(seg_dev_[d].p, sg.data(), sizeof(i64) * sg.size(), cudaMemcpyHostToDevice,
                                   stream_));
        }
        STL_CUDA(cudaStreamSynchronize(stream_));
        core[d].assign(ids.size(), 0);
        for (i64 c : support_.core[d]) core[d][c] = 1;
      }
      upload_masks({core});
      if (segmented()) {
        // one set of sums per segment, over its core pixels
        K_ = segments();
        kcount_.assign(K_, std::vector<i64>(levels_, 0));
        for (int d = 0; d < levels_; ++d) {
          const auto& sg = support_.seg[d];
          int k = 0;
          for (i64 c : support_.core[d]) {
            while (c >= sg[k + 1]) ++k;
            ++kcount_[k][d];
          }
        }
      }
    }
    for (int n = 0; n < levels_; ++n) {
      ConvSpec cs;
      cs.nside = opt_.nside >> n; cs.ksz = opt_.ksz; cs.G = L; cs.gauge = 0;
      cs.tensor_cores = opt_.tensor_cores;
      if (grid_mode()) {
        cs.d_grid = ids_dev_[n].as<i64>();
        cs.n_in = npix(n);
        cs.eps = kBindEps;
        cs.symmetric = false;
        if (segmented()) {
          cs.d_seg = seg_dev_[n].as<i64>();
          cs.nseg = segments();
        }
      }
      build_conv(cs, ker, dtype_of(n), conv_[n], stream_);
      operator_bytes_ += conv_[n].bytes();
    }
    for (int d = 0; d + 1 < levels_; ++d) {
      DecSpec ds;
      ds.nside = opt_.nside >> d;
      if (grid_mode()) {
        ds.d_ids = ids_dev_[d].as<i64>();
        ds.n_in = npix(d);
        ds.d_out = ids_dev_[d + 1].as<i64>();
        ds.n_out = npix(d + 1);
        ds.symmetric = false;
        if (segmented()) {
          ds.d_seg_in = seg_dev_[d].as<i64>();
          ds.d_seg_out = seg_dev_[d + 1].as<i64>();
          ds.nseg = segments();
        }
      }
      build_dec(ds, dtype_of(d + 1), dec_[d], stream_);  // FP64 weights into an FP64 level
      operator_bytes_ += dec_[d].bytes();
    }
    // fields
    X_.resize(levels_); Z_.resize(levels_); Mod_.resize(levels_); Br_.resize(levels_);
    gMod_.resize(levels_); gX_.resize(levels_);
    shapes_.resize(levels_);
    size_t max_part = 0, max_gz = 0, max_gbr = 0;
    // field store: z and the branches of every level kept, or one buffer each
    // (the largest level's) recomputed per level in the reverse sweep
    {
      size_t keep = 0, zmax = 0, bmax = 0;
      for (int n = 0; n < levels_; ++n) {
        const size_t e = esz(n), N = (size_t)npix(n);
        keep += e * 2 * B * L * N + e * 2 * B * (n + 1) * L * L * N;
        zmax = std::max(zmax, e * 2 * B * L * N);
        bmax = std::max(bmax, e * 2 * B * (n + 1) * L * L * N);
      }
      keep_bytes_ = keep;
      recompute_ = opt_.recompute;
      if (opt_.fields_auto) {  // keep them when they fit the free memory with a quarter to spare
        size_t free_b = 0, total_b = 0;
        STL_CUDA(cudaMemGetInfo(&free_b, &total_b));
        recompute_ = keep > free_b / 4 * 3;
      }
      if (recompute_) {
        Zs_.alloc(zmax);
        Brs_.alloc(bmax);
        field_bytes_ += Zs_.bytes + Brs_.bytes;
      }
    }
    for (int n = 0; n < levels_; ++n) {
      i64 N = npix(n);
      const size_t e = esz(n);
      X_[n].alloc(e * B * N + 16);  // padded: the products stage their maps in 16-byte units
      if (!recompute_) Z_[n].alloc(e * 2 * B * L * N);
      Mod_[n].alloc(e * B * (n + 1) * L * N);
      if (!recompute_) Br_[n].alloc(e * 2 * B * (n + 1) * L * L * N);
      gMod_[n].alloc(e * B * (n + 1) * L * N);
      gX_[n].alloc(e * B * N);
      shapes_[n] = product_shape(n, L, B, N, e);
      if (segmented()) segment_ranges(shapes_[n], support_.seg[n]);
      max_part = std::max(max_part, (size_t)B * L * shapes_[n].blocks * shapes_[n].slots);
      if (opt_.cross)
        max_part = std::max(max_part, (size_t)cross_blocks(N) * vb_ * L * cross_slots(shapes_[n].K));
      max_gz = std::max(max_gz, e * 2 * B * L * N);
      max_gbr = std::max(max_gbr, e * 2 * B * (n + 1) * L * L * N);
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
      total_sums += opt_.cross ? (size_t)vb_ * L * cross_slots(shapes_[n].K) : (size_t)B * L * shapes_[n].slots;
    }
    total_sums_ = total_sums;
    if (segmented()) upload_ranges();
    plan_tables();
    size_mask_buffers();
    gZ_.alloc(max_gz);
    gBr_.alloc(max_gbr);
    err_.alloc(sizeof(int));
    STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_));
    // per-row constants of the fields: maps [level][B], moduli [level][B][L],
    // branch rows of one level, and the partial sums of their means
    xc_.alloc(sizeof(double) * levels_ * B);
    zc_.alloc(sizeof(double) * levels_ * B * L);
    rc_.alloc(sizeof(double) * B * levels_ * L);
    mpart_.alloc(sizeof(double) * kMeansBlocks * B * L);
    in_f64_.alloc(sizeof(double) * B * npix(0));
    field_bytes_ += partials_.bytes + sums_.bytes + gZ_.bytes + gBr_.bytes + in_f64_.bytes;
    if (!hi(0)) {  // FP32 level 0: the rounding residuals of its deviations
      xr_.alloc(sizeof(float) * B * npix(0));
      STL_CUDA(cudaMemsetAsync(xr_.p, 0, xr_.bytes, stream_));
      field_bytes_ += xr_.bytes;
    }
    // partial sums of the row-centric adjoint
    {
      size_t cap = 0;
      for (int n = 0; n < levels_; ++n)
        cap = std::max(cap, adjoint_part_bytes(conv_[n], esz(n), B * (n + 1) * L));
      if (cap) adj_part_.alloc(cap);
      adj_.part = adj_part_.p;
      adj_.capacity = cap;
      field_bytes_ += adj_part_.bytes;
    }
    STL_CUDA(cudaStreamSynchronize(stream_));
    tune();
    ready_ = true;
    ++graph_epoch_;
    timers.build_s += ms_since(t0) / 1000.0;
  }

  void load_host(const double* x) override {
    prepare();
    size_t n = (size_t)opt_.B * npix(0);
    if (io_.to_device(in_f64_.p, x, n * 8, stream_, true))
      throw std::runtime_error("input map contains non-finite values");
    load_maps(in_f64_.as<double>());
  }

  // level-0 maps (map-major, device) -> constants [B] and pixel-major
  // deviations; the pyramid levels carry the same constants
  template <typename Tin>
  void load_maps(const Tin* x) {
    const int B = opt_.B;
    const i64 N = npix(0);
    prof_.launch(Profiler::ELEM, 3, B * N * (2.0 * sizeof(Tin) + esz(0)), 0.0, stream_, [&] {
      row_means<Tin>(x, false, false, N, B, mpart_.as<double>(), xc_.as<double>(), stream_);
      typed(0, [&](auto t) {
        using U = typename decltype(t)::type;
        to_pixel_major<Tin, U>(x, X_[0].as<U>(), N, B, stream_, xc_.as<double>(), xr_.as<U>());
      });
    });
    for (int d = 1; d < levels_; ++d)
      STL_CUDA(cudaMemcpyAsync(xc_.as<double>() + d * B, xc_.p, sizeof(double) * B, cudaMemcpyDeviceToDevice,
                               stream_));
    loaded_ = true;
    levels_given_ = false;
  }

  void load_levels(const double* x) override {
    prepare();
    size_t off = 0;
    for (int d = 0; d < levels_; ++d) {
      const size_t n = (size_t)opt_.B * npix(d);
      STL_CUDA(cudaMemcpyAsync(in_f64_.p, x + off, n * 8, cudaMemcpyHostToDevice, stream_));
      double* c = xc_.as<double>() + (size_t)d * opt_.B;
      row_means<double>(in_f64_.as<double>(), false, false, npix(d), opt_.B, mpart_.as<double>(), c, stream_);
      typed(d, [&](auto t) {
        using U = typename decltype(t)::type;
        to_pixel_major<double, U>(in_f64_.as<double>(), X_[d].as<U>(), npix(d), opt_.B, stream_, c,
                                  d == 0 ? xr_.as<U>() : nullptr);
      });
      STL_CUDA(cudaStreamSynchronize(stream_));  // the staging buffer is reused for the next level
      off += n;
    }
    loaded_ = true;
    levels_given_ = true;
  }

  void load_device_levels(const double* const* x) override {
    prepare();
    for (int d = 0; d < levels_; ++d) {
      double* c = xc_.as<double>() + (size_t)d * opt_.B;
      prof_.launch(Profiler::ELEM, 3, opt_.B * npix(d) * (2.0 * 8 + esz(d)), 0.0, stream_, [&] {
        row_means<double>(x[d], false, false, npix(d), opt_.B, mpart_.as<double>(), c, stream_);
        typed(d, [&](auto t) {
          using U = typename decltype(t)::type;
          to_pixel_major<double, U>(x[d], X_[d].as<U>(), npix(d), opt_.B, stream_, c, d == 0 ? xr_.as<U>() : nullptr);
        });
      });
    }
    loaded_ = true;
    levels_given_ = true;
  }

  void load_device(const void* x, bool f32) override {
    prepare();
    if (f32) load_maps(static_cast<const float*>(x));
    else load_maps(static_cast<const double*>(x));
  }

  // the level-0 deviations in FP64 (FP32 fields: with their residuals) and
  // their constants
  void save_state(std::vector<double>& st) override {
    const size_t n = (size_t)opt_.B * npix(0);
    st.resize(n + opt_.B);
    if (xr_.p) join_f64(X_[0].as<float>(), xr_.as<float>(), in_f64_.as<double>(), (i64)n, stream_);
    else
      typed(0, [&](auto t) {
        using U = typename decltype(t)::type;
        convert<U, double>(X_[0].as<U>(), in_f64_.as<double>(), (i64)n, stream_);
      });
    STL_CUDA(cudaMemcpyAsync(st.data(), in_f64_.p, n * 8, cudaMemcpyDeviceToHost, stream_));
    STL_CUDA(cudaMemcpyAsync(st.data() + n, xc_.p, sizeof(double) * opt_.B, cudaMemcpyDeviceToHost, stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }
  void load_state(const std::vector<double>& st) override {
    prepare();
    const size_t n = (size_t)opt_.B * npix(0);
    if (st.size() != n + (size_t)opt_.B) throw std::runtime_error("checkpoint of another configuration");
    STL_CUDA(cudaMemcpyAsync(in_f64_.p, st.data(), n * 8, cudaMemcpyHostToDevice, stream_));
    if (xr_.p) split_f64(in_f64_.as<double>(), X_[0].as<float>(), xr_.as<float>(), (i64)n, stream_);
    else
      typed(0, [&](auto t) {
        using U = typename decltype(t)::type;
        convert<double, U>(in_f64_.as<double>(), X_[0].as<U>(), (i64)n, stream_);
      });
    for (int d = 0; d < levels_; ++d)
      STL_CUDA(cudaMemcpyAsync(xc_.as<double>() + (size_t)d * opt_.B, st.data() + n, sizeof(double) * opt_.B,
                               cudaMemcpyHostToDevice, stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
    loaded_ = true;
    levels_given_ = false;
  }

  void save_input(std::vector<double>& x) override {
    i64 n = (i64)opt_.B * npix(0);
    if (xr_.p) {  // deviations and residuals in FP64 (pixel-major), then map-major plus the constants
      const i64 N = npix(0);
      const int B = opt_.B;
      std::vector<double> d(n), c(B);
      join_f64(X_[0].as<float>(), xr_.as<float>(), in_f64_.as<double>(), n, stream_);
      STL_CUDA(cudaMemcpyAsync(d.data(), in_f64_.p, n * 8, cudaMemcpyDeviceToHost, stream_));
      STL_CUDA(cudaMemcpyAsync(c.data(), xc_.p, sizeof(double) * B, cudaMemcpyDeviceToHost, stream_));
      STL_CUDA(cudaStreamSynchronize(stream_));
      x.resize(n);
      for (int b = 0; b < B; ++b)
        for (i64 p = 0; p < N; ++p) x[(size_t)b * N + p] = d[(size_t)p * B + b] + c[b];
      return;
    }
    typed(0, [&](auto t) {
      using U = typename decltype(t)::type;
      to_map_major<U, double>(X_[0].as<U>(), in_f64_.as<double>(), npix(0), opt_.B, stream_, xc_.as<double>());
    });
    x.resize(n);
    STL_CUDA(cudaMemcpyAsync(x.data(), in_f64_.p, n * 8, cudaMemcpyDeviceToHost, stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  void forward(bool moments, double* values, double* var) override {
    if (!loaded_) throw std::runtime_error("forward before the maps were loaded");
    auto t0 = std::chrono::steady_clock::now();
    const int B = opt_.B;
    const size_t nv = (size_t)vb_ * K_ * plan_.size();
    in_graph(gfwd_, (moments ? 1 : 0) + (levels_given_ ? 2 : 0), [&] {
      forward_sweep(moments);
      // the coefficients (and variances) of every map and mask, from the sums
      prof_.launch(Profiler::ELEM, 1, 16.0 * nv, 0.0, stream_, [&] {
        assemble_values(sums_.as<double>(), total_sums_, plan_dev_.as<PlanSlots>(), (int)plan_.size(),
                        counts_dev_.as<double>(), levels_, vb_, K_, vals_dev_.as<double>(),
                        moments ? var_dev_.as<double>() : nullptr, stream_);
      });
    });
    cudaStream_t s = stream_;
    STL_CUDA(cudaMemcpyAsync(values, vals_dev_.p, 16 * nv, cudaMemcpyDeviceToHost, s));
    if (moments && var) STL_CUDA(cudaMemcpyAsync(var, var_dev_.p, 8 * nv, cudaMemcpyDeviceToHost, s));
    int err = 0;
    STL_CUDA(cudaMemcpyAsync(&err, err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    prof_.collect();
    if (err) {
      STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), s));
      throw std::runtime_error(wait_timeout_message(err, "the forward sweep"));
    }
    forward_done_ = true;
    timers.forward_ms += ms_since(t0);
    timers.forwards += 1;
  }

  // the forward launches: pyramid, then every level's fields and sums
  void forward_sweep(bool moments) {
    const int B = opt_.B;
    cudaStream_t s = stream_;
    for (int d = 0; d + 1 < levels_ && !levels_given_; ++d)
      prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[d], B, false), dec_flops(dec_[d], B, false), s, [&] {
        typed(d, [&](auto ti) {
          typed(d + 1, [&](auto to) {
            using Ui = typename decltype(ti)::type;
            using Uo = typename decltype(to)::type;
            dec_apply<Ui, Uo>(dec_[d], false, X_[d].as<Ui>(), B, 0, X_[d + 1].as<Uo>(), B, 0, 1, B, false, s,
                              tile(d, T_DEC_X));
          });
        });
      });
    for (int n = 0; n < levels_; ++n)
      typed(n, [&](auto t) { forward_level<typename decltype(t)::type>(n, moments); });
  }

  void set_objective(const double* target, const double* weights) override {
    prepare();
    const size_t nv = (size_t)vb_ * K_ * plan_.size(), np = plan_.size();
    target_dev_.alloc(16 * nv);
    STL_CUDA(cudaMemcpyAsync(target_dev_.p, target, 16 * nv, cudaMemcpyHostToDevice, stream_));
    weights_dev_.release();
    if (weights) {
      weights_dev_.alloc(8 * np);
      STL_CUDA(cudaMemcpyAsync(weights_dev_.p, weights, 8 * np, cudaMemcpyHostToDevice, stream_));
    }
    STL_CUDA(cudaStreamSynchronize(stream_));
    objective_set_ = true;
  }

  void objective(const double* x, double* g, double* loss) override {
    if (!objective_set_) throw std::runtime_error("objective before set_objective");
    cudaStream_t s = stream_;
    const int B = opt_.B;
    load_maps(x);
    forward_sweep(false);
    const i64 nv = (i64)vb_ * K_ * plan_.size();
    prof_.launch(Profiler::ELEM, 1, 16.0 * nv, 0.0, s, [&] {
      assemble_values(sums_.as<double>(), total_sums_, plan_dev_.as<PlanSlots>(), (int)plan_.size(),
                      counts_dev_.as<double>(), levels_, vb_, K_, vals_dev_.as<double>(), nullptr, s);
    });
    objective_terms(vals_dev_.as<double>(), target_dev_.as<double>(),
                    weights_dev_.p ? weights_dev_.as<double>() : nullptr, nv, (int)plan_.size(),
                    cot_dev_.as<double>(), loss, s);
    reverse_launches();
    typed(0, [&](auto t) {
      using U = typename decltype(t)::type;
      to_map_major<U, double>(gX_[0].as<U>(), g, npix(0), B, s);
    });
    forward_done_ = true;
  }

  int* error_flag() override { return err_.as<int>(); }

  template <typename U>
  void forward_level(int n, bool moments) {
    const int L = opt_.L, B = opt_.B;
    cudaStream_t s = stream_;
    const i64 N = npix(n);
    U* mod = Mod_[n].as<U>();
    const ConvOp& op = conv_[n];
    prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, B, true, false), conv_flops(op, B), s, [&] {
      conv_forward<U>(op, X_[n].as<U>(), B, zf<U>(n), nullptr, 0, 0, 0, s, err_.as<int>(),
                      xc_.as<double>() + (size_t)n * B, tile(n, T_FWD_Z));
    });
    // |z| as deviations from their means per (map, orientation)
    double* zc = zc_.as<double>() + (size_t)n * B * L;
    prof_.launch(Profiler::ELEM, 3, (double)N * B * L * (2 * 2 * sizeof(U) + sizeof(U)), 0.0, s, [&] {
      row_means<U>(zf<U>(n), true, true, N, B * L, mpart_.as<double>(), zc, s);
      moduli_deviations<U>(zf<U>(n), N, B, L, zc, mod, B * (n + 1) * L, (n + 1) * L, n * L, s);
    });
    if (n > 0)
      prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n - 1], B * n * L, false), dec_flops(dec_[n - 1], B * n * L, false),
                   s, [&] {
                     typed(n - 1, [&](auto ti) {
                       using Ui = typename decltype(ti)::type;
                       dec_apply<Ui, U>(dec_[n - 1], false, Mod_[n - 1].as<Ui>(), B * n * L, n * L, mod,
                                        B * (n + 1) * L, (n + 1) * L, B, n * L, false, s, tile(n, T_DEC_MOD));
                     });
                   });
    const int R = B * (n + 1) * L;
    prof_.launch(Profiler::ELEM, 1, 16.0 * B * L, 0.0, s,
                 [&] { branch_constants(zc_.as<double>(), n, B, L, rc_.as<double>(), s); });
    prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, R, true, false), conv_flops(op, R), s, [&] {
      conv_forward<U>(op, mod, R, brf<U>(n), nullptr, 0, 0, 0, s, err_.as<int>(), rc_.as<double>(),
                      tile(n, T_FWD_BR));
    });
    const ProductShape& sh = shapes_[n];
    const double E = sh.K * (sh.K + 1) / 2.0;
    if (opt_.cross) {  // the cross terms of each channel pair only
      for (int k = 0; k < launch_sets(); ++k)
        prof_.launch(Profiler::PROD_FWD, 2, (double)B * L * N * sh.K * 2 * sizeof(U),
                     (double)vb_ * L * N * sh.K * sh.K * 8.0, s, [&] {
                       cross_forward<U>(sh.K, N, B, zf<U>(n), brf<U>(n), mask(k, n), moments,
                                        partials_.as<double>(), cross_blocks(N),
                                        sums_.as<double>() + k * total_sums_ + sum_off_[n], s);
                     });
      return;
    }
    for (int k = 0; k < launch_sets(); ++k)
      prof_.launch(Profiler::PROD_FWD, 2, (double)B * L * N * sh.K * 2 * sizeof(U), (double)B * L * N * E * 10.0, s,
                   [&] {
                     products_forward<U>(sh, zf<U>(n), brf<U>(n), n == 0 ? X_[0].as<U>() : nullptr,
                                         n == 0 ? xr_.as<U>() : nullptr, xc_.as<double>(), mask(k, n), partials_.as<double>(),
                                         sums_.as<double>() + k * total_sums_ + sum_off_[n], err_.as<int>(), s,
                                         moments);
                   });
  }

  void reverse_host(const double* cot, double* out) override {
    reverse_impl(cot);
    i64 n = (i64)opt_.B * npix(0);
    if (!hi(0)) {  // FP32 gradients: moved as floats and widened on the host (exact)
      prof_.launch(Profiler::ELEM, 1, n * (4.0 + esz(0)), 0.0, stream_, [&] {
        to_map_major<float, float>(gX_[0].as<float>(), in_f64_.as<float>(), npix(0), opt_.B, stream_);
      });
      io_.to_host_widen(out, in_f64_.as<float>(), (size_t)n, stream_);
      return;
    }
    prof_.launch(Profiler::ELEM, 1, n * (8.0 + esz(0)), 0.0, stream_, [&] {
      typed(0, [&](auto t) {
        using U = typename decltype(t)::type;
        to_map_major<U, double>(gX_[0].as<U>(), in_f64_.as<double>(), npix(0), opt_.B, stream_);
      });
    });
    io_.to_host(out, in_f64_.p, n * 8, stream_);
  }

  void reverse_device(const double* cot, void* out, bool f32) override {
    reverse_impl(cot);
    i64 n = (i64)opt_.B * npix(0);
    prof_.launch(Profiler::ELEM, 1, n * ((f32 ? 4.0 : 8.0) + esz(0)), 0.0, stream_, [&] {
      typed(0, [&](auto t) {
        using U = typename decltype(t)::type;
        if (f32) to_map_major<U, float>(gX_[0].as<U>(), static_cast<float*>(out), npix(0), opt_.B, stream_);
        else to_map_major<U, double>(gX_[0].as<U>(), static_cast<double*>(out), npix(0), opt_.B, stream_);
      });
    });
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  size_t host_to_device(void* dst, const void* src, size_t n, bool check) override {
    return io_.to_device(dst, src, n, stream_, check);
  }
  void device_to_host(void* dst, const void* src, size_t n) override { io_.to_host(dst, src, n, stream_); }

  void reverse_levels(const double* cot, double* const* out) override {
    if (!levels_given_) throw std::runtime_error("per-level cotangents need maps given at every level");
    reverse_impl(cot);
    for (int d = 0; d < levels_; ++d)
      prof_.launch(Profiler::ELEM, 1, (double)opt_.B * npix(d) * (8.0 + esz(d)), 0.0, stream_, [&] {
        typed(d, [&](auto t) {
          using U = typename decltype(t)::type;
          to_map_major<U, double>(gX_[d].as<U>(), out[d], npix(d), opt_.B, stream_);
        });
      });
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  std::vector<KernelStat> kernel_stats() const override {
    return std::vector<KernelStat>(prof_.stat, prof_.stat + Profiler::NCAT);
  }
  void reset_kernel_stats() override { prof_.reset(); }
  void set_profiling(bool on) override { prof_.on = on; }
  bool profiling() const override { return prof_.on; }
  std::vector<double> mean_slots() const override {
    std::vector<double> v;
    for (const auto& c : conv_) v.push_back(c.mean_slots);
    return v;
  }
  std::vector<std::array<int, 8>> tile_heights() const override { return tiles_; }
  void operator_rows(int level, int kind, std::vector<int64_t>& out, std::vector<double>& weight,
                     int& width) override {
    prepare();
    if (grid_mode()) throw std::runtime_error("operator tables are exported for full-sky engines");
    if (level < 0 || level >= levels_ || kind < 0 || kind > 1 || (kind == 1 && level + 1 >= levels_))
      throw std::runtime_error("no such operator");
    cudaStream_t s = stream_;
    auto fetch = [&](const DevMem& m, auto* tag) {
      using V = std::remove_pointer_t<decltype(tag)>;
      std::vector<V> h(m.bytes / sizeof(V));
      if (m.bytes) STL_CUDA(cudaMemcpyAsync(h.data(), m.p, m.bytes, cudaMemcpyDeviceToHost, s));
      return h;
    };
    auto fetch_real = [&](const DevMem& m, DType t) {
      std::vector<double> h;
      if (t == DType::F64) {
        auto v = fetch(m, (double*)nullptr);
        STL_CUDA(cudaStreamSynchronize(s));
        h.assign(v.begin(), v.end());
      } else {
        auto v = fetch(m, (float*)nullptr);
        STL_CUDA(cudaStreamSynchronize(s));
        h.assign(v.begin(), v.end());
      }
      return h;
    };
    auto rotp = [](i64 u, int k, int o2) {
      return ((4 * (u >> o2) + k) << o2) | (u & ((i64(1) << o2) - 1));
    };
    auto rotc = [](i64 c, int k, int o2) {
      const i64 f = c >> o2;
      return (((f & ~i64(3)) | ((f + k) & 3)) << o2) | (c & ((i64(1) << o2) - 1));
    };
    // per stored row: (cell, weight) entries; the weight of a wavelet cell is
    // its largest |coefficient|, of a decimation column |w|
    std::vector<std::vector<std::pair<int64_t, double>>> rows;
    int nk = 1, o2_row = 0, o2_cell = 0;
    auto cmax = [](const double* c) {
      double m = 0.0;
      for (int j = 0; j < 8; ++j) m = std::max(m, std::fabs(c[j]));
      return m;
    };
    if (kind == 0) {
      const ConvOp& op = conv_[level];
      nk = op.nk; o2_row = o2_cell = op.o2;
      rows.resize(op.n_rep);
      if (op.mma) {
        auto lc = fetch(op.m_lc, (uint16_t*)nullptr);
        auto cells = fetch(op.m_cells, (int32_t*)nullptr);
        auto rch = fetch(op.m_rowch, (uint8_t*)nullptr);
        auto coef = fetch_real(op.m_coef, DType::F32);
        for (i64 u = 0; u < op.n_rep; ++u) {
          const i64 tile = u / kMmaRows, ul = u % kMmaRows;
          for (int c = 0; c < rch[u]; ++c)
            for (int p = 0; p < 8; ++p) {
              const int pl = lc[((tile * (op.m_S / 8) + c) * kMmaRows + ul) * 8 + p];
              const int32_t cell = cells[tile * op.m_pc + pl];
              if (cell >= 0) rows[u].push_back({cell, cmax(&coef[((i64)(8 * c + p) * op.n_rep + u) * 8])});
            }
        }
      } else {
        auto cell = fetch(op.cell, (int32_t*)nullptr);
        auto coef = fetch_real(op.coef, op.dtype);
        for (i64 u = 0; u < op.n_rep; ++u)
          for (int sl = 0; sl < op.S; ++sl)
            rows[u].push_back({cell[(i64)sl * op.n_rep + u], cmax(&coef[((i64)sl * op.n_rep + u) * 8])});
      }
    } else {
      const DecOp& op = dec_[level];
      nk = op.nk; o2_row = op.co2; o2_cell = op.o2;
      rows.resize(op.n_rep_out);
      auto col = fetch(op.col, (int32_t*)nullptr);
      auto w = fetch_real(op.w, op.dtype);
      for (i64 u = 0; u < op.n_rep_out; ++u)
        for (int e = 0; e < op.W; ++e) {
          const double v = w[(i64)e * op.n_rep_out + u];
          if (v != 0.0) rows[u].push_back({col[(i64)e * op.n_rep_out + u], std::fabs(v)});
        }
    }
    // distinct cells (a padding slot repeats a real cell with zero
    // coefficients: the largest weight is kept)
    width = 0;
    for (auto& r : rows) {
      std::sort(r.begin(), r.end());
      std::vector<std::pair<int64_t, double>> m;
      for (const auto& e : r) {
        if (!m.empty() && m.back().first == e.first) m.back().second = std::max(m.back().second, e.second);
        else m.push_back(e);
      }
      r.swap(m);
      width = std::max(width, (int)r.size());
    }
    const i64 npx = (i64)rows.size() * nk;
    out.assign((size_t)npx * width, -1);
    weight.assign((size_t)npx * width, 0.0);
    for (i64 u = 0; u < (i64)rows.size(); ++u)
      for (int k = 0; k < nk; ++k) {
        const i64 p = nk == 4 ? rotp(u, k, o2_row) : u;
        std::vector<std::pair<int64_t, double>> r;
        for (const auto& e : rows[u]) r.push_back({nk == 4 ? rotc(e.first, k, o2_cell) : e.first, e.second});
        std::sort(r.begin(), r.end());
        for (size_t j = 0; j < r.size(); ++j) {
          out[(size_t)p * width + j] = r[j].first;
          weight[(size_t)p * width + j] = r[j].second;
        }
      }
  }

  bool recomputes() const override { return recompute_; }
  size_t kept_field_bytes() const override { return keep_bytes_; }

  std::vector<std::array<int, 4>> operator_layout() const override {
    std::vector<std::array<int, 4>> v;
    for (const auto& c : conv_)
      v.push_back({c.mma ? c.m_S : c.S, c.mma ? c.m_pc : c.max_tile_cells,
                   c.mma_adj ? 3 : c.mma ? 2 : c.colored ? 1 : 0, c.mma_adj ? c.m_wl : 0});
    return v;
  }

 private:
  // Algorithmic traffic of one wavelet launch over R rows: the used
  // coefficients of the stored rows (2L values and a 4-byte cell index per
  // cell read; a quarter of the rows on the full sky), the input rows read
  // once, the complex outputs written once (plus |z|, or the
  // read-modify-write of an accumulated adjoint).
  double conv_bytes(const ConvOp& op, int R, bool fwd, bool extra) const {
    const double s = op.dtype == DType::F64 ? 8.0 : 4.0, N = (double)op.n_rows, D = op.mean_slots;
    double coef = (double)op.n_rep * D * (8.0 * s + 4.0);
    double field = fwd ? R * N * s + R * N * 8.0 * s : R * N * 8.0 * s + R * N * s;
    if (extra) field += fwd ? R * N * 4.0 * s : R * N * s;
    return coef + field;
  }
  double conv_flops(const ConvOp& op, int R) const { return 2.0 * 8.0 * R * (double)op.n_rows * op.mean_slots; }
  double dec_bytes(const DecOp& op, int R, bool transpose) const {
    const double s = op.dtype == DType::F64 ? 8.0 : 4.0;
    double nnz = op.mean_w * (double)op.n_rep_out;  // the stored rows (a quarter on the full sky) are read
    return nnz * (s + 4.0) + R * (double)(op.n_in + op.n_out) * s;
    (void)transpose;
  }
  double dec_flops(const DecOp& op, int R, bool) const { return 2.0 * R * op.mean_w * (double)op.n_out; }

  // where a plan coefficient's sums live: level, l3 row, and the slots of
  // its real part, imaginary part (-1: exactly zero) and second moment
  struct Loc {
    int level, l3, re, im, second;
    int conj = 0;  // the coefficient is the conjugate of the sum
  };

  // cross terms (the cross_slots layout of kernels.cu): S1 the rn term, S2
  // G[z][z], terms in channel order (0, 1) G[r][q] and in order (1, 0)
  // conj(G[q][r]), r and q the operand entries (branch (d, l) at d L + l, z
  // last) of channels 0 and 1 (operands of engine.rs:956-984)
  Loc locate_cross(const Coef& c) const {
    const int L = opt_.L, n = c.native, K = (n + 1) * L + 1, z = K - 1, K2 = K * K;
    Loc l{n, 0, 0, 0, 0, 0};
    auto entry = [&](int e, bool conj) {
      l.re = 2 * e;
      l.im = 2 * e + 1;
      l.second = 2 * K2 + 2 + e;
      l.conj = conj ? 1 : 0;
    };
    switch (c.family) {
      case S1: l.l3 = c.l1; l.re = 2 * K2; l.im = 2 * K2 + 1; l.second = 3 * K2 + 2; break;
      case S2: l.l3 = c.l1; entry(z * K + z, false); break;
      case S3: {
        const int r = c.j1 * L + c.l1;
        l.l3 = c.l3;
        if (c.c1 == 0) entry(r * K + z, false);
        else entry(z * K + r, true);
        break;
      }
      case S4: {
        const int r = c.j1 * L + c.l1, q = c.j2 * L + c.l2;
        l.l3 = c.l3;
        if (c.c1 == 0) entry(r * K + q, false);
        else entry(q * K + r, true);
        break;
      }
      default: throw std::runtime_error("cross plans hold S1-S4 only");
    }
    return l;
  }

  // Sums of the products kernel per (b, l3) (kernels.cu): 4 x 4 Gram blocks
  // (d1 <= d2) of the branches, 4 x 1 blocks (d, z), then the per-pixel sums.
  Loc locate(const Coef& c) const {
    if (opt_.cross) return locate_cross(c);
    const int L = opt_.L;
    const int n = c.native, nd = n + 1;
    const int nBB = nd * (nd + 1) / 2, zb = nBB * 48 + nd * 12;
    auto tblock = [&](int d1, int d2) { return d1 * nd - d1 * (d1 - 1) / 2 + (d2 - d1); };
    Loc l{n, 0, 0, 0, 0, 0};
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

  void reverse_impl(const double* cot) {
    if (!forward_done_) throw std::runtime_error("vjp before forward");
    io_.to_device(cot_dev_.p, cot, 16 * (size_t)vb_ * K_ * plan_.size(), stream_);
    reverse_sweep();
  }

  // the reverse sweep from the coefficient cotangents in cot_dev_
  void reverse_sweep() {
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = stream_;
    in_graph(grev_, levels_given_ ? 1 : 0, [&] { reverse_launches(); });
    int err = 0;
    STL_CUDA(cudaMemcpyAsync(&err, err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    STL_CUDA(cudaStreamSynchronize(s));
    prof_.collect();
    if (err) {
      STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), s));
      throw std::runtime_error(wait_timeout_message(err, "the reverse sweep"));
    }
    timers.reverse_ms += ms_since(t0);
    timers.reverses += 1;
  }

  // the reverse launches: cotangent matrices, then the levels descending and
  // the mean / variance terms into gX_[0]
  void reverse_launches() {
    const int L = opt_.L, B = opt_.B;
    const int np = (int)plan_.size();
    cudaStream_t s = stream_;
    // per level and mask: cotangent matrices and S1 scales in the level's
    // field type; the mean and variance scales
    for (int n = 0; n < levels_; ++n)
      prof_.launch(Profiler::ELEM, 1, (double)K_ * B * (L * shapes_[n].K * shapes_[n].K + L) * 16.0, 0.0, s, [&] {
        typed(n, [&](auto t) {
          using U = typename decltype(t)::type;
          unsigned char* base = stage_dev_.as<unsigned char>();
          build_cotangents<U>(cot_dev_.as<double>(), np, vb_, K_, counts_dev_.as<double>(), levels_, n, shapes_[n].K,
                              L, cotsrc_dev_.as<CotSources>() + cotsrc_off_[n],
                              cotsrc_dev_.as<CotSources>() + cotsrc_off_[n] + (size_t)L * shapes_[n].K * shapes_[n].K,
                              reinterpret_cast<U*>(base + stage_m_[(size_t)n * K_]),
                              reinterpret_cast<U*>(base + stage_s_[(size_t)n * K_]), s, opt_.cross);
        });
      });
    if (!opt_.cross)
      prof_.launch(Profiler::ELEM, 1, 16.0 * B * K_ * 2, 0.0, s, [&] {
        build_mean_var(cot_dev_.as<double>(), np, B, K_, counts_dev_.as<double>(), levels_, i_mean_, i_var_,
                       mv_.as<double>(), s);
      });
    for (int n = levels_ - 1; n >= 0; --n)
      typed(n, [&](auto t) { reverse_level<typename decltype(t)::type>(n); });
    for (int k = 0; k < launch_sets() && !opt_.cross; ++k)  // the cross plan has no mean or variance
      prof_.launch(Profiler::ELEM, 1, (double)B * npix(0) * 3 * esz(0), (double)B * npix(0) * 2.0, s, [&] {
        typed(0, [&](auto t) {
          using U = typename decltype(t)::type;
          mean_var_grad<U>(X_[0].as<U>(), xc_.as<double>(), mask(k, 0), mv_.as<double>() + (size_t)k * 2 * B, B,
                           npix(0), gX_[0].as<U>(), s, segmented() ? seg_dev_[0].as<i64>() : nullptr, K_);
        });
      });
  }

  // one level of the reverse sweep (field type U); M: the level's cotangent
  // matrices [B][L][K][K], s1: the auto-S1 scales [B][L]
  template <typename U>
  void reverse_level(int n) {
    const int L = opt_.L, B = opt_.B;
    cudaStream_t s = stream_;
    const i64 N = npix(n);
    const ProductShape& sh = shapes_[n];
    const ConvOp& op = conv_[n];
    U* gmod = gMod_[n].as<U>();
    if (n + 1 < levels_)
      prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n], B * (n + 1) * L, true), dec_flops(dec_[n], B * (n + 1) * L, true),
                   s, [&] {
                     typed(n + 1, [&](auto ti) {
                       using Ui = typename decltype(ti)::type;
                       dec_apply<Ui, U>(dec_[n], true, gMod_[n + 1].as<Ui>(), B * (n + 2) * L, (n + 2) * L, gmod,
                                        B * (n + 1) * L, (n + 1) * L, B, (n + 1) * L, false, s, tile(n, T_DECT_MOD));
                     });
                   });
    else
      STL_CUDA(cudaMemsetAsync(gmod, 0, gMod_[n].bytes, s));
    if (recompute_) {
      // the level's z and branches again, from the kept maps and stored
      // moduli (the forward's launches on the same inputs: identical values)
      const int Rb = B * (n + 1) * L;
      prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, B, true, false), conv_flops(op, B), s, [&] {
        conv_forward<U>(op, X_[n].as<U>(), B, zf<U>(n), nullptr, 0, 0, 0, s, err_.as<int>(),
                        xc_.as<double>() + (size_t)n * B, tile(n, T_FWD_Z));
      });
      prof_.launch(Profiler::ELEM, 1, 16.0 * B * L, 0.0, s,
                   [&] { branch_constants(zc_.as<double>(), n, B, L, rc_.as<double>(), s); });
      prof_.launch(Profiler::CONV_FWD, 1, conv_bytes(op, Rb, true, false), conv_flops(op, Rb), s, [&] {
        conv_forward<U>(op, Mod_[n].as<U>(), Rb, brf<U>(n), nullptr, 0, 0, 0, s, err_.as<int>(), rc_.as<double>(),
                        tile(n, T_FWD_BR));
      });
    }
    // cotangent matrices and S1 scales in the field precision, one set per
    // mask, staged for every level before the sweep; the products VJP of
    // mask k > 0 adds to that of the masks before it
    const double sz = sizeof(U);
    for (int k = 0; k < launch_sets(); ++k) {
      const U* Mdev = reinterpret_cast<const U*>(stage_dev_.as<unsigned char>() + stage_m_[(size_t)n * K_ + k]);
      const U* sdev = reinterpret_cast<const U*>(stage_dev_.as<unsigned char>() + stage_s_[(size_t)n * K_ + k]);
      prof_.launch(Profiler::PROD_REV, 1, (double)B * L * N * sh.K * 4 * sz, (double)B * L * N * sh.K * sh.K * 8.0,
                   s, [&] {
                     if (opt_.cross)
                       cross_reverse<U>(sh.K, N, B, zf<U>(n), brf<U>(n), Mdev, sdev, mask(k, n), k > 0,
                                        gZ_.as<U>(), gBr_.as<U>(), s);
                     else
                       products_reverse<U>(sh, zf<U>(n), brf<U>(n), Mdev, sdev, mask(k, n), k > 0,
                                           gZ_.as<U>(), gBr_.as<U>(), s);
                   });
    }
    const int R = B * (n + 1) * L;
    prof_.launch(Profiler::CONV_ADJ, adjoint_tiles_usable(op, sizeof(U), R, adj_ptr()) ? 2 : 1,
                 conv_bytes(op, R, false, true), conv_flops(op, R), s,
                 [&] {
                   conv_adjoint<U>(op, gBr_.as<U>(), R, gmod, true, s, adj_ptr(), err_.as<int>(), nullptr,
                                   tile(n, T_ADJ_BR));
                 });
    // the modulus VJP of z (gZ += gmod z / |z|): inside the coloured adjoint
    // of z when the operator has it, else its own pass
    ModulusAdd<U> madd;
    madd.z = zf<U>(n);
    madd.g = gmod + n * L;
    madd.g_pix = B * (n + 1) * L;
    madd.g_row = (n + 1) * L;
    const bool fuse = conv_adjoint_fuses_modulus(op, sizeof(U), B, adj_ptr(), err_.as<int>());
    if (!fuse)
      prof_.launch(Profiler::ELEM, 1, (double)B * L * N * 5 * sz, (double)B * L * N * 6.0, s, [&] {
        modulus_vjp_add<U>(zf<U>(n), gmod + n * L, B * (n + 1) * L, (n + 1) * L, gZ_.as<U>(), N, B, L, s);
      });
    prof_.launch(Profiler::CONV_ADJ, adjoint_tiles_usable(op, sizeof(U), B, adj_ptr()) ? 2 : 1,
                 conv_bytes(op, B, false, false), conv_flops(op, B), s, [&] {
                   conv_adjoint<U>(op, gZ_.as<U>(), B, gX_[n].as<U>(), false, s, adj_ptr(), err_.as<int>(),
                                   fuse ? &madd : nullptr, tile(n, T_ADJ_Z));
                 });
    if (n + 1 < levels_ && !levels_given_)  // maps given per level: no chain through the decimation
      prof_.launch(Profiler::DEC, 1, dec_bytes(dec_[n], B, true) + (double)B * N * sz, dec_flops(dec_[n], B, true), s,
                   [&] {
                     typed(n + 1, [&](auto ti) {
                       using Ui = typename decltype(ti)::type;
                       dec_apply<Ui, U>(dec_[n], true, gX_[n + 1].as<Ui>(), B, 0, gX_[n].as<U>(), B, 0, 1, B, true,
                                        s, tile(n, T_DECT_X));
                     });
                   });
  }

  // buffers whose size follows the number of masks: the sums, the
  // coefficients, their variances and cotangents, the staged cotangent
  // matrices (per level the masks' matrices one after the other, then their
  // S1 scales: a segmented launch reads all of them) and the mask counts
  void size_mask_buffers() {
    ++graph_epoch_;  // the sweeps' buffers move: capture them again
    const int L = opt_.L, B = opt_.B;
    const size_t nv = (size_t)vb_ * K_ * plan_.size();
    sums_.alloc(sizeof(double) * total_sums_ * K_);
    mv_.alloc(sizeof(double) * 2 * B * K_);
    vals_dev_.alloc(16 * nv);
    var_dev_.alloc(8 * nv);
    cot_dev_.alloc(16 * nv);
    stage_m_.assign((size_t)levels_ * K_, 0);
    stage_s_.assign((size_t)levels_ * K_, 0);
    size_t bytes = 0;
    auto align = [](size_t v) { return (v + 255) & ~(size_t)255; };
    for (int n = 0; n < levels_; ++n) {
      // with cross: one matrix per channel pair (batch entry), complex cross-S1 scales
      const size_t ms = esz(n) * 2 * vb_ * L * shapes_[n].K * shapes_[n].K, ss = esz(n) * vb_ * L * (opt_.cross ? 2 : 1);
      for (int k = 0; k < K_; ++k) stage_m_[(size_t)n * K_ + k] = bytes + k * ms;
      bytes = align(bytes + K_ * ms);
      for (int k = 0; k < K_; ++k) stage_s_[(size_t)n * K_ + k] = bytes + k * ss;
      bytes = align(bytes + K_ * ss);
    }
    stage_dev_.alloc(bytes);
    std::vector<double> counts((size_t)K_ * levels_);
    for (int k = 0; k < K_; ++k)
      for (int n = 0; n < levels_; ++n) counts[(size_t)k * levels_ + n] = (double)count(k, n);
    counts_dev_.alloc(sizeof(double) * counts.size());
    STL_CUDA(cudaMemcpyAsync(counts_dev_.p, counts.data(), sizeof(double) * counts.size(), cudaMemcpyHostToDevice,
                             stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  // where every plan coefficient's sums live, and the sources of every
  // cotangent matrix entry (the adjoint of the assembly: the S3 and S4
  // terms enter (r, q) as g and (q, r) as conj(g), S2 the diagonal z entry
  // as 2 Re g, engine.rs:1062-1113)
  void plan_tables() {
    const int L = opt_.L;
    const size_t np = plan_.size();
    std::vector<PlanSlots> ps(np);
    for (size_t i = 0; i < np; ++i) {
      const Loc& l = map_[i];
      const ProductShape& sh = shapes_[l.level];
      const int row = opt_.cross ? cross_slots(sh.K) : sh.slots;  // doubles per (map or pair, l3)
      ps[i] = PlanSlots{l.level, (int32_t)(sum_off_[l.level] + (size_t)l.l3 * row), L * row, l.re, l.im,
                        l.second, l.conj};
    }
    plan_dev_.alloc(sizeof(PlanSlots) * np);
    STL_CUDA(cudaMemcpyAsync(plan_dev_.p, ps.data(), sizeof(PlanSlots) * np, cudaMemcpyHostToDevice, stream_));
    cotsrc_off_.assign(levels_ + 1, 0);
    for (int n = 0; n < levels_; ++n)
      cotsrc_off_[n + 1] = cotsrc_off_[n] + (size_t)L * shapes_[n].K * shapes_[n].K + L;
    std::vector<CotSources> src(cotsrc_off_[levels_], CotSources{-1, -1, 0, 0});
    for (size_t i = 0; i < np; ++i) {
      const Coef& c = plan_[i];
      const int n = c.native, Kd = shapes_[n].K, z = Kd - 1;
      CotSources* base = src.data() + cotsrc_off_[n];
      const size_t E = (size_t)L * Kd * Kd;
      auto put = [&](size_t e, int mode) {
        CotSources& x = base[e];
        if (x.i0 < 0) { x.i0 = (int32_t)i; x.m0 = mode; }
        else if (x.i1 < 0) { x.i1 = (int32_t)i; x.m1 = mode; }
        else throw std::runtime_error("a cotangent entry with more than two sources");
      };
      if (opt_.cross) {  // the cotangents of G (the cross S1's complex)
        switch (c.family) {
          case S1: put(E + c.l1, 0); break;
          case S2: put(((size_t)c.l1 * Kd + z) * Kd + z, 0); break;
          case S3: {
            const int r = c.j1 * L + c.l1;
            if (c.c1 == 0) put(((size_t)c.l3 * Kd + r) * Kd + z, 0);
            else put(((size_t)c.l3 * Kd + z) * Kd + r, 1);
            break;
          }
          case S4: {
            const int r = c.j1 * L + c.l1, q = c.j2 * L + c.l2;
            if (c.c1 == 0) put(((size_t)c.l3 * Kd + r) * Kd + q, 0);
            else put(((size_t)c.l3 * Kd + q) * Kd + r, 1);
            break;
          }
          default: throw std::runtime_error("cross plans hold S1-S4 only");
        }
        continue;
      }
      switch (c.family) {
        case MEAN: i_mean_ = (int)i; break;
        case VAR: i_var_ = (int)i; break;
        case S1: put(E + c.l1, 0); break;
        case S2: put(((size_t)c.l1 * Kd + z) * Kd + z, 2); break;
        case S3: {
          const int r = c.j1 * L + c.l1;
          put(((size_t)c.l3 * Kd + r) * Kd + z, 0);
          put(((size_t)c.l3 * Kd + z) * Kd + r, 1);
          break;
        }
        case S4: {
          const int r = c.j1 * L + c.l1, q = c.j2 * L + c.l2;
          put(((size_t)c.l3 * Kd + r) * Kd + q, 0);
          put(((size_t)c.l3 * Kd + q) * Kd + r, 1);
          break;
        }
      }
    }
    cotsrc_dev_.alloc(sizeof(CotSources) * src.size());
    STL_CUDA(cudaMemcpyAsync(cotsrc_dev_.p, src.data(), sizeof(CotSources) * src.size(), cudaMemcpyHostToDevice,
                             stream_));
    STL_CUDA(cudaStreamSynchronize(stream_));
  }

  Profiler prof_;
  bool ready_ = false, loaded_ = false, forward_done_ = false;
  bool levels_given_ = false;  // X_[d] for d > 0 were loaded, not decimated
  std::vector<ConvOp> conv_;
  std::vector<DecOp> dec_;
  std::vector<DevMem> X_, Z_, Mod_, Br_, gMod_, gX_;
  // Sweeps as CUDA graphs: the launches of a sweep are captured on a private
  // stream at the first sweep of a configuration (key: the sweep's variant;
  // epoch: bumped whenever buffers, masks or tile heights change) and the
  // graph is launched into the engine's stream from then on.  Replays add the
  // captured launches' accounting.  Off while profiling (CUDA events need the
  // launches one by one) or with "graphs": false.
  struct SweepGraph {
    cudaGraphExec_t exec = nullptr;
    long key = -1;
    KernelStat delta[Profiler::NCAT];
    void reset() {
      if (exec) cudaGraphExecDestroy(exec);
      exec = nullptr;
      key = -1;
    }
    ~SweepGraph() { reset(); }
  };
  SweepGraph gfwd_, grev_;
  long graph_epoch_ = 0;
  cudaStream_t capture_stream_ = nullptr;
  template <typename F>
  void in_graph(SweepGraph& g, int variant, F&& launches) {
    if (!opt_.graphs || prof_.on) {
      launches();
      return;
    }
    const long key = graph_epoch_ * 8 + variant;
    if (!(g.exec && g.key == key)) {
      g.reset();
      if (!capture_stream_) STL_CUDA(cudaStreamCreateWithFlags(&capture_stream_, cudaStreamNonBlocking));
      KernelStat before[Profiler::NCAT];
      std::copy(prof_.stat, prof_.stat + Profiler::NCAT, before);
      cudaStream_t user = stream_;
      stream_ = capture_stream_;
      cudaGraph_t graph = nullptr;
      STL_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      try {
        launches();
      } catch (...) {
        cudaStreamEndCapture(stream_, &graph);
        if (graph) cudaGraphDestroy(graph);
        stream_ = user;
        throw;
      }
      const cudaError_t ec = cudaStreamEndCapture(stream_, &graph);
      stream_ = user;
      STL_CUDA(ec);
      const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      STL_CUDA(ei);
      g.key = key;
      for (int c = 0; c < Profiler::NCAT; ++c) {  // the capture counted the launches once: keep that
        g.delta[c].launches = prof_.stat[c].launches - before[c].launches;
        g.delta[c].calls = prof_.stat[c].calls - before[c].calls;
        g.delta[c].bytes = prof_.stat[c].bytes - before[c].bytes;
        g.delta[c].flops = prof_.stat[c].flops - before[c].flops;
      }
    } else {
      for (int c = 0; c < Profiler::NCAT; ++c) {
        prof_.stat[c].launches += g.delta[c].launches;
        prof_.stat[c].calls += g.delta[c].calls;
        prof_.stat[c].bytes += g.delta[c].bytes;
        prof_.stat[c].flops += g.delta[c].flops;
      }
    }
    STL_CUDA(cudaGraphLaunch(g.exec, stream_));
  }

  // recompute field store: the one z and branch buffer of every level
  bool recompute_ = false;
  size_t keep_bytes_ = 0;  // z and branches of every level (the kept store)
  DevMem Zs_, Brs_;
  template <typename U> U* zf(int n) { return recompute_ ? Zs_.as<U>() : Z_[n].as<U>(); }
  template <typename U> U* brf(int n) { return recompute_ ? Brs_.as<U>() : Br_[n].as<U>(); }
  std::vector<ProductShape> shapes_;
  std::vector<size_t> sum_off_;
  DevMem partials_, sums_, gZ_, gBr_, mv_, in_f64_, err_, roles_;
  DevMem stage_dev_;                      // cotangent matrices and S1 scales of every level
  std::vector<size_t> stage_m_, stage_s_;  // byte offsets per (level, mask)
  DevMem plan_dev_, counts_dev_, vals_dev_, var_dev_, cot_dev_, cotsrc_dev_;
  std::vector<size_t> cotsrc_off_;  // per level: first cotangent source entry
  int i_mean_ = -1, i_var_ = -1;    // plan entries of the mean and the variance
  DevMem target_dev_, weights_dev_;  // the synthesis objective
  HostStage io_;                     // large host <-> device copies
  bool objective_set_ = false;
  DevMem xc_, zc_, rc_, mpart_;  // field constants (see row_means in kernels.cu)
  // FP32 level 0: the rounding residuals of the deviations X_[0], so that the
  // map sums (the mean and variance) are those of the FP64 maps
  DevMem xr_;
  std::vector<DevMem> ids_dev_;  // grid mode: supports per level
  // averaging masks [k][level] (grid mode: the core; none: every pixel) and
  // their pixel counts
  int K_ = 1;
  std::vector<std::vector<DevMem>> kmask_;
  std::vector<std::vector<i64>> kcount_;
  size_t total_sums_ = 0;
  const uint8_t* mask(int k, int n) const {
    return kmask_.empty() ? nullptr : kmask_[kmask_.size() == 1 ? 0 : k][n].as<uint8_t>();
  }
  // tile heights per level and launch (0: the default)
  enum { T_FWD_Z, T_FWD_BR, T_ADJ_BR, T_ADJ_Z, T_DEC_X, T_DEC_MOD, T_DECT_MOD, T_DECT_X };
  std::vector<std::array<int, 8>> tiles_;
  int tile(int n, int k) const { return tiles_.empty() ? 0 : tiles_[n][k]; }

  // The tile heights, by timing: every valid height of a launch runs once to
  // warm up and three times between CUDA events, on the engine's own
  // buffers (cleared first: the timing reads zeros), and the fastest is
  // kept.  The choice does not change any result.  A process-wide table
  // keyed by the launch's geometry spares engines of the same shapes the
  // timing.
  void tune() {
    tiles_.assign(levels_, std::array<int, 8>{});
    if (!opt_.autotune) return;
    const int L = opt_.L, B = opt_.B;
    cudaStream_t s = stream_;
    for (int n = 0; n < levels_; ++n)
      for (DevMem* f : {&X_[n], &Z_[n], &Mod_[n], &Br_[n], &gMod_[n], &gX_[n]})
        if (f->p) STL_CUDA(cudaMemsetAsync(f->p, 0, f->bytes, s));
    for (DevMem* f : {&Zs_, &Brs_})
      if (f->p) STL_CUDA(cudaMemsetAsync(f->p, 0, f->bytes, s));
    STL_CUDA(cudaMemsetAsync(gZ_.p, 0, gZ_.bytes, s));
    STL_CUDA(cudaMemsetAsync(gBr_.p, 0, gBr_.bytes, s));
    for (DevMem* c : {&xc_, &zc_, &rc_}) STL_CUDA(cudaMemsetAsync(c->p, 0, c->bytes, s));
    int dev = 0;
    STL_CUDA(cudaGetDevice(&dev));
    cudaEvent_t ea, eb;
    STL_CUDA(cudaEventCreate(&ea));
    STL_CUDA(cudaEventCreate(&eb));
    auto pick = [&](const char* what, const ConvOp* op, const DecOp* dop, int R, const std::vector<int>& cand,
                    const std::function<void(int)>& run) -> int {
      if (cand.size() < 2) return 0;
      std::ostringstream k;
      k << dev << '|' << what << '|' << opt_.fp32 << '|' << R << '|' << B;
      if (op) k << '|' << op->n_rep << '|' << op->S << '|' << op->nk << '|' << op->colored << '|' << op->max_tile_cells;
      if (dop) k << '|' << dop->n_rep_out << '|' << dop->n_rep_in << '|' << dop->W << '|' << dop->WT << '|' << dop->nk;
      const std::string key = k.str();
      {
        std::lock_guard<std::mutex> g(tune_mu());
        load_tune_file(opt_.tune_cache);
        auto it = tune_cache().find(key);  // a height that is not valid here is timed again
        if (it != tune_cache().end() && std::find(cand.begin(), cand.end(), it->second) != cand.end()) {
          record_tune(opt_.tune_cache, key, it->second);
          return it->second;
        }
      }
      int best = cand.back();
      float best_ms = 0.f;
      for (int c : cand) {
        run(c);
        STL_CUDA(cudaEventRecord(ea, s));
        for (int r = 0; r < 3; ++r) run(c);
        STL_CUDA(cudaEventRecord(eb, s));
        STL_CUDA(cudaEventSynchronize(eb));
        float ms = 0.f;
        STL_CUDA(cudaEventElapsedTime(&ms, ea, eb));
        if (c == cand.front() || ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
      std::lock_guard<std::mutex> g(tune_mu());
      tune_cache()[key] = best;
      record_tune(opt_.tune_cache, key, best);
      return best;
    };
    try {
      for (int n = 0; n < levels_; ++n)
        typed(n, [&](auto t) {
          using U = typename decltype(t)::type;
          const ConvOp& op = conv_[n];
          const size_t e = esz(n);
          const int R = B * (n + 1) * L;
          int* err = err_.as<int>();
          U* mod = Mod_[n].as<U>();
          U* gmod = gMod_[n].as<U>();
          tiles_[n][T_FWD_Z] = pick("fz", &op, nullptr, B, conv_forward_choices(op, e, B, true), [&](int rb) {
            conv_forward<U>(op, X_[n].as<U>(), B, zf<U>(n), nullptr, 0, 0, 0, s, err,
                            xc_.as<double>() + (size_t)n * B, rb);
          });
          tiles_[n][T_FWD_BR] = pick("fb", &op, nullptr, R, conv_forward_choices(op, e, R, true), [&](int rb) {
            conv_forward<U>(op, mod, R, brf<U>(n), nullptr, 0, 0, 0, s, err, rc_.as<double>(), rb);
          });
          tiles_[n][T_ADJ_BR] = pick("ab", &op, nullptr, R, conv_adjoint_choices(op, e, R, adj_ptr()), [&](int rb) {
            conv_adjoint<U>(op, gBr_.as<U>(), R, gmod, true, s, adj_ptr(), err, nullptr, rb);
          });
          ModulusAdd<U> madd;
          madd.z = zf<U>(n);
          madd.g = gmod + n * L;
          madd.g_pix = B * (n + 1) * L;
          madd.g_row = (n + 1) * L;
          const bool fuse = conv_adjoint_fuses_modulus(op, e, B, adj_ptr(), err);
          tiles_[n][T_ADJ_Z] = pick(fuse ? "azm" : "az", &op, nullptr, B, conv_adjoint_choices(op, e, B, adj_ptr()),
                                    [&](int rb) {
                                      conv_adjoint<U>(op, gZ_.as<U>(), B, gX_[n].as<U>(), false, s, adj_ptr(), err,
                                                      fuse ? &madd : nullptr, rb);
                                    });
          if (n > 0)
            typed(n - 1, [&](auto ti) {
              using Ui = typename decltype(ti)::type;
              tiles_[n][T_DEC_MOD] =
                  pick("dm", nullptr, &dec_[n - 1], n * L, dec_choices(esz(n - 1), n * L), [&](int rb) {
                    dec_apply<Ui, U>(dec_[n - 1], false, Mod_[n - 1].as<Ui>(), B * n * L, n * L, mod, B * (n + 1) * L,
                                     (n + 1) * L, B, n * L, false, s, rb);
                  });
            });
          if (n + 1 < levels_)
            typed(n + 1, [&](auto tn) {
              using Un = typename decltype(tn)::type;
              tiles_[n][T_DEC_X] = pick("dx", nullptr, &dec_[n], B, dec_choices(e, B), [&](int rb) {
                dec_apply<U, Un>(dec_[n], false, X_[n].as<U>(), B, 0, X_[n + 1].as<Un>(), B, 0, 1, B, false, s, rb);
              });
              tiles_[n][T_DECT_MOD] =
                  pick("tm", nullptr, &dec_[n], (n + 1) * L, dec_choices(esz(n + 1), (n + 1) * L), [&](int rb) {
                    dec_apply<Un, U>(dec_[n], true, gMod_[n + 1].as<Un>(), B * (n + 2) * L, (n + 2) * L, gmod,
                                     B * (n + 1) * L, (n + 1) * L, B, (n + 1) * L, false, s, rb);
                  });
              tiles_[n][T_DECT_X] = pick("tx", nullptr, &dec_[n], B, dec_choices(esz(n + 1), B), [&](int rb) {
                dec_apply<Un, U>(dec_[n], true, gX_[n + 1].as<Un>(), B, 0, gX_[n].as<U>(), B, 0, 1, B, true, s, rb);
              });
            });
        });
    } catch (...) {
      cudaEventDestroy(ea);
      cudaEventDestroy(eb);
      throw;
    }
    STL_CUDA(cudaEventDestroy(ea));
    STL_CUDA(cudaEventDestroy(eb));
    STL_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), s));
    STL_CUDA(cudaStreamSynchronize(s));
  }
  static std::mutex& tune_mu() {
    static std::mutex m;
    return m;
  }
  static std::map<std::string, int>& tune_cache() {
    static std::map<std::string, int> c;
    return c;
  }
  // keys a cache file holds (read or appended by this process)
  static std::map<std::string, std::set<std::string>>& file_keys() {
    static std::map<std::string, std::set<std::string>> k;
    return k;
  }
  // the heights a cache file holds (once per file and process; a missing
  // file is an empty cache; malformed lines are skipped)
  static void load_tune_file(const std::string& path) {
    static std::set<std::string> read;
    if (path.empty() || read.count(path)) return;
    read.insert(path);
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
      const size_t tab = line.rfind('\t');
      if (tab == std::string::npos) continue;
      const int h = std::atoi(line.c_str() + tab + 1);
      if (h != 1 && h != 2 && h != 4) continue;
      tune_cache()[line.substr(0, tab)] = h;
      file_keys()[path].insert(line.substr(0, tab));
    }
  }
  // a height an engine uses into its cache file, one line per launch key:
  // key, tab, height (appended once)
  static void record_tune(const std::string& path, const std::string& key, int h) {
    if (path.empty() || !file_keys()[path].insert(key).second) return;
    std::ofstream f(path, std::ios::app);
    if (f) f << key << '\t' << h << '\n';
  }

  // several regions: one launch covers the sums of all of them
  bool segmented() const { return grid_mode() && segments() > 1; }
  int launch_sets() const { return segmented() ? 1 : K_; }
  std::vector<DevMem> seg_dev_;  // segment starts per level (device)
  DevMem ranges_;                // the products' range tables of every level
  // the range tables of the products to the device
  void upload_ranges() {
    size_t bytes = 0;
    auto add = [&](size_t b) { size_t o = bytes; bytes += (b + 255) & ~(size_t)255; return o; };
    std::vector<std::array<size_t, 4>> off(levels_);
    for (int n = 0; n < levels_; ++n) {
      const ProductShape& sh = shapes_[n];
      off[n] = {add(sizeof(i64) * sh.blk.size()), add(sizeof(i64) * sh.rev_blk.size()),
                add(sizeof(int32_t) * sh.rev_seg.size()), add(sizeof(int32_t) * sh.seg_blk.size())};
    }
    ranges_.alloc(bytes);
    unsigned char* base = ranges_.as<unsigned char>();
    for (int n = 0; n < levels_; ++n) {
      ProductShape& sh = shapes_[n];
      auto put = [&](size_t o, const void* src, size_t b) {
        STL_CUDA(cudaMemcpyAsync(base + o, src, b, cudaMemcpyHostToDevice, stream_));
      };
      put(off[n][0], sh.blk.data(), sizeof(i64) * sh.blk.size());
      put(off[n][1], sh.rev_blk.data(), sizeof(i64) * sh.rev_blk.size());
      put(off[n][2], sh.rev_seg.data(), sizeof(int32_t) * sh.rev_seg.size());
      put(off[n][3], sh.seg_blk.data(), sizeof(int32_t) * sh.seg_blk.size());
      sh.d_blk = reinterpret_cast<const i64*>(base + off[n][0]);
      sh.d_rev_blk = reinterpret_cast<const i64*>(base + off[n][1]);
      sh.d_rev_seg = reinterpret_cast<const int32_t*>(base + off[n][2]);
      sh.d_seg_blk = reinterpret_cast<const int32_t*>(base + off[n][3]);
      sh.seg_stride = total_sums_;
    }
    STL_CUDA(cudaStreamSynchronize(stream_));
  }
  i64 count(int k, int n) const { return kcount_.empty() ? npix(n) : kcount_[k][n]; }
  DevMem adj_part_;
  AdjScratch adj_;
  const AdjScratch* adj_ptr() const { return adj_.part ? &adj_ : nullptr; }
  std::vector<Loc> map_;
};

std::unique_ptr<Engine> Engine::create_patch(const Options& o, const Support& s) {
  if (o.fp32) return std::unique_ptr<Engine>(new EngineImpl<float>(o, &s));
  return std::unique_ptr<Engine>(new EngineImpl<double>(o, &s));
}

std::unique_ptr<Engine> Engine::create(const Options& o) {
  if (o.fp32) return std::unique_ptr<Engine>(new EngineImpl<float>(o));
  return std::unique_ptr<Engine>(new EngineImpl<double>(o));
}

}  // namespace stl
