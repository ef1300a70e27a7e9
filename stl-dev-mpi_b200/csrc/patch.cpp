// Disc patches behind the stlp_patch_* entry points (crates/stl-bridge/src/
// lib.rs:743-1176): the statistics of maps known on spherical discs only.
//
// A disc's support (level 0: the NESTED pixels whose centre lies within the
// angle R of the centre; level d + 1: the parents of level d) and its core
// (the pixels within the core radius, then their parents) are built on the
// host (crates/stl-core/src/disc.rs:62-140); every selected disc then runs
// on a grid-mode engine (engine.cu): wavelets bound to the support with the
// binding threshold 1e-9, decimations restricted to it, coefficients
// averaged over the core.  Supports are cached by (centre, radius, core);
// each selected disc has its own engine (a disc selected twice gets two),
// built at its first forward.  The discs' engines run concurrently: host
// threads take discs in turn, each thread launching on its own stream, so
// the many small launches of different discs overlap on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <functional>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "healpix.cuh"
#include "json.hpp"
#include "scatcov.hpp"
#include "../../include/stl_b200.h"

namespace stl {
void set_error(const std::string& msg);
}

using namespace stl;

namespace {

constexpr double kPi = 3.14159265358979323846;

void pixel_vector(i64 pix, i64 nside, double v[3]) {
  double theta, phi;
  pix2ang_nest(pix, nside, theta, phi);
  const double s = std::sin(theta);
  v[0] = s * std::cos(phi);
  v[1] = s * std::sin(phi);
  v[2] = std::cos(theta);
}

// atan2(|u x v|, u . v): accurate at every separation (disc.rs:53-59)
double angle(const double u[3], const double v[3]) {
  const double c0 = u[1] * v[2] - u[2] * v[1], c1 = u[2] * v[0] - u[0] * v[2], c2 = u[0] * v[1] - u[1] * v[0];
  return std::atan2(std::sqrt(c0 * c0 + c1 * c1 + c2 * c2), u[0] * v[0] + u[1] * v[1] + u[2] * v[2]);
}

// Sorted pixels of nside whose centre is within `radius` of the unit vector
// c: descent from the 12 base pixels keeping the cells whose centre is
// within radius plus a bound of the cell's angular radius (1.5 / ns at
// nside ns), the exact test at the finest level.
std::vector<i64> disc_pixels(i64 nside, const double c[3], double radius) {
  std::vector<i64> out;
  if (radius >= kPi) {
    out.resize(npix_of(nside));
    for (i64 p = 0; p < (i64)out.size(); ++p) out[p] = p;
    return out;
  }
  const int order = order_of(nside);
  std::vector<i64> cells(12);
  for (int f = 0; f < 12; ++f) cells[f] = f;
  for (int k = 0; k <= order; ++k) {
    const i64 ns = i64(1) << k;
    const double slack = k == order ? 0.0 : 1.5 / (double)ns;
    std::vector<i64> next;
    for (i64 p : cells) {
      double v[3];
      pixel_vector(p, ns, v);
      if (angle(c, v) <= radius + slack) {
        if (k == order) next.push_back(p);
        else
          for (int q = 0; q < 4; ++q) next.push_back(4 * p + q);
      }
    }
    cells.swap(next);
  }
  std::sort(cells.begin(), cells.end());
  return cells;
}

std::vector<i64> parents(const std::vector<i64>& ids) {
  std::vector<i64> out;
  for (i64 p : ids)
    if (out.empty() || out.back() != (p >> 2)) out.push_back(p >> 2);
  return out;  // ids sorted: parents sorted and unique
}

Support disc_support(i64 nside, int levels, const double c[3], double radius, double core) {
  Support s;
  s.ids.push_back(disc_pixels(nside, c, radius));
  if (s.ids[0].empty()) throw std::runtime_error("empty disc support");
  for (int d = 1; d < levels; ++d) s.ids.push_back(parents(s.ids[d - 1]));
  std::vector<i64> cc;
  const bool has_core = core > 0.0 && core < radius;
  if (has_core) {
    for (i64 p : s.ids[0]) {
      double v[3];
      pixel_vector(p, nside, v);
      if (angle(c, v) <= core) cc.push_back(p);
    }
    if (cc.empty()) throw std::runtime_error("the core holds no pixel centre");
  }
  for (int d = 0; d < levels; ++d) {
    std::vector<i64> pos;
    if (!has_core) {
      pos.resize(s.ids[d].size());
      for (size_t i = 0; i < pos.size(); ++i) pos[i] = (i64)i;
    } else {
      size_t j = 0;
      for (i64 p : cc) {  // both sorted
        while (s.ids[d][j] < p) ++j;
        pos.push_back((i64)j);
      }
      cc = parents(cc);
    }
    s.core.push_back(std::move(pos));
  }
  return s;
}

struct Key {
  uint64_t v[5];
  bool operator<(const Key& o) const { return std::memcmp(v, o.v, sizeof(v)) < 0; }
  bool operator==(const Key& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};

uint64_t bits(double x) {
  uint64_t b;
  std::memcpy(&b, &x, 8);
  return b;
}

struct CachedDisc {
  Support support;
  std::vector<std::unique_ptr<Engine>> engines;  // one per occurrence in the selection
};

template <typename R, typename F>
R guard(R fail, F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    stl::set_error(e.what());
  } catch (...) {
    stl::set_error("unknown native failure");
  }
  return fail;
}

void require(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

}  // namespace

struct StlpPatchHandle {
  Options opt;
  std::vector<Coef> plan;
  int levels = 0;
  size_t capacity = 256;
  int threads = 1;
  std::map<Key, std::shared_ptr<CachedDisc>> cache;
  std::deque<Key> order;
  long hits = 0, misses = 0;
  std::vector<std::pair<std::shared_ptr<CachedDisc>, int>> selected;  // disc, occurrence
  bool has_current = false;
  uint64_t current = 0;
  int nstreams = 8;
  std::vector<cudaStream_t> streams;
  ~StlpPatchHandle() {
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
  }

  // the engine of selected disc i, built (on stream s) at its first use;
  // the caller has sized the disc's engine list (reserve_engines)
  Engine& engine(size_t i, cudaStream_t s = nullptr) {
    auto& d = *selected[i].first;
    const int k = selected[i].second;
    if (!d.engines[k]) {
      Options o = opt;
      o.B = 1;
      if (cudaSetDevice(opt.device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
      std::unique_ptr<Engine> e = Engine::create_patch(o, d.support);
      e->set_stream(s);
      e->prepare();
      d.engines[k] = std::move(e);
    }
    return *d.engines[k];
  }
  void reserve_engines() {
    for (auto& sel : selected)
      while ((int)sel.first->engines.size() <= sel.second) sel.first->engines.push_back(nullptr);
  }
  size_t size(size_t i) const { return selected[i].first->support.ids[0].size(); }
  // f(disc index, its engine) for every selected disc: up to nstreams
  // threads take the discs in turn, each on its own non-blocking stream
  // (building a disc's engine there at its first use); the first error is
  // rethrown once every thread has stopped.
  void for_discs(const std::function<void(size_t, Engine&)>& f) {
    reserve_engines();
    if (cudaSetDevice(opt.device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
      throw std::runtime_error("device synchronisation before the disc sweep failed");
    const int T = (int)std::min<size_t>((size_t)std::max(1, nstreams), selected.size());
    while ((int)streams.size() < T) {
      cudaStream_t st;
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        throw std::runtime_error("stream creation failed");
      streams.push_back(st);
    }
    std::atomic<size_t> next{0};
    std::vector<std::string> errors(T);
    auto work = [&](int t) {
      try {
        if (cudaSetDevice(opt.device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
        for (size_t i = next++; i < selected.size(); i = next++) {
          Engine& e = engine(i, streams[t]);
          e.set_stream(streams[t]);
          f(i, e);
        }
      } catch (const std::exception& ex) {
        errors[t] = ex.what();
        next = selected.size();
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    for (const auto& e : errors)
      if (!e.empty()) throw std::runtime_error(e);
  }
  size_t total() const {
    size_t t = 0;
    for (size_t i = 0; i < selected.size(); ++i) t += size(i);
    return t;
  }
};

extern "C" {

StlpPatchHandle* stlp_patch_new(const char* config) {
  return guard<StlpPatchHandle*>(nullptr, [&]() -> StlpPatchHandle* {
    const Json v = Json::parse(config && *config ? config : "{}");
    std::unique_ptr<StlpPatchHandle> h(new StlpPatchHandle);
    h->opt.nside = v.integer("nside", 128);
    h->opt.J = (int)v.integer("j", 7);
    h->opt.ksz = (int)v.integer("kernel", 5);
    h->opt.L = (int)v.integer("orientations", 4);
    h->opt.device = (int)v.integer("device", 0);
    h->opt.B = 1;
    const std::string backend = v.string("backend", "gpu");
    require(backend == "gpu", "the B200 patch engine runs on the GPU only (backend \"gpu\")");
    require(!v.boolean("cross", false), "cross-channel statistics are not built in the B200 patch engine");
    const std::string dtype = v.string("dtype", "float64");
    require(dtype == "float64" || dtype == "float32", "dtype must be float64 or float32");
    h->opt.fp32 = dtype == "float32";
    h->capacity = (size_t)v.integer("cache", 256);
    const long long t = v.integer("threads", 0);
    h->threads = t > 0 ? (int)t : std::max(1, (int)std::thread::hardware_concurrency());
    h->nstreams = (int)v.integer("streams", 8);
    require(h->nstreams >= 1 && h->nstreams <= 64, "streams must be 1 to 64");
    // validates nside, J, L, kernel as the full-sky engine does
    std::unique_ptr<Engine> probe = Engine::create(h->opt);
    h->plan = probe->plan();
    h->levels = probe->levels();
    return h.release();
  });
}

void stlp_patch_free(StlpPatchHandle* h) { delete h; }

char* stlp_patch_info(StlpPatchHandle* h) {
  return guard<char*>(nullptr, [&]() -> char* {
    require(h != nullptr, "null handle");
    std::ostringstream js;
    js << "{\"version\": \"stl-b200-patch-0.1\", \"nside\": " << h->opt.nside << ", \"j\": " << h->opt.J
       << ", \"levels\": " << h->levels << ", \"channels\": 1, \"cross\": false, \"dtype\": \""
       << (h->opt.fp32 ? "float32" : "float64") << "\", \"fewer\": false, \"threads\": " << h->threads
       << ", \"backend\": \"gpu\", \"cache\": {\"capacity\": " << h->capacity << ", \"entries\": " << h->cache.size()
       << ", \"hits\": " << h->hits << ", \"misses\": " << h->misses << "}, \"selected\": [";
    for (size_t i = 0; i < h->selected.size(); ++i) js << (i ? ", " : "") << h->size(i);
    js << "], \"plan\": [";
    for (size_t i = 0; i < h->plan.size(); ++i) {
      const Coef& c = h->plan[i];
      auto opt = [](int x) { return x < 0 ? std::string("null") : std::to_string(x); };
      js << (i ? ", " : "") << "{\"index\": " << i << ", \"family\": \"" << family_name(c.family)
         << "\", \"native_dg\": " << c.native << ", \"c1\": " << c.c1 << ", \"c2\": " << c.c2 << ", \"j1\": "
         << opt(c.j1) << ", \"j2\": " << opt(c.j2) << ", \"j3\": " << opt(c.j3) << ", \"l1\": " << opt(c.l1)
         << ", \"l2\": " << opt(c.l2) << ", \"l3\": " << opt(c.l3) << "}";
    }
    js << "]}";
    const std::string s = js.str();
    char* out = (char*)std::malloc(s.size() + 1);
    std::memcpy(out, s.c_str(), s.size() + 1);
    return out;
  });
}

int stlp_pixel_vectors(size_t nside, const int64_t* ids, size_t n, double* out) {
  return guard<int>(-1, [&] {
    require(nside > 0 && (nside & (nside - 1)) == 0, "nside must be a power of two");
    require(n == 0 || (ids && out), "null argument");
    for (size_t i = 0; i < n; ++i) {
      require(ids[i] >= 0 && ids[i] < npix_of((i64)nside), "pixel index out of range");
      pixel_vector(ids[i], (i64)nside, out + 3 * i);
    }
    return 0;
  });
}

static int select_discs(StlpPatchHandle* h, const double* centres, size_t b, const double* radii,
                        const double* cores, size_t* counts) {
    require(h != nullptr && centres != nullptr && counts != nullptr, "null argument");
    h->has_current = false;
    h->selected.clear();
    require(b > 0, "empty batch");
    std::vector<Key> keys(b);
    std::vector<std::array<double, 3>> unit(b);
    std::vector<double> rad(b), cor(b);
    for (size_t i = 0; i < b; ++i) {
      rad[i] = radii[i];
      require(std::isfinite(rad[i]) && rad[i] > 0.0, "disc radius must be positive");
      cor[i] = (std::isfinite(cores[i]) && cores[i] > 0.0 && cores[i] < rad[i]) ? cores[i] : -1.0;
      const double* c = centres + 3 * i;
      const double nrm = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      require(nrm > 0.0 && std::isfinite(nrm), "disc centre must be a nonzero finite vector");
      unit[i] = {c[0] / nrm, c[1] / nrm, c[2] / nrm};
      keys[i] = Key{{bits(unit[i][0]), bits(unit[i][1]), bits(unit[i][2]), bits(rad[i]), bits(cor[i])}};
    }
    // supports of the discs not cached, built on the host threads
    std::vector<size_t> missing;
    std::map<Key, size_t> first;
    for (size_t i = 0; i < b; ++i) {
      if (h->cache.count(keys[i]) || first.count(keys[i])) {
        ++h->hits;
      } else {
        ++h->misses;
        first[keys[i]] = i;
        missing.push_back(i);
      }
    }
    std::vector<Support> built(missing.size());
    std::vector<std::string> errors(missing.size());
    auto work = [&](size_t k0, size_t k1) {
      for (size_t k = k0; k < k1; ++k) {
        try {
          const size_t i = missing[k];
          built[k] = disc_support(h->opt.nside, h->levels, unit[i].data(), rad[i], cor[i]);
        } catch (const std::exception& e) {
          errors[k] = e.what();
        }
      }
    };
    const size_t t = std::min<size_t>((size_t)h->threads, std::max<size_t>(missing.size(), 1));
    std::vector<std::thread> pool;
    const size_t per = (missing.size() + t - 1) / t;
    for (size_t q = 0; q < t; ++q) {
      const size_t k0 = std::min(missing.size(), q * per), k1 = std::min(missing.size(), (q + 1) * per);
      if (k0 < k1) pool.emplace_back(work, k0, k1);
    }
    for (auto& th : pool) th.join();
    for (const auto& e : errors)
      if (!e.empty()) throw std::runtime_error(e);
    for (size_t k = 0; k < missing.size(); ++k) {
      auto d = std::make_shared<CachedDisc>();
      d->support = std::move(built[k]);
      h->cache[keys[missing[k]]] = d;
      h->order.push_back(keys[missing[k]]);
    }
    std::map<Key, int> seen;
    for (size_t i = 0; i < b; ++i) h->selected.push_back({h->cache.at(keys[i]), seen[keys[i]]++});
    // the cache keeps the last `capacity` discs (selected ones stay alive here)
    while (h->cache.size() > h->capacity && !h->order.empty()) {
      h->cache.erase(h->order.front());
      h->order.pop_front();
    }
    for (size_t i = 0; i < b; ++i) counts[i] = h->size(i);
    return 0;
}

int stlp_patch_select(StlpPatchHandle* h, const double* centres, size_t b, double radius, double core,
                      size_t* counts) {
  return guard<int>(-1, [&] {
    std::vector<double> r(b, radius), c(b, core);
    return select_discs(h, centres, b, r.data(), c.data(), counts);
  });
}

int stlp_patch_select_radii(StlpPatchHandle* h, const double* centres, size_t b, const double* radii,
                            const double* cores, size_t* counts) {
  return guard<int>(-1, [&] {
    require(radii != nullptr, "null argument");
    std::vector<double> c(b, 0.0);
    if (cores) c.assign(cores, cores + b);
    return select_discs(h, centres, b, radii, c.data(), counts);
  });
}

int stlp_patch_ids(StlpPatchHandle* h, size_t i, int64_t* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && out != nullptr, "null argument");
    require(i < h->selected.size(), "disc index out of range");
    const auto& ids = h->selected[i].first->support.ids[0];
    std::memcpy(out, ids.data(), ids.size() * sizeof(int64_t));
    return 0;
  });
}

int stlp_patch_core_pixels(StlpPatchHandle* h, size_t* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && out != nullptr, "null argument");
    for (size_t i = 0; i < h->selected.size(); ++i)
      for (int n = 0; n < h->levels; ++n) out[i * h->levels + n] = h->selected[i].first->support.core[n].size();
    return 0;
  });
}

static int patch_forward(StlpPatchHandle* h, const double* x_host, uint64_t x_dev, size_t n, uint64_t generation,
                         bool moments, double* out, double* var) {
  require(h != nullptr && out != nullptr, "null argument");
  require(!moments || var != nullptr, "moments need a variance buffer");
  h->has_current = false;
  require(!h->selected.empty(), "no disc selected");
  require(n == h->total(), "input shape mismatch");
  const size_t np = h->plan.size();
  std::vector<size_t> off(h->selected.size() + 1, 0);
  for (size_t i = 0; i < h->selected.size(); ++i) off[i + 1] = off[i] + h->size(i);
  if (x_host)
    for (size_t q = 0; q < n; ++q) require(std::isfinite(x_host[q]), "input patch contains non-finite values");
  h->for_discs([&](size_t i, Engine& e) {
    if (x_host) e.load_host(x_host + off[i]);
    else e.load_device(reinterpret_cast<const double*>(x_dev) + off[i], false);
    e.forward(moments, out + 2 * i * np, moments ? var + i * np : nullptr);
  });
  h->has_current = true;
  h->current = generation;
  return 0;
}

int stlp_patch_forward(StlpPatchHandle* h, const double* x, size_t n, uint64_t generation, bool moments, double* out,
                       double* var) {
  return guard<int>(-1, [&] {
    require(x != nullptr, "null argument");
    return patch_forward(h, x, 0, n, generation, moments, out, var);
  });
}

int stlp_patch_forward_device(StlpPatchHandle* h, uint64_t x, size_t n, uint64_t generation, bool moments,
                              double* out, double* var) {
  return guard<int>(-1, [&] {
    require(x != 0, "null device address");
    return patch_forward(h, nullptr, x, n, generation, moments, out, var);
  });
}

static int patch_vjp(StlpPatchHandle* h, const double* cot, size_t n, uint64_t generation, double* out_host,
                     uint64_t out_dev) {
  require(h != nullptr && cot != nullptr, "null argument");
  require(h->has_current && h->current == generation, "stale forward state");
  const size_t np = h->plan.size();
  require(n == h->selected.size() * np, "cotangent shape mismatch");
  std::vector<size_t> off(h->selected.size() + 1, 0);
  for (size_t i = 0; i < h->selected.size(); ++i) off[i + 1] = off[i] + h->size(i);
  h->for_discs([&](size_t i, Engine& e) {
    if (out_host) e.reverse_host(cot + 2 * i * np, out_host + off[i]);
    else e.reverse_device(cot + 2 * i * np, reinterpret_cast<double*>(out_dev) + off[i], false);
  });
  return 0;
}

int stlp_patch_vjp(StlpPatchHandle* h, const double* cot, size_t n, uint64_t generation, double* out) {
  return guard<int>(-1, [&] {
    require(out != nullptr, "null argument");
    return patch_vjp(h, cot, n, generation, out, 0);
  });
}

int stlp_patch_vjp_device(StlpPatchHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t out) {
  return guard<int>(-1, [&] {
    require(out != 0, "null device address");
    return patch_vjp(h, cot, n, generation, nullptr, out);
  });
}

}  // extern "C"
