// Disc patches behind the stlp_patch_* entry points (crates/stl-bridge/src/
// lib.rs:743-1176): the statistics of maps known on spherical discs only.
//
// A disc's support (level 0: the NESTED pixels whose centre lies within the
// angle R of the centre; level d + 1: the parents of level d) and its core
// (the pixels within the core radius, then their parents) are built on the
// host (crates/stl-core/src/disc.rs:62-140) and cached by (centre, radius,
// core).  The selected discs then run batched: consecutive discs, up to
// group_pixels level-0 pixels in all, form one grid-mode engine (engine.cu)
// whose support is the concatenation of their supports, one segment per
// disc -- wavelets bound to the disc's support with the binding threshold
// 1e-9, decimations restricted to it, coefficients averaged over its core
// -- so that every kernel of a sweep is one launch over all the discs of a
// group.  The engines of a selection are built at its first forward and
// kept while the same discs are selected again.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
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
};

// the supports of discs one after the other, one segment each
Support concatenate(const std::vector<const Support*>& discs, int levels) {
  Support s;
  s.ids.resize(levels);
  s.core.resize(levels);
  s.seg.resize(levels);
  for (int d = 0; d < levels; ++d) {
    s.seg[d].push_back(0);
    for (const Support* q : discs) {
      const i64 off = (i64)s.ids[d].size();
      s.ids[d].insert(s.ids[d].end(), q->ids[d].begin(), q->ids[d].end());
      for (i64 c : q->core[d]) s.core[d].push_back(off + c);
      s.seg[d].push_back((i64)s.ids[d].size());
    }
  }
  return s;
}

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
  i64 group_pixels = i64(1) << 23;  // level-0 pixels of one batched engine (at least one disc)
  std::map<Key, std::shared_ptr<CachedDisc>> cache;
  std::deque<Key> order;
  long hits = 0, misses = 0;
  std::vector<std::shared_ptr<CachedDisc>> selected;
  std::vector<Key> selected_keys;
  // consecutive selected discs first .. first + count - 1, level-0 pixels
  // from offset, in one segmented engine
  struct Group {
    size_t first = 0, count = 0;
    i64 offset = 0;
    std::unique_ptr<Engine> engine;
  };
  std::vector<Group> groups;
  std::vector<Key> group_keys;  // the selection the groups were built for
  bool has_current = false;
  uint64_t current = 0;
  bool profile = false;  // time every launch of the engines (CUDA events)

  size_t size(size_t i) const { return selected[i]->support.ids[0].size(); }
  size_t total() const {
    size_t t = 0;
    for (size_t i = 0; i < selected.size(); ++i) t += size(i);
    return t;
  }
  // the engines of the current selection, built at its first use
  std::vector<Group>& engines() {
    if (!groups.empty() && group_keys == selected_keys) return groups;
    groups.clear();
    group_keys.clear();
    if (cudaSetDevice(opt.device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
    i64 off = 0;
    for (size_t i = 0; i < selected.size();) {
      Group g;
      g.first = i;
      g.offset = off;
      i64 px = 0;
      std::vector<const Support*> discs;
      while (i < selected.size() && (discs.empty() || px + (i64)size(i) <= group_pixels)) {
        discs.push_back(&selected[i]->support);
        px += (i64)size(i);
        ++i;
      }
      g.count = discs.size();
      off += px;
      Options o = opt;
      o.B = 1;
      g.engine = Engine::create_patch(o, concatenate(discs, levels));
      g.engine->set_profiling(profile);
      g.engine->prepare();
      groups.push_back(std::move(g));
    }
    group_keys = selected_keys;
    return groups;
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
    h->group_pixels = (i64)v.integer("group_pixels", (long long)h->group_pixels);
    h->profile = v.boolean("profile", false);
    h->opt.autotune = v.boolean("autotune", true);
    h->opt.graphs = v.boolean("graphs", true);
    h->opt.tune_cache = v.string("autotune_cache", "");
    require(h->group_pixels >= 1, "group_pixels must be positive");
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
       << ", \"group_pixels\": " << h->group_pixels << ", \"groups\": " << h->groups.size();
    // the engines' timers and kernel classes, summed
    double fwd = 0.0, rev = 0.0, build = 0.0;
    std::vector<KernelStat> ks;
    for (const auto& g : h->groups) {
      fwd += g.engine->timers.forward_ms;
      rev += g.engine->timers.reverse_ms;
      build += g.engine->timers.build_s;
      auto k = g.engine->kernel_stats();
      if (ks.empty()) ks = k;
      else
        for (size_t i = 0; i < ks.size() && i < k.size(); ++i) {
          ks[i].launches += k[i].launches;
          ks[i].calls += k[i].calls;
          ks[i].ms += k[i].ms;
          ks[i].bytes += k[i].bytes;
          ks[i].flops += k[i].flops;
        }
    }
    js << ", \"timers\": {\"build_s\": " << build << ", \"forward_ms\": " << fwd << ", \"reverse_ms\": " << rev
       << "}, \"kernels\": [";
    for (size_t i = 0; i < ks.size(); ++i)
      js << (i ? ", " : "") << "{\"name\": \"" << ks[i].name << "\", \"launches\": " << ks[i].launches
         << ", \"calls\": " << ks[i].calls << ", \"ms\": " << ks[i].ms << ", \"bytes\": " << ks[i].bytes << "}";
    js << "]";
    js
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
    h->selected_keys.clear();
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
    for (size_t i = 0; i < b; ++i) h->selected.push_back(h->cache.at(keys[i]));
    h->selected_keys = keys;
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
    const auto& ids = h->selected[i]->support.ids[0];
    std::memcpy(out, ids.data(), ids.size() * sizeof(int64_t));
    return 0;
  });
}

int stlp_patch_core_pixels(StlpPatchHandle* h, size_t* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && out != nullptr, "null argument");
    for (size_t i = 0; i < h->selected.size(); ++i)
      for (int n = 0; n < h->levels; ++n) out[i * h->levels + n] = h->selected[i]->support.core[n].size();
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
  for (auto& g : h->engines()) {  // every group's upload counts non-finite values (load_host)
    Engine& e = *g.engine;
    if (x_host) e.load_host(x_host + g.offset);
    else e.load_device(reinterpret_cast<const double*>(x_dev) + g.offset, false);
    e.forward(moments, out + 2 * g.first * np, moments ? var + g.first * np : nullptr);
  }
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
  for (auto& g : h->engines()) {
    Engine& e = *g.engine;
    if (out_host) e.reverse_host(cot + 2 * g.first * np, out_host + g.offset);
    else e.reverse_device(cot + 2 * g.first * np, reinterpret_cast<double*>(out_dev) + g.offset, false);
  }
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
