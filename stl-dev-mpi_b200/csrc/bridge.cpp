// C ABI of the B200 ScatCov engine: the `stlp_*` entry points of the
// reference's stl-bridge (crates/stl-bridge/src/lib.rs), same names, types
// and conventions, so that its Python binding (python/stl_ensemble/
// stl_port/native.py) loads this library through STL_NATIVE_LIBRARY.
//
// Conventions kept from the reference: maps are f64 NESTED [batch, 12
// nside^2]; complex values and cotangents are interleaved (re, im); the
// gradient is that of Re sum(conj(cotangent) * values); every forward
// state carries an identity (handle, generation, member, objective) that
// stlp_vjp and stlp_restore check; failures return -1 / NULL and
// stlp_last_error() holds the message (thread-local, owned by the
// library).  Additions: device-pointer forward/VJP (f32 or f64 maps),
// the caller's CUDA stream, and an explicit prepare.
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>

#include "engine.cuh"
#include "json.hpp"
#include "lbfgs.hpp"
#include "scatcov.hpp"
#include "spin.hpp"
#include "../../include/stl_b200.h"

using namespace stl;

namespace {

const char* kVersion = "stl-b200-0.1 (abi 2026-11-09-v12)";
thread_local std::string g_error;
std::atomic<uint64_t> g_next_id{1};

struct Identity {
  uint64_t owner = 0, generation = 0, member = 0, objective = 0;
  bool operator==(const Identity& o) const {
    return owner == o.owner && generation == o.generation && member == o.member && objective == o.objective;
  }
};

template <typename R, typename F>
R guard(R fail, F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_error = e.what();
  } catch (...) {
    g_error = "unknown native failure";
  }
  return fail;
}

void require(bool ok, const std::string& msg) {
  if (!ok) throw std::runtime_error(msg);
}

std::string jstr(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') { o += '\\'; o += c; }
    else if (c == '\n') o += "\\n";
    else o += c;
  }
  return o + "\"";
}

}  // namespace

namespace stl {
void set_error(const std::string& msg) { g_error = msg; }
long long synthesize_device(Engine& e, double* x, size_t n, const double* target, const double* weights,
                            const lbfgs::Options& o, std::vector<double>* losses);
}  // namespace stl

struct StlpHandle {
  std::unique_ptr<Engine> engine;
  // spin 2: (Q, U) maps through the spin front end; the engine's batch is
  // twice the handle's (chi_E and chi_B of every map)
  std::unique_ptr<SpinFront> spin;
  uint64_t id = 0;
  bool has_current = false;
  Identity current;
  int device = 0;
  size_t input_len() const {
    return spin ? spin->input_len() : (size_t)engine->options().B * (size_t)engine->npix(0);
  }
  // B K np: K masks (1 without)
  size_t values_len() const {
    return (size_t)engine->value_batch() * std::max(1, engine->nmasks()) * engine->plan().size();
  }
  void activate() { STL_CUDA(cudaSetDevice(device)); }
};

struct StlpSnapshot {
  Identity identity;
  uint64_t owner = 0;
  std::vector<double> maps;
};

extern "C" {

const char* stlp_last_error(void) { return g_error.c_str(); }

void stlp_string_free(char* p) { free(p); }

StlpHandle* stlp_new(const char* config) {
  return guard<StlpHandle*>(nullptr, [&]() -> StlpHandle* {
    Json v = Json::parse(config);
    require(v.kind == Json::Object, "config must be a JSON object");
    Options o;
    o.nside = v.integer("nside", 128);
    o.J = (int)v.integer("j", 7);
    o.B = (int)v.integer("batch", 1);
    o.ksz = (int)v.integer("kernel", 5);
    o.L = (int)v.integer("orientations", 4);
    o.device = (int)v.integer("device", 0);
    std::string backend = v.string("backend", "gpu");
    require(backend == "gpu",
            "backend '" + backend + "' is not built in this library: it is the B200 engine (use backend \"gpu\")");
    std::string dtype = v.string("dtype", "float64");
    require(dtype == "float64" || dtype == "float32", "dtype must be float64 or float32");
    o.fp32 = dtype == "float32";
    o.autotune = v.boolean("autotune", true);
    o.graphs = v.boolean("graphs", true);  // the sweeps as CUDA graphs
    if (const Json* tcv = v.get("tensor_cores")) {  // true / false, or "forward", "all", "none"
      if (tcv->kind == Json::Bool) o.tensor_cores = tcv->b ? 1 : 0;
      else if (tcv->kind == Json::String && (tcv->str == "none" || tcv->str == "forward" || tcv->str == "all"))
        o.tensor_cores = tcv->str == "none" ? 0 : tcv->str == "forward" ? 1 : 2;
      else if (tcv->kind != Json::Null)
        throw std::runtime_error("tensor_cores must be a boolean or one of \"none\", \"forward\", \"all\"");
    }
    o.tune_cache = v.string("autotune_cache", "");
    o.cross = v.boolean("cross", false);  // two channels, the plan of their cross terms (lib.rs:238-245)
    const std::string fields = v.string("fields", "keep");  // lib.rs:273-345: auto | keep | recompute
    require(fields == "keep" || fields == "recompute" || fields == "auto", "fields must be auto, keep or recompute");
    o.recompute = fields == "recompute";
    o.fields_auto = fields == "auto";
    // spin 2 (lib.rs:301-319): "spin" 0 or 2, "spin_kernel" 3, 5, 7 or 9,
    // "spin_pyramid" scalar (default) or transported, "spin_a" 0 or 2 (cross)
    const long long spin = v.integer("spin", 0);
    require(spin == 0 || spin == 2, "spin must be 0 or 2, not " + std::to_string(spin));
    const std::string pyramid = v.string("spin_pyramid", "scalar");
    require(pyramid == "scalar" || pyramid == "transported",
            "spin_pyramid must be transported or scalar, not " + jstr(pyramid));
    const int spin_a = (int)v.integer("spin_a", 2);
    require(spin_a == 0 || spin_a == 2, "spin_a must be 0 or 2");
    const int spin_kernel = (int)v.integer("spin_kernel", 5);
    require(o.nside > 0 && (o.nside & (o.nside - 1)) == 0, "nside must be a power of two");
    SpinConfig sc;
    if (spin == 2) {
      require(!o.cross || pyramid == "scalar", "spin 2: cross statistics need the scalar pyramid");
      require(spin_kernel == 3 || spin_kernel == 5 || spin_kernel == 7 || spin_kernel == 9,
              "spin_kernel must be 3, 5, 7 or 9");
      sc.nside = o.nside;
      sc.levels = o.J;
      sc.kernel = spin_kernel;
      sc.transported = pyramid == "transported";
      sc.cross = o.cross;
      sc.spin_a = spin_a;
      sc.batch = o.B;
      o.B = 2 * o.B;  // the engine sees chi_E and chi_B of every map as two of its maps
    }
    auto h = std::make_unique<StlpHandle>();
    h->engine = Engine::create(o);
    h->device = o.device;
    h->id = g_next_id.fetch_add(1);
    if (spin == 2) h->spin = SpinFront::create(sc, h->engine->stream());
    return h.release();
  });
}

void stlp_free(StlpHandle* h) {
  if (!h) return;
  try {
    h->activate();
  } catch (...) {
  }
  delete h;
}

int stlp_prepare(StlpHandle* h) {
  return guard<int>(-1, [&] {
    require(h != nullptr, "null handle");
    h->activate();
    h->engine->prepare();
    if (h->spin) h->spin->prepare();
    return 0;
  });
}

int stlp_profile(StlpHandle* h, int on, int reset) {
  return guard<int>(-1, [&] {
    require(h != nullptr, "null handle");
    h->activate();
    if (reset) h->engine->reset_kernel_stats();
    h->engine->set_profiling(on != 0);
    return 0;
  });
}

int stlp_set_stream(StlpHandle* h, uint64_t stream) {
  return guard<int>(-1, [&] {
    require(h != nullptr, "null handle");
    h->engine->set_stream(reinterpret_cast<cudaStream_t>(stream));
    if (h->spin) h->spin->set_stream(reinterpret_cast<cudaStream_t>(stream));
    return 0;
  });
}

char* stlp_info(StlpHandle* h) {
  return guard<char*>(nullptr, [&]() -> char* {
    require(h != nullptr, "null handle");
    const Engine& e = *h->engine;
    const Options& o = e.options();
    std::ostringstream js;
    js.precision(17);
    js << "{\"version\": " << jstr(kVersion) << ", \"engine\": \"b200\", \"nside\": " << o.nside
       << ", \"j\": " << o.J << ", \"batch\": " << e.value_batch() << ", \"channels\": " << e.channels()
       << ", \"cross\": " << (o.cross ? "true" : "false")
       << ", \"dtype\": " << jstr(o.fp32 ? "float32 fields, float64 sums/complex128" : "float64/complex128")
       << ", \"fewer\": false, \"orientations\": " << o.L << ", \"kernel\": " << o.ksz
       << ", \"levels\": " << e.levels() << ", \"masks\": " << e.nmasks() << ", \"spin\": " << (h->spin ? 2 : 0)
       << ", \"device\": " << o.device
       << ", \"conv\": \"folded-stencil\", \"fields\": "
       << jstr(e.recomputes() ? "recompute" : "keep");
    if (h->spin) {
      const SpinConfig& sc = h->spin->config();
      js << ", \"spin_kernel\": " << sc.kernel << ", \"spin_pyramid\": " << jstr(sc.transported ? "transported" : "scalar")
         << ", \"spin_a\": " << (sc.cross ? std::to_string(sc.spin_a) : std::string("null"))
         << ", \"spin_bytes\": " << h->spin->bytes() << ", \"spin_batch\": " << sc.batch;
    }
    js << ", \"device_memory\": {\"operator_bytes\": " << e.operator_bytes() << ", \"field_bytes\": " << e.field_bytes()
       << ", \"live_bytes\": " << device_bytes_live() << ", \"peak_bytes\": " << device_bytes_peak()
       << ", \"kept_field_bytes\": " << e.kept_field_bytes() << "}";
    js << ", \"timers\": {\"build_s\": " << e.timers.build_s << ", \"forward_ms\": " << e.timers.forward_ms
       << ", \"reverse_ms\": " << e.timers.reverse_ms << ", \"forwards\": " << e.timers.forwards
       << ", \"reverses\": " << e.timers.reverses << "}";
    js << ", \"kernels\": [";
    auto ks = e.kernel_stats();
    for (size_t i = 0; i < ks.size(); ++i)
      js << (i ? ", " : "") << "{\"name\": " << jstr(ks[i].name) << ", \"launches\": " << ks[i].launches
         << ", \"calls\": " << ks[i].calls
         << ", \"ms\": " << ks[i].ms << ", \"bytes\": " << ks[i].bytes << ", \"flops\": " << ks[i].flops << "}";
    js << "], \"mean_cells_per_row\": [";
    auto ms = e.mean_slots();
    for (size_t i = 0; i < ms.size(); ++i) js << (i ? ", " : "") << ms[i];
    js << "], \"operators\": [";
    auto ol = e.operator_layout();
    for (size_t i = 0; i < ol.size(); ++i)
      js << (i ? ", " : "") << "{\"slots\": " << ol[i][0] << ", \"tile_cells\": " << ol[i][1]
         << ", \"coloured\": " << (ol[i][2] == 1 || ol[i][2] == 2 ? "true" : "false") << ", \"layout\": \""
         << (ol[i][2] == 3 ? "tensor_cores" : ol[i][2] == 2 ? "tensor_cores+coloured" : ol[i][2] == 1 ? "coloured" : "rows")
         << "\", \"warp_cells\": "
         << ol[i][3] << "}";
    js << "], \"tile_heights\": [";
    auto th = e.tile_heights();
    for (size_t i = 0; i < th.size(); ++i) {
      js << (i ? ", " : "") << "[";
      for (size_t k = 0; k < th[i].size(); ++k) js << (k ? ", " : "") << th[i][k];
      js << "]";
    }
    js << "]";
    js << ", \"plan\": [";
    const auto& plan = e.plan();
    auto opt = [](int v) { return v < 0 ? std::string("null") : std::to_string(v); };
    for (size_t i = 0; i < plan.size(); ++i) {
      const Coef& c = plan[i];
      if (i) js << ", ";
      js << "{\"index\": " << i << ", \"family\": \"" << family_name(c.family) << "\", \"native_dg\": " << c.native
         << ", \"c1\": " << c.c1 << ", \"c2\": " << c.c2 << ", \"j1\": " << opt(c.j1) << ", \"j2\": " << opt(c.j2)
         << ", \"j3\": " << opt(c.j3) << ", \"l1\": " << opt(c.l1) << ", \"l2\": " << opt(c.l2)
         << ", \"l3\": " << opt(c.l3) << "}";
    }
    js << "]}";
    std::string s = js.str();
    char* out = (char*)malloc(s.size() + 1);
    std::memcpy(out, s.c_str(), s.size() + 1);
    return out;
  });
}

int stlp_native_pixels(StlpHandle* h, size_t* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && out != nullptr, "null argument");
    const auto& plan = h->engine->plan();
    const int K = std::max(1, h->engine->nmasks());
    for (int k = 0; k < K; ++k)
      for (size_t i = 0; i < plan.size(); ++i)
        out[k * plan.size() + i] = (size_t)(h->engine->nmasks() ? h->engine->mask_count(k, plan[i].native)
                                                               : h->engine->npix(plan[i].native));
    return 0;
  });
}

int stlp_memory(size_t* live, size_t* peak, int reset_peak) {
  return guard<int>(-1, [&] {
    if (reset_peak) device_bytes_reset_peak();
    if (live) *live = device_bytes_live();
    if (peak) *peak = device_bytes_peak();
    return 0;
  });
}

int stlp_operator_rows(StlpHandle* h, size_t level, int kind, int64_t* out, double* weight, size_t width,
                       size_t* needed) {
  return guard<int>(-1, [&] {
    require(h != nullptr && needed != nullptr, "null argument");
    std::vector<int64_t> rows;
    std::vector<double> wts;
    int w = 0;
    h->engine->operator_rows((int)level, kind, rows, wts, w);
    *needed = (size_t)w;
    if (out && width >= (size_t)w && w > 0) {
      const size_t n = rows.size() / (size_t)w;
      for (size_t r = 0; r < n; ++r) {
        std::copy(rows.begin() + r * w, rows.begin() + (r + 1) * w, out + r * width);
        std::fill(out + r * width + w, out + (r + 1) * width, (int64_t)-1);
        if (weight) {
          std::copy(wts.begin() + r * w, wts.begin() + (r + 1) * w, weight + r * width);
          std::fill(weight + r * width + w, weight + (r + 1) * width, 0.0);
        }
      }
    }
    return 0;
  });
}

int stlp_set_masks(StlpHandle* h, const double* weights, size_t k) {
  return guard<int>(-1, [&] {
    require(h != nullptr, "null handle");
    require(k == 0 || weights != nullptr, "null mask weights");
    h->has_current = false;
    h->activate();
    if (h->spin && k > 0) h->engine->set_mask_levels(h->spin->mask_levels(weights, k));  // eroded, every level
    else h->engine->set_masks(weights, k);
    return 0;
  });
}

static int forward_common(StlpHandle* h, uint64_t generation, uint64_t member, uint64_t objective, bool moments,
                          double* out, double* var) {
  h->engine->forward(moments, out, var);
  h->current = Identity{h->id, generation, member, objective};
  h->has_current = true;
  return 0;
}

int stlp_forward(StlpHandle* h, const double* x, size_t n, uint64_t generation, uint64_t member, uint64_t objective,
                 bool moments, double* out, double* var) {
  return guard<int>(-1, [&] {
    require(h != nullptr && x != nullptr && out != nullptr, "null argument");
    require(n == h->input_len(), "input shape mismatch");
    require(!moments || var != nullptr, "moments need a variance buffer");
    // small inputs are checked here; larger ones while their copy to the
    // device is staged (load_host), on several host threads
    if (n < (size_t(1) << 19))
      for (size_t i = 0; i < n; ++i) require(std::isfinite(x[i]), "input map contains non-finite values");
    h->activate();
    h->has_current = false;
    if (h->spin) h->spin->load_host(*h->engine, x);
    else h->engine->load_host(x);
    return forward_common(h, generation, member, objective, moments, out, var);
  });
}

int stlp_forward_device(StlpHandle* h, uint64_t x, size_t n, int f32, uint64_t generation, uint64_t member,
                        uint64_t objective, bool moments, double* out, double* var) {
  return guard<int>(-1, [&] {
    require(h != nullptr && x != 0 && out != nullptr, "null argument");
    require(n == h->input_len(), "input shape mismatch");
    require(!moments || var != nullptr, "moments need a variance buffer");
    h->activate();
    h->has_current = false;
    if (h->spin) h->spin->load_device(*h->engine, reinterpret_cast<const void*>(x), f32 != 0);
    else h->engine->load_device(reinterpret_cast<const void*>(x), f32 != 0);
    return forward_common(h, generation, member, objective, moments, out, var);
  });
}

static void check_identity(StlpHandle* h, uint64_t generation, uint64_t member, uint64_t objective, size_t n) {
  require(h->has_current && h->current == Identity{h->id, generation, member, objective},
          "stale, wrong-member or wrong-objective forward state");
  require(n == h->values_len(), "cotangent shape mismatch");
}

int stlp_vjp(StlpHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t member, uint64_t objective,
             double* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && cot != nullptr && out != nullptr, "null argument");
    check_identity(h, generation, member, objective, n);
    h->activate();
    if (h->spin) h->spin->reverse_host(*h->engine, cot, out);
    else h->engine->reverse_host(cot, out);
    return 0;
  });
}

int stlp_vjp_device(StlpHandle* h, const double* cot, size_t n, uint64_t generation, uint64_t member,
                    uint64_t objective, uint64_t out, int f32) {
  return guard<int>(-1, [&] {
    require(h != nullptr && cot != nullptr && out != 0, "null argument");
    check_identity(h, generation, member, objective, n);
    h->activate();
    if (h->spin) h->spin->reverse_device(*h->engine, cot, reinterpret_cast<void*>(out), f32 != 0);
    else h->engine->reverse_device(cot, reinterpret_cast<void*>(out), f32 != 0);
    return 0;
  });
}

int64_t stlp_synthesize_device(StlpHandle* h, uint64_t x, size_t n, const double* target, size_t n_target,
                               const double* weights, const char* options, double* losses, size_t n_losses) {
  return guard<int64_t>(-1, [&]() -> int64_t {
    require(h != nullptr && x != 0 && target != nullptr, "null argument");
    require(!h->spin, "the device synthesis takes scalar maps: spin-2 handles synthesise through stlp_lbfgs");
    require(n == h->input_len(), "map shape mismatch");
    require(n_target == h->values_len(), "target shape mismatch");
    const lbfgs::Options o = lbfgs::parse_options(options);
    h->activate();
    h->has_current = false;  // the engine's forward state moves with the iterate
    std::vector<double> hist;
    const long long evals = synthesize_device(*h->engine, reinterpret_cast<double*>(x), n, target, weights, o,
                                              losses ? &hist : nullptr);
    if (losses) std::copy(hist.begin(), hist.begin() + std::min(hist.size(), n_losses), losses);
    return evals;
  });
}

StlpSnapshot* stlp_checkpoint(StlpHandle* h) {
  return guard<StlpSnapshot*>(nullptr, [&]() -> StlpSnapshot* {
    require(h != nullptr, "null handle");
    require(h->has_current, "checkpoint requires a forward state");
    h->activate();
    auto s = std::make_unique<StlpSnapshot>();
    s->identity = h->current;
    s->owner = h->id;
    if (h->spin) h->spin->save_input(s->maps);  // the (Q, U) maps: the front end runs again at restore
    else h->engine->save_state(s->maps);
    return s.release();
  });
}

void stlp_checkpoint_free(StlpSnapshot* s) { delete s; }

size_t stlp_checkpoint_bytes(const StlpSnapshot* s) { return s ? s->maps.size() * sizeof(double) : 0; }

int stlp_restore(StlpHandle* h, const StlpSnapshot* s, uint64_t generation, uint64_t member, uint64_t objective) {
  return guard<int>(-1, [&] {
    require(h != nullptr && s != nullptr, "null argument");
    require(s->owner == h->id && s->identity == Identity{h->id, generation, member, objective},
            "stale, wrong-member, wrong-objective or foreign checkpoint");
    h->activate();
    h->has_current = false;
    // The forward state is recomputed from the saved maps: the sweeps are
    // deterministic, so the restored fields equal the checkpointed ones.
    if (h->spin) {
      require(s->maps.size() == h->input_len(), "checkpoint of another configuration");
      h->spin->load_host(*h->engine, s->maps.data());
    } else {
      h->engine->load_state(s->maps);
    }
    std::vector<double> values(2 * h->values_len());
    h->engine->forward(false, values.data(), nullptr);
    h->current = s->identity;
    h->has_current = true;
    return 0;
  });
}

int stlp_forward_levels(StlpHandle* h, const double* x, size_t n, double* out) {
  return guard<int>(-1, [&] {
    require(h != nullptr && x != nullptr && out != nullptr, "null argument");
    size_t want = 0;
    for (int d = 0; d < h->engine->levels(); ++d) want += (size_t)h->engine->options().B * h->engine->npix(d);
    require(n == want, "input shape mismatch");
    for (size_t i = 0; i < n; ++i) require(std::isfinite(x[i]), "input map contains non-finite values");
    h->activate();
    h->has_current = false;  // a validation sweep: no vjp or checkpoint follows it
    h->engine->load_levels(x);
    h->engine->forward(false, out, nullptr);
    return 0;
  });
}

int stlp_spin_fields(StlpHandle* h, const double* x, size_t n, size_t level, double* qu, double* chi) {
  return guard<int>(-1, [&] {
    require(h != nullptr && x != nullptr && qu != nullptr && chi != nullptr, "null argument");
    require(h->spin != nullptr, "not a spin-2 handle");
    require(!h->spin->config().cross, "spin fields of auto handles only");
    require(n == h->input_len(), "input shape mismatch");
    const int levels = h->spin->config().transported ? h->engine->levels() : 1;
    require(level < (size_t)levels, "level out of range");
    for (size_t i = 0; i < n; ++i) require(std::isfinite(x[i]), "input map contains non-finite values");
    h->activate();
    h->spin->fields(x, (int)level, qu, chi);
    return 0;
  });
}

int stlp_spin_rows(StlpHandle* h, size_t level, int kind, int64_t* cells, double* weights, size_t width,
                   size_t* needed) {
  return guard<int>(-1, [&] {
    require(h != nullptr && needed != nullptr, "null argument");
    require(h->spin != nullptr, "not a spin-2 handle");
    require(kind == 0 || kind == 1, "kind must be 0 (stencil) or 1 (transported means)");
    h->activate();
    std::vector<int64_t> c;
    std::vector<double> w;
    int wd = 0;
    h->spin->export_rows((int)level, kind, c, w, wd);
    *needed = (size_t)wd;
    if (cells && width >= (size_t)wd && wd > 0) {
      const size_t rows = c.size() / (size_t)wd;
      for (size_t r = 0; r < rows; ++r) {
        std::copy(c.begin() + r * wd, c.begin() + (r + 1) * wd, cells + r * width);
        std::fill(cells + r * width + wd, cells + (r + 1) * width, (int64_t)-1);
        if (weights) {
          std::copy(w.begin() + 2 * r * wd, w.begin() + 2 * (r + 1) * wd, weights + 2 * r * width);
          std::fill(weights + 2 * (r * width + wd), weights + 2 * (r + 1) * width, 0.0);
        }
      }
    }
    return 0;
  });
}

}  // extern "C"
