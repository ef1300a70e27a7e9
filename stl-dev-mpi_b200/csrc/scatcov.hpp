// Host interface of the B200 ScatCov engine (one GPU, one handle).
//
// The engine mirrors the reference's `Evaluator` contract
// (crates/stl-core/src/engine.rs:254-271): forward(x) -> statistics of a
// batch of maps (optionally with the spatial variance of every
// coefficient's terms), then gradient(cotangent) -> the level-0 map
// cotangent of Re sum(conj(cotangent) * values).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace stl {

typedef int64_t i64;
enum class DType;

// crates/stl-core/src/plan.rs:4-68; unused indices are -1
enum Family { MEAN = 0, VAR = 1, S1 = 2, S2 = 3, S3 = 4, S4 = 5 };
struct Coef {
  int family, native, c1, c2, j1, j2, j3, l1, l2, l3;
};
const char* family_name(int f);
// build_plan of one channel, dg(j) = j, all families (plan.rs:80-158)
std::vector<Coef> build_plan(int J, int L);
// the cross terms of two channels (c1 != c2) of build_plan with two
// channels, in its order (plan.rs:80-158 filtered as the bridge's plan_of,
// crates/stl-bridge/src/lib.rs:238-245)
std::vector<Coef> build_plan_cross(int J, int L);

struct Options {
  i64 nside = 128;
  int J = 7;
  int B = 1;
  int L = 4;
  int ksz = 5;
  bool fp32 = false;  // compute precision of the fields (sums are FP64 in both)
  int device = 0;
  bool autotune = true;  // time the tile heights of the wavelet and decimation launches at prepare
  // FP32 full-sky wavelets on the tensor cores (3xTF32 mma.sync): 0 none
  // (the CUDA-core kernels of the coloured layout, the default: as fast,
  // a single layout, closer to FP64), 1 the forward (the adjoint on the
  // CUDA cores), 2 forward and adjoint
  int tensor_cores = 0;
  // Two channels and the plan of their cross terms only (c1 != c2: S1 of the
  // root-normalised z, S2, S3 and S4 in both channel orders), maps
  // [B][2][N]; the fields then hold 2 B maps (map 2 b + c).
  bool cross = false;
  // Field store (the reference's `fields`, crates/stl-gpu/src/engine.rs:
  // 174-204): keep every level's wavelet outputs z and branches from the
  // forward for the reverse sweep, or recompute them per level in the
  // reverse (one buffer of the largest level each; the stored moduli and
  // the maps of the pyramid stay).  Results are identical either way.
  bool recompute = false;
  bool fields_auto = false;  // recompute only when keeping them would not fit the device's free memory
  std::string tune_cache;  // file of tile heights already timed (read, then extended); empty: none
  // the launches of a forward or reverse sweep as one CUDA graph, captured at
  // the first sweep of a configuration and replayed (not while profiling)
  bool graphs = true;
};

struct Timers {
  double build_s = 0, forward_ms = 0, reverse_ms = 0;
  int forwards = 0, reverses = 0;
};

// Per kernel class: launches, device time (CUDA events on the engine's
// stream, only while profiling is on) and algorithmic bytes / flops of the
// launches (the minimal traffic and work of the operation, not the
// kernel's actual traffic).
struct KernelStat {
  const char* name;
  long launches = 0;
  long calls = 0;  // operations (a call may take more than one kernel launch)
  double ms = 0.0, bytes = 0.0, flops = 0.0;
};

// Sky regions of the engine's grid mode (disc patches): per level the NESTED
// ids of the support (level d + 1: the parents of level d) and the
// ascending positions in them of the pixels the coefficients average (the
// core).  The support may hold several regions one after the other
// (segments): seg[d] gives their starts in ids[d] and, last, its size
// (empty: one region).  Every segment is sorted and unique; the wavelets
// and decimations of a segment read its own cells only, and every segment
// has its own coefficients, averaged over its own core pixels.
struct Support {
  std::vector<std::vector<int64_t>> ids;
  std::vector<std::vector<int64_t>> core;
  std::vector<std::vector<int64_t>> seg;
};

class Engine {
 public:
  static std::unique_ptr<Engine> create(const Options& o);
  // Grid mode: the fields live on the support only, the wavelets are bound
  // to it (binding threshold 1e-9), the decimations restricted to it, and
  // the coefficients average the core.  Batch 1.
  static std::unique_ptr<Engine> create_patch(const Options& o, const Support& s);
  virtual ~Engine() = default;

  const Options& options() const { return opt_; }
  const std::vector<Coef>& plan() const { return plan_; }
  int levels() const { return levels_; }
  // maps of the values and cotangents (the batch; options().B counts the
  // fields' maps, two per batch entry with cross)
  int value_batch() const { return vb_; }
  int channels() const { return opt_.cross ? 2 : 1; }
  i64 npix(int d) const { return npix_[d]; }
  // pixels a coefficient of native level d averages
  i64 ncore(int d) const { return ncore_[d]; }
  bool grid_mode() const { return !support_.ids.empty(); }
  // regions of the support (1 on the full sky)
  int segments() const { return support_.seg.empty() ? 1 : (int)support_.seg[0].size() - 1; }
  const Support& support() const { return support_; }
  bool fp32() const { return opt_.fp32; }

  void set_stream(cudaStream_t s) { stream_ = s; }
  cudaStream_t stream() const { return stream_; }

  // Builds the device operators of every level (first use does it too).
  virtual void prepare() = 0;
  // Loads maps [B][N_0] from host (f64) or device memory (f64 or f32).
  virtual void load_host(const double* x) = 0;
  virtual void load_device(const void* x, bool f32) = 0;
  // Maps given at every level (host f64, the concatenation over d of
  // [B][npix(d)]): the next forward uses them instead of the decimation
  // pyramid of level 0.
  virtual void load_levels(const double* x) = 0;
  // Maps given at every level on the device (map-major f64 [B][N_d] each,
  // d = 0 .. levels - 1): the decimation of the maps is skipped (the spin-2
  // transported pyramid feeds its own fields of every level)
  virtual void load_device_levels(const double* const* x) = 0;
  // Averages over k masks (level-0 indicators [k][npix(0)], nonzero: in the
  // mask) from the next forward on, or over every pixel (k = 0); values,
  // variances and cotangents are then [B][K][np].
  virtual void set_masks(const double* w, size_t k) = 0;
  // masks given at every level: [k][level][pixel] indicators, level d + 1
  // not derived from level d (the spin-2 front end erodes them itself)
  virtual void set_mask_levels(const std::vector<std::vector<std::vector<uint8_t>>>& levels) = 0;
  virtual int nmasks() const = 0;                   // 0: no masks
  virtual i64 mask_count(int k, int n) const = 0;   // pixels mask k averages at level n
  // Forward sweep on the loaded maps: values [B][np] complex (interleaved),
  // var [B][np] when moments.  Host outputs; the call synchronises.
  virtual void forward(bool moments, double* values, double* var) = 0;
  // After forward: map cotangent of Re sum(conj(cot) * values), cot [B][np]
  // complex interleaved (host).  Output to host f64 or device f64/f32.
  virtual void reverse_host(const double* cot, double* out) = 0;
  virtual void reverse_device(const double* cot, void* out, bool f32) = 0;
  // After a forward of maps given at every level: the map cotangent of every
  // level (its own terms, without the chain through the decimations),
  // map-major f64 [B][N_d] into the device buffers out[d]
  virtual void reverse_levels(const double* cot, double* const* out) = 0;
  // Large host <-> device copies on the engine's stream through its pinned
  // staging (pageable host memory, several host threads): to the device,
  // returning the non-finite doubles counted on the way when check; to the
  // host, synchronising.
  virtual size_t host_to_device(void* dst, const void* src, size_t n, bool check) = 0;
  virtual void device_to_host(void* dst, const void* src, size_t n) = 0;
  // The synthesis objective on the device: loss = sum_o w_(o mod np)
  // |S_o(x) - T_o|^2 over the coefficients [B][K][np] of the maps x (f64
  // [B][N_0], device), its gradient into g (f64, device) and the loss into
  // *loss (one f64, device), every step on the engine's stream with no host
  // synchronisation (a CUDA graph may capture it; the first call, outside a
  // capture, sets the kernels' attributes).  set_objective copies the
  // target [B][K][np] complex and weights [np] (null: 1) to the device.
  // Failed bounded waits set *error_flag().
  virtual void set_objective(const double* target, const double* weights) = 0;
  virtual void objective(const double* x, double* g, double* loss) = 0;
  virtual int* error_flag() = 0;
  // Device level-0 maps of the last load (T), for checkpoints.
  virtual void save_input(std::vector<double>& x) = 0;
  // exact copy of the loaded level-0 state (fields are stored as deviations
  // from per-map constants) and its restoration
  virtual void save_state(std::vector<double>& state) = 0;
  virtual void load_state(const std::vector<double>& state) = 0;

  size_t operator_bytes() const { return operator_bytes_; }
  size_t field_bytes() const { return field_bytes_; }
  Timers timers;

  // Kernel statistics since the last reset; profiling adds a pair of CUDA
  // events around every launch.
  virtual std::vector<KernelStat> kernel_stats() const = 0;
  virtual void reset_kernel_stats() = 0;
  virtual void set_profiling(bool on) = 0;
  virtual bool profiling() const = 0;
  // Mean cells read per row of each level's wavelet operator.
  virtual std::vector<double> mean_slots() const = 0;
  // Per level: slots per stored row, most cells of a tile, coloured layout (0/1).
  virtual std::vector<std::array<int, 4>> operator_layout() const = 0;
  virtual bool recomputes() const = 0;  // the field store in use (after prepare)
  virtual size_t kept_field_bytes() const = 0;  // bytes of z and branches of every level (after prepare)
  // The integer tables of the operators, for exact checks: kind 0, the
  // sorted distinct input cells of every output pixel of level `level`'s
  // wavelet (weight: the cell's largest |coefficient|); kind 1, the sorted
  // fine cells of nonzero weight of every coarse pixel of the decimation
  // from level `level` to `level` + 1 (weight: |w|).  Rows of the full level
  // in pixel order, padded with -1 (weight 0) to the widest (width).
  virtual void operator_rows(int level, int kind, std::vector<int64_t>& out, std::vector<double>& weight,
                             int& width) = 0;
  // Per level, the tile heights (rows of the field a thread takes) chosen
  // for: the wavelet of the maps, of the moduli, their adjoints, the
  // decimation of the maps (to the next level), of the moduli (from the
  // level before), their transposes (from the next level); 0: the default.
  virtual std::vector<std::array<int, 8>> tile_heights() const = 0;

 protected:
  explicit Engine(const Options& o, const Support* s = nullptr);
  Options opt_;
  std::vector<Coef> plan_;
  int levels_ = 1;
  int vb_ = 1;
  Support support_;
  std::vector<i64> npix_, ncore_;
  cudaStream_t stream_ = nullptr;
  size_t operator_bytes_ = 0, field_bytes_ = 0;
};

}  // namespace stl
