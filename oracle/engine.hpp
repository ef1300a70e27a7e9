// CPU FP64 restatement of the reference's ScatCov engine (full sky).
// TEST INFRASTRUCTURE ONLY: the oracle of the CUDA engine (see healpix_ops.hpp).
//
// The reference evaluates the statistics block by block with halos
// (crates/stl-core/src/engine.rs); its blocks are exact on their
// interiors, so the full-sky sweep below computes the same values up to
// the summation order.
#pragma once
#include "healpix_ops.hpp"
#include <map>
#include <utility>

namespace orc {

enum Family { MEAN = 0, VAR = 1, S1 = 2, S2 = 3, S3 = 4, S4 = 5 };

// crates/stl-core/src/plan.rs:47-68 (unused indices are -1)
struct Coef {
  int family, native, c1, c2, j1, j2, j3, l1, l2, l3;
};

// build_plan (plan.rs:80-158), all families; cross_only keeps the pairs
// c1 != c2 (the bridge's `cross` plan, stl-bridge/src/lib.rs plan_of).
std::vector<Coef> build_plan(int J, int L, const std::vector<int>& j_to_dg, int C, bool cross_only);

struct Masks {  // crates/stl-core/src/mask.rs
  std::vector<std::vector<std::vector<double>>> weights;  // [K][levels][N_n]
  std::vector<std::vector<i64>> counts;                    // [K][levels]
};

struct Engine {
  i64 nside0 = 0;
  int J = 0, L = 4, ksz = 5, B = 1, C = 1, levels = 1;
  bool fewer = false;
  Gauge gauge = Gauge::Cosmo;
  std::vector<int> j_to_dg;
  std::vector<double> ker;  // [L][2][P], f32-rounded
  std::vector<ConvOp> conv;
  std::vector<Csr> down, downT;  // level d -> d + 1, and transposes
  std::vector<Coef> plan;
  bool has_masks = false;
  Masks masks;
  // forward state
  std::vector<std::vector<double>> maps;                         // [BC][N_d]
  std::vector<std::vector<cplx>> z;                              // [BC][L][N_n]
  std::map<std::pair<int, int>, std::vector<double>> m;          // (d, n): [BC][L][N_n]
  std::map<std::pair<int, int>, std::vector<cplx>> br;           // (d, n): [BC][L][L][N_n]

  i64 npix(int n) const { return 12 * (nside0 >> n) * (nside0 >> n); }
  int K() const { return has_masks ? (int)masks.weights.size() : 1; }
  void init(i64 nside, int J, int L, int ksz, Gauge gauge, int B, int C, bool fewer, const std::vector<int>& dg,
            bool cross_only, size_t cache_budget);
  void set_masks(const double* w0, i64 K);
  // masks given at every level ([K][levels][N_n] indicators, mask.rs:75-82)
  void set_mask_levels(const double* w, i64 K);
  void load(const double* x);
  void load_levels(const double* x);
  // values [B][K][np] complex; second [B][K][np] when moments
  void forward(std::vector<cplx>& values, std::vector<double>* second);
  // maps gradient of every level [levels][BC][N_d]
  std::vector<std::vector<double>> reverse(const std::vector<cplx>& cot);
  // g0 [BC][N_0] and bands (engine.rs:730-779)
  void analysis_vjp(std::vector<std::vector<double>> mg, std::vector<double>& g0,
                    std::vector<std::vector<double>>& bands);
  std::vector<double> decimate(int d, const std::vector<double>& x, i64 rows) const;
  std::vector<double> decimate_adjoint(int d, const std::vector<double>& g, i64 rows) const;
};

}  // namespace orc
