// Spin-2 front end of the B200 ScatCov engine: the polarisation P = Q + iU of
// level 0 becomes the spin-0 fields chi = chi_E + i chi_B = -(d_x - i d_y)^2 P
// (pixel units of the level) that the scalar engine takes as maps, two per
// input map (rows 2 b and 2 b + 1: chi_E and chi_B of map b).  The
// counterpart of the reference's crates/stl-core/src/spin.rs, used as its
// bridge uses it (crates/stl-bridge/src/lib.rs:139-240, 474-600):
//
//  * scalar pyramid (default): chi of level 0 only, decimated by the
//    engine's own scalar pyramid;
//  * transported pyramid: P_j the mean of the four children of P_{j-1}
//    turned into the parent's frame by parallel transport, chi_j of every
//    level given to the engine, which then skips its decimation of the maps;
//  * cross pairs (scalar pyramid): (a, b) with b a (Q, U) field and a
//    another one (spin_a 2) or a scalar map T (spin_a 0); the engine's cross
//    plan on the channel pairs (chi_a^E, chi_b^E) and (chi_a^B, chi_b^B), or
//    (T, chi_b^E) and (T, chi_b^B).
//
// The operators are built on the device in FP64 at the first use (one warp
// per stored row: the cells within kernel / 2 rings, the weighted least-norm
// weights exact on the polynomials of degree 2 rings by a Cholesky solve,
// the transport rotation e^{-2 i psi}), for the rows of faces 0, 4 and 8 only: a rotation
// of the sky by a quarter turn maps faces f to 4 (f / 4) + (f + 1) % 4 and
// leaves every weight unchanged (the weights are relative to the pixels'
// own frames), so the rows of the other faces are those rotations.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "scatcov.hpp"

namespace stl {

struct SpinConfig {
  i64 nside = 0;
  int levels = 1;         // engine levels (the transported pyramid builds them all)
  int kernel = 5;         // stencil side: 3, 5, 7 or 9 (rings = kernel / 2)
  bool transported = false;
  bool cross = false;     // pairs (a, b), scalar pyramid only
  int spin_a = 2;         // cross: 2 a (Q, U), 0 a scalar map T
  int batch = 1;          // input maps (pairs with cross)
};

class SpinFront {
 public:
  static std::unique_ptr<SpinFront> create(const SpinConfig& c, cudaStream_t s);
  virtual ~SpinFront() = default;

  // f64 values of the input maps: [batch, 2, npix] (cross: the first fields
  // [batch, 1 or 2, npix], then the second [batch, 2, npix])
  virtual size_t input_len() const = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  // The spin front of the maps x (host f64, or device f64 / f32) into the
  // engine's maps, then loaded into e; throws on non-finite input.
  virtual void load_host(Engine& e, const double* x) = 0;
  virtual void load_device(Engine& e, const void* x, bool f32) = 0;
  // The input cotangent of the engine's reverse sweep for cot (the values'
  // cotangents, host), to host f64 (out_host) or device memory.
  virtual void reverse_host(Engine& e, const double* cot, double* out) = 0;
  virtual void reverse_device(Engine& e, const double* cot, void* out, bool f32) = 0;
  // (Q, U) of `level` (transported means) and its (chi_E, chi_B), each
  // [batch, 2, npix(level)], for host maps x [batch, 2, npix] (no cross)
  virtual void fields(const double* x, int level, double* qu, double* chi) = 0;
  // The masks of every level of the valid data w [k, npix] (nonzero: valid):
  // the rows whose stencil reads valid data only, then eroded up the
  // pyramid (lib.rs:396-454)
  virtual std::vector<std::vector<std::vector<uint8_t>>> mask_levels(const double* w, size_t k) = 0;
  // the staged input maps of the last load (host copy, for checkpoints)
  virtual void save_input(std::vector<double>& x) = 0;
  virtual size_t bytes() const = 0;  // operators (0 before they are built)
  // builds the operators now (otherwise at the first use)
  virtual void prepare() = 0;
  // Operator rows of level `level` for exact checks: kind 0 the stencil
  // (cells and complex weights of every pixel, [npix][width]), kind 1 the
  // transported means (the 4 children's weights of every coarse pixel)
  virtual void export_rows(int level, int kind, std::vector<int64_t>& cells, std::vector<double>& w,
                           int& width) = 0;
  const SpinConfig& config() const { return cfg_; }

 protected:
  SpinConfig cfg_;
};

}  // namespace stl
