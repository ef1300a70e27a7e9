// C entry points of the map files (mapio.hpp): NESTED .npy and HEALPix FITS
// maps read whole or by pixel range, written whole or in pieces.  Status 0
// on success, -1 with stlp_last_error() set otherwise.
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "mapio.hpp"

namespace stl {
void set_error(const std::string& msg);
}

namespace {

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    stl::set_error(e.what());
  } catch (...) {
    stl::set_error("unknown native failure");
  }
  return -1;
}

std::string path_of(const char* p) {
  if (!p || !*p) throw std::runtime_error("null or empty path");
  return std::string(p);
}

}  // namespace

extern "C" {

int stlp_map_len(const char* path, size_t* n) {
  return guarded([&] {
    if (!n) throw std::runtime_error("null argument");
    *n = stl::mapio::map_len(path_of(path));
  });
}

int stlp_npy_shape(const char* path, size_t* shape, size_t max_dims, size_t* ndim) {
  return guarded([&] {
    if (!ndim || (max_dims && !shape)) throw std::runtime_error("null argument");
    const std::vector<size_t> s = stl::mapio::npy_shape(path_of(path));
    *ndim = s.size();
    if (s.size() > max_dims) throw std::runtime_error("the array has more axes than the buffer holds");
    for (size_t i = 0; i < s.size(); ++i) shape[i] = s[i];
  });
}

int stlp_map_read(const char* path, double* out, size_t n) {
  return guarded([&] {
    if (!out && n) throw std::runtime_error("null argument");
    const std::vector<double> v = stl::mapio::read_map(path_of(path));
    if (v.size() != n)
      throw std::runtime_error(std::string(path) + ": the map holds " + std::to_string(v.size()) + " values, not " +
                               std::to_string(n));
    if (n) std::memcpy(out, v.data(), n * sizeof(double));
  });
}

int stlp_map_read_range(const char* path, size_t start, size_t end, double* out) {
  return guarded([&] {
    if (!out && end > start) throw std::runtime_error("null argument");
    const std::vector<double> v = stl::mapio::read_map_range(path_of(path), start, end);
    if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(double));
  });
}

int stlp_npy_write(const char* path, const double* values, const size_t* shape, size_t ndim) {
  return guarded([&] {
    if ((!values || !shape) && ndim) throw std::runtime_error("null argument");
    stl::mapio::write_npy(path_of(path), values, std::vector<size_t>(shape, shape + ndim));
  });
}

int stlp_fits_write(const char* path, const double* values, size_t n, const char* column, int dbl) {
  return guarded([&] {
    if (!values || !column) throw std::runtime_error("null argument");
    stl::mapio::write_healpix_fits(path_of(path), values, n, column, dbl != 0);
  });
}

int stlp_map_create(const char* path, size_t n, const char* column, int dbl) {
  return guarded([&] {
    if (!column) throw std::runtime_error("null argument");
    stl::mapio::create_map(path_of(path), n, column, dbl != 0);
  });
}

int stlp_map_write(const char* path, size_t start, const double* values, size_t count, int dbl) {
  return guarded([&] {
    if (!values && count) throw std::runtime_error("null argument");
    stl::mapio::write_piece(path_of(path), start, values, count, dbl != 0);
  });
}

}  // extern "C"
