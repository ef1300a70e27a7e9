// Host-side parts of the large host <-> device copies (the engine's staging
// through pinned buffers): a plain copy, a copy that counts non-finite
// doubles, and floats widened to doubles.  The destinations are written with
// streaming stores where the CPU has AVX: a buffer of hundreds of MB is not
// read back soon, and ordinary stores would first read every destination
// line into the cache, a third more memory traffic on the host.
#include "hostcopy.hpp"

#include <immintrin.h>

#include <cmath>
#include <cstdint>
#include <cstring>

namespace stl {
namespace {

bool has_avx() {
  static const bool v = [] {
    __builtin_cpu_init();  // the CPU model, also when called from another constructor
    return __builtin_cpu_supports("avx") != 0;
  }();
  return v;
}

bool aligned32(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31) == 0; }

size_t count_nonfinite_scalar(const char* src, size_t n) {
  size_t bad = 0;
  for (size_t i = 0; i + 8 <= n; i += 8) {
    uint64_t v;
    std::memcpy(&v, src + i, 8);
    bad += (v & 0x7FF0000000000000ull) == 0x7FF0000000000000ull;  // exponent all ones: inf or nan
  }
  return bad;
}

size_t copy_scalar(char* dst, const char* src, size_t n, bool check) {
  const size_t bad = check ? count_nonfinite_scalar(src, n) : 0;
  std::memcpy(dst, src, n);
  return bad;
}

__attribute__((target("avx"))) size_t copy_avx(char* dst, const char* src, size_t n, bool check) {
  size_t i = 0, bad = 0;
  // 8-byte steps until the destination is 32-byte aligned
  while (i + 8 <= n && !aligned32(dst + i)) {
    bad += check ? count_nonfinite_scalar(src + i, 8) : 0;
    std::memcpy(dst + i, src + i, 8);
    i += 8;
  }
  const __m256d absmask = _mm256_castsi256_pd(_mm256_set1_epi64x(0x7FFFFFFFFFFFFFFFll));
  const __m256d inf = _mm256_set1_pd(INFINITY);
  for (; i + 64 <= n; i += 64) {
    const __m256d a = _mm256_loadu_pd(reinterpret_cast<const double*>(src + i));
    const __m256d b = _mm256_loadu_pd(reinterpret_cast<const double*>(src + i + 32));
    if (check) {  // |v| not below inf (unordered included): inf or nan
      bad += (size_t)__builtin_popcount(_mm256_movemask_pd(_mm256_cmp_pd(_mm256_and_pd(a, absmask), inf, _CMP_NLT_UQ)));
      bad += (size_t)__builtin_popcount(_mm256_movemask_pd(_mm256_cmp_pd(_mm256_and_pd(b, absmask), inf, _CMP_NLT_UQ)));
    }
    _mm256_stream_pd(reinterpret_cast<double*>(dst + i), a);
    _mm256_stream_pd(reinterpret_cast<double*>(dst + i + 32), b);
  }
  _mm_sfence();  // the streamed lines are visible before the caller signals completion
  if (i < n) bad += copy_scalar(dst + i, src + i, n - i, check);
  return bad;
}

__attribute__((target("avx"))) void widen_avx(double* dst, const float* src, size_t m) {
  size_t i = 0;
  for (; i < m && !aligned32(dst + i); ++i) dst[i] = (double)src[i];
  for (; i + 8 <= m; i += 8) {
    _mm256_stream_pd(dst + i, _mm256_cvtps_pd(_mm_loadu_ps(src + i)));
    _mm256_stream_pd(dst + i + 4, _mm256_cvtps_pd(_mm_loadu_ps(src + i + 4)));
  }
  _mm_sfence();
  for (; i < m; ++i) dst[i] = (double)src[i];
}

}  // namespace

size_t host_copy(void* dst, const void* src, size_t n, bool check) {
  char* d = static_cast<char*>(dst);
  const char* s = static_cast<const char*>(src);
  return has_avx() ? copy_avx(d, s, n, check) : copy_scalar(d, s, n, check);
}

void host_widen(double* dst, const float* src, size_t m) {
  if (has_avx()) {
    widen_avx(dst, src, m);
    return;
  }
  for (size_t i = 0; i < m; ++i) dst[i] = (double)src[i];
}

}  // namespace stl
