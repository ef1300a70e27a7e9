// Host-side copies of large buffers (compiled by the host compiler alone).
#pragma once
#include <cstddef>

namespace stl {

// dst[0, n) = src[0, n); with check (n a multiple of 8): the number of
// non-finite doubles among the copied bytes
size_t host_copy(void* dst, const void* src, size_t n, bool check);
// dst[i] = (double)src[i] for i < m (exact)
void host_widen(double* dst, const float* src, size_t m);

}  // namespace stl
