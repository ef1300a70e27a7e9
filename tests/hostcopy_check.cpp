// Checks of the host copies behind the staged host <-> device transfers:
// copies with non-finite counting at every alignment, floats widened to
// doubles, odd byte counts; exits nonzero on a mismatch.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "hostcopy.hpp"

int main() {
  std::mt19937_64 rng(1);
  int fails = 0;
  for (int t = 0; t < 300; ++t) {
    // doubles with inf / nan planted, source and destination at 8-byte offsets
    const size_t n = (rng() % 5000) * 8;
    const size_t so = (rng() % 4) * 8, dofs = (rng() % 4) * 8;
    std::vector<double> src(n / 8 + 8), dst(n / 8 + 8, -1.0);
    for (auto& v : src) v = (double)(rng() % 1000) - 500.0;
    for (size_t i = 0; i < n / 8; ++i)
      if (rng() % 50 == 0) src[so / 8 + i] = (i & 1) ? INFINITY : NAN;
    size_t nb = 0;
    for (size_t i = 0; i < n / 8; ++i) nb += !std::isfinite(src[so / 8 + i]);
    const size_t bad = stl::host_copy((char*)dst.data() + dofs, (const char*)src.data() + so, n, true);
    if (bad != nb || std::memcmp((char*)dst.data() + dofs, (const char*)src.data() + so, n)) {
      ++fails;
      std::printf("copy: n %zu, %zu non-finite counted, %zu planted\n", n, bad, nb);
    }
    // floats to doubles, the destination at every double offset; no write past the end
    const size_t m = rng() % 3000 + 1, off = rng() % 4;
    std::vector<float> f(m);
    std::vector<double> d(m + 8, -7.0);
    for (auto& v : f) v = (float)((double)(rng() % 100000) / 7.0);
    stl::host_widen(d.data() + off, f.data(), m);
    for (size_t i = 0; i < m; ++i)
      if (d[off + i] != (double)f[i]) {
        ++fails;
        std::printf("widen: element %zu\n", i);
        break;
      }
    if (d[off + m] != -7.0 || (off && d[off - 1] != -7.0)) {
      ++fails;
      std::printf("widen: write outside the destination\n");
    }
    // any byte count, byte offsets, no check
    const size_t nbytes = rng() % 4000 + 1;
    std::vector<char> a(nbytes + 64), b(nbytes + 64, 0);
    for (auto& c : a) c = (char)rng();
    stl::host_copy(b.data() + 1, a.data() + 3, nbytes, false);
    if (std::memcmp(b.data() + 1, a.data() + 3, nbytes)) {
      ++fails;
      std::printf("bytes: n %zu\n", nbytes);
    }
  }
  std::printf("fails %d\n", fails);
  return fails != 0;
}
