// CPU FP64 restatement of the reference's HEALPix geometry and operators.
// TEST INFRASTRUCTURE ONLY (see healpix_ops.hpp).
#include "healpix_ops.hpp"

#include <atomic>
#include <cstdlib>
#include <stdexcept>
#include <thread>

namespace orc {

// ---------------------------------------------------------------------------
// threads
static int g_threads = 0;
int num_threads() {
  if (g_threads <= 0) {
    const char* e = std::getenv("STL_ORACLE_THREADS");
    int n = e ? std::atoi(e) : 0;
    if (n <= 0) n = (int)std::max(1u, std::thread::hardware_concurrency());
    g_threads = n;
  }
  return g_threads;
}
void set_num_threads(int n) { g_threads = n; }

void parallel_chunks(i64 n, const std::function<void(i64, i64, int)>& f) {
  int t = num_threads();
  if (n <= 0) return;
  if (t <= 1 || n < 2) { f(0, n, 0); return; }
  i64 nt = std::min<i64>(t, n);
  std::vector<std::thread> pool;
  for (i64 w = 0; w < nt; ++w) {
    i64 a = n * w / nt, b = n * (w + 1) / nt;
    pool.emplace_back([&, a, b, w] { f(a, b, (int)w); });
  }
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// HEALPix primitives (crates/stl-core/src/healpix.rs)
static const i64 JRLL[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
static const i64 JPLL[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

static inline i64 compress_bits(i64 v) {  // healpix.rs:53-61
  uint64_t u = (uint64_t)v & 0x5555555555555555ULL;
  u = (u | (u >> 1)) & 0x3333333333333333ULL;
  u = (u | (u >> 2)) & 0x0F0F0F0F0F0F0F0FULL;
  u = (u | (u >> 4)) & 0x00FF00FF00FF00FFULL;
  u = (u | (u >> 8)) & 0x0000FFFF0000FFFFULL;
  return (i64)((u | (u >> 16)) & 0x00000000FFFFFFFFULL);
}
static inline i64 spread_bits(i64 v) {  // healpix.rs:63-71
  uint64_t u = (uint64_t)v & 0x00000000FFFFFFFFULL;
  u = (u | (u << 16)) & 0x0000FFFF0000FFFFULL;
  u = (u | (u << 8)) & 0x00FF00FF00FF00FFULL;
  u = (u | (u << 4)) & 0x0F0F0F0F0F0F0F0FULL;
  u = (u | (u << 2)) & 0x3333333333333333ULL;
  return (i64)((u | (u << 1)) & 0x5555555555555555ULL);
}

void nest2xyf(i64 pix, int order, i64& ix, i64& iy, i64& face) {  // healpix.rs:74-79
  face = pix >> (2 * order);
  i64 local = pix & ((i64(1) << (2 * order)) - 1);
  ix = compress_bits(local);
  iy = compress_bits(local >> 1);
}

i64 xyf2nest(i64 ix, i64 iy, i64 face, int order) {  // healpix.rs:82-85
  return (face << (2 * order)) + spread_bits(ix) + (spread_bits(iy) << 1);
}

void xyf2ang(i64 ix, i64 iy, i64 face, i64 nside, double& theta, double& phi) {  // healpix.rs:88-127
  i64 jr = JRLL[face] * nside - ix - iy - 1;
  double ns = (double)nside;
  double fact2 = 4.0 / (12.0 * ns * ns);
  double fact1 = 2.0 / (3.0 * ns);
  bool north = jr < nside, south = jr > 3 * nside;
  i64 nr = north ? jr : (south ? 4 * nside - jr : nside);
  i64 kshift = (north || south) ? 0 : ((jr - nside) & 1);
  double nrf = (double)nr;
  if (north || south) {
    double tmp = nrf * nrf * fact2;
    double z_cap = 1.0 - tmp;
    double sth_cap = std::sqrt(tmp * (2.0 - tmp));
    double theta_cap = std::atan2(sth_cap, z_cap);
    theta = north ? theta_cap : PI - theta_cap;
  } else {
    theta = std::acos((2.0 * ns - (double)jr) * fact1);
  }
  i64 jp = floor_div(JPLL[face] * nr + ix - iy + 1 + kshift, 2);
  if (jp > 4 * nr) jp -= 4 * nr;
  if (jp < 1) jp += 4 * nr;
  phi = ((double)jp - ((double)kshift + 1.0) * 0.5) * (0.5 * PI / nrf);
}

void pix2ang_nest(i64 pix, i64 nside, double& theta, double& phi) {
  i64 ix, iy, f;
  nest2xyf(pix, order_of(nside), ix, iy, f);
  xyf2ang(ix, iy, f, nside, theta, phi);
}

void centre_lonlat(i64 pix, i64 nside, double& lon, double& lat) {  // healpix.rs:140-143
  double theta, phi;
  pix2ang_nest(pix, nside, theta, phi);
  lon = deg2rad(rad2deg(phi));
  lat = deg2rad(90.0 - rad2deg(theta));
}

static i64 isqrt(i64 v) {  // healpix.rs:145-154
  i64 r = (i64)std::sqrt((double)v);
  if (r * r > v) r -= 1;
  if ((r + 1) * (r + 1) <= v) r += 1;
  return r;
}

i64 ring2nest(i64 pix, int order) {  // healpix.rs:157-210
  i64 nside = i64(1) << order;
  i64 np = npix(nside);
  i64 ncap = 2 * nside * (nside - 1);
  i64 nl2 = 2 * nside;
  i64 iring, iphi, kshift, nr, face;
  if (pix < ncap) {
    i64 ir = (1 + isqrt(1 + 2 * pix)) >> 1;
    i64 ip = pix + 1 - 2 * ir * (ir - 1);
    iring = ir; iphi = ip; kshift = 0; nr = ir;
    face = floor_div(ip - 1, std::max<i64>(ir, 1));
  } else if (pix < np - ncap) {
    i64 ip = pix - ncap;
    i64 tmp = ip >> (order + 2);
    i64 ir = tmp + nside;
    i64 ip2 = ip - tmp * 4 * nside + 1;
    i64 ire = ir - nside + 1;
    i64 irm = nl2 + 2 - ire;
    i64 ifm = (ip2 - floor_div(ire, 2) + nside - 1) >> order;
    i64 ifp = (ip2 - floor_div(irm, 2) + nside - 1) >> order;
    iring = ir; iphi = ip2; kshift = (ir + nside) & 1; nr = nside;
    face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : ifm + 8);
  } else {
    i64 ip = np - pix;
    i64 ir = (1 + isqrt(2 * ip - 1)) >> 1;
    i64 ip2 = 4 * ir + 1 - (ip - 2 * ir * (ir - 1));
    iring = 2 * nl2 - ir; iphi = ip2; kshift = 0; nr = ir;
    face = 8 + floor_div(ip2 - 1, std::max<i64>(ir, 1));
  }
  i64 irt = iring - JRLL[face] * nside + 1;
  i64 ipt = 2 * iphi - JPLL[face] * nr - kshift - 1;
  if (ipt >= nl2) ipt -= 8 * nside;
  i64 ix = (ipt - irt) >> 1;
  i64 iy = (-ipt - irt) >> 1;
  return xyf2nest(ix, iy, face, order);
}

static i64 ring_above(double z, i64 nside) {  // healpix.rs:216-229
  double az = std::fabs(z);
  double ns = (double)nside;
  if (az <= 2.0 / 3.0) return (i64)std::trunc(ns * (2.0 - 1.5 * z));
  i64 iring = (i64)std::trunc(ns * std::sqrt(3.0 * (1.0 - az)));
  return z > 0.0 ? iring : 4 * nside - iring - 1;
}

static void ring_info(i64 ring, i64 nside, i64& startpix, i64& ringpix, double& theta, bool& shifted) {
  // healpix.rs:232-259
  i64 ncap = 2 * nside * (nside - 1);
  i64 np = npix(nside);
  double ns = (double)nside;
  double fact1 = 2.0 / (3.0 * ns);
  double fact2 = 1.0 / (3.0 * ns * ns);
  i64 northring = ring > 2 * nside ? 4 * nside - ring : ring;
  if (northring < nside) {
    double nrf = (double)northring;
    double tmp = nrf * nrf * fact2;
    theta = std::atan2(std::sqrt(tmp * (2.0 - tmp)), 1.0 - tmp);
    ringpix = 4 * northring;
    shifted = true;
    startpix = 2 * northring * (northring - 1);
  } else {
    theta = std::acos((double)(2 * nside - northring) * fact1);
    ringpix = 4 * nside;
    shifted = ((northring - nside) & 1) == 0;
    startpix = ncap + (northring - nside) * 4 * nside;
  }
  if (northring != ring) {
    theta = PI - theta;
    startpix = np - startpix - ringpix;
  }
}

static void ring_pair(double phi, i64 ring, i64 nside, i64& p0, i64& p1, double& w0, double& w1, double& th) {
  // healpix.rs:262-280
  i64 sp, nr; bool shifted;
  ring_info(ring, nside, sp, nr, th, shifted);
  double dphi = (2.0 * PI) / (double)nr;
  double half = shifted ? 0.5 : 0.0;
  double tmp = phi / dphi - half;
  i64 i1 = (i64)std::trunc(tmp);
  if (tmp < 0.0) i1 -= 1;
  double ww = (phi - ((double)i1 + half) * dphi) / dphi;
  i64 i2 = i1 + 1;
  if (i1 < 0) i1 += nr;
  if (i2 >= nr) i2 -= nr;
  p0 = sp + i1; p1 = sp + i2; w0 = 1.0 - ww; w1 = ww;
}

void get_interpol_ring(double theta, double phi, i64 nside, i64 out_pix[4], double out_w[4]) {
  // healpix.rs:283-324
  i64 np = npix(nside);
  double z = std::cos(theta);
  i64 ir1 = ring_above(z, nside);
  i64 ir2 = ir1 + 1;
  i64 pix[4] = {0, 0, 0, 0};
  double wgt[4] = {0, 0, 0, 0};
  i64 p0, p1, p2, p3; double w0, w1, w2, w3, theta1, theta2;
  ring_pair(phi, std::max<i64>(ir1, 1), nside, p0, p1, w0, w1, theta1);
  if (ir1 > 0) { pix[0] = p0; pix[1] = p1; wgt[0] = w0; wgt[1] = w1; }
  ring_pair(phi, std::min<i64>(ir2, 4 * nside - 1), nside, p2, p3, w2, w3, theta2);
  if (ir2 < 4 * nside) { pix[2] = p2; pix[3] = p3; wgt[2] = w2; wgt[3] = w3; }
  bool north = ir1 == 0;
  bool south = ir2 == 4 * nside && !north;
  if (north) {
    double wn = theta / theta2;
    double facn = (1.0 - wn) * 0.25;
    out_pix[0] = (pix[2] + 2) & 3; out_pix[1] = (pix[3] + 2) & 3; out_pix[2] = pix[2]; out_pix[3] = pix[3];
    out_w[0] = facn; out_w[1] = facn; out_w[2] = wgt[2] * wn + facn; out_w[3] = wgt[3] * wn + facn;
  } else if (south) {
    double ws = (theta - theta1) / (PI - theta1);
    double facs = ws * 0.25;
    out_pix[0] = pix[0]; out_pix[1] = pix[1];
    out_pix[2] = ((pix[0] + 2) & 3) + np - 4; out_pix[3] = ((pix[1] + 2) & 3) + np - 4;
    out_w[0] = wgt[0] * (1.0 - ws) + facs; out_w[1] = wgt[1] * (1.0 - ws) + facs; out_w[2] = facs; out_w[3] = facs;
  } else {
    double wm = (theta - theta1) / (theta2 - theta1);
    for (int i = 0; i < 4; ++i) out_pix[i] = pix[i];
    out_w[0] = wgt[0] * (1.0 - wm); out_w[1] = wgt[1] * (1.0 - wm); out_w[2] = wgt[2] * wm; out_w[3] = wgt[3] * wm;
  }
}

static inline double norm3(const double v[3]) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

void interp_weights_nested(const double v[3], int order, i64 pix[4], double w[4]) {  // healpix.rs:336-347
  double n = std::max(norm3(v), 1e-12);
  double vn[3] = {v[0] / n, v[1] / n, v[2] / n};
  double theta = std::acos(std::min(1.0, std::max(-1.0, vn[2])));
  double phi = remainder(std::atan2(vn[1], vn[0]), 2.0 * PI);
  double lon_deg = rad2deg(phi);
  double lat_deg = 90.0 - rad2deg(theta);
  double theta2 = deg2rad(90.0 - lat_deg);
  double phi2 = remainder(deg2rad(lon_deg), 2.0 * PI);
  i64 rp[4];
  get_interpol_ring(theta2, phi2, i64(1) << order, rp, w);
  for (int i = 0; i < 4; ++i) pix[i] = ring2nest(rp[i], order);
}

// ---------------------------------------------------------------------------
// stencil + wavelet (stencil.rs, wavelet.rs, conv.rs:167-172)
std::vector<std::array<double, 3>> local_kernel_grid(int ksz, i64 nside) {  // stencil.rs:33-47
  i64 half = ksz / 2;
  double ns = (double)nside;
  double alpha_pix = std::sqrt(4.0 * PI / (12.0 * ns * ns));
  std::vector<std::array<double, 3>> out;
  for (i64 i = 0; i < ksz; ++i)
    for (i64 j = 0; j < ksz; ++j) {
      i64 x = j - half, y = i - half;
      double dtheta = std::sqrt((double)(x * x + y * y)) * alpha_pix;
      double dphi = std::atan2((double)y, (double)x);
      out.push_back({std::sin(dtheta) * std::cos(dphi), std::sin(dtheta) * std::sin(dphi), std::cos(dtheta)});
    }
  return out;
}

static Mat3 matmul(const Mat3& a, const Mat3& b) {
  Mat3 c{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
  return c;
}

std::vector<Mat3> rotation_matrices(double theta, double phi, int G, Gauge gauge) {  // stencil.rs:51-88
  double ct = std::cos(theta), st = std::sin(theta), cp = std::cos(phi), sp = std::sin(phi);
  Mat3 base = {{{cp * ct, -sp, cp * st}, {sp * ct, cp, sp * st}, {-st, 0.0, ct}}};
  double n0[3] = {base[0][2], base[1][2], base[2][2]};
  double nn = std::max(norm3(n0), 1e-12);
  double n[3] = {n0[0] / nn, n0[1] / nn, n0[2] / nn};
  double alpha_base, sign_g;
  if (gauge == Gauge::Cosmo) {
    if (theta > PI / 2.0) { alpha_base = phi; sign_g = -1.0; } else { alpha_base = -phi; sign_g = 1.0; }
  } else { alpha_base = 0.0; sign_g = 1.0; }
  double skew[3][3] = {{0.0, -n[2], n[1]}, {n[2], 0.0, -n[0]}, {-n[1], n[0], 0.0}};
  double step = PI / (double)G;
  std::vector<Mat3> out;
  for (int g = 0; g < G; ++g) {
    double alpha = alpha_base + sign_g * ((double)g * step);
    double ca = std::cos(alpha), sa = std::sin(alpha);
    Mat3 rg{};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double eye = (i == j) ? 1.0 : 0.0;
        rg[i][j] = eye * ca + skew[i][j] * sa + n[i] * n[j] * (1.0 - ca);
      }
    out.push_back(matmul(rg, base));
  }
  return out;
}

std::vector<cplx> wavelet_kernel(int ksz, double sigma) {  // wavelet.rs:11-26
  auto c = [&](int i) { return (double)i - ((double)ksz - 1.0) / 2.0; };
  std::vector<cplx> k;
  for (int i = 0; i < ksz; ++i)
    for (int j = 0; j < ksz; ++j) {
      double x = c(j), y = c(i);
      double mother = std::exp(-(x * x + y * y) / (2.0 * sigma * sigma));
      double angle = 0.5 * PI * x;
      k.emplace_back(std::cos(angle) * mother, std::sin(angle) * mother);
    }
  double n = (double)k.size();
  double sr = 0.0, si = 0.0;
  for (auto& v : k) { sr += v.real(); si += v.imag(); }
  double mr = sr / n, mi = si / n;
  for (auto& v : k) v = cplx(v.real() - mr, v.imag() - mi);
  double l1 = 0.0;
  for (auto& v : k) l1 += std::hypot(v.real(), v.imag());
  for (auto& v : k) v = cplx(v.real() / l1, v.imag() / l1);
  return k;
}

std::vector<double> wavelet_weights(int ksz) {  // wavelet.rs:142-145
  auto k = wavelet_kernel(ksz, 1.0);
  std::vector<double> out;
  for (auto& v : k) out.push_back(v.real());
  for (auto& v : k) out.push_back(v.imag());
  return out;
}

std::vector<double> shared_kernel(const std::vector<double>& weights, int G, int P) {  // conv.rs:167-172
  std::vector<double> out;
  for (int g = 0; g < G; ++g)
    for (int i = 0; i < 2 * P; ++i) out.push_back((double)(float)weights[i]);
  return out;
}

// ---------------------------------------------------------------------------
// face frames (dia.rs:24-101; the HEALPix C++ neighbour tables)
static const int8_t NB_FACE[9][12] = {
    {8, 9, 10, 11, -1, -1, -1, -1, 10, 11, 8, 9}, {5, 6, 7, 4, 8, 9, 10, 11, 9, 10, 11, 8},
    {-1, -1, -1, -1, 5, 6, 7, 4, -1, -1, -1, -1}, {4, 5, 6, 7, 11, 8, 9, 10, 11, 8, 9, 10},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},       {1, 2, 3, 0, 0, 1, 2, 3, 5, 6, 7, 4},
    {-1, -1, -1, -1, 7, 4, 5, 6, -1, -1, -1, -1}, {3, 0, 1, 2, 3, 0, 1, 2, 4, 5, 6, 7},
    {2, 3, 0, 1, -1, -1, -1, -1, 0, 1, 2, 3}};
static const uint8_t NB_SWAP[9][3] = {{0, 0, 3}, {0, 0, 6}, {0, 0, 0}, {0, 0, 5}, {0, 0, 0},
                                      {5, 0, 0}, {0, 0, 0}, {6, 0, 0}, {3, 0, 0}};

bool ext_pix(i64 face, i64 ex, i64 ey, i64 nside, int order, i64& out) {
  i64 x = ex, y = ey;
  int nb = 4;
  if (x < 0) { x += nside; nb -= 1; } else if (x >= nside) { x -= nside; nb += 1; }
  if (y < 0) { y += nside; nb -= 3; } else if (y >= nside) { y -= nside; nb += 3; }
  int f = NB_FACE[nb][face];
  if (f < 0) return false;
  int bits = NB_SWAP[nb][face >> 2];
  if (bits & 1) x = nside - x - 1;
  if (bits & 2) y = nside - y - 1;
  if (bits & 4) std::swap(x, y);
  out = xyf2nest(x, y, f, order);
  return true;
}

bool rel_offset(i64 row, i64 cell, i64 nside, int order, i64& dx, i64& dy) {
  i64 x, y, f, xq, yq, fq;
  nest2xyf(row, order, x, y, f);
  nest2xyf(cell, order, xq, yq, fq);
  if (fq == f) { dx = xq - x; dy = yq - y; return true; }
  int nb = -1;
  for (int k = 0; k < 9; ++k)
    if (k != 4 && NB_FACE[k][f] == fq) { nb = k; break; }
  if (nb < 0) return false;
  int bits = NB_SWAP[nb][f >> 2];
  i64 a = xq, b = yq;
  if (bits & 4) std::swap(a, b);
  if (bits & 2) b = nside - b - 1;
  if (bits & 1) a = nside - a - 1;
  i64 xdir = nb % 3 - 1, ydir = nb / 3 - 1;
  dx = a + xdir * nside - x;
  dy = b + ydir * nside - y;
  return true;
}

// ---------------------------------------------------------------------------
// neighbourhoods (neighbours.rs)
std::vector<i64> kth_neighbourhood_set(i64 id, i64 nside, int k) {
  int order = order_of(nside);
  i64 x, y, f;
  nest2xyf(id, order, x, y, f);
  std::vector<i64> out;
  for (i64 dy = -k; dy <= k; ++dy)
    for (i64 dx = -k; dx <= k; ++dx) {
      i64 q;
      if (ext_pix(f, x + dx, y + dy, nside, order, q)) out.push_back(q);
    }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

std::vector<i64> parents(const std::vector<i64>& ids) {
  std::vector<i64> out;
  for (i64 v : ids) out.push_back(floor_div(v, 4));
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

std::vector<i64> children(const std::vector<i64>& ids) {
  std::vector<i64> out;
  for (i64 v : ids)
    for (int c = 0; c < 4; ++c) out.push_back(4 * v + c);
  return out;
}

std::vector<i64> dilate(const std::vector<i64>& ids, i64 nside, int rings) {
  if (rings == 0) return ids;
  if ((i64)rings >= nside) {
    std::vector<i64> all(npix(nside));
    for (i64 i = 0; i < (i64)all.size(); ++i) all[i] = i;
    return all;
  }
  std::vector<i64> out;
  for (i64 v : ids) {
    auto nb = kth_neighbourhood_set(v, nside, rings);
    out.insert(out.end(), nb.begin(), nb.end());
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

std::vector<i64> dilate_fine(const std::vector<i64>& ids, i64 nside, int rings) {
  if (nside < 4 || rings <= 1) return dilate(ids, nside, rings);
  return children(dilate(parents(ids), nside / 2, rings / 2 + 1));
}

// ---------------------------------------------------------------------------
// bound stencils (conv.rs:73-135)
static inline i64 search(const i64* grid, i64 n, i64 v) {
  if (!grid) return (v >= 0 && v < n) ? v : -1;
  const i64* p = std::lower_bound(grid, grid + n, v);
  return (p != grid + n && *p == v) ? (i64)(p - grid) : -1;
}

void bind_rows(const i64* grid, i64 ngrid, const i64* rows, i64 nrows, i64 nside, int ksz, int G, Gauge gauge,
               double eps, Bound& out, i64 row0) {
  int order = order_of(nside);
  int P = ksz * ksz;
  int p_ref = (ksz / 2) * (ksz + 1);
  auto stencil = local_kernel_grid(ksz, nside);
  out.K = nrows; out.G = G; out.P = P;
  out.pos.assign((size_t)nrows * G * P * 4, 0);
  out.w.assign((size_t)nrows * G * P * 4, 0.0);
  out.complete.assign(nrows, 1);
  std::vector<std::array<i64, 4>> idx(P);
  std::vector<std::array<double, 4>> wt(P);
  for (i64 k = 0; k < nrows; ++k) {
    i64 id = rows ? rows[k] : row0 + k;
    double theta, phi;
    pix2ang_nest(id, nside, theta, phi);
    theta = deg2rad(90.0 - rad2deg(PI / 2.0 - theta));
    phi = deg2rad(rad2deg(phi));
    auto rots = rotation_matrices(theta, phi, G, gauge);
    for (int g = 0; g < G; ++g) {
      const Mat3& r = rots[g];
      for (int p = 0; p < P; ++p) {
        const auto& v = stencil[p];
        double a[3] = {r[0][0] * v[0] + r[0][1] * v[1] + r[0][2] * v[2],
                       r[1][0] * v[0] + r[1][1] * v[1] + r[1][2] * v[2],
                       r[2][0] * v[0] + r[2][1] * v[1] + r[2][2] * v[2]};
        interp_weights_nested(a, order, idx[p].data(), wt[p].data());
      }
      for (int p = 0; p < P; ++p) {
        const i64* ix = idx[p].data();
        const double* wx = wt[p].data();
        i64 found[4];
        auto bind = [&](const i64* ixx, const double* wxx) {
          for (int n = 0; n < 4; ++n) {
            found[n] = search(grid, ngrid, ixx[n]);
            if (eps > 0.0 && wxx[n] <= eps) found[n] = -1;
          }
        };
        bind(ix, wx);
        if (found[0] < 0 && found[1] < 0 && found[2] < 0 && found[3] < 0) {
          ix = idx[p_ref].data();
          wx = wt[p_ref].data();
          bind(ix, wx);
        }
        double w[4];
        for (int n = 0; n < 4; ++n) w[n] = wx[n] * (found[n] >= 0 ? 1.0 : 0.0);
        double colsum = w[0] + w[1] + w[2] + w[3];
        if (colsum == 0.0) {
          w[0] = found[0] >= 0 ? 1.0 : 0.0;
          colsum = w[0] + w[1] + w[2] + w[3];
        }
        for (int n = 0; n < 4; ++n) {
          size_t a = (((size_t)k * G + g) * P + p) * 4 + n;
          out.w[a] = w[n] / std::max(colsum, 1e-12);
          out.pos[a] = (int32_t)(found[n] >= 0 ? found[n] : 0);
          if (found[n] < 0) out.complete[k] = 0;
        }
      }
    }
  }
}

void ConvOp::init(std::vector<i64> grid_, std::vector<i64> rows_, i64 nside_, int ksz_, int G_, Gauge gauge_,
                  double eps_, size_t cache_budget_bytes) {
  grid = std::move(grid_);
  rows = std::move(rows_);
  nside = nside_; ksz = ksz_; G = G_; gauge = gauge_; eps = eps_;
  n_in = grid.empty() ? npix(nside) : (i64)grid.size();
  n_rows = rows.empty() ? (grid.empty() ? npix(nside) : (i64)grid.size()) : (i64)rows.size();
  size_t bytes = (size_t)n_rows * G * ksz * ksz * 4 * 12;
  cached = bytes <= cache_budget_bytes;
  if (cached) {
    whole.K = n_rows; whole.G = G; whole.P = ksz * ksz;
    whole.pos.resize((size_t)n_rows * G * whole.P * 4);
    whole.w.resize(whole.pos.size());
    whole.complete.resize(n_rows);
    parallel_chunks(n_rows, [&](i64 a, i64 b, int) {
      Bound part;
      chunk(a, b, nullptr, part);
      size_t per = (size_t)G * whole.P * 4;
      std::copy(part.pos.begin(), part.pos.end(), whole.pos.begin() + a * per);
      std::copy(part.w.begin(), part.w.end(), whole.w.begin() + a * per);
      std::copy(part.complete.begin(), part.complete.end(), whole.complete.begin() + a);
    });
  }
}

void ConvOp::chunk(i64 k0, i64 k1, const std::vector<i64>* sel, Bound& b) const {
  std::vector<i64> ids(k1 - k0);
  for (i64 i = k0; i < k1; ++i) {
    i64 r = sel ? (*sel)[i] : i;
    ids[i - k0] = rows.empty() ? (grid.empty() ? r : grid[r]) : rows[r];
  }
  bind_rows(grid.empty() ? nullptr : grid.data(), n_in, ids.data(), k1 - k0, nside, ksz, G, gauge, eps, b);
}

// y [R][G*2][K] with K = |sel| (or all rows); ker [G][2][P]
void ConvOp::forward(const std::vector<double>& ker, const double* x, i64 R, double* y,
                     const std::vector<i64>* sel) const {
  i64 K = sel ? (i64)sel->size() : n_rows;
  int P = ksz * ksz;
  parallel_chunks(K, [&](i64 a, i64 b, int) {
    const i64 step = 1024;
    Bound local;
    std::vector<double> gathered(P);
    for (i64 c0 = a; c0 < b; c0 += step) {
      i64 c1 = std::min(b, c0 + step);
      const Bound* geo;
      i64 base;
      if (cached && !sel) { geo = &whole; base = c0; }
      else if (cached) { geo = &whole; base = -1; }
      else { chunk(c0, c1, sel, local); geo = &local; base = 0; }
      for (i64 r = 0; r < R; ++r) {
        const double* xs = x + r * n_in;
        for (int g = 0; g < G; ++g)
          for (i64 i = c0; i < c1; ++i) {
            i64 k = (base < 0) ? (*sel)[i] : (i - c0 + base);
            for (int p = 0; p < P; ++p) {
              double acc = 0.0;
              size_t e = (((size_t)k * G + g) * P + p) * 4;
              for (int n = 0; n < 4; ++n) acc += xs[geo->pos[e + n]] * geo->w[e + n];
              gathered[p] = acc;
            }
            for (int o = 0; o < 2; ++o) {
              double s = 0.0;
              const double* kk = &ker[((size_t)g * 2 + o) * P];
              for (int p = 0; p < P; ++p) s += gathered[p] * kk[p];
              y[((r * G + g) * 2 + o) * K + i] = s;
            }
          }
      }
    }
  });
}

void ConvOp::adjoint_add(const std::vector<double>& ker, const double* gy, i64 R, double* gx,
                         const std::vector<i64>* sel) const {
  i64 K = sel ? (i64)sel->size() : n_rows;
  int P = ksz * ksz;
  int nt = num_threads();
  i64 nw = std::min<i64>(nt, std::max<i64>(K, 1));
  std::vector<std::vector<double>> part(nw);
  parallel_chunks(K, [&](i64 a, i64 b, int w) {
    std::vector<double>& acc = part[w];
    acc.assign((size_t)R * n_in, 0.0);
    const i64 step = 1024;
    Bound local;
    std::vector<double> taps(P);
    for (i64 c0 = a; c0 < b; c0 += step) {
      i64 c1 = std::min(b, c0 + step);
      const Bound* geo;
      i64 base;
      if (cached && !sel) { geo = &whole; base = c0; }
      else if (cached) { geo = &whole; base = -1; }
      else { chunk(c0, c1, sel, local); geo = &local; base = 0; }
      for (i64 r = 0; r < R; ++r) {
        double* dst = acc.data() + r * n_in;
        for (int g = 0; g < G; ++g)
          for (i64 i = c0; i < c1; ++i) {
            i64 k = (base < 0) ? (*sel)[i] : (i - c0 + base);
            double g0 = gy[((r * G + g) * 2 + 0) * K + i], g1 = gy[((r * G + g) * 2 + 1) * K + i];
            const double* k0 = &ker[((size_t)g * 2 + 0) * P];
            const double* k1 = &ker[((size_t)g * 2 + 1) * P];
            for (int p = 0; p < P; ++p) taps[p] = g0 * k0[p] + g1 * k1[p];
            for (int n = 0; n < 4; ++n)
              for (int p = 0; p < P; ++p) {
                size_t e = (((size_t)k * G + g) * P + p) * 4 + n;
                dst[geo->pos[e]] += taps[p] * geo->w[e];
              }
          }
      }
    }
  });
  for (i64 w = 0; w < nw; ++w) {
    if (part[w].empty()) continue;
    const double* s = part[w].data();
    for (size_t i = 0; i < (size_t)R * n_in; ++i) gx[i] += s[i];
  }
}

// ---------------------------------------------------------------------------
// smooth decimation (decimation.rs)
Csr Csr::transpose() const {  // decimation.rs:70-91
  Csr t;
  std::vector<i64> count(n_cols + 1, 0);
  for (i64 c : indices) count[c + 1] += 1;
  for (i64 i = 0; i < n_cols; ++i) count[i + 1] += count[i];
  t.indptr = count;
  std::vector<i64> next = count;
  t.indices.assign(indices.size(), 0);
  t.values.assign(values.size(), 0.0);
  for (i64 r = 0; r < n_rows; ++r)
    for (i64 e = indptr[r]; e < indptr[r + 1]; ++e) {
      i64 c = indices[e];
      t.indices[next[c]] = r;
      t.values[next[c]] = values[e];
      next[c] += 1;
    }
  t.n_rows = n_cols; t.n_cols = n_rows;
  return t;
}

void Csr::apply(const double* x, double* y) const {
  for (i64 r = 0; r < n_rows; ++r) {
    double s = 0.0;
    for (i64 e = indptr[r]; e < indptr[r + 1]; ++e) s += values[e] * x[indices[e]];
    y[r] = s;
  }
}

static inline double haversine(double lat1, double lon1, double lat2, double lon2) {  // decimation.rs:121-128
  double dlat = 0.5 * (lat2 - lat1);
  double dlon = 0.5 * (lon2 - lon1);
  double sa = std::sin(dlat), so = std::sin(dlon);
  double a = std::min(1.0, std::max(0.0, sa * sa + std::cos(lat1) * std::cos(lat2) * (so * so)));
  return 2.0 * std::asin(std::sqrt(a));
}

std::vector<i64> smooth_decimation(const i64* ids, i64 n, i64 nside, Csr& out) {  // decimation.rs:134-201
  const bool full = ids == nullptr;
  if (full) n = npix(nside);
  double pix_deg = std::sqrt(4.0 * PI / (double)npix(nside)) * (180.0 / PI);
  double radius = (3.0 * pix_deg) * (PI / 180.0);
  double sigma = radius / 2.0;
  std::vector<i64> coarse;
  if (full) {
    coarse.resize(npix(nside / 2));
    for (i64 i = 0; i < (i64)coarse.size(); ++i) coarse[i] = i;
  } else {
    std::vector<i64> v(ids, ids + n);
    coarse = parents(v);
  }
  i64 nc = (i64)coarse.size();
  i64 cn = nside / 2;
  std::vector<std::vector<i64>> rcols(nc);
  std::vector<std::vector<double>> rvals(nc);
  parallel_chunks(nc, [&](i64 a, i64 b, int) {
    for (i64 r = a; r < b; ++r) {
      i64 c = coarse[r];
      std::vector<i64> cols;
      if (cn >= 4) {
        for (i64 v : kth_neighbourhood_set(c, cn, 2))
          for (int ch = 0; ch < 4; ++ch) {
            i64 q = search(full ? nullptr : ids, n, 4 * v + ch);
            if (q >= 0) cols.push_back(q);
          }
      } else {
        for (i64 v = 0; v < npix(nside); ++v) {
          i64 q = search(full ? nullptr : ids, n, v);
          if (q >= 0) cols.push_back(q);
        }
      }
      std::sort(cols.begin(), cols.end());
      cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
      double lon_c, lat_c;
      centre_lonlat(c, nside / 2, lon_c, lat_c);
      std::vector<double> w(cols.size());
      for (size_t i = 0; i < cols.size(); ++i) {
        i64 f = full ? cols[i] : ids[cols[i]];
        double lon_f, lat_f;
        centre_lonlat(f, nside, lon_f, lat_f);
        double gamma = haversine(lat_c, lon_c, lat_f, lon_f);
        double t = gamma / sigma;
        w[i] = gamma > radius ? 0.0 : std::exp(-0.5 * (t * t));
      }
      double row_sum = 0.0;
      for (double v : w) row_sum += v;
      if (row_sum <= 0.0 && !w.empty()) {
        double u = 1.0 / (double)w.size();
        for (double& v : w) v = u;
        row_sum = 0.0;
        for (double v : w) row_sum += v;
      }
      double scale = std::max(row_sum, 1e-300);
      for (size_t i = 0; i < cols.size(); ++i) {
        double v = w[i] / scale;
        if (v != 0.0) { rcols[r].push_back(cols[i]); rvals[r].push_back(v); }
      }
    }
  });
  out.n_rows = nc; out.n_cols = n;
  out.indptr.assign(1, 0);
  out.indices.clear(); out.values.clear();
  for (i64 r = 0; r < nc; ++r) {
    out.indices.insert(out.indices.end(), rcols[r].begin(), rcols[r].end());
    out.values.insert(out.values.end(), rvals[r].begin(), rvals[r].end());
    out.indptr.push_back((i64)out.indices.size());
  }
  return coarse;
}

}  // namespace orc
