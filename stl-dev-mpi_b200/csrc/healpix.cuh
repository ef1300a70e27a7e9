// HEALPix primitives in FP64, usable on the host and on the device.
//
// The formulas follow the reference's crates/stl-core/src/healpix.rs
// (NESTED <-> (x, y, face), pixel centres, RING -> NESTED, the bilinear
// interpolation of the HEALPix C++ library), stencil.rs (tangent stencil,
// rotations, gauges) and dia.rs (extended face frames), keeping their
// floating-point operation order.  On the device, the transcendental
// functions are CUDA's, within a few ulps of the host's.
#pragma once
#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define HD __host__ __device__ __forceinline__
#else
#define HD inline
#endif

namespace stl {

typedef int64_t i64;

constexpr double kPi = 3.141592653589793115997963468544185161590576171875;
constexpr double kRad2Deg = 57.295779513082320876798154814105170332405472466564;
constexpr double kDeg2Rad = 0.017453292519943295769236907684886127134428718885417;

HD double rad2deg(double x) { return x * kRad2Deg; }
HD double deg2rad(double x) { return x * kDeg2Rad; }
HD double py_remainder(double a, double b) {  // healpix.rs:33-39
  double m = fmod(a, b);
  if (m != 0.0 && ((b < 0.0) != (m < 0.0))) m += b;
  return m;
}
HD i64 floor_div(i64 a, i64 b) {
  i64 q = a / b;
  if ((a % b) < 0) q -= 1;
  return q;
}
HD int order_of(i64 nside) {
  int o = 0;
  while ((i64(1) << o) < nside) ++o;
  return o;
}
HD i64 npix_of(i64 nside) { return 12 * nside * nside; }

HD i64 jrll(i64 f) { return f < 4 ? 2 : (f < 8 ? 3 : 4); }
HD i64 jpll(i64 f) {
  const int t[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};
  return t[f];
}

HD i64 compress_bits(i64 v) {
  uint64_t u = (uint64_t)v & 0x5555555555555555ULL;
  u = (u | (u >> 1)) & 0x3333333333333333ULL;
  u = (u | (u >> 2)) & 0x0F0F0F0F0F0F0F0FULL;
  u = (u | (u >> 4)) & 0x00FF00FF00FF00FFULL;
  u = (u | (u >> 8)) & 0x0000FFFF0000FFFFULL;
  return (i64)((u | (u >> 16)) & 0x00000000FFFFFFFFULL);
}
HD i64 spread_bits(i64 v) {
  uint64_t u = (uint64_t)v & 0x00000000FFFFFFFFULL;
  u = (u | (u << 16)) & 0x0000FFFF0000FFFFULL;
  u = (u | (u << 8)) & 0x00FF00FF00FF00FFULL;
  u = (u | (u << 4)) & 0x0F0F0F0F0F0F0F0FULL;
  u = (u | (u << 2)) & 0x3333333333333333ULL;
  return (i64)((u | (u << 1)) & 0x5555555555555555ULL);
}

HD void nest2xyf(i64 pix, int order, i64& ix, i64& iy, i64& face) {
  face = pix >> (2 * order);
  i64 local = pix & ((i64(1) << (2 * order)) - 1);
  ix = compress_bits(local);
  iy = compress_bits(local >> 1);
}
HD i64 xyf2nest(i64 ix, i64 iy, i64 face, int order) {
  return (face << (2 * order)) + spread_bits(ix) + (spread_bits(iy) << 1);
}

// colatitude / longitude of a pixel centre (healpix.rs:88-127)
HD void xyf2ang(i64 ix, i64 iy, i64 face, i64 nside, double& theta, double& phi) {
  i64 jr = jrll(face) * nside - ix - iy - 1;
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
    double sth_cap = sqrt(tmp * (2.0 - tmp));
    double theta_cap = atan2(sth_cap, z_cap);
    theta = north ? theta_cap : kPi - theta_cap;
  } else {
    theta = acos((2.0 * ns - (double)jr) * fact1);
  }
  i64 jp = floor_div(jpll(face) * nr + ix - iy + 1 + kshift, 2);
  if (jp > 4 * nr) jp -= 4 * nr;
  if (jp < 1) jp += 4 * nr;
  phi = ((double)jp - ((double)kshift + 1.0) * 0.5) * (0.5 * kPi / nrf);
}

HD void pix2ang_nest(i64 pix, i64 nside, double& theta, double& phi) {
  i64 ix, iy, f;
  nest2xyf(pix, order_of(nside), ix, iy, f);
  xyf2ang(ix, iy, f, nside, theta, phi);
}

// longitude / latitude through degrees (healpix.rs:140-143)
HD void centre_lonlat(i64 pix, i64 nside, double& lon, double& lat) {
  double theta, phi;
  pix2ang_nest(pix, nside, theta, phi);
  lon = deg2rad(rad2deg(phi));
  lat = deg2rad(90.0 - rad2deg(theta));
}

HD i64 isqrt_i64(i64 v) {
  i64 r = (i64)sqrt((double)v);
  if (r * r > v) r -= 1;
  if ((r + 1) * (r + 1) <= v) r += 1;
  return r;
}

HD i64 ring2nest(i64 pix, int order) {  // healpix.rs:157-210
  i64 nside = i64(1) << order;
  i64 np = npix_of(nside);
  i64 ncap = 2 * nside * (nside - 1);
  i64 nl2 = 2 * nside;
  i64 iring, iphi, kshift, nr, face;
  if (pix < ncap) {
    i64 ir = (1 + isqrt_i64(1 + 2 * pix)) >> 1;
    i64 ip = pix + 1 - 2 * ir * (ir - 1);
    iring = ir; iphi = ip; kshift = 0; nr = ir;
    face = floor_div(ip - 1, ir > 1 ? ir : 1);
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
    i64 ir = (1 + isqrt_i64(2 * ip - 1)) >> 1;
    i64 ip2 = 4 * ir + 1 - (ip - 2 * ir * (ir - 1));
    iring = 2 * nl2 - ir; iphi = ip2; kshift = 0; nr = ir;
    face = 8 + floor_div(ip2 - 1, ir > 1 ? ir : 1);
  }
  i64 irt = iring - jrll(face) * nside + 1;
  i64 ipt = 2 * iphi - jpll(face) * nr - kshift - 1;
  if (ipt >= nl2) ipt -= 8 * nside;
  i64 ix = (ipt - irt) >> 1;
  i64 iy = (-ipt - irt) >> 1;
  return xyf2nest(ix, iy, face, order);
}

HD i64 ring_above(double z, i64 nside) {
  double az = fabs(z);
  double ns = (double)nside;
  if (az <= 2.0 / 3.0) return (i64)trunc(ns * (2.0 - 1.5 * z));
  i64 iring = (i64)trunc(ns * sqrt(3.0 * (1.0 - az)));
  return z > 0.0 ? iring : 4 * nside - iring - 1;
}

HD void ring_info(i64 ring, i64 nside, i64& startpix, i64& ringpix, double& theta, bool& shifted) {
  i64 ncap = 2 * nside * (nside - 1);
  i64 np = npix_of(nside);
  double ns = (double)nside;
  double fact1 = 2.0 / (3.0 * ns);
  double fact2 = 1.0 / (3.0 * ns * ns);
  i64 northring = ring > 2 * nside ? 4 * nside - ring : ring;
  if (northring < nside) {
    double nrf = (double)northring;
    double tmp = nrf * nrf * fact2;
    theta = atan2(sqrt(tmp * (2.0 - tmp)), 1.0 - tmp);
    ringpix = 4 * northring;
    shifted = true;
    startpix = 2 * northring * (northring - 1);
  } else {
    theta = acos((double)(2 * nside - northring) * fact1);
    ringpix = 4 * nside;
    shifted = ((northring - nside) & 1) == 0;
    startpix = ncap + (northring - nside) * 4 * nside;
  }
  if (northring != ring) {
    theta = kPi - theta;
    startpix = np - startpix - ringpix;
  }
}

HD void ring_pair(double phi, i64 ring, i64 nside, i64& p0, i64& p1, double& w0, double& w1, double& th) {
  i64 sp, nr;
  bool shifted;
  ring_info(ring, nside, sp, nr, th, shifted);
  double dphi = (2.0 * kPi) / (double)nr;
  double half = shifted ? 0.5 : 0.0;
  double tmp = phi / dphi - half;
  i64 i1 = (i64)trunc(tmp);
  if (tmp < 0.0) i1 -= 1;
  double ww = (phi - ((double)i1 + half) * dphi) / dphi;
  i64 i2 = i1 + 1;
  if (i1 < 0) i1 += nr;
  if (i2 >= nr) i2 -= nr;
  p0 = sp + i1; p1 = sp + i2; w0 = 1.0 - ww; w1 = ww;
}

// four RING pixels and weights of a direction (healpix.rs:283-324)
HD void get_interpol_ring(double theta, double phi, i64 nside, i64 out_pix[4], double out_w[4]) {
  i64 np = npix_of(nside);
  double z = cos(theta);
  i64 ir1 = ring_above(z, nside);
  i64 ir2 = ir1 + 1;
  i64 pix[4] = {0, 0, 0, 0};
  double wgt[4] = {0, 0, 0, 0};
  i64 p0, p1, p2, p3;
  double w0, w1, w2, w3, theta1, theta2;
  ring_pair(phi, ir1 > 1 ? ir1 : 1, nside, p0, p1, w0, w1, theta1);
  if (ir1 > 0) { pix[0] = p0; pix[1] = p1; wgt[0] = w0; wgt[1] = w1; }
  ring_pair(phi, ir2 < 4 * nside - 1 ? ir2 : 4 * nside - 1, nside, p2, p3, w2, w3, theta2);
  if (ir2 < 4 * nside) { pix[2] = p2; pix[3] = p3; wgt[2] = w2; wgt[3] = w3; }
  bool north = ir1 == 0;
  bool south = ir2 == 4 * nside && !north;
  if (north) {
    double wn = theta / theta2;
    double facn = (1.0 - wn) * 0.25;
    out_pix[0] = (pix[2] + 2) & 3; out_pix[1] = (pix[3] + 2) & 3; out_pix[2] = pix[2]; out_pix[3] = pix[3];
    out_w[0] = facn; out_w[1] = facn; out_w[2] = wgt[2] * wn + facn; out_w[3] = wgt[3] * wn + facn;
  } else if (south) {
    double ws = (theta - theta1) / (kPi - theta1);
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

// four NESTED pixels and weights of a direction, through degrees (healpix.rs:336-347)
HD void interp_weights_nested(const double v[3], int order, i64 pix[4], double w[4]) {
  double nrm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double n = nrm > 1e-12 ? nrm : 1e-12;
  double vn[3] = {v[0] / n, v[1] / n, v[2] / n};
  double c = vn[2] < -1.0 ? -1.0 : (vn[2] > 1.0 ? 1.0 : vn[2]);
  double theta = acos(c);
  double phi = py_remainder(atan2(vn[1], vn[0]), 2.0 * kPi);
  double lon_deg = rad2deg(phi);
  double lat_deg = 90.0 - rad2deg(theta);
  double theta2 = deg2rad(90.0 - lat_deg);
  double phi2 = py_remainder(deg2rad(lon_deg), 2.0 * kPi);
  i64 rp[4];
  get_interpol_ring(theta2, phi2, i64(1) << order, rp, w);
  for (int i = 0; i < 4; ++i) pix[i] = ring2nest(rp[i], order);
}

// Rotation of gauge g taking the north-pole stencil to (theta, phi)
// (stencil.rs:51-88); gauge 0 = cosmo, 1 = phi.  Row-major 3 x 3.
HD void rotation_matrix(double theta, double phi, int g, int G, int gauge, double out[9]) {
  double ct = cos(theta), st = sin(theta), cp = cos(phi), sp = sin(phi);
  double base[9] = {cp * ct, -sp, cp * st, sp * ct, cp, sp * st, -st, 0.0, ct};
  double n0[3] = {base[2], base[5], base[8]};
  double nn0 = sqrt(n0[0] * n0[0] + n0[1] * n0[1] + n0[2] * n0[2]);
  double nn = nn0 > 1e-12 ? nn0 : 1e-12;
  double n[3] = {n0[0] / nn, n0[1] / nn, n0[2] / nn};
  double alpha_base, sign_g;
  if (gauge == 0) {
    if (theta > kPi / 2.0) { alpha_base = phi; sign_g = -1.0; } else { alpha_base = -phi; sign_g = 1.0; }
  } else { alpha_base = 0.0; sign_g = 1.0; }
  double skew[9] = {0.0, -n[2], n[1], n[2], 0.0, -n[0], -n[1], n[0], 0.0};
  double step = kPi / (double)G;
  double alpha = alpha_base + sign_g * ((double)g * step);
  double ca = cos(alpha), sa = sin(alpha);
  double rg[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double eye = (i == j) ? 1.0 : 0.0;
      rg[3 * i + j] = eye * ca + skew[3 * i + j] * sa + n[i] * n[j] * (1.0 - ca);
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      out[3 * i + j] = rg[3 * i] * base[j] + rg[3 * i + 1] * base[3 + j] + rg[3 * i + 2] * base[6 + j];
}

// pixel at the extended coordinates (ex, ey) of `face` (dia.rs:46-77);
// false in the quadrant missing at a vertex of three faces
HD bool ext_pix(i64 face, i64 ex, i64 ey, i64 nside, int order, i64& out) {
  const signed char NB_FACE[9][12] = {
      {8, 9, 10, 11, -1, -1, -1, -1, 10, 11, 8, 9}, {5, 6, 7, 4, 8, 9, 10, 11, 9, 10, 11, 8},
      {-1, -1, -1, -1, 5, 6, 7, 4, -1, -1, -1, -1}, {4, 5, 6, 7, 11, 8, 9, 10, 11, 8, 9, 10},
      {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},       {1, 2, 3, 0, 0, 1, 2, 3, 5, 6, 7, 4},
      {-1, -1, -1, -1, 7, 4, 5, 6, -1, -1, -1, -1}, {3, 0, 1, 2, 3, 0, 1, 2, 4, 5, 6, 7},
      {2, 3, 0, 1, -1, -1, -1, -1, 0, 1, 2, 3}};
  const unsigned char NB_SWAP[9][3] = {{0, 0, 3}, {0, 0, 6}, {0, 0, 0}, {0, 0, 5}, {0, 0, 0},
                                       {5, 0, 0}, {0, 0, 0}, {6, 0, 0}, {3, 0, 0}};
  i64 x = ex, y = ey;
  int nb = 4;
  if (x < 0) { x += nside; nb -= 1; } else if (x >= nside) { x -= nside; nb += 1; }
  if (y < 0) { y += nside; nb -= 3; } else if (y >= nside) { y -= nside; nb += 3; }
  int f = NB_FACE[nb][face];
  if (f < 0) return false;
  int bits = NB_SWAP[nb][face >> 2];
  if (bits & 1) x = nside - x - 1;
  if (bits & 2) y = nside - y - 1;
  if (bits & 4) { i64 t = x; x = y; y = t; }
  out = xyf2nest(x, y, f, order);
  return true;
}

}  // namespace stl
