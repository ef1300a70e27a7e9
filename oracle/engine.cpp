// CPU FP64 restatement of the reference's ScatCov engine (full sky).
// TEST INFRASTRUCTURE ONLY (see engine.hpp).
#include "engine.hpp"

#include <set>
#include <stdexcept>

namespace orc {

std::vector<Coef> build_plan(int J, int L, const std::vector<int>& dg, int C, bool cross_only) {
  // crates/stl-core/src/plan.rs:80-158 (all families, every pair crossed)
  std::vector<Coef> plan;
  auto mk = [](int fam, int nat, int c1, int c2) { return Coef{fam, nat, c1, c2, -1, -1, -1, -1, -1, -1}; };
  for (int fam : {MEAN, VAR})
    for (int c = 0; c < C; ++c) plan.push_back(mk(fam, 0, c, c));
  for (int j3 = 0; j3 < J; ++j3) {
    int d = dg[j3];
    for (int c1 = 0; c1 < C; ++c1)
      for (int c2 = c1; c2 < C; ++c2) {
        for (int fam : {S1, S2})
          for (int l = 0; l < L; ++l) {
            Coef c = mk(fam, d, c1, c2);
            c.j1 = j3; c.l1 = l;
            plan.push_back(c);
          }
        std::vector<std::pair<int, int>> pairs = {{c1, c2}};
        if (c1 != c2) pairs.push_back({c2, c1});
        for (auto [ca, cb] : pairs)
          for (int j2 = 0; j2 <= j3; ++j2) {
            for (int l2 = 0; l2 < L; ++l2)
              for (int l3 = 0; l3 < L; ++l3) {
                Coef c = mk(S3, d, ca, cb);
                c.j1 = j2; c.j3 = j3; c.l1 = l2; c.l3 = l3;
                plan.push_back(c);
              }
            for (int j1 = 0; j1 <= j2; ++j1)
              for (int l1 = 0; l1 < L; ++l1)
                for (int l2 = 0; l2 < L; ++l2)
                  for (int l3 = 0; l3 < L; ++l3) {
                    Coef c = mk(S4, d, ca, cb);
                    c.j1 = j1; c.j2 = j2; c.j3 = j3; c.l1 = l1; c.l2 = l2; c.l3 = l3;
                    plan.push_back(c);
                  }
          }
      }
  }
  std::stable_sort(plan.begin(), plan.end(), [](const Coef& a, const Coef& b) { return a.native < b.native; });
  if (cross_only) {
    std::vector<Coef> out;
    for (auto& c : plan)
      if (c.c1 != c.c2) out.push_back(c);
    return out;
  }
  return plan;
}

void Engine::init(i64 nside, int J_, int L_, int ksz_, Gauge gauge_, int B_, int C_, bool fewer_,
                  const std::vector<int>& dg, bool cross_only, size_t cache_budget) {
  nside0 = nside; J = J_; L = L_; ksz = ksz_; gauge = gauge_; B = B_; C = C_; fewer = fewer_;
  j_to_dg = dg;
  if ((int)j_to_dg.size() != J) {
    j_to_dg.resize(J);
    for (int j = 0; j < J; ++j) j_to_dg[j] = j;
  }
  levels = 1 + *std::max_element(j_to_dg.begin(), j_to_dg.end());
  if ((nside0 >> (levels - 1)) < 1) throw std::runtime_error("too many levels for nside");
  int P = ksz * ksz;
  ker = shared_kernel(wavelet_weights(ksz), L, P);
  plan = build_plan(J, L, j_to_dg, C, cross_only);
  conv.resize(levels);
  size_t per_level = cache_budget / (size_t)levels;
  for (int n = 0; n < levels; ++n) conv[n].init({}, {}, nside0 >> n, ksz, L, gauge, 0.0, per_level);
  down.resize(levels > 0 ? levels - 1 : 0);
  downT.resize(down.size());
  for (int d = 0; d + 1 < levels; ++d) {
    smooth_decimation(nullptr, 0, nside0 >> d, down[d]);
    downT[d] = down[d].transpose();
  }
}

void Engine::set_masks(const double* w0, i64 Kc) {  // mask.rs:203-228
  if (Kc <= 0) { has_masks = false; masks = Masks(); return; }
  masks = Masks();
  i64 n0 = npix(0);
  for (i64 k = 0; k < Kc; ++k) {
    std::vector<double> level(n0);
    for (i64 i = 0; i < n0; ++i) level[i] = w0[k * n0 + i] != 0.0 ? 1.0 : 0.0;
    std::vector<std::vector<double>> per;
    std::vector<i64> cnt;
    for (int n = 0; n < levels; ++n) {
      if (n > 0) {
        std::vector<double> next(level.size() / 4);
        for (size_t i = 0; i < next.size(); ++i)
          next[i] = (level[4 * i] != 0 || level[4 * i + 1] != 0 || level[4 * i + 2] != 0 || level[4 * i + 3] != 0) ? 1.0 : 0.0;
        level = next;
      }
      i64 c = 0;
      for (double v : level) c += v != 0.0;
      if (c == 0) throw std::runtime_error("empty mask");
      cnt.push_back(c);
      per.push_back(level);
    }
    masks.weights.push_back(per);
    masks.counts.push_back(cnt);
  }
  has_masks = true;
}

void Engine::set_mask_levels(const double* w, i64 Kc) {  // mask.rs:75-82
  if (Kc <= 0) { has_masks = false; masks = Masks(); return; }
  masks = Masks();
  for (i64 k = 0; k < Kc; ++k) {
    std::vector<std::vector<double>> per;
    std::vector<i64> cnt;
    for (int n = 0; n < levels; ++n) {
      std::vector<double> level(npix(n));
      i64 c = 0;
      for (i64 i = 0; i < npix(n); ++i) {
        level[i] = w[i] != 0.0 ? 1.0 : 0.0;
        c += w[i] != 0.0;
      }
      w += npix(n);
      if (c == 0) throw std::runtime_error("empty mask at some level");
      cnt.push_back(c);
      per.push_back(level);
    }
    masks.weights.push_back(per);
    masks.counts.push_back(cnt);
  }
  has_masks = true;
}

std::vector<double> Engine::decimate(int d, const std::vector<double>& x, i64 rows) const {
  i64 n = down[d].n_cols, nc = down[d].n_rows;
  std::vector<double> y((size_t)rows * nc);
  parallel_chunks(rows, [&](i64 a, i64 b, int) {
    for (i64 r = a; r < b; ++r) down[d].apply(x.data() + r * n, y.data() + r * nc);
  });
  return y;
}

std::vector<double> Engine::decimate_adjoint(int d, const std::vector<double>& g, i64 rows) const {
  i64 n = down[d].n_cols, nc = down[d].n_rows;
  std::vector<double> y((size_t)rows * n);
  parallel_chunks(rows, [&](i64 a, i64 b, int) {
    for (i64 r = a; r < b; ++r) downT[d].apply(g.data() + r * nc, y.data() + r * n);
  });
  return y;
}

void Engine::load(const double* x) {  // engine.rs:337-347 and decimate_levels
  i64 bc = (i64)B * C;
  maps.assign(1, std::vector<double>(x, x + bc * npix(0)));
  for (int d = 0; d + 1 < levels; ++d) maps.push_back(decimate(d, maps[d], bc));
  z.clear(); m.clear(); br.clear();
}

void Engine::load_levels(const double* x) {  // engine.rs:354-369
  i64 bc = (i64)B * C;
  maps.clear();
  for (int d = 0; d < levels; ++d) {
    maps.emplace_back(x, x + bc * npix(d));
    x += bc * npix(d);
  }
  z.clear(); m.clear(); br.clear();
}

static inline double normc(cplx v) { return std::hypot(v.real(), v.imag()); }
static inline cplx cmul(cplx a, cplx b) {  // num-complex Mul
  return cplx(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}
static inline cplx cconj(cplx a) { return cplx(a.real(), -a.imag()); }
static inline cplx cdivr(cplx a, double r) { return cplx(a.real() / r, a.imag() / r); }
static inline cplx rmulc(double r, cplx a) { return cplx(r * a.real(), r * a.imag()); }
static inline cplx root_normalise(cplx z) { return cdivr(z, std::sqrt(normc(z) + 1e-8)); }  // engine.rs:41-43

// Operands [B][N_n] of a coefficient (engine.rs:956-984, on the whole level)
struct Operands {
  std::vector<cplx> a, b;
};

static void operands(const Engine& e, const Coef& c, Operands& op) {
  int n = c.native;
  i64 N = e.npix(n);
  int L = e.L, C = e.C;
  op.a.assign((size_t)e.B * N, cplx(0, 0));
  op.b.clear();
  auto z_core = [&](std::vector<cplx>& out, int ch, int ang) {
    out.resize((size_t)e.B * N);
    for (int b = 0; b < e.B; ++b)
      for (i64 p = 0; p < N; ++p) out[b * N + p] = e.z[n][(((size_t)b * C + ch) * L + ang) * N + p];
  };
  auto map_core = [&](std::vector<cplx>& out, int level, int ch) {
    i64 Nl = e.npix(level);
    out.resize((size_t)e.B * N);
    for (int b = 0; b < e.B; ++b)
      for (i64 p = 0; p < N; ++p) out[b * N + p] = cplx(e.maps[level][((size_t)b * C + ch) * Nl + p], 0.0);
  };
  auto branch_core = [&](std::vector<cplx>& out, int d, int ch, int l1, int l3) {
    const auto& v = e.br.at({d, n});
    out.resize((size_t)e.B * N);
    for (int b = 0; b < e.B; ++b)
      for (i64 p = 0; p < N; ++p) out[b * N + p] = v[((((size_t)b * C + ch) * L + l1) * L + l3) * N + p];
  };
  auto modulus_core = [&](std::vector<cplx>& out, int d, int ch, int l1) {
    const auto& v = e.m.at({d, n});
    out.resize((size_t)e.B * N);
    for (int b = 0; b < e.B; ++b)
      for (i64 p = 0; p < N; ++p) out[b * N + p] = cplx(v[(((size_t)b * C + ch) * L + l1) * N + p], 0.0);
  };
  const auto& dg = e.j_to_dg;
  switch (c.family) {
    case MEAN:
    case VAR: map_core(op.a, 0, c.c1); break;
    case S1:
    case S2: z_core(op.a, c.c1, c.l1); z_core(op.b, c.c2, c.l1); break;
    case S3:
      if (!e.fewer) { branch_core(op.a, dg[c.j1], c.c1, c.l1, c.l3); z_core(op.b, c.c2, c.l3); }
      else { map_core(op.a, n, c.c1); branch_core(op.b, dg[c.j1], c.c2, c.l1, c.l3); }
      break;
    case S4:
      if (e.fewer) modulus_core(op.a, dg[c.j1], c.c1, c.l1);
      else branch_core(op.a, dg[c.j1], c.c1, c.l1, c.l3);
      branch_core(op.b, dg[c.j2], c.c2, c.l2, c.l3);
      break;
  }
}

// term f_p of a coefficient (engine.rs:1194-1215)
static inline cplx term(const Coef& c, cplx a, cplx b) {
  switch (c.family) {
    case MEAN: return a;
    case VAR: { double r = normc(a); return cplx(r * r, 0.0); }
    case S2:
      if (c.c1 == c.c2) { double r = normc(a); return cplx(r * r, 0.0); }
      return cmul(a, cconj(b));
    case S1:
      if (c.c1 == c.c2) return cplx(normc(a), 0.0);
      return cmul(root_normalise(a), cconj(root_normalise(b)));
    default: return cmul(a, cconj(b));
  }
}

// |f_p|^2 of the terms whose mean is the coefficient (engine.rs:1219-1240)
static inline double term_second(const Coef& c, cplx a, cplx b) {
  switch (c.family) {
    case MEAN: return std::norm(a);
    case VAR: { double r = normc(a); double s = r * r; return s * s; }
    case S2:
      if (c.c1 == c.c2) { double r = normc(a); double s = r * r; return s * s; }
      return std::norm(cmul(a, cconj(b)));
    case S1:
      if (c.c1 == c.c2) return std::norm(a);
      return std::norm(cmul(root_normalise(a), cconj(root_normalise(b))));
    default: return std::norm(cmul(a, cconj(b)));
  }
}

void Engine::forward(std::vector<cplx>& values, std::vector<double>* second) {
  int Kc = K();
  i64 np = (i64)plan.size();
  i64 bc = (i64)B * C;
  values.assign((size_t)B * Kc * np, cplx(0, 0));
  if (second) second->assign((size_t)B * Kc * np, 0.0);
  z.assign(levels, {});
  m.clear(); br.clear();
  std::vector<std::set<int>> need(levels);
  for (auto& c : plan) {
    if (c.family == S3) need[c.native].insert(j_to_dg[c.j1]);
    if (c.family == S4) {
      if (!fewer) need[c.native].insert(j_to_dg[c.j1]);
      need[c.native].insert(j_to_dg[c.j2]);
    }
  }
  for (int n = 0; n < levels; ++n) {
    i64 N = npix(n);
    std::vector<double> y((size_t)bc * L * 2 * N);
    conv[n].forward(ker, maps[n].data(), bc, y.data());
    auto& zn = z[n];
    zn.resize((size_t)bc * L * N);
    std::vector<double> mod((size_t)bc * L * N);
    for (i64 r = 0; r < bc * L; ++r)
      for (i64 p = 0; p < N; ++p) {
        cplx v(y[(r * 2 + 0) * N + p], y[(r * 2 + 1) * N + p]);
        zn[r * N + p] = v;
        mod[r * N + p] = normc(v);
      }
    m[{n, n}] = mod;
    for (int d = 0; d < n; ++d) m[{d, n}] = decimate(n - 1, m.at({d, n - 1}), bc * L);
    for (int d : need[n]) {
      const auto& src = m.at({d, n});
      std::vector<double> yb((size_t)bc * L * L * 2 * N);
      conv[n].forward(ker, src.data(), bc * L, yb.data());
      std::vector<cplx> v((size_t)bc * L * L * N);
      for (i64 r = 0; r < bc * L * L; ++r)
        for (i64 p = 0; p < N; ++p) v[r * N + p] = cplx(yb[(r * 2 + 0) * N + p], yb[(r * 2 + 1) * N + p]);
      br[{d, n}] = std::move(v);
    }
    // coefficient sums native at level n
    std::vector<i64> idx;
    for (i64 i = 0; i < np; ++i)
      if (plan[i].native == n) idx.push_back(i);
    parallel_chunks((i64)idx.size(), [&](i64 a0, i64 a1, int) {
      Operands op;
      for (i64 t = a0; t < a1; ++t) {
        i64 i = idx[t];
        const Coef& c = plan[i];
        operands(*this, c, op);
        for (int b = 0; b < B; ++b)
          for (int k = 0; k < Kc; ++k) {
            const double* w = has_masks ? masks.weights[k][n].data() : nullptr;
            double total = has_masks ? (double)masks.counts[k][n] : (double)N;
            double sr = 0.0, si = 0.0, s2 = 0.0;
            for (i64 p = 0; p < N; ++p) {
              if (w && w[p] == 0.0) continue;
              cplx av = op.a[b * N + p];
              cplx bv = op.b.empty() ? cplx(0, 0) : op.b[b * N + p];
              cplx f = term(c, av, bv);
              sr += f.real(); si += f.imag();
              if (second) s2 += term_second(c, av, bv);
            }
            values[((size_t)b * Kc + k) * np + i] = cplx(sr / total, si / total);
            if (second) (*second)[((size_t)b * Kc + k) * np + i] = s2 / total;
          }
      }
    });
  }
}

// modulus VJP (local.rs:289-298)
static inline cplx modvjp(cplx v, double g) {
  double mag = normc(v);
  return cdivr(rmulc(g, v), mag == 0.0 ? 1.0 : mag);
}
// root_modulus_vjp (engine.rs:46-56)
static inline cplx root_modvjp(cplx v, cplx g) {
  double r = normc(v);
  double radial = cmul(cconj(g), v).real();
  double mag = r == 0.0 ? 1.0 : r;
  cplx t1 = cdivr(g, std::sqrt(r + 1e-8));
  cplx t2 = cdivr(rmulc(0.5 * radial / std::pow(r + 1e-8, 1.5), v), mag);
  return t1 - t2;
}

std::vector<std::vector<double>> Engine::reverse(const std::vector<cplx>& cot) {
  int Kc = K();
  i64 np = (i64)plan.size();
  i64 bc = (i64)B * C;
  if ((i64)cot.size() != (i64)B * Kc * np) throw std::runtime_error("cotangent shape mismatch");
  std::vector<bool> active(np, false);
  for (i64 i = 0; i < np; ++i)
    for (i64 r = 0; r < (i64)B * Kc; ++r)
      if (cot[r * np + i] != cplx(0, 0)) active[i] = true;
  std::vector<std::vector<double>> mg(levels);
  for (int d = 0; d < levels; ++d) mg[d].assign((size_t)bc * npix(d), 0.0);
  std::map<int, std::vector<double>> gmod_next;  // cotangents of m[d][n + 1], d <= n
  const auto& dg = j_to_dg;
  for (int n = levels - 1; n >= 0; --n) {
    i64 N = npix(n);
    std::map<int, std::vector<double>> gmod;  // cotangents of m[d][n], d <= n
    for (auto& kv : gmod_next) gmod[kv.first] = decimate_adjoint(n, kv.second, bc * L);
    std::vector<cplx> gz((size_t)bc * L * N, cplx(0, 0));
    bool gz_any = false;
    std::map<int, std::vector<cplx>> gbr;
    auto add_z = [&](int ch, int ang, int b, const std::vector<cplx>& v) {
      cplx* row = &gz[(((size_t)b * C + ch) * L + ang) * N];
      for (i64 p = 0; p < N; ++p) row[p] += v[p];
      gz_any = true;
    };
    auto add_branch = [&](int d, int ch, int l1, int l3, int b, const std::vector<cplx>& v) {
      auto& slot = gbr[d];
      if (slot.empty()) slot.assign((size_t)bc * L * L * N, cplx(0, 0));
      cplx* row = &slot[((((size_t)b * C + ch) * L + l1) * L + l3) * N];
      for (i64 p = 0; p < N; ++p) row[p] += v[p];
    };
    auto add_map = [&](int level, int ch, int b, const std::vector<cplx>& v) {
      i64 Nl = npix(level);
      double* row = &mg[level][((size_t)b * C + ch) * Nl];
      for (i64 p = 0; p < N; ++p) row[p] += v[p].real();
    };
    auto add_mod = [&](int d, int ch, int l1, int b, const std::vector<cplx>& v) {
      auto& slot = gmod[d];
      if (slot.empty()) slot.assign((size_t)bc * L * N, 0.0);
      double* row = &slot[(((size_t)b * C + ch) * L + l1) * N];
      for (i64 p = 0; p < N; ++p) row[p] += v[p].real();
    };
    Operands op;
    std::vector<cplx> ga(N), gb(N);
    for (i64 i = 0; i < np; ++i) {
      const Coef& c = plan[i];
      if (c.native != n || !active[i]) continue;
      operands(*this, c, op);
      for (int b = 0; b < B; ++b) {
        std::fill(ga.begin(), ga.end(), cplx(0, 0));
        std::fill(gb.begin(), gb.end(), cplx(0, 0));
        bool any = false;
        for (int k = 0; k < Kc; ++k) {
          cplx g = cot[((size_t)b * Kc + k) * np + i];
          if (g == cplx(0, 0)) continue;
          any = true;
          const double* w = has_masks ? masks.weights[k][n].data() : nullptr;
          double nt = has_masks ? (double)masks.counts[k][n] : (double)N;
          for (i64 p = 0; p < N; ++p) {  // operand_cotangents (engine.rs:1247-1277)
            if (w && w[p] == 0.0) continue;
            cplx a = op.a[b * N + p];
            cplx bv = op.b.empty() ? cplx(0, 0) : op.b[b * N + p];
            switch (c.family) {
              case MEAN: ga[p] += cplx(g.real() / nt, 0.0); break;
              case VAR: ga[p] += cplx(2.0 * g.real() * a.real() / nt, 0.0); break;
              case S1:
                if (c.c1 == c.c2) { ga[p] += modvjp(a, g.real() / nt); break; }
                ga[p] += root_modvjp(a, cdivr(cmul(g, root_normalise(bv)), nt));
                gb[p] += root_modvjp(bv, cdivr(cmul(cconj(g), root_normalise(a)), nt));
                break;
              case S2:
                if (c.c1 == c.c2) { ga[p] += cdivr(rmulc(2.0 * g.real(), a), nt); break; }
                ga[p] += cdivr(cmul(g, bv), nt);
                gb[p] += cdivr(cmul(cconj(g), a), nt);
                break;
              default:
                ga[p] += cdivr(cmul(g, bv), nt);
                gb[p] += cdivr(cmul(cconj(g), a), nt);
            }
          }
        }
        if (!any) continue;
        // apply_cotangents (engine.rs:1077-1113)
        switch (c.family) {
          case MEAN:
          case VAR: add_map(0, c.c1, b, ga); break;
          case S1:
          case S2:
            add_z(c.c1, c.l1, b, ga);
            if (c.c1 != c.c2) add_z(c.c2, c.l1, b, gb);
            break;
          case S3:
            if (fewer) { add_map(n, c.c1, b, ga); add_branch(dg[c.j1], c.c2, c.l1, c.l3, b, gb); }
            else { add_branch(dg[c.j1], c.c1, c.l1, c.l3, b, ga); add_z(c.c2, c.l3, b, gb); }
            break;
          case S4:
            if (fewer) add_mod(dg[c.j1], c.c1, c.l1, b, ga);
            else add_branch(dg[c.j1], c.c1, c.l1, c.l3, b, ga);
            add_branch(dg[c.j2], c.c2, c.l2, c.l3, b, gb);
            break;
        }
      }
    }
    // second-wavelet cotangents -> modulus cotangents (engine.rs:1121-1129)
    for (auto& kv : gbr) {
      int d = kv.first;
      std::vector<double> gy((size_t)bc * L * L * 2 * N);
      for (i64 r = 0; r < bc * L * L; ++r)
        for (i64 p = 0; p < N; ++p) {
          gy[(r * 2 + 0) * N + p] = kv.second[r * N + p].real();
          gy[(r * 2 + 1) * N + p] = kv.second[r * N + p].imag();
        }
      auto& slot = gmod[d];
      if (slot.empty()) slot.assign((size_t)bc * L * N, 0.0);
      conv[n].adjoint_add(ker, gy.data(), bc * L, slot.data());
    }
    // own modulus -> z (engine.rs:1131-1167)
    auto it = gmod.find(n);
    if (it != gmod.end()) {
      for (size_t q = 0; q < gz.size(); ++q) gz[q] += modvjp(z[n][q], it->second[q]);
      gz_any = true;
      gmod.erase(it);
    }
    // wavelet adjoint -> map cotangent of level n
    if (gz_any) {
      std::vector<double> gy((size_t)bc * L * 2 * N);
      for (i64 r = 0; r < bc * L; ++r)
        for (i64 p = 0; p < N; ++p) {
          gy[(r * 2 + 0) * N + p] = gz[r * N + p].real();
          gy[(r * 2 + 1) * N + p] = gz[r * N + p].imag();
        }
      conv[n].adjoint_add(ker, gy.data(), bc, mg[n].data());
    }
    gmod_next = std::move(gmod);
    if (n == 0) gmod_next.clear();
  }
  return mg;
}

void Engine::analysis_vjp(std::vector<std::vector<double>> mg, std::vector<double>& g0,
                          std::vector<std::vector<double>>& bands) {  // engine.rs:730-779
  i64 bc = (i64)B * C;
  for (int d = levels - 1; d >= 1; --d) {
    auto back = decimate_adjoint(d - 1, mg[d], bc);
    for (size_t i = 0; i < back.size(); ++i) mg[d - 1][i] += back[i];
  }
  g0 = mg[0];
  bands.assign(1, g0);
  for (int d = 0; d + 1 < levels; ++d) {
    const auto& fine = bands.back();
    i64 nf = npix(d), ncs = npix(d + 1);
    std::vector<double> coarse((size_t)bc * ncs, 0.0);
    for (i64 r = 0; r < bc; ++r)
      for (i64 p = 0; p < nf; ++p) coarse[r * ncs + p / 4] += fine[r * nf + p];
    bands.push_back(coarse);
  }
}

}  // namespace orc
