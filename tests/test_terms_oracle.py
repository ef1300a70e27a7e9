"""The oracle of the synthesis objective terms (oracle/terms.py) against
independent restatements, on the CPU.

The reference checks its device terms against host expressions written as
loops (crates/stl-gpu/tests/terms.rs:45-186): the sort as a sort by value in
f64 total order then by position, the 4-children pyramid, its detail
moments, the level-power and kurtosis gradients (with and without the chain
factor) and the marginal term.  Here the vectorised oracle meets the same
loops in plain Python (small sizes), on inputs built like the reference's
(heavy tails, ties, signed zeros, subnormals and extremes), with the same
bars: the gradients and the sort exact, the moments and losses to 1e-13.
The kappa table is checked against scipy's cubic Hermite spline.
"""
from __future__ import annotations

import struct
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import terms as T  # noqa: E402


def noise(seed: int, n: int) -> np.ndarray:
    """xorshift64 uniform values in [-0.5, 0.5) (the reference tests' generator)."""
    state = (seed | 1) & 0xFFFFFFFFFFFFFFFF
    out = np.empty(n)
    for i in range(n):
        state ^= (state << 13) & 0xFFFFFFFFFFFFFFFF
        state ^= state >> 7
        state ^= (state << 17) & 0xFFFFFFFFFFFFFFFF
        out[i] = (state >> 11) / float(1 << 53) - 0.5
    return out


def field(seed: int, n: int) -> np.ndarray:
    """Heavy-tailed values with ties, signed zeros and a few extremes."""
    v = noise(seed, n)
    out = v * v * v * 40.0 + np.where(np.arange(n) % 1013 == 0, 9.0, 0.0)
    special = {0: 0.0, 1: -0.0, 2: 0.25, 3: -1e300, 4: 1e-310}
    for i in range(n):
        r = i % 97
        if r in special:
            out[i] = special[r]
    return out


def total_key(v: float) -> int:
    b = struct.unpack("<Q", struct.pack("<d", v))[0]
    return (~b) & 0xFFFFFFFFFFFFFFFF if b >> 63 else b | (1 << 63)


@pytest.mark.parametrize("n", [1, 7, 2047, 2048, 2049, 30001])
def test_sort_is_total_order_then_position(n):
    x = field(n + 3, n)
    want = sorted(range(n), key=lambda i: (total_key(float(x[i])), i))
    assert T.sort_positions(x).tolist() == want


def test_sort_orders_nans_and_zeros():
    x = np.array([np.nan, np.copysign(np.nan, -1.0), 0.0, -0.0, np.inf, -np.inf, 1.0, -1.0, 0.0])
    order = T.sort_positions(x).tolist()
    # -NaN, -inf, -1, -0, +0 (positions 2 then 8), 1, inf, +NaN
    assert order == [1, 5, 7, 3, 2, 8, 6, 4, 0]


def host_pyramid(row, levels):
    """Details and sum of squares per level as the reference's host loop."""
    cur = list(row)
    out = []
    for _ in range(levels):
        parents = []
        for k in range(0, len(cur), 4):
            s = 0.0
            for v in cur[k:k + 4]:
                s += v
            parents.append(s / 4.0)
        d = [cur[i] - parents[i // 4] for i in range(len(cur))]
        s2 = 0.0
        for v in d:
            s2 += v * v
        out.append((d, s2))
        cur = parents
    return out


def test_pyramid_terms_match_host_loops():
    rows, depth = 2, 4
    n = 4 ** 5
    x = np.stack([np.clip(field(11 + r, n), -50.0, 50.0) for r in range(rows)])
    dk = 1.0 + noise(5, rows * n).reshape(rows, n)
    g0 = noise(9, rows * n).reshape(rows, n)
    lv = T.pyramid(x, depth)
    host = [host_pyramid(x[r].tolist(), depth) for r in range(rows)]

    mom = T.detail_moments(lv)
    for r in range(rows):
        for m in range(depth):
            d, s2 = host[r][m]
            s4 = 0.0
            for v in d:
                s4 += v * v * v * v
            assert abs(mom[r, m, 0] - s2) <= 1e-13 * s2
            assert abs(mom[r, m, 1] - s4) <= 1e-13 * s4

    coef = np.array([[0.3 + 0.01 * (r * depth + m) for m in range(depth)] for r in range(rows)])
    got = T.level_power_grad(lv, coef, g0)
    for r in range(rows):
        for i in range(0, n, 37):
            acc = 0.0
            for m in range(depth):
                acc += coef[r, m] * host[r][m][0][i >> (2 * m)]
            assert got[r, i] == g0[r, i] + acc

    lev = [0, 2, 3]
    cf = np.array([[[0.7 - 0.05 * k, 3.0 + 0.1 * k, 0.2 + 0.01 * k] for k in range(r * 3, r * 3 + 3)]
                   for r in range(rows)])
    for chain in (False, True):
        got = T.kurtosis_grad(lv, lev, cf, g0, dk if chain else None)
        for r in range(rows):
            for i in range(0, n, 29):
                acc = 0.0
                for t, m in enumerate(lev):
                    d = host[r][m][0]
                    j = i >> (2 * m)
                    sib = d[j & ~3:(j & ~3) + 4]
                    c = 0.0
                    for v in sib:
                        c += v * v * v
                    c /= 4.0
                    co, kn, vv = cf[r, t]
                    acc += co * (d[j] * d[j] * d[j] - c - kn * vv * d[j])
                want = g0[r, i] + acc * dk[r, i] if chain else g0[r, i] + acc
                assert got[r, i] == want

    want = g0 + x * dk
    assert np.array_equal(T.add_product(g0, x, dk), want)
    assert np.array_equal(T.add_product(g0, x), g0 + x)


def test_pyramid_rejects_misaligned_rows():
    with pytest.raises(ValueError):
        T.pyramid(np.zeros((1, 40)), 2)
    lv = T.pyramid(np.zeros((1, 64)), 2)
    with pytest.raises(ValueError):
        T.level_power_grad(lv, np.zeros((1, 3)), np.zeros((1, 64)))
    with pytest.raises(ValueError):
        T.kurtosis_grad(lv, [2], np.zeros((1, 1, 3)), np.zeros((1, 64)))


def test_marginal_matches_host_loop():
    n = 2003
    x = field(21, n)
    f = field(22, n)
    t = f[np.array(sorted(range(n), key=lambda i: (total_key(float(f[i])), i)))]
    idx = sorted(range(n), key=lambda i: (total_key(float(x[i])), i))
    coef = 2.0 * 0.37 / n
    g0 = noise(4, n)
    want = g0.copy()
    loss = 0.0
    for q, p in enumerate(idx):
        d = x[p] - t[q]
        loss += d * d
        want[p] += coef * d
    got, got_loss = T.marginal_row(x, T.sort_positions(x), t, coef, g0)
    assert abs(got_loss - loss) <= 1e-13 * loss
    assert np.array_equal(got, want)


def test_kappa_table_is_the_hermite_cubic():
    interp = pytest.importorskip("scipy.interpolate")
    kx = np.array([-3.0, -1.0, -0.2, 0.5, 2.0, 4.0])
    ky = np.array([-2.5, -0.9, -0.1, 0.6, 1.5, 2.2])
    kd = np.array([0.9, 1.1, 1.2, 0.8, 0.5, 0.3])
    gm, gs, km, ks = 0.1, 1.7, 0.05, 1.3
    x = np.linspace(-4.0, 4.0, 2001)
    k, dk = T.kappa_pchip(x, kx, ky, kd, gm, gs, km, ks)
    t = x * gs + gm
    spl = interp.CubicHermiteSpline(kx, ky, kd)
    inside = (t > kx[0]) & (t < kx[-1])
    assert np.allclose(k[inside], (spl(t[inside]) - km) / ks, rtol=1e-12, atol=1e-12)
    assert np.allclose(dk[inside], spl.derivative()(t[inside]) * gs / ks, rtol=1e-11, atol=1e-11)
    lo, hi = t <= kx[0], t >= kx[-1]
    assert np.array_equal(k[lo], (ky[0] + kd[0] * (t[lo] - kx[0]) - km) / ks)
    assert np.array_equal(k[hi], (ky[-1] + kd[-1] * (t[hi] - kx[-1]) - km) / ks)
    assert np.all(dk[lo] == kd[0] * gs / ks) and np.all(dk[hi] == kd[-1] * gs / ks)
    with pytest.raises(ValueError):
        T.kappa_pchip(x, kx[:1], ky[:1], kd[:1], gm, gs, km, ks)
