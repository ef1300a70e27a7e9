"""FP64 objective terms of the synthesis on the CPU: the oracle of the device terms.

TEST INFRASTRUCTURE ONLY (the checker of a device implementation of these
terms; nothing in the product imports it).  A numpy restatement of the terms
the reference evaluates on the device for ``stl-synth`` / the CLI ensemble
objective (crates/stl-gpu/src/terms.rs, kernels in crates/stl-gpu/src/
kernels.cu:1454-1625), written as the host expressions its tests check them
against (crates/stl-gpu/tests/terms.rs:45-186):

* the standardised kappa transform of a monotone cubic (PCHIP) table and its
  derivative (terms.rs:36-58, kernels.cu:1454-1485);
* the 4-children pyramid of NESTED rows (means of four children), its details
  d = child - parent and their moments (sum d^2, sum d^4) per level
  (terms.rs:78-145, kernels.cu:1487-1530);
* the level-power gradient g += sum_n coef[r, n] d_n[i >> 2n] and the
  kurtosis gradient g += dk * sum_k coef (d^3 - c - K V d), c the mean of d^3
  over the four siblings (terms.rs:148-184, kernels.cu:1532-1579);
* the stable sort of a row in f64 total order, ties in position order
  (terms.rs:187-258, kernels.cu:1609-1623), the pixel-marginal term of a
  row against a sorted target (terms.rs:260-269) and g += a b (terms.rs:271-275).

Every product is rounded on its own and the sums run in the order the host
expressions use (numpy element-wise operations do not fuse), so the gradients
are the host's bit for bit and the moments and losses equal them to rounding.
"""
from __future__ import annotations

import numpy as np


def total_order_keys(x: np.ndarray) -> np.ndarray:
    """u64 keys that order as f64 total order (-NaN < -inf < ... < -0 < +0 <
    ... < +inf < +NaN): the sign bit set flips every bit, else sets the sign
    bit (kernels.cu:1617-1623)."""
    b = np.ascontiguousarray(x, dtype=np.float64).view(np.uint64)
    neg = (b >> np.uint64(63)) != 0
    return np.where(neg, ~b, b | np.uint64(1 << 63))


def sort_positions(x: np.ndarray) -> np.ndarray:
    """Positions of the values of one row in increasing total order, ties in
    position order (the reference's stable radix sort, terms.rs:230-258)."""
    return np.argsort(total_order_keys(x), kind="stable").astype(np.uint32)


def kappa_pchip(x, kx, ky, kd, gm, gs, km, ks):
    """kappa = (f(x gs + gm) - km) / ks and its derivative in x, f the cubic
    Hermite interpolant of the knots kx (increasing), values ky and slopes kd,
    continued linearly outside [kx[0], kx[-1]] (kernels.cu:1454-1485)."""
    x = np.asarray(x, dtype=np.float64)
    kx, ky, kd = (np.asarray(a, dtype=np.float64) for a in (kx, ky, kd))
    if kx.size < 2 or ky.size != kx.size or kd.size != kx.size:
        raise ValueError("the table needs at least two knots, values and slopes of one length")
    t = x * gs + gm
    v = np.empty_like(t)
    dv = np.empty_like(t)
    lo, hi = t <= kx[0], t >= kx[-1]
    v[lo] = ky[0] + kd[0] * (t[lo] - kx[0])
    dv[lo] = kd[0]
    v[hi] = ky[-1] + kd[-1] * (t[hi] - kx[-1])
    dv[hi] = kd[-1]
    mid = ~(lo | hi)
    tm = t[mid]
    j = np.searchsorted(kx, tm, side="right") - 1  # the last knot <= t
    h = kx[j + 1] - kx[j]
    u = (tm - kx[j]) / h
    y0, y1, d0, d1 = ky[j], ky[j + 1], kd[j] * h, kd[j + 1] * h
    u2, u3 = u * u, u * u * u
    v[mid] = (2.0 * u3 - 3.0 * u2 + 1.0) * y0 + (u3 - 2.0 * u2 + u) * d0 + (3.0 * u2 - 2.0 * u3) * y1 + (u3 - u2) * d1
    w = (6.0 * u2 - 6.0 * u) * (y0 - y1) + (3.0 * u2 - 4.0 * u + 1.0) * d0 + (3.0 * u2 - 2.0 * u) * d1
    dv[mid] = w / h
    return (v - km) / ks, dv * gs / ks


def quad_means(x: np.ndarray) -> np.ndarray:
    """Parents of rows [R, 4m] of NESTED cells: ((c0 + c1) + c2 + c3) / 4."""
    c = np.asarray(x, dtype=np.float64).reshape(x.shape[0], -1, 4)
    return (((c[:, :, 0] + c[:, :, 1]) + c[:, :, 2]) + c[:, :, 3]) / 4.0


def pyramid(x: np.ndarray, depth: int) -> list[np.ndarray]:
    """Levels 0..depth of rows x [R, len] (level 0 the rows; len a multiple of
    4^depth, terms.rs:88-102)."""
    x = np.asarray(x, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] % (1 << (2 * depth)):
        raise ValueError("rows not aligned on the pyramid")
    out = [x]
    for _ in range(depth):
        out.append(quad_means(out[-1]))
    return out


def details(levels: list[np.ndarray], n: int) -> np.ndarray:
    """d_n = level n - its parent, [R, len >> 2n]."""
    return levels[n] - np.repeat(levels[n + 1], 4, axis=1)


def detail_moments(levels: list[np.ndarray]) -> np.ndarray:
    """(sum d^2, sum d^4) of every row and level n < depth, [R, depth, 2]
    (terms.rs:117-138; equal to the device's chunked tree sums to rounding)."""
    depth = len(levels) - 1
    out = np.zeros((levels[0].shape[0], depth, 2))
    for n in range(depth):
        d = details(levels, n)
        out[:, n, 0] = (d * d).sum(axis=1)
        out[:, n, 1] = (d * d * d * d).sum(axis=1)
    return out


def level_power_grad(levels: list[np.ndarray], coef: np.ndarray, g: np.ndarray) -> np.ndarray:
    """g + sum_{n < L} coef[r, n] d_n[r, i >> 2n], the sum from 0 in level order
    and added to g last (kernels.cu:1532-1551; coef [R, L], L <= depth)."""
    coef = np.asarray(coef, dtype=np.float64)
    R, L = coef.shape
    if L > len(levels) - 1:
        raise ValueError("more level-power levels than the pyramid holds")
    acc = np.zeros_like(levels[0])
    for n in range(L):
        d = np.repeat(details(levels, n), 1 << (2 * n), axis=1)
        acc = acc + coef[:, n:n + 1] * d
    return g + acc


def kurtosis_grad(levels: list[np.ndarray], lev, cf: np.ndarray, g: np.ndarray, dk=None) -> np.ndarray:
    """g + dk * sum_k coef (d^3 - c - (K V) d) over the levels lev[k], d the
    level's detail of the pixel, c = (e0^3 + e1^3 + e2^3 + e3^3) / 4 over its
    four siblings, cf [R, len(lev), 3] = (coef, K, V) (kernels.cu:1553-1578;
    dk None: g + the sum)."""
    cf = np.asarray(cf, dtype=np.float64).reshape(levels[0].shape[0], len(lev), 3)
    acc = np.zeros_like(levels[0])
    for k, n in enumerate(lev):
        if not 0 <= n < len(levels) - 1:
            raise ValueError("kurtosis level outside the pyramid")
        d = details(levels, n)
        e = d.reshape(d.shape[0], -1, 4)
        e3 = e * e * e
        c = (((e3[:, :, 0] + e3[:, :, 1]) + e3[:, :, 2]) + e3[:, :, 3]) / 4.0
        c = np.repeat(c, 4, axis=1)
        kv = cf[:, k, 1:2] * cf[:, k, 2:3]
        term = cf[:, k, 0:1] * (((d * d * d) - c) - kv * d)
        acc = acc + np.repeat(term, 1 << (2 * n), axis=1)
    return g + (acc * dk if dk is not None else acc)


def marginal_row(x: np.ndarray, perm: np.ndarray, t_sorted: np.ndarray, coef: float, g: np.ndarray):
    """The pixel marginal of one row: d_q = x[perm[q]] - t[q]; returns (g with
    g[perm[q]] += coef d_q, sum d_q^2) (kernels.cu:1586-1607)."""
    d = x[perm] - t_sorted
    out = np.array(g, dtype=np.float64, copy=True)
    out[perm] = out[perm] + coef * d
    return out, float((d * d).sum())


def add_product(g: np.ndarray, a: np.ndarray, b=None) -> np.ndarray:
    """g + a b (b None: g + a) (kernels.cu:1580-1585)."""
    return g + (a * b if b is not None else a)
