"""The spin-2 oracle (oracle/spin.py, a restatement of crates/stl-core/src/spin.rs)
checked on the CPU.

The reference holds no fixture of this front end; its own tests pin it by
properties (spin.rs:435-482: adjoints, complex linearity; python/stl_ensemble/
tests/test_spin.py: finite differences in both pyramid modes, level 0 shared by
both, eroded masks, the cross pairs, and a smooth pure-E field against the exact
operator).  The same properties are checked here, the pure-E case analytically:
for P = eth^2 f with f = P_l(cos theta) (Q = sin^2 theta P_l''(cos theta), U = 0,
a pure E field) the operator -(d_x - i d_y)^2 in pixel units gives
chi = -(4 pi / N) (l + 2)(l + 1) l (l - 1) f, and chi_B = 0.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import oracle as O  # noqa: E402
import spin as S  # noqa: E402

NSIDE, J = 16, 3


def _maps(batch, seed=0, nside=NSIDE):
    return np.random.default_rng(seed).normal(size=(batch, 2, 12 * nside ** 2))


def _lcg_fields(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.5, 0.5, size=n)


def test_pyramid_adjoint():
    """<y, A x> = <A^T y, x> over the transported pyramid (spin.rs:444-455)."""
    p = S.SpinPyramid(8, 3, 5)
    x = _lcg_fields(2 * 2 * 768, 7).reshape(2, 2, 768)
    y = p.forward(x)
    rng = np.random.default_rng(8)
    g = [rng.uniform(-0.5, 0.5, size=v.shape) for v in y]
    lhs = sum(float((a * b).sum()) for a, b in zip(y, g))
    rhs = float((x * p.adjoint(g)).sum())
    assert abs(lhs - rhs) < 1e-12 * max(abs(lhs), 1.0)


def test_complex_linearity():
    """A uniform phase on P turns chi by the same phase (spin.rs:458-475)."""
    e = S.eth_bar2(4, 5)
    x = _lcg_fields(2 * 192, 3).reshape(1, 2, 192)
    r = np.exp(2j * 0.3)
    p = (x[0, 0] + 1j * x[0, 1]) * r
    y, yr = e.apply(x)[0], e.apply(np.stack([p.real, p.imag])[None])[0]
    c = (y[0] + 1j * y[1]) * r
    assert np.abs(c.real - yr[0]).max() < 1e-12 and np.abs(c.imag - yr[1]).max() < 1e-12


@pytest.mark.parametrize("kernel,widths", [(3, (8, 9)), (5, (21, 25)), (7, (40, 49)), (9, (65, 81))])
def test_stencil_supports(kernel, widths):
    """Rows read the cells within kernel // 2 rings (fewer at the face corners)."""
    ptr, col, w = S.eth_bar2(8, kernel).export()
    n = np.diff(ptr)
    assert (n.min(), n.max()) == widths
    for r in (0, 100, 767):
        assert sorted(col[ptr[r]:ptr[r + 1]].tolist()) == sorted(O.kth_neighbourhood(r, 8, kernel // 2).tolist())


def test_singular_level_is_refused():
    """nside 1 has too few pixels for even the quadratic fit (spin.rs:330-332)."""
    with pytest.raises(ValueError, match="singular"):
        S.eth_bar2(1, 5)


def test_transported_decimation_weights():
    """Each parent is the mean of its four children turned by e^{-2 i psi}."""
    ptr, col, w = S.spin_decimation(16).export()
    assert np.array_equal(ptr, 4 * np.arange(ptr.size))
    assert np.array_equal(col, np.arange(col.size))
    assert np.allclose(np.abs(w), 0.25, rtol=0, atol=1e-15)


def _pure_mode(nside, l, b_mode):
    n = 12 * nside ** 2
    mu = np.cos(O.centres(nside, np.arange(n))[3])
    f = {4: (35 * mu ** 4 - 30 * mu ** 2 + 3) / 8, 3: (5 * mu ** 3 - 3 * mu) / 2}[l]
    f2 = {4: (420 * mu ** 2 - 60) / 8, 3: 15 * mu}[l]
    p = (1 - mu ** 2) * f2
    qu = np.stack([0 * p, p]) if b_mode else np.stack([p, 0 * p])
    return f, qu[None]


@pytest.mark.parametrize("nside,tol", [(16, 5e-3), (32, 5e-4)])
@pytest.mark.parametrize("l", [3, 4])
@pytest.mark.parametrize("b_mode", [False, True])
def test_smooth_pure_mode_against_exact_operator(nside, tol, l, b_mode):
    f, qu = _pure_mode(nside, l, b_mode)
    chi = S.eth_bar2(nside, 5).apply(qu)[0]
    on, off = (chi[1], chi[0]) if b_mode else (chi[0], chi[1])
    exact = -(4 * np.pi / f.size) * (l + 2) * (l + 1) * l * (l - 1) * f
    assert np.linalg.norm(on - exact) <= tol * np.linalg.norm(exact)
    assert np.linalg.norm(off) <= tol * np.linalg.norm(exact)


def test_transported_mean_of_smooth_field():
    """The transported mean of a smooth spin-2 field is the field at the parent
    to O(h^2), in the parent's frame."""
    _, fine = _pure_mode(32, 4, False)
    _, coarse = _pure_mode(16, 4, False)
    got = S.spin_decimation(32).apply(fine)[0]
    assert np.linalg.norm(got - coarse[0]) <= 2e-2 * np.linalg.norm(coarse[0])


def _fd(f, x, d, h=1e-5):
    return (f(x + h * d) - f(x - h * d)) / (2 * h)


@pytest.mark.parametrize("mode", ["transported", "scalar"])
def test_vjp_finite_differences(mode):
    e = S.SpinOracle(NSIDE, J, batch=2, pyramid=mode)
    x = _maps(2)
    rng = np.random.default_rng(1)
    v = e.forward(x)
    assert v.shape == (2, 2, len(e.plan))
    c = rng.normal(size=v.shape) + 1j * rng.normal(size=v.shape)
    g = e.vjp(c)
    assert g.shape == x.shape
    for _ in range(2):
        d = rng.normal(size=x.shape)
        fd = _fd(lambda y: float(np.real(np.sum(np.conj(c) * e.forward(y)))), x, d)
        an = float(np.sum(g * d))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-6), (fd, an)


def test_level0_shared_by_both_pyramids():
    x = _maps(1, 3)
    va = S.SpinOracle(NSIDE, J, pyramid="transported").forward(x)
    vb = S.SpinOracle(NSIDE, J, pyramid="scalar").forward(x)
    plan = S.SpinOracle(NSIDE, J).plan
    lev0 = [i for i, c in enumerate(plan) if c["native_dg"] == 0 and c["family"] in ("mean", "var", "S1", "S2")]
    assert lev0
    assert np.allclose(va[..., lev0], vb[..., lev0], rtol=1e-12, atol=0)


def test_masks_eroded():
    e = S.SpinOracle(NSIDE, J, pyramid="transported")
    w = np.ones(12 * NSIDE ** 2)
    w[:200] = 0.0
    e.set_masks(w[None])
    counts = e.native_pixels()
    plan = e.plan
    s1 = [i for i, c in enumerate(plan) if c["family"] == "S1" and c["l1"] == 0]
    full = [12 * (NSIDE >> plan[i]["j1"]) ** 2 for i in s1]
    assert all(counts[0, i] < n for i, n in zip(s1, full))
    x = _maps(1, 4)
    for level in range(J):
        _, a = e.fields(x, level)
        _, b = e.fields(x * w, level)
        changed = np.abs(a - b).max((0, 1)) > 0
        assert 0 < changed.sum() <= full[level] - counts[0, s1[level]]


@pytest.mark.parametrize("mode", ["scalar", "transported"])
def test_small_mask_keeps_coarse_levels(mode):
    n = 12 * 32 ** 2
    w = np.zeros(n)
    w[:n // 48] = 1.0
    e = S.SpinOracle(32, 4, pyramid=mode)
    e.set_masks(w[None])
    assert (e.native_pixels() > 0).all()
    e.forward(np.random.default_rng(12).normal(size=(1, 2, n)))


def _cross_inputs(spin_a, seed):
    rng = np.random.default_rng(seed)
    n = 12 * NSIDE ** 2
    a = rng.normal(size=(2, 2, n)) if spin_a == 2 else rng.normal(size=(2, n))
    return a, rng.normal(size=(2, 2, n))


@pytest.mark.parametrize("spin_a", [2, 0])
def test_cross_vjp(spin_a):
    e = S.SpinOracle(NSIDE, J, batch=2, cross=True, spin_a=spin_a)
    a, b = _cross_inputs(spin_a, 8)
    rng = np.random.default_rng(7)
    v = e.forward((a, b))
    c = rng.normal(size=v.shape) + 1j * rng.normal(size=v.shape)
    ga, gb = e.vjp(c)
    assert ga.shape == a.shape and gb.shape == b.shape
    da, db = rng.normal(size=a.shape), rng.normal(size=b.shape)
    f = lambda s: float(np.real(np.sum(np.conj(c) * e.forward((a + s * da, b + s * db)))))  # noqa: E731
    fd = (f(1e-5) - f(-1e-5)) / 2e-5
    an = float(np.sum(ga * da) + np.sum(gb * db))
    assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-6), (fd, an)


@pytest.mark.parametrize("spin_a", [2, 0])
def test_cross_is_scalar_cross_of_chi(spin_a):
    auto = S.SpinOracle(NSIDE, J, batch=2)
    sc = O.OracleEngine(NSIDE, J, batch=2, channels=2, cross_only=True)
    e = S.SpinOracle(NSIDE, J, batch=2, cross=True, spin_a=spin_a)
    a, b = _cross_inputs(spin_a, 9)
    v = e.forward((a, b))
    chi_b = auto.fields(b, 0)[1]
    chi_a = auto.fields(a, 0)[1] if spin_a == 2 else np.stack([a, a], 1)
    for k in range(2):
        ref = sc.forward(np.stack([chi_a[:, k], chi_b[:, k]], 1))
        assert np.abs(v[:, k] - ref).max() <= 1e-12 * np.abs(ref).max()
