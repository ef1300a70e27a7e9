"""Spin-2 front end on the GPU against the oracle (oracle/spin.py, a restatement
of crates/stl-core/src/spin.rs with the bridge's use of it).

The operators are built on the device; their cells must equal the oracle's
exactly (integer work) and their weights agree to rounding (the device's
sin, cos, exp and atan2 against the host's libm, through a Cholesky solve).
The statistics and gradients of both pyramids and of the cross pairs follow
the reference's own GPU-versus-CPU bars (python/stl_ensemble/tests/
test_spin.py:165-190: values 1e-12, gradients 1e-11 of the largest).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import spin as S  # noqa: E402

pytestmark = pytest.mark.gpu

NSIDE, J = 16, 3


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def _maps(batch, seed=0, nside=NSIDE):
    return np.random.default_rng(seed).normal(size=(batch, 2, 12 * nside ** 2))


def _rows_match(cells, w, ptr, col, wo):
    """Cells as sets per row (exact), weights matched by cell; the worst weight
    difference relative to the row's largest weight."""
    worst = 0.0
    for r in range(cells.shape[0]):
        mine = cells[r][cells[r] >= 0]
        ref = col[ptr[r]:ptr[r + 1]]
        assert np.array_equal(np.sort(mine), np.sort(ref)), r
        a = dict(zip(mine.tolist(), w[r][:mine.size]))
        b = dict(zip(ref.tolist(), wo[ptr[r]:ptr[r + 1]]))
        scale = max(abs(v) for v in b.values())
        worst = max(worst, max(abs(a[c] - b[c]) for c in b) / scale)
    return worst


# The weights solve the normal equations of the monomials up to degree
# kernel - 1 (15 to 45 of them); their conditioning grows with the degree, so
# the few-ulp differences of the device's trigonometry from the host's libm
# reach the weights at these bounds (measured: 1.6e-14, 2.6e-13, 4.1e-12,
# 2.7e-10 of a row's largest weight).
WEIGHT_TOL = {3: 1e-13, 5: 2e-12, 7: 4e-11, 9: 2e-9}


@pytest.mark.parametrize("nside,kernel", [(16, 5), (16, 3), (8, 7), (8, 9), (32, 5), (4, 9), (2, 5)])
def test_stencil_rows_match_oracle(stl, nside, kernel):
    e = stl.NativeEngine(nside, 1, spin=2, spin_kernel=kernel)
    cells, w = e.spin_rows(0, "stencil")
    ptr, col, wo = S.eth_bar2(nside, kernel).export()
    worst = _rows_match(cells, w, ptr, col, wo)
    print(f"nside {nside} kernel {kernel}: worst weight difference {worst:.2e} of the row's largest")
    assert worst <= WEIGHT_TOL[kernel]


def test_transported_rows_match_oracle(stl):
    e = stl.NativeEngine(32, 4, spin=2, spin_pyramid="transported")
    for level in range(4):
        cells, w = e.spin_rows(level, "stencil")
        ptr, col, wo = S.eth_bar2(32 >> level, 5).export()
        assert _rows_match(cells, w, ptr, col, wo) <= WEIGHT_TOL[5]
    for level in range(3):
        cells, w = e.spin_rows(level, "means")
        ptr, col, wo = S.spin_decimation(32 >> level).export()
        assert np.array_equal(cells, col.reshape(-1, 4))
        assert np.abs(w - wo.reshape(-1, 4)).max() <= 1e-14


def test_singular_level_is_refused(stl):
    """nside 1 is too small for the fit (the reference panics there as well)."""
    e = stl.NativeEngine(16, 5, spin=2, spin_pyramid="transported")
    with pytest.raises(RuntimeError, match="singular"):
        e.forward(_maps(1))


@pytest.mark.parametrize("mode", ["scalar", "transported"])
def test_values_and_gradients_match_oracle(stl, mode):
    x = _maps(2, 5)
    e = stl.NativeEngine(NSIDE, J, batch=2, spin=2, spin_pyramid=mode)
    o = S.SpinOracle(NSIDE, J, batch=2, pyramid=mode)
    v, _ = e.forward(x)
    vo = o.forward(x)
    assert v.shape == vo.shape == (2, 2, e.ncoeff)
    assert np.abs(v - vo).max() <= 1e-12 * np.abs(vo).max(), np.abs(v - vo).max()
    cot = np.random.default_rng(6).normal(size=v.shape) + 1j * np.random.default_rng(7).normal(size=v.shape)
    g, go = e.vjp(cot), o.vjp(cot)
    assert g.shape == x.shape
    assert np.abs(g - go).max() <= 1e-11 * np.abs(go).max(), np.abs(g - go).max()


def test_level0_shared_by_both_pyramids(stl):
    x = _maps(1, 3)
    a = stl.NativeEngine(NSIDE, J, spin=2, spin_pyramid="transported")
    b = stl.NativeEngine(NSIDE, J, spin=2)
    va, vb = a.forward(x)[0], b.forward(x)[0]
    lev0 = [i for i, c in enumerate(a.plan) if c["native_dg"] == 0 and c["family"] in ("mean", "var", "S1", "S2")]
    assert np.allclose(va[..., lev0], vb[..., lev0], rtol=1e-12, atol=0)


@pytest.mark.parametrize("spin_a", [2, 0])
def test_cross_pairs_match_oracle(stl, spin_a):
    rng = np.random.default_rng(10)
    n = 12 * NSIDE ** 2
    a = rng.normal(size=(2, 2, n)) if spin_a == 2 else rng.normal(size=(2, n))
    b = rng.normal(size=(2, 2, n))
    e = stl.NativeEngine(NSIDE, J, batch=2, spin=2, cross=True, spin_a=spin_a)
    o = S.SpinOracle(NSIDE, J, batch=2, cross=True, spin_a=spin_a)
    v = e.forward_cross(a, b)[0]
    vo = o.forward((a, b))
    assert np.abs(v - vo).max() <= 1e-12 * np.abs(vo).max()
    cot = rng.normal(size=v.shape) + 0j
    for x, y in zip(e.vjp_cross(cot), o.vjp(cot)):
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= 1e-11 * np.abs(y).max()


@pytest.mark.parametrize("mode", ["scalar", "transported"])
def test_eroded_masks_match_oracle(stl, mode):
    w = np.ones(12 * NSIDE ** 2)
    w[:200] = 0.0
    w[2000:2100] = 0.0
    e = stl.NativeEngine(NSIDE, J, batch=1, spin=2, spin_pyramid=mode)
    o = S.SpinOracle(NSIDE, J, batch=1, pyramid=mode)
    e.set_masks(w[None])
    o.set_masks(w[None])
    assert np.array_equal(e.native_pixels(), o.native_pixels())
    x = _maps(1, 4)
    v, vo = e.forward(x)[0], o.forward(x)
    assert v.shape == vo.shape == (1, 2, 1, e.ncoeff)
    assert np.abs(v - vo).max() <= 1e-12 * np.abs(vo).max()


@pytest.mark.parametrize("mode", ["scalar", "transported"])
def test_small_mask_keeps_coarse_levels(stl, mode):
    n = 12 * 32 ** 2
    w = np.zeros(n)
    w[:n // 48] = 1.0
    e = stl.NativeEngine(32, 4, spin=2, spin_pyramid=mode)
    o = S.SpinOracle(32, 4, pyramid=mode)
    e.set_masks(w[None])
    o.set_masks(w[None])
    assert (e.native_pixels() > 0).all()
    assert np.array_equal(e.native_pixels(), o.native_pixels())
    e.forward(np.random.default_rng(12).normal(size=(1, 2, n)))


def test_spin_fields_match_oracle(stl):
    x = _maps(2, 8)
    e = stl.NativeEngine(NSIDE, J, batch=2, spin=2, spin_pyramid="transported")
    o = S.SpinOracle(NSIDE, J, batch=2, pyramid="transported")
    for level in range(J):
        qu, chi = e.spin_fields(x, level)
        quo, chio = o.fields(x, level)
        assert np.abs(qu - quo).max() <= 1e-14 * np.abs(quo).max()
        assert np.abs(chi - chio).max() <= 1e-12 * np.abs(chio).max()


def test_fp32_within_family_tolerance(stl):
    """FP32 fields against the engine's FP64 path on the same maps (the 1e-6
    family criterion of the headline), both pyramids."""
    x = _maps(2, 9, nside=64)
    for mode in ("scalar", "transported"):
        v32 = stl.NativeEngine(64, 4, batch=2, spin=2, spin_pyramid=mode, dtype="float32").forward(x)[0]
        v64 = stl.NativeEngine(64, 4, batch=2, spin=2, spin_pyramid=mode).forward(x)[0]
        assert np.isfinite(v32).all()
        scale = np.abs(v64).max(axis=-1, keepdims=True)
        err = np.maximum(np.abs((v32 - v64).real), np.abs((v32 - v64).imag))
        assert (err <= 1e-6 * scale + 1e-6 * np.abs(v64)).all(), mode


def test_checkpoint_restore(stl):
    e = stl.NativeEngine(NSIDE, J, batch=1, spin=2, spin_pyramid="transported")
    x, y = _maps(1, 1), _maps(1, 2)
    v, _ = e.forward(x, generation=1)
    snap = e.checkpoint()
    e.forward(y, generation=2)
    cot = np.ones_like(v)
    e.restore(snap, generation=1)
    g = e.vjp(cot, generation=1)
    ref = stl.NativeEngine(NSIDE, J, batch=1, spin=2, spin_pyramid="transported")
    ref.forward(x, generation=1)
    assert np.array_equal(g, ref.vjp(cot, generation=1))


def test_device_tensors_and_bit_reproducible(stl):
    import torch
    x = _maps(2, 11)
    e = stl.NativeEngine(NSIDE, J, batch=2, spin=2, spin_pyramid="transported")
    v_host = e.forward(x)[0]
    v_dev, _ = e.forward_tensor(torch.tensor(x, device="cuda"))
    assert np.array_equal(v_host, v_dev)
    cot = np.random.default_rng(3).normal(size=v_host.shape) + 0j
    g_dev = torch.empty(x.shape, dtype=torch.float64, device="cuda")
    e.vjp_tensor(cot, g_dev)
    e.forward(x)
    assert np.array_equal(e.vjp(cot), g_dev.cpu().numpy())


@pytest.mark.parametrize("kernel,tol", [(3, 1e-12), (7, 1e-10), (9, 1e-8)])
def test_other_stencils_match_oracle(stl, kernel, tol):
    """Kernels 3, 7 and 9: statistics and gradients against the oracle, the bar
    scaled by the weights' conditioning (the operator rows' bounds above)."""
    x = _maps(1, 13)
    e = stl.NativeEngine(NSIDE, J, spin=2, spin_kernel=kernel, spin_pyramid="transported")
    o = S.SpinOracle(NSIDE, J, kernel=kernel, pyramid="transported")
    v, vo = e.forward(x)[0], o.forward(x)
    assert np.abs(v - vo).max() <= tol * np.abs(vo).max()
    cot = np.random.default_rng(14).normal(size=v.shape) + 0j
    assert np.abs(e.vjp(cot) - o.vjp(cot)).max() <= 10 * tol * np.abs(o.vjp(cot)).max()


def test_cross_pairs_with_masks_match_oracle(stl):
    """Cross pairs (spin_a 2) with eroded masks: the scalar-pyramid erosion of
    both channels' level-0 stencil."""
    rng = np.random.default_rng(15)
    n = 12 * NSIDE ** 2
    a, b = rng.normal(size=(2, 2, n)), rng.normal(size=(2, 2, n))
    w = np.ones((2, n))
    w[0, :300] = 0.0
    w[1, 1500:1900] = 0.0
    e = stl.NativeEngine(NSIDE, J, batch=2, spin=2, cross=True)
    o = S.SpinOracle(NSIDE, J, batch=2, cross=True)
    e.set_masks(w)
    o.set_masks(w)
    assert np.array_equal(e.native_pixels(), o.native_pixels())
    v, vo = e.forward_cross(a, b)[0], o.forward((a, b))
    assert v.shape == vo.shape == (2, 2, 2, e.ncoeff)
    assert np.abs(v - vo).max() <= 1e-12 * np.abs(vo).max()
    cot = rng.normal(size=v.shape) + 0j
    for x, y in zip(e.vjp_cross(cot), o.vjp(cot)):
        assert np.abs(x - y).max() <= 1e-11 * np.abs(y).max()


def test_fp32_cross_pairs_within_tolerance(stl):
    """FP32 cross pairs (spin_a 0: a scalar T with (Q, U)) against FP64."""
    rng = np.random.default_rng(16)
    n = 12 * 64 ** 2
    a, b = rng.normal(size=(2, n)), rng.normal(size=(2, 2, n))
    v32 = stl.NativeEngine(64, 4, batch=2, spin=2, cross=True, spin_a=0, dtype="float32").forward_cross(a, b)[0]
    v64 = stl.NativeEngine(64, 4, batch=2, spin=2, cross=True, spin_a=0).forward_cross(a, b)[0]
    scale = np.abs(v64).max(axis=-1, keepdims=True)
    err = np.maximum(np.abs((v32 - v64).real), np.abs((v32 - v64).imag))
    assert (err <= 1e-6 * scale + 1e-6 * np.abs(v64)).all()
