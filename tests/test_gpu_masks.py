"""Masked averages of the CUDA engine (stlp_set_masks) against the FP64 oracle.

The reference's mask test (crates/stl-core/tests/mask.rs:38-97) evaluates K
masks at once (the whole sky and two latitude cuts) and checks values,
variances and the map cotangent against a per-mask evaluation with the mask
as the core, at 1e-11 abs + 1e-10 rel; the whole-sky mask must equal the
unmasked engine.  Here the FP64 engine is held to those tolerances against
the C++ oracle's masked engine, and the FP32 engine to the FP32 criterion of
the unmasked parity tests (rtol 1e-6, atol 1e-6 of the family's largest |S|).
"""
import numpy as np
import pytest

import oracle as O
from conftest import close_ratio

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def latitude_cut(nside, b_deg):
    """NESTED ids of the pixels with |z| > sin(b) (mask.rs:34-36)."""
    ids = np.arange(12 * nside * nside, dtype=np.int64)
    theta = O.centres(nside, ids)[3]
    return ids[np.abs(np.cos(theta)) > np.sin(np.radians(b_deg))]


def mask_sets(nside):
    return [np.arange(12 * nside * nside), latitude_cut(nside, 20.0), latitude_cut(nside, 45.0)]


def indicators(nside, sets):
    w = np.zeros((len(sets), 12 * nside * nside))
    for k, s in enumerate(sets):
        w[k, s] = 1.0
    return w


@pytest.mark.parametrize("nside,J,B", [(16, 3, 2), (64, 5, 2)])
def test_fp64_masks_match_oracle(stl, nside, J, B):
    rng = np.random.default_rng(40 + nside)
    x = np.exp(rng.standard_normal((B, 12 * nside * nside)) - 0.5)
    sets = mask_sets(nside)
    e = stl.NativeEngine(nside, J, batch=B, dtype="float64")
    full, full_var = e.forward(x, moments=True)
    e.set_masks(sets)
    assert e.nmasks == len(sets) and e.info()["masks"] == len(sets)
    values, var = e.forward(x, moments=True)
    assert values.shape == (B, len(sets), e.ncoeff) and var.shape == values.shape

    o = O.OracleEngine(nside, J, batch=B)
    o.set_masks(indicators(nside, sets))
    ref, ref_var = o.forward(x, moments=True)
    assert close_ratio(values.real, ref.real, 1e-11, 1e-10) <= 1.0
    assert close_ratio(values.imag, ref.imag, 1e-11, 1e-10) <= 1.0
    assert close_ratio(var, ref_var, 1e-11, 1e-10) <= 1.0
    # the whole-sky mask is the unmasked engine
    assert close_ratio(values[:, 0], full, 1e-13, 1e-12) <= 1.0
    assert close_ratio(var[:, 0], full_var, 1e-13, 1e-12) <= 1.0
    np.testing.assert_array_equal(e.native_pixels(), o.native_pixels())

    cot = rng.standard_normal(values.shape) + 1j * rng.standard_normal(values.shape)
    g_ref = o.vjp(cot)
    grad = e.vjp(cot)
    assert close_ratio(grad, g_ref, 1e-10 * np.max(np.abs(g_ref)), 0.0) <= 1.0
    e.close()


def test_fp32_masks_within_1e6(stl):
    nside, J, B = 64, 5, 2
    rng = np.random.default_rng(41)
    x = np.exp(rng.standard_normal((B, 12 * nside * nside)) - 0.5).astype(np.float32).astype(np.float64)
    sets = mask_sets(nside)[1:]
    o = O.OracleEngine(nside, J, batch=B)
    o.set_masks(indicators(nside, sets))
    ref = o.forward(x)
    e = stl.NativeEngine(nside, J, batch=B, dtype="float32")
    e.set_masks(indicators(nside, sets))
    values, _ = e.forward(x)
    fam = np.array([c["family"] for c in e.plan])
    lev = np.array([c["native_dg"] for c in e.plan])
    scale = np.zeros(ref.shape)
    for f in set(fam):
        for n in set(lev):
            sel = (fam == f) & (lev == n)
            if sel.any():
                scale[..., sel] = np.max(np.abs(ref[..., sel]), axis=-1, keepdims=True)
    for part in (np.real, np.imag):
        err = np.abs(part(values) - part(ref))
        assert np.max(err / (1e-6 * scale + 1e-6 * np.abs(part(ref)))) <= 1.0
    cot = rng.standard_normal(values.shape) + 1j * rng.standard_normal(values.shape)
    assert np.max(np.abs(e.vjp(cot) - o.vjp(cot))) <= 1e-5 * np.max(np.abs(o.vjp(cot)))
    e.close()


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("moments", [False, True])
def test_fp32_map_sums_are_those_of_the_fp64_maps(stl, masked, moments):
    """FP32 fields hold the maps' deviations from their means rounded to FP32;
    the map sums add the rounding residuals back, so a mean near zero (1e-7
    against deviations of 1, on the sky or under a latitude mask) keeps the
    FP64 engine's value to 1e-6 of itself, and the variance to 1e-12."""
    nside, J, B = 64, 4, 2
    rng = np.random.default_rng(44)
    g = rng.standard_normal((B, 12 * nside * nside))
    cut = latitude_cut(nside, 20.0)
    over = g[:, cut] if masked else g
    x = g - over.mean(axis=1, keepdims=True) + 1e-7 * (1.0 + np.arange(B))[:, None]
    e32 = stl.NativeEngine(nside, J, batch=B, dtype="float32")
    e64 = stl.NativeEngine(nside, J, batch=B, dtype="float64")
    if masked:
        e32.set_masks([cut])
        e64.set_masks([cut])
    v32, var32 = e32.forward(x, moments=moments)
    v64, var64 = e64.forward(x, moments=moments)
    fam = [c["family"] for c in e32.plan]
    im, iv = fam.index("mean"), fam.index("var")
    m32, m64 = v32[..., im].real, v64[..., im].real
    assert np.max(np.abs(m64)) < 1e-6
    assert np.max(np.abs(m32 - m64) / np.abs(m64)) <= 1e-6
    assert np.max(np.abs(v32[..., iv] - v64[..., iv]) / np.abs(v64[..., iv])) <= 1e-12
    if moments:
        assert np.max(np.abs(var32[..., im] - var64[..., im]) / var64[..., im]) <= 1e-9
    e32.close()
    e64.close()


def test_masks_reset_and_refusals(stl):
    nside, J = 16, 3
    rng = np.random.default_rng(42)
    x = rng.standard_normal((1, 12 * nside * nside))
    e = stl.NativeEngine(nside, J, dtype="float64")
    full, _ = e.forward(x)
    e.set_masks([latitude_cut(nside, 30.0)])
    masked, _ = e.forward(x)
    assert masked.shape == (1, 1, e.ncoeff)
    e.set_masks(None)
    assert e.nmasks == 0
    again, _ = e.forward(x)
    np.testing.assert_array_equal(again, full)
    with pytest.raises(ValueError, match="out of range"):
        e.set_masks([np.array([12 * nside * nside])])
    with pytest.raises(RuntimeError, match="empty mask"):
        e.set_masks(np.zeros((1, 12 * nside * nside)))
    e.close()
