"""Cross statistics of two channels (config "cross"; maps [B, 2, N], the
plan of the cross terms only) against the FP64 oracle's cross-only engine
and against the cross coefficients of the reference's two-channel fixture
(stats_n32_J4_L4_k5_C2_B1_full_b512: values of the full two-channel plan,
matched by coefficient), to the reference's tolerances (values 1e-11 +
1e-10 rel, tests/stats.rs:175-190); masks included; FP32 within the 1e-6
family criterion of FP64."""
import json

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, close_ratio

pytestmark = pytest.mark.gpu

KEYS = ("family", "native_dg", "c1", "c2", "j1", "j2", "j3", "l1", "l2", "l3")


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def _maps(rng, B, nside):
    """Two correlated lognormal channels (a shared field plus noise), so the cross terms are not small."""
    npix = 12 * nside * nside
    g = rng.standard_normal((B, 1, npix))
    return np.exp(0.7 * g + 0.5 * rng.standard_normal((B, 2, npix)) - 0.5)


@pytest.mark.parametrize("nside,J,B", [(16, 3, 2), (32, 4, 1)])
def test_fp64_cross_matches_oracle(stl, nside, J, B):
    rng = np.random.default_rng(60 + nside)
    x = _maps(rng, B, nside)
    e = stl.NativeEngine(nside, J, batch=B, dtype="float64", cross=True)
    v, var = e.forward(x, moments=True)
    o = O.OracleEngine(nside, J, batch=B, channels=2, cross_only=True)
    ref, ref_var = o.forward(x, moments=True)
    assert v.shape == ref.shape == (B, e.ncoeff)
    assert close_ratio(v.real, ref.real, 1e-11, 1e-10) <= 1.0
    assert close_ratio(v.imag, ref.imag, 1e-11, 1e-10) <= 1.0
    assert close_ratio(var, ref_var, 1e-11, 1e-10) <= 1.0
    cot = rng.standard_normal(v.shape) + 1j * rng.standard_normal(v.shape)
    g = e.vjp(cot)
    gr = o.vjp(cot).reshape(B, 2, -1)
    assert g.shape == (B, 2, 12 * nside * nside)
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))
    e.close()


def test_fp64_cross_matches_the_two_channel_fixture(stl):
    d = GOLDEN / "stats" / "stats_n32_J4_L4_k5_C2_B1_full_b512"
    meta = json.loads((d / "meta.json").read_text())
    x = np.load(d / "map0.npy")
    want = np.load(d / "values_re.npy")[0] + 1j * np.load(d / "values_im.npy")[0]
    plan = json.loads((d / "plan.json").read_text())  # rows [family, native_dg, c1, c2, j1, j2, j3, l1, l2, l3]
    index = {tuple(c): i for i, c in enumerate(plan)}
    e = stl.NativeEngine(meta["nside"], meta["J"], batch=1, dtype="float64", cross=True)
    v, _ = e.forward(x)
    pick = np.array([index[tuple(c[k] for k in KEYS)] for c in e.plan])
    assert close_ratio(v[0].real, want[pick].real, 1e-11, 1e-10) <= 1.0
    assert close_ratio(v[0].imag, want[pick].imag, 1e-11, 1e-10) <= 1.0
    e.close()


def test_cross_with_masks(stl):
    nside, J, B = 16, 3, 1
    rng = np.random.default_rng(61)
    x = _maps(rng, B, nside)
    theta = O.centres(nside, np.arange(12 * nside * nside))[3]
    w = np.stack([np.ones(12 * nside * nside), (np.abs(np.cos(theta)) > 0.4).astype(float)])
    e = stl.NativeEngine(nside, J, batch=B, dtype="float64", cross=True)
    e.set_masks(w)
    v, var = e.forward(x, moments=True)
    o = O.OracleEngine(nside, J, batch=B, channels=2, cross_only=True)
    o.set_masks(w)
    ref, ref_var = o.forward(x, moments=True)
    assert v.shape == (B, 2, e.ncoeff)
    assert close_ratio(v, ref, 1e-11, 1e-10) <= 1.0 and close_ratio(var, ref_var, 1e-11, 1e-10) <= 1.0
    cot = rng.standard_normal(v.shape) + 1j * rng.standard_normal(v.shape)
    gr = o.vjp(cot).reshape(B, 2, -1)
    assert np.max(np.abs(e.vjp(cot) - gr)) <= 1e-10 * np.max(np.abs(gr))
    e.close()


def test_fp32_cross_within_1e6(stl):
    nside, J, B = 64, 5, 2
    rng = np.random.default_rng(62)
    x = _maps(rng, B, nside).astype(np.float32).astype(np.float64)
    e64 = stl.NativeEngine(nside, J, batch=B, dtype="float64", cross=True)
    e32 = stl.NativeEngine(nside, J, batch=B, dtype="float32", cross=True)
    r, _ = e64.forward(x)
    a, _ = e32.forward(x)
    fam = np.array([c["family"] for c in e64.plan])
    lev = np.array([c["native_dg"] for c in e64.plan])
    for f in set(fam):
        for n in set(lev):
            sel = (fam == f) & (lev == n)
            if not sel.any():
                continue
            scale = np.max(np.abs(r[:, sel]), axis=-1, keepdims=True)
            for part in (np.real, np.imag):
                assert np.max(np.abs(part(a[:, sel]) - part(r[:, sel])) / (1e-6 * scale + 1e-6 * np.abs(part(r[:, sel])))) <= 1.0
    cot = rng.standard_normal(r.shape) + 1j * rng.standard_normal(r.shape)
    g64, g32 = e64.vjp(cot), e32.vjp(cot)
    # the cross S1's rn(z) = z / sqrt(|z| + 1e-8) has a gradient ~ |z|^-1/2 that
    # magnifies FP32 rounding where |z| is small (6e-5 measured here)
    assert np.max(np.abs(g32 - g64)) <= 1e-4 * np.max(np.abs(g64))
    e64.close()
    e32.close()
