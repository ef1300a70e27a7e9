"""The patch engine (stlp_patch_*) against the disc oracle and the full-sky
engine: disc supports bit-exact, a disc of radius pi equal to the full sky,
cored discs equal to the oracle's disc model (FP64 to the reference's
tolerances), several discs in one batch, FP32 within the 1e-6 criterion."""
import numpy as np
import pytest

import disc as D
from conftest import close_ratio

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def test_supports_and_cores_are_exact(stl):
    nside, J = 32, 4
    pe = stl.PatchEngine(nside, J)
    centres = np.array([100, 5000, 12287], dtype=np.int64)
    ids = pe.select(centres, 20.0, 12.0)
    vec = pe.centre_vectors(centres)
    assert np.allclose(vec, D.pixel_vectors(nside, centres), rtol=0, atol=1e-15)
    for k, c in enumerate(vec):
        disc = D.Disc(nside, J, c, np.radians(20.0), np.radians(12.0))
        assert np.array_equal(ids[k], disc.ids[0])
        core = np.array(disc.core_pixels(), dtype=np.float64)
        assert np.array_equal(pe.native_pixels[k], core[pe._native])


def test_full_disc_equals_full_sky(stl):
    nside, J = 16, 3
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (1, 12 * nside * nside))
    e = stl.NativeEngine(nside, J, dtype="float64")
    v_ref, var_ref = e.forward(x, moments=True)
    cot = rng.uniform(-1, 1, v_ref.shape) + 1j * rng.uniform(-1, 1, v_ref.shape)
    g_ref = e.vjp(cot)
    pe = stl.PatchEngine(nside, J)
    pe.select(np.array([[0.3, -0.2, 0.9]]), 180.0)
    assert pe.ids[0].size == 12 * nside * nside
    v, var = pe.forward(x, moments=True, generation=4)
    assert close_ratio(v, v_ref, 1e-11, 1e-10) <= 1.0
    assert close_ratio(var, var_ref, 1e-11, 1e-10) <= 1.0
    g = pe.vjp(cot, generation=4)
    assert np.max(np.abs(g - g_ref)) <= 1e-10 * np.max(np.abs(g_ref))


@pytest.mark.parametrize("core", [None, 35.0])
def test_cored_discs_match_the_disc_oracle(stl, core):
    nside, J = 16, 3
    centres = np.array([700, 2000, 700], dtype=np.int64)  # the first disc twice
    pe = stl.PatchEngine(nside, J)
    ids = pe.select(centres, 50.0, core)
    rng = np.random.default_rng(3)
    patches = [rng.uniform(-1, 1, i.size) for i in ids]
    v, var = pe.forward(patches, moments=True, generation=1)
    cot = rng.uniform(-1, 1, v.shape) + 1j * rng.uniform(-1, 1, v.shape)
    g = pe.vjp(cot, generation=1)
    model = D.DiscModel(J)
    for k, c in enumerate(pe.centre_vectors(centres)):
        disc = D.Disc(nside, J, c, np.radians(50.0), None if core is None else np.radians(core))
        vr, varr = model.forward(disc, patches[k], moments=True)
        assert close_ratio(v[k], vr, 1e-11, 1e-10) <= 1.0
        assert close_ratio(var[k], varr, 1e-11, 1e-10) <= 1.0
        gr = model.reverse(disc, cot[k])
        assert np.max(np.abs(g[k] - gr)) <= 1e-10 * np.max(np.abs(gr))
    with pytest.raises(RuntimeError, match="stale"):
        pe.vjp(cot, generation=2)


def test_fp32_disc_within_1e6(stl):
    nside, J = 64, 4
    centre = np.array([1234], dtype=np.int64)
    p32 = stl.PatchEngine(nside, J, dtype="float32")
    p64 = stl.PatchEngine(nside, J, dtype="float64")
    ids = p32.select(centre, 30.0, 20.0)
    p64.select(centre, 30.0, 20.0)
    x = np.exp(np.random.default_rng(5).standard_normal(ids[0].size) - 0.5).astype(np.float32).astype(np.float64)
    v32, _ = p32.forward([x], moments=False)
    v64, _ = p64.forward([x], moments=False)
    fam = np.array([c["family"] for c in p64.plan])
    lev = np.array([c["native_dg"] for c in p64.plan])
    worst = 0.0
    for f in set(fam):
        for n in set(lev):
            sel = (fam == f) & (lev == n)
            if sel.any():
                r, a = v64[0, sel], v32[0, sel]
                scale = np.max(np.abs(r))
                for part in (np.real, np.imag):
                    worst = max(worst, float(np.max(np.abs(part(a) - part(r)) / (1e-6 * scale + 1e-6 * np.abs(part(r))))))
    print(f"patch FP32 vs FP64: worst ratio to the 1e-6 family tolerance {worst:.3f}")
    assert worst <= 1.0
