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


@pytest.mark.parametrize("moments", [False, True])
def test_fp32_disc_means_near_zero(stl, moments):
    """Disc values whose mean is near zero (1e-7 against values of 1): the FP32
    engine's mean of each disc is the FP64 engine's to 1e-6 of itself (the
    map sums take the FP32 deviations with their rounding residuals), and
    every other coefficient within the 1e-6 family criterion."""
    nside, J = 128, 4
    centres = np.array([100, 30000, 70000, 150000, 190000], dtype=np.int64)
    p32 = stl.PatchEngine(nside, J, dtype="float32")
    p64 = stl.PatchEngine(nside, J, dtype="float64")
    ids = p32.select(centres, 12.0)
    p64.select(centres, 12.0)
    rng = np.random.default_rng(9)
    xs = []
    for k, i in enumerate(ids):
        v = rng.standard_normal(i.size)
        xs.append(v - v.mean() + 1e-7 * (k + 1))
    v32, var32 = p32.forward(xs, moments=moments)
    v64, var64 = p64.forward(xs, moments=moments)
    fam = np.array([c["family"] for c in p64.plan])
    lev = np.array([c["native_dg"] for c in p64.plan])
    im = int(np.flatnonzero(fam == "mean")[0])
    assert np.max(np.abs(v64[:, im])) < 1e-6
    assert np.max(np.abs(v32[:, im].real - v64[:, im].real) / np.abs(v64[:, im].real)) <= 1e-6
    worst = 0.0
    for f in set(fam):
        for n in set(lev):
            sel = (fam == f) & (lev == n)
            if sel.any():
                r, a = v64[:, sel], v32[:, sel]
                scale = np.max(np.abs(r), axis=1, keepdims=True)
                for part in (np.real, np.imag):
                    worst = max(worst, float(np.max(np.abs(part(a) - part(r)) / (1e-6 * scale + 1e-6 * np.abs(part(r))))))
    assert worst <= 1.0
    if moments:
        assert np.max(np.abs(var32[:, im] - var64[:, im]) / var64[:, im]) <= 1e-9


def test_batched_discs_match_one_engine_per_disc(stl):
    """Discs of different sizes (one selected twice, cores on some) in one
    segmented engine, in two groups, and one engine per disc: the same
    statistics and cotangents (FP64, summation order only), and the FP32
    batch within the 1e-6 criterion of the FP64 one."""
    nside, J = 64, 4
    centres = np.array([10, 9000, 30000, 47000, 9000, 21000, 300], dtype=np.int64)
    radii = np.array([9.0, 25.0, 14.0, 30.0, 25.0, 6.0, 18.0])
    cores = np.array([0.0, 15.0, 0.0, 20.0, 15.0, 0.0, 10.0])
    rng = np.random.default_rng(11)
    runs = {}
    for name, kw in (("batch", {}), ("single", {"group_pixels": 1}), ("groups", {"group_pixels": 6000}),
                     ("batch32", {"dtype": "float32"})):
        pe = stl.PatchEngine(nside, J, **({"dtype": "float64"} | kw))
        ids = pe.select(centres, radii, cores)
        if name == "batch":
            patches = [np.exp(rng.standard_normal(i.size) - 0.5).astype(np.float32).astype(np.float64) for i in ids]
            cot = rng.uniform(-1, 1, (len(ids), pe.ncoeff)) + 1j * rng.uniform(-1, 1, (len(ids), pe.ncoeff))
        v, var = pe.forward(patches, moments=True, generation=3)
        g = pe.vjp(cot, generation=3)
        runs[name] = (v, var, g, pe.info()["groups"])
        plan = pe.plan
        pe.close()
    assert runs["batch"][3] == 1 and runs["single"][3] == len(centres) and 1 < runs["groups"][3] < len(centres)
    v, var, g, _ = runs["batch"]
    for name in ("single", "groups"):
        v2, var2, g2, _ = runs[name]
        assert close_ratio(v2, v, 1e-13, 1e-12) <= 1.0
        assert close_ratio(var2, var, 1e-13, 1e-12) <= 1.0
        for a, b in zip(g2, g):
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    v32 = runs["batch32"][0]
    fam = np.array([c["family"] for c in plan])
    lev = np.array([c["native_dg"] for c in plan])
    for k in range(len(centres)):
        for f in set(fam):
            for n in set(lev):
                sel = (fam == f) & (lev == n)
                if not sel.any():
                    continue
                r, a = v[k, sel], v32[k, sel]
                scale = np.max(np.abs(r))
                for part in (np.real, np.imag):
                    assert np.max(np.abs(part(a) - part(r)) / (1e-6 * scale + 1e-6 * np.abs(part(r)))) <= 1.0
        assert np.max(np.abs(runs["batch32"][2][k] - g[k])) <= 1e-5 * np.max(np.abs(g[k]))


def test_vjp_into_a_kept_array_and_the_reused_input_buffer(stl):
    """vjp(out=) writes the same gradients into the caller's array (the
    patches returned are views of it), forward(out=) the same statistics;
    a second forward of other values through the reused packing buffer
    equals a fresh engine's."""
    nside, J = 32, 3
    centres = np.array([100, 5000], dtype=np.int64)
    pe = stl.PatchEngine(nside, J, dtype="float64")
    ids = pe.select(centres, 20.0)
    rng = np.random.default_rng(2)
    xa = [rng.standard_normal(i.size) for i in ids]
    xb = [rng.standard_normal(i.size) for i in ids]
    va, _ = pe.forward(xa, moments=False, generation=1)
    cot = rng.standard_normal(va.shape) + 1j * rng.standard_normal(va.shape)
    ga = pe.vjp(cot, generation=1)
    out = np.empty(sum(i.size for i in ids))
    gb = pe.vjp(cot, generation=1, out=out)
    for a, b in zip(ga, gb):
        np.testing.assert_array_equal(a, b)
    assert all(np.shares_memory(b, out) for b in gb)
    with pytest.raises(ValueError):
        pe.vjp(cot, generation=1, out=np.empty(3))
    vb, _ = pe.forward(xb, moments=False, generation=2)
    kept = np.empty_like(vb)
    vk, _ = pe.forward(xb, moments=False, generation=3, out=kept)
    assert vk is kept
    np.testing.assert_array_equal(vk, vb)
    with pytest.raises(ValueError):
        pe.forward(xb, moments=False, generation=4, out=np.empty((1, 1), np.complex128))
    fresh = stl.PatchEngine(nside, J, dtype="float64")
    fresh.select(centres, 20.0)
    vb2, _ = fresh.forward(xb, moments=False, generation=1)
    np.testing.assert_array_equal(vb, vb2)
    pe.close()
    fresh.close()


def test_config4_subset_batched_equals_one_engine_per_disc(stl):
    """32 discs of the ragged workload of config 4 (nside 512, J 5, centres
    uniform on the sphere, pixel counts log-uniform in [1024, 65536]): the
    segmented engine holding all of them gives every disc's statistics and
    gradients as an engine of its own does (FP64; the same kernels over
    segment-bounded tables)."""
    nside, J, n = 512, 5, 32
    rng = np.random.default_rng(3)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    counts = np.exp(rng.uniform(np.log(1024.0), np.log(65536.0), n))
    omega = 4.0 * np.pi / (12.0 * nside * nside)
    radii = np.degrees(np.arccos(1.0 - counts * omega / (2.0 * np.pi)))
    batched = stl.PatchEngine(nside, J, dtype="float64", autotune=False)
    single = stl.PatchEngine(nside, J, dtype="float64", autotune=False, group_pixels=1)
    ids = batched.select(v, radii)
    assert [i.size for i in single.select(v, radii)] == [i.size for i in ids]
    xs = [np.random.default_rng(100 + k).standard_normal(i.size) for k, i in enumerate(ids)]
    vb, varb = batched.forward(xs, generation=1)
    vs, vars_ = single.forward(xs, generation=1)
    assert close_ratio(vb, vs, 1e-11, 1e-10) <= 1.0
    assert close_ratio(varb, vars_, 1e-11, 1e-10) <= 1.0
    cot = rng.standard_normal(vb.shape) + 1j * rng.standard_normal(vb.shape)
    gb = batched.vjp(cot, generation=1)
    gs = single.vjp(cot, generation=1)
    for a, b in zip(gb, gs):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))
    assert batched.info()["groups"] == 1 and single.info()["groups"] == n
