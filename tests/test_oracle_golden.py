"""The FP64 CPU oracle against the reference's golden fixtures.

Mirrors the reference's own tests: crates/stl-core/tests/geometry.rs
(centres, ring2nest, interpolation, rotations, kernel grid, convolution
geometry + forward, decimation weights, neighbourhoods), tests/block.rs
(wavelet kernel) and tests/stats.rs (statistics, stored moduli, per-level
map cotangents and band cotangents of all 8 stats cases, with the same
tolerances).  Passing these pins the oracle the CUDA engine is checked
against.
"""
import numpy as np
import pytest

import oracle as O
from conftest import cases, close_ratio

TOL = 1e-12  # geometry.rs:17


def weight_tol(nside):  # geometry.rs:72-74
    return max(TOL, 1e-14 * nside)


def conv_noise(ids, nside):  # tests/common/mod.rs:85-89
    th = O.centres(nside, ids)[3]
    s = np.maximum(np.sin(th), 1.0 / nside)
    return np.maximum(1e-12, np.finfo(float).eps * 128.0 * nside / s)


def as_operator(pix, w):
    m = {}
    for p, v in zip(pix, w):
        m[int(p)] = m.get(int(p), 0.0) + float(v)
    return m


def same_operator(a, b, tol):
    return all(abs(a.get(k, 0.0) - b.get(k, 0.0)) <= tol for k in set(a) | set(b))


@pytest.mark.parametrize("case", cases("geometry", "centres"), ids=lambda c: c.name)
def test_centres(case):
    ix, iy, f, th, ph, lo, la = O.centres(case["nside"], case.npy("ids"))
    assert np.array_equal(ix, case.npy("ix")) and np.array_equal(iy, case.npy("iy"))
    assert np.array_equal(f, case.npy("face"))
    for mine, name in [(th, "theta"), (ph, "phi"), (lo, "lon"), (la, "lat")]:
        assert np.max(np.abs(mine - case.npy(name))) <= 1e-14


@pytest.mark.parametrize("case", cases("geometry", "ring2nest"), ids=lambda c: c.name)
def test_ring2nest(case):
    assert np.array_equal(O.ring2nest(case["order"], case.npy("ring")), case.npy("nest"))


@pytest.mark.parametrize("case", cases("geometry", "interp"), ids=lambda c: c.name)
def test_interpolation(case):
    nside = case["nside"]
    order = int(np.log2(nside))
    p, w = O.interp_ring(nside, case.npy("theta"), case.npy("phi"))
    pr, wr = case.npy("pix_ring").reshape(-1, 4), case.npy("w_ring").reshape(-1, 4)
    p2, w2 = O.interp_nested(order, case.npy("vecs"))
    pn, wn = case.npy("pix_nest").reshape(-1, 4), case.npy("w_nest").reshape(-1, 4)
    for i in range(len(p)):
        assert same_operator(as_operator(p[i], w[i]), as_operator(pr[i], wr[i]), TOL), i
        assert same_operator(as_operator(p2[i], w2[i]), as_operator(pn[i], wn[i]), weight_tol(nside)), i


@pytest.mark.parametrize("case", cases("geometry", "rotation"), ids=lambda c: c.name)
def test_rotations(case):
    r = O.rotations(case.npy("theta"), case.npy("phi"), case["G"], case["gauge"])
    assert np.max(np.abs(r.ravel() - case.npy("R").ravel())) <= 1e-14


@pytest.mark.parametrize("case", cases("geometry", "kernel_grid"), ids=lambda c: c.name)
def test_kernel_grid(case):
    v = O.kernel_grid(case["kernel_sz"], case["nside"])
    assert np.max(np.abs(v.ravel() - case.npy("vec").ravel())) <= 1e-15


@pytest.mark.parametrize("case", cases("block", "wavelet"), ids=lambda c: c.name)
def test_wavelet_kernel(case):
    w = O.wavelet_weights(case["kernel_sz"])
    assert np.max(np.abs(w - case.npy("weights").ravel())) <= 1e-15


@pytest.mark.parametrize("case", cases("geometry", "conv"), ids=lambda c: c.name)
def test_convolution_geometry_and_forward(case):
    nside, ksz, G, gauge = case["nside"], case["kernel_sz"], case["G"], case["gauge"]
    ids = case.npy("ids")
    pos, w, complete = O.bind(ids, nside, ksz, G, gauge)
    assert np.array_equal(complete, case.npy("complete").astype(bool))
    weights = case.npy("weights").ravel()
    f32 = np.tile(weights.astype(np.float32).astype(np.float64), G)
    assert np.array_equal(f32, case.npy("weight_f32").ravel())
    if case.has("pos_safe"):  # raw binding as operators on complete rows
        shape = (4, G, len(ids), ksz * ksz)
        rp, rw = case.npy("pos_safe").reshape(shape), case.npy("w_norm").reshape(shape)
        for k in np.nonzero(complete)[0]:
            for g in range(G):
                for t in range(ksz * ksz):
                    assert same_operator(as_operator(pos[:, g, k, t], w[:, g, k, t]),
                                         as_operator(rp[:, g, k, t], rw[:, g, k, t]), weight_tol(nside))
    y = O.conv_forward(case.npy("x").reshape(1, -1), nside, ksz, G, gauge, grid=ids, weights=weights)
    y = y.reshape(2 * G, -1)
    ref = case.npy("y").reshape(2 * G, -1)
    ratio = np.max((np.abs(y - ref) / conv_noise(ids, nside))[:, complete])
    assert ratio <= 1.0, ratio


@pytest.mark.parametrize("case", cases("geometry", "down"), ids=lambda c: c.name)
def test_decimation_weights(case):
    coarse, indptr, indices, values = O.smooth_decimation(case.npy("ids"), case["nside"])
    assert np.array_equal(coarse, case.npy("coarse_ids"))
    rows = np.repeat(np.arange(len(coarse)), np.diff(indptr))
    assert np.array_equal(rows, case.npy("rows"))
    assert np.array_equal(indices, case.npy("cols"))
    assert np.max(np.abs(values - case.npy("values"))) <= TOL


@pytest.mark.parametrize("case", cases("geometry", "neighbours"), ids=lambda c: c.name)
def test_neighbourhoods_as_sets(case):
    """kth_neighbourhood restated on the face frames: same cell sets as cdshealpix 0.10.1."""
    nb, ids = case.npy("neighbours"), case.npy("ids")
    for i, pid in enumerate(ids):
        expected = sorted(int(v) for v in nb[i] if v >= 0)
        assert sorted(O.kth_neighbourhood(pid, case["nside"], case["k"]).tolist()) == expected, pid


FAMILY = {"mean": 0, "var": 1, "S1": 2, "S2": 3, "S3": 4, "S4": 5}


def oracle_for(case):
    return O.OracleEngine(case["nside"], case["J"], L=case["L"], kernel=case["kernel_sz"], batch=case["batch"],
                          channels=case["channels"], fewer=case["fewer"], j_to_dg=case["j_to_dg"],
                          gauge=case["gauge"])


@pytest.mark.parametrize("case", cases("stats", "stats"), ids=lambda c: c.name)
def test_statistics_and_gradients(case):
    """tests/stats.rs:165-209 on the full-sky oracle."""
    import json
    e = oracle_for(case)
    plan = json.loads((case.dir / "plan.json").read_text())
    rows = [[FAMILY[r[0]]] + [-1 if v is None else v for v in r[1:]] for r in plan]
    assert np.array_equal(np.array(rows), e.plan_rows)
    values = e.forward(case.npy("map0"))
    for d in range(e.levels):
        assert np.max(np.abs(e.map(d).ravel() - case.npy(f"map{d}").ravel())) <= 1e-12
        for n in range(d + 1, e.levels):
            assert np.max(np.abs(e.m(d, n).ravel() - case.npy(f"m{d}_{n}").ravel())) <= 1e-12
    ref = case.complex("values").reshape(values.shape)
    assert close_ratio(values.real, ref.real, 1e-11, 1e-10) <= 1.0
    assert close_ratio(values.imag, ref.imag, 1e-11, 1e-10) <= 1.0
    mg = e.reverse(case.complex("gradient").reshape(values.shape))
    for d in range(e.levels):
        assert close_ratio(mg[d], case.npy(f"maps_gradient{d}"), 1e-10, 1e-9) <= 1.0
    _, bands = e.analysis()
    for d in range(e.levels):
        assert close_ratio(bands[d], case.npy(f"band_gradient{d}"), 1e-10, 1e-9) <= 1.0


def test_gradient_matches_finite_difference():
    """tests/stats.rs:76-108: directional derivative vs central difference, rel <= 1e-7."""
    case = next(c for c in cases("stats", "stats") if c.name == "stats_n16_J3_L2_k3_C2_B2_full_b64")
    e = oracle_for(case)
    x = case.npy("map0").ravel()
    g = case.complex("gradient").reshape(e.batch, e.ncoeff)
    e.forward(x)
    grad = e.vjp(g).ravel()
    v = np.random.default_rng(5).random(x.size) - 0.5
    pairing = lambda y: float(np.sum((np.conj(g) * e.forward(y)).real))
    eps = 1e-5
    fd = (pairing(x + eps * v) - pairing(x - eps * v)) / (2 * eps)
    exact = float(grad @ v)
    assert abs(fd - exact) / abs(exact) <= 1e-7


def test_spatial_variance_of_mean_and_var():
    """tests/stats.rs:138-163: moments of mean/var are the variances of x and x^2."""
    case = next(c for c in cases("stats", "stats") if c.name == "stats_n16_J3_L2_k3_C2_B2_full_b64")
    e = oracle_for(case)
    x = case.npy("map0").reshape(e.batch, e.channels, -1)
    v1 = e.forward(x)
    v2, var = e.forward(x, moments=True)
    assert np.array_equal(v1, v2)
    for i, c in enumerate(e.plan()):
        if c["family"] not in ("mean", "var"):
            continue
        for b in range(e.batch):
            f = x[b, c["c1"]] if c["family"] == "mean" else x[b, c["c1"]] ** 2
            expect = np.mean((f - f.mean()) ** 2)
            assert abs(var[b, i] - expect) <= 1e-12 * expect
    assert np.all(var >= 0)


def test_mask_of_whole_sky_equals_full_sky():
    """A mask holding every pixel averages like the full sky (crates/stl-core/tests/mask.rs)."""
    e = O.OracleEngine(16, 3)
    x = np.random.default_rng(0).standard_normal(12 * 16 * 16)
    full = e.forward(x)
    e.set_masks(np.ones((2, x.size)))
    masked = e.forward(x)
    assert masked.shape == (1, 2, e.ncoeff)
    assert np.max(np.abs(masked[:, 0] - full)) <= 1e-14
    assert np.max(np.abs(masked[:, 1] - full)) <= 1e-14


def test_oracle_forward_levels_on_fixture_pyramid():
    """The oracle's forward_levels on the fixture's level maps gives the golden values."""
    case = next(c for c in cases("stats", "stats") if c.name == "stats_n16_J3_L4_k5_C1_B1_full_b256")
    o = O.OracleEngine(16, 3)
    levels = [case.npy(f"map{d}").reshape(1, -1) for d in range(3)]
    values = o.forward_levels(levels)
    ref = case.complex("values").reshape(values.shape)
    assert close_ratio(values, ref, 1e-11, 1e-10) <= 1.0
