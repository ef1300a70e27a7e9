"""The disc-patch oracle (oracle/disc.py) pinned as the reference pins its disc
model (crates/stl-core/tests/disc.rs): disc pixels against a brute-force
selection, a disc of radius pi against the full-sky oracle (itself pinned to
the reference's fixtures), and the VJP against central finite differences."""
import numpy as np
import pytest

import disc as D
import oracle as O
from conftest import close_ratio


def test_disc_pixels_are_the_centres_within_the_radius():
    nside = 32
    centre = D.pixel_vectors(nside, [1234])[0]
    got = D.disc_pixels(nside, centre, 0.3)
    v = D.pixel_vectors(nside, np.arange(12 * nside * nside))
    brute = np.nonzero(np.arccos(np.clip(v @ centre, -1.0, 1.0)) <= 0.3)[0]
    assert np.array_equal(got, brute)
    assert D.disc_pixels(nside, centre, np.pi).size == 12 * nside * nside


def test_full_disc_equals_full_sky():
    nside, J = 16, 3
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, 12 * nside * nside)
    disc = D.Disc(nside, J, [0.3, -0.2, 0.9], np.pi)
    m = D.DiscModel(J)
    v, var = m.forward(disc, x, moments=True)
    o = O.OracleEngine(nside, J)
    vr, varr = o.forward(x[None], moments=True)
    assert close_ratio(v, vr[0], 1e-11, 1e-10) <= 1.0
    assert close_ratio(var, varr[0], 1e-11, 1e-10) <= 1.0
    cot = rng.uniform(-1, 1, v.size) + 1j * rng.uniform(-1, 1, v.size)
    g, gr = m.reverse(disc, cot), o.vjp(cot[None])[0]
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))


@pytest.mark.parametrize("core", [None, 35.0])
def test_disc_gradient_matches_finite_differences(core):
    nside, J = 16, 3
    disc = D.Disc(nside, J, D.pixel_vectors(nside, [700])[0], np.radians(50.0),
                  None if core is None else np.radians(core))
    if core is not None:
        assert disc.core_pixels()[0] < disc.ids[0].size
    m = D.DiscModel(J)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, disc.ids[0].size)
    m.forward(disc, x)
    cot = rng.uniform(-1, 1, len(m.plan)) + 1j * rng.uniform(-1, 1, len(m.plan))
    g = m.reverse(disc, cot)
    f = lambda y: float(np.sum((np.conj(cot) * m.forward(disc, y)).real))
    for trial in range(3):
        d = np.random.default_rng(1000 + trial).uniform(-1, 1, x.size)
        h = 1e-5
        fd = (f(x + h * d) - f(x - h * d)) / (2 * h)
        an = float(g @ d)
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1.0)


def test_masked_oracle_equals_full_sky_discs_with_the_mask_as_core():
    """K masks at once against one whole-sky disc per mask whose core is the
    mask (crates/stl-core/tests/mask.rs:38-97): values, variances and the
    summed map cotangent."""
    nside, J, B = 16, 3, 2
    npix = 12 * nside * nside
    theta = O.centres(nside, np.arange(npix))[3]
    sets = [np.arange(npix)] + [np.nonzero(np.abs(np.cos(theta)) > np.sin(np.radians(b)))[0] for b in (20.0, 45.0)]
    w = np.zeros((len(sets), npix))
    for k, s in enumerate(sets):
        w[k, s] = 1.0
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (B, npix))
    o = O.OracleEngine(nside, J, batch=B)
    o.set_masks(w)
    v, var = o.forward(x, moments=True)
    cot = rng.uniform(-1, 1, v.shape) + 1j * rng.uniform(-1, 1, v.shape)
    g = o.vjp(cot)
    m = D.DiscModel(J)
    g_ref = np.zeros_like(x)
    for k, s in enumerate(sets):
        disc = D.Disc(nside, J, [0.0, 0.0, 1.0], np.pi)
        core, cc = [], s
        for n in range(J):
            core.append(np.searchsorted(disc.ids[n], cc))
            cc = np.unique(cc >> 2)
        disc.core = core
        for b in range(B):
            vr, varr = m.forward(disc, x[b], moments=True)
            assert close_ratio(v[b, k], vr, 1e-11, 1e-10) <= 1.0
            assert close_ratio(var[b, k], varr, 1e-11, 1e-10) <= 1.0
            g_ref[b] += m.reverse(disc, cot[b, k])
    assert np.max(np.abs(g - g_ref)) <= 1e-10 * np.max(np.abs(g_ref))
