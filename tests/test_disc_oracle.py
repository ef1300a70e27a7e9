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
