"""The synthesis objective's terms on the device (stlp_terms_*) against the
FP64 oracle of oracle/terms.py, which its CPU tests pin to the host loops of
the reference's tests (crates/stl-gpu/tests/terms.rs): the sort's permutation
exactly (total order, ties by position), the pyramid levels and the
level-power, kurtosis, marginal and add-product gradients bit for bit, the
detail moments and the marginal's loss to 1e-13 relative (chunked sums)."""
import numpy as np
import pytest

import terms as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def cuda(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def awkward(seed, n):
    """Heavy-tailed values with repeats, signed zeros, infinities, NaNs of
    both signs, subnormals and huge magnitudes."""
    rng = np.random.default_rng(seed)
    x = rng.standard_t(2.0, n) * 3.0
    x[rng.random(n) < 0.05] = 0.5   # repeats: their order is their positions'
    x[rng.random(n) < 0.05] = -2.25
    special = np.array([0.0, -0.0, 1.5, -1.5, np.inf, -np.inf, np.nan, -np.nan, 5e-324, -5e-324, 1e300, -1e300])
    pick = rng.random(n) < 0.08
    x[pick] = special[rng.integers(0, special.size, int(pick.sum()))]
    return x


@pytest.mark.parametrize("n", [1, 7, 4095, 4096, 4097, 300_001, 1 << 20])
def test_sort_is_the_stable_total_order(stl, n):
    x = awkward(n, n)
    t = stl.Terms(sort=n)
    perm = t.sort(cuda(x)).cpu().numpy().astype(np.int64)
    np.testing.assert_array_equal(perm, T.sort_positions(x))
    t.close()


@pytest.fixture(scope="module")
def pyr(stl):
    rows, length, depth = 3, 4 ** 7, 6
    rng = np.random.default_rng(21)
    x = np.clip(rng.standard_t(3.0, (rows, length)) * 4.0, -50.0, 50.0)
    x[:, ::97] = 0.25
    t = stl.Terms(rows=rows, length=length, depth=depth)
    xd = cuda(x)
    t.pyramid(xd)
    return t, x, xd, T.pyramid(x, depth)


def test_pyramid_levels_bit_exact(pyr):
    t, x, xd, levels = pyr
    import torch
    # the device levels through the level-power gradient of one level at a time:
    # coef 1 on level n alone gives d_n = level n - its parent, exactly
    for n in range(t.depth):
        coef = np.zeros((t.rows, t.depth))
        coef[:, n] = 1.0
        g = torch.zeros_like(xd)
        t.level_power_grad(xd, coef[:, : n + 1], g)
        want = T.level_power_grad(levels, coef[:, : n + 1], np.zeros_like(x))
        np.testing.assert_array_equal(g.cpu().numpy(), want)


def test_detail_moments(pyr):
    t, x, xd, levels = pyr
    got = t.moments(xd)
    want = T.detail_moments(levels)
    assert np.all(np.abs(got - want) <= 1e-13 * np.abs(want))


def test_level_power_gradient(pyr):
    t, x, xd, levels = pyr
    coef = 0.3 + 0.01 * np.arange(t.rows * t.depth).reshape(t.rows, t.depth)
    g0 = np.random.default_rng(9).standard_normal(x.shape)
    g = cuda(g0)
    t.level_power_grad(xd, coef, g)
    np.testing.assert_array_equal(g.cpu().numpy(), T.level_power_grad(levels, coef, g0))


@pytest.mark.parametrize("chain", [False, True])
def test_kurtosis_gradient(pyr, chain):
    t, x, xd, levels = pyr
    lev = [0, 2, 5]
    k = np.arange(t.rows * len(lev), dtype=np.float64).reshape(t.rows, len(lev))
    cf = np.stack([0.7 - 0.05 * k, 3.0 + 0.1 * k, 0.2 + 0.01 * k], axis=-1)
    rng = np.random.default_rng(4)
    g0 = rng.standard_normal(x.shape)
    dk = 1.0 + 0.5 * rng.standard_normal(x.shape) if chain else None
    g = cuda(g0)
    t.kurtosis_grad(xd, lev, cf, g, None if dk is None else cuda(dk))
    np.testing.assert_array_equal(g.cpu().numpy(), T.kurtosis_grad(levels, lev, cf, g0, dk))


def test_marginal_and_add_product(stl):
    n = 300_001
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n) * 2.0
    target = np.sort(rng.standard_normal(n))
    g0 = rng.standard_normal(n)
    t = stl.Terms(length=n, sort=n)
    xd = cuda(x)
    perm = t.sort(xd)
    g = cuda(g0)
    s = t.marginal(xd, perm, cuda(target), 2.0 / n, g)
    want_g, want_s = T.marginal_row(x, T.sort_positions(x), target, 2.0 / n, g0)
    np.testing.assert_array_equal(g.cpu().numpy(), want_g)
    assert abs(s - want_s) <= 1e-13 * want_s
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    t.add_product(g, cuda(a), cuda(b))
    np.testing.assert_array_equal(g.cpu().numpy(), T.add_product(want_g, a, b))
    t.add_product(g, cuda(a))
    np.testing.assert_array_equal(g.cpu().numpy(), T.add_product(T.add_product(want_g, a, b), a))


def test_kappa_transform(stl):
    kx = np.linspace(-3.0, 4.0, 41)
    ky = np.tanh(kx) + 0.1 * kx
    kd = 1.0 / np.cosh(kx) ** 2 + 0.1
    x = np.random.default_rng(6).standard_normal(200_000) * 2.5
    x[:5] = [kx[0], kx[-1], kx[7], -100.0, 100.0]
    gm, gs, km, ks = 0.2, 1.3, 0.05, 0.9
    t = stl.Terms()
    t.kappa_table(kx, ky, kd)
    k, dk = t.kappa(cuda(x), gm, gs, km, ks)
    wk, wdk = T.kappa_pchip(x, kx, ky, kd, gm, gs, km, ks)
    np.testing.assert_array_equal(k.cpu().numpy(), wk)
    np.testing.assert_array_equal(dk.cpu().numpy(), wdk)
