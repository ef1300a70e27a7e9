"""Synthesis (L-BFGS over the GPU engine's forward + VJP) against the same
optimiser over the FP64 CPU oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def test_fp64_synthesis_follows_oracle(stl):
    nside, J = 16, 3
    rng = np.random.default_rng(8)
    target_map = np.exp(rng.standard_normal((1, 12 * nside * nside)) - 0.5)
    x0 = rng.standard_normal((1, 12 * nside * nside)) * target_map.std() + target_map.mean()
    o = O.OracleEngine(nside, J)
    e = stl.NativeEngine(nside, J, dtype="float64")
    target = o.forward(target_map)

    def oracle_fun(x):
        r = o.forward(x.reshape(1, -1)) - target
        return float(np.sum(r.real ** 2 + r.imag ** 2)), o.vjp(2.0 * r).reshape(x.shape)

    opts = dict(max_iter=6, history_size=5)
    _, ref = stl.native_lbfgs(oracle_fun, x0.copy(), opts)
    x, rep = stl.native_lbfgs(stl.synthesis_objective(e, target), x0.copy(), opts)
    got, want = np.array(rep["loss_history"]), np.array(ref["loss_history"])
    assert len(got) == len(want)
    assert np.max(np.abs(got - want) / want) <= 1e-8
    assert got.min() < 0.9 * got[0]


def test_fp32_synthesis_decreases_loss(stl):
    nside, J = 32, 4
    rng = np.random.default_rng(9)
    target_map = np.exp(rng.standard_normal((1, 12 * nside * nside)) - 0.5)
    x0 = rng.standard_normal((1, 12 * nside * nside)) * target_map.std() + target_map.mean()
    e = stl.NativeEngine(nside, J, dtype="float32")
    target, _ = e.forward(target_map)
    x, rep = stl.native_lbfgs(stl.synthesis_objective(e, target), x0.copy(), dict(max_iter=15))
    h = np.array(rep["loss_history"])
    assert np.isfinite(h).all() and h.min() < 0.5 * h[0]
