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


def test_device_synthesis_follows_host_lbfgs(stl):
    """stlp_synthesize_device (iterate, gradients and history in device memory)
    takes the steps of the host L-BFGS over the same FP64 engine: the same loss
    after every evaluation, up to the order of the dot-product sums."""
    import torch
    nside, J = 16, 3
    rng = np.random.default_rng(10)
    target_map = np.exp(rng.standard_normal((1, 12 * nside * nside)) - 0.5)
    x0 = rng.standard_normal((1, 12 * nside * nside)) * target_map.std() + target_map.mean()
    e = stl.NativeEngine(nside, J, dtype="float64")
    target, _ = e.forward(target_map)
    w = 1.0 / (1.0 + np.arange(e.ncoeff) % 7)
    opts = dict(max_iter=8, history_size=4)
    xh, rep = stl.native_lbfgs(stl.synthesis_objective(e, target, weights=w), x0.copy(), opts)
    xd = torch.tensor(x0, device="cuda")
    n, losses = e.synthesize(xd, target, weights=w, options=opts)
    want = np.array(rep["loss_history"])
    assert n == len(want) == len(losses)
    assert np.max(np.abs(losses - want) / want) <= 1e-9
    assert np.max(np.abs(xd.cpu().numpy() - xh)) <= 1e-9 * np.max(np.abs(xh))
    # the handle's forward state was cleared: a vjp needs a new forward
    with pytest.raises(RuntimeError, match="stale"):
        e.vjp(np.zeros((1, e.ncoeff), complex), generation=0)


def test_device_synthesis_refuses_bad_shapes(stl):
    import torch
    e = stl.NativeEngine(16, 3, dtype="float32")
    x = torch.zeros(1, 12 * 16 * 16, device="cuda", dtype=torch.float64)
    with pytest.raises(RuntimeError, match="target shape mismatch"):
        e.synthesize(x, np.zeros(e.ncoeff - 1, complex))
    with pytest.raises(ValueError, match="CUDA float64"):
        e.synthesize(x.float(), np.zeros(e.ncoeff, complex))
    e.close()


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_graph_iterations_equal_step_by_step(stl, dtype):
    """Iterations 2 on as one CUDA graph launch each (the default) take the
    same steps as the step-by-step device path: the same losses after every
    evaluation and the same iterate, bit for bit (same reductions, same
    order); with FP64 both follow the host L-BFGS."""
    import torch
    nside, J = 32, 4
    rng = np.random.default_rng(12)
    target_map = np.exp(rng.standard_normal((1, 12 * nside * nside)) - 0.5)
    x0 = rng.standard_normal((1, 12 * nside * nside)) * target_map.std() + target_map.mean()
    e = stl.NativeEngine(nside, J, dtype=dtype)
    target, var = e.forward(target_map, moments=True)
    w = 1.0 / np.maximum(var.reshape(-1), 1e-12 * var.max())
    opts = dict(max_iter=12, history_size=4)
    runs = {}
    for graph in (False, True):
        xd = torch.tensor(x0, device="cuda")
        n, losses = e.synthesize(xd, target, weights=w, options=dict(opts, graph=graph))
        runs[graph] = (n, losses, xd.cpu().numpy())
    assert runs[True][0] == runs[False][0] > 12
    np.testing.assert_array_equal(runs[True][1], runs[False][1])
    np.testing.assert_array_equal(runs[True][2], runs[False][2])
    assert runs[True][1][-1] < 0.5 * runs[True][1][0]
    if dtype == "float64":
        xh, rep = stl.native_lbfgs(stl.synthesis_objective(e, target, weights=w), x0.copy(), opts)
        want = np.array(rep["loss_history"])
        assert len(want) == runs[True][0]
        assert np.max(np.abs(runs[True][1] - want) / want) <= 1e-9
    e.close()
