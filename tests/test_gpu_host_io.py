"""Host buffers through the C ABI (stlp_forward / stlp_vjp): large maps and
gradients cross through pinned chunks filled and drained by host threads.
The results equal those of the device-tensor entry points bit for bit, for
buffers of several chunks and for one smaller than a chunk, and so does the
gradient written into a caller's array (vjp out=)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


@pytest.mark.parametrize("nside,batch", [(512, 4), (128, 2)])
def test_host_buffers_equal_device_tensors(stl, nside, batch):
    import torch
    J = 4
    rng = np.random.default_rng(31)
    x = np.exp(rng.standard_normal((batch, 12 * nside * nside)) - 0.5)
    e = stl.NativeEngine(nside, J, batch=batch, dtype="float32", autotune=False)
    v_host, _ = e.forward(x, generation=1)
    cot = rng.standard_normal(v_host.shape) + 1j * rng.standard_normal(v_host.shape)
    g_host = e.vjp(cot, generation=1)
    # into a caller's array, twice (the second call overwrites the first)
    out = np.full_like(x, np.nan)
    for _ in range(2):
        g_out = e.vjp(cot, generation=1, out=out)
        assert np.shares_memory(g_out, out)
        np.testing.assert_array_equal(g_out, g_host)
    with pytest.raises(ValueError):
        e.vjp(cot, generation=1, out=np.empty(3))
    xt = torch.tensor(x, dtype=torch.float64, device="cuda")
    v_dev, _ = e.forward_tensor(xt, generation=2)
    g_dev = torch.empty_like(xt)
    e.vjp_tensor(cot, g_dev, generation=2)
    np.testing.assert_array_equal(v_host, v_dev)
    np.testing.assert_array_equal(g_host, g_dev.cpu().numpy())
    assert g_host.shape == x.shape and np.isfinite(g_host).all()
    e.close()


def test_non_finite_large_input_is_refused(stl):
    """A NaN in maps too large for the host-side scan is found while the maps
    are copied: ValueError, and the engine stays usable."""
    nside, J, batch = 512, 3, 2
    rng = np.random.default_rng(32)
    x = rng.standard_normal((batch, 12 * nside * nside))
    e = stl.NativeEngine(nside, J, batch=batch, dtype="float32", autotune=False)
    bad = x.copy()
    bad[1, 2_500_000] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        e.forward(bad, generation=1)
    bad[1, 2_500_000] = np.inf
    with pytest.raises(ValueError, match="non-finite"):
        e.forward(bad, generation=1)
    v, _ = e.forward(x, generation=2)
    assert np.isfinite(v).all()
    e.close()
