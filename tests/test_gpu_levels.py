"""stlp_forward_levels (maps given at every level, no decimation of level 0)
against the oracle and the reference's fixture pyramid."""
import numpy as np
import pytest

import oracle as O
from conftest import cases, close_ratio

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stl():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200
    return stl_b200


def test_fixture_pyramid_reproduces_values(stl):
    """The fixture's maps at every level are the decimation pyramid of map0:
    the statistics from them equal the golden values (tests/stats.rs tolerances)."""
    case = next(c for c in cases("stats", "stats") if c.name == "stats_n16_J3_L4_k5_C1_B1_full_b256")
    e = stl.NativeEngine(16, 3, dtype="float64")
    levels = [case.npy(f"map{d}").reshape(1, -1) for d in range(3)]
    values = e.forward_levels(levels)
    ref = case.complex("values").reshape(values.shape)
    assert close_ratio(values, ref, 1e-11, 1e-10) <= 1.0


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_independent_levels_match_oracle(stl, dtype):
    nside, J, B = 32, 4, 2
    rng = np.random.default_rng(21)
    levels = [rng.standard_normal((B, 12 * (nside >> d) ** 2)) for d in range(J)]
    if dtype == "float32":
        levels = [v.astype(np.float32).astype(np.float64) for v in levels]
    ref = O.OracleEngine(nside, J, batch=B).forward_levels(levels)
    e = stl.NativeEngine(nside, J, batch=B, dtype=dtype)
    values = e.forward_levels(levels)
    if dtype == "float64":
        assert close_ratio(values, ref, 1e-11, 1e-10) <= 1.0
    else:
        assert np.max(np.abs(values - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_no_vjp_after_levels_and_shape_checked(stl):
    nside, J = 16, 3
    e = stl.NativeEngine(nside, J, dtype="float64")
    rng = np.random.default_rng(2)
    levels = [rng.standard_normal((1, 12 * (nside >> d) ** 2)) for d in range(J)]
    v = e.forward_levels(levels)
    with pytest.raises(RuntimeError):
        e.vjp(np.ones_like(v))
    with pytest.raises(RuntimeError, match="shape"):
        e.forward_levels(levels[:2])
    # a regular forward afterwards decimates level 0 again
    x = levels[0]
    o = O.OracleEngine(nside, J)
    assert close_ratio(e.forward(x)[0], o.forward(x), 1e-11, 1e-10) <= 1.0
