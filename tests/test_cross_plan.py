"""The cross plan of two channels (config "cross"): the coefficients the
library lists are the oracle's cross-only plan, in its order (the reference's
plan_of with cross, crates/stl-bridge/src/lib.rs:238-245), and the handle
reports two channels.  No GPU needed: the plan comes from stlp_info."""
import oracle as O
import pytest


@pytest.fixture(scope="module")
def stl():
    import stl_b200
    return stl_b200


@pytest.mark.parametrize("J", [1, 3, 5])
def test_cross_plan_matches_oracle(stl, J):
    e = stl.NativeEngine(16 if J < 5 else 32, J, batch=2, cross=True)
    info = e.info()
    assert info["channels"] == 2 and info["cross"] is True and info["batch"] == 2
    want = O.build_plan(J, 4, channels=2, cross_only=True)
    got = info["plan"]
    assert len(got) == len(want) == e.ncoeff
    keys = ("family", "native_dg", "c1", "c2", "j1", "j2", "j3", "l1", "l2", "l3")
    for a, b in zip(got, want):
        assert tuple(a[k] for k in keys) == tuple(b[k] for k in keys)
    assert all(c["c1"] != c["c2"] for c in got)
    e.close()
