"""The C ABI boundary on the CPU: the library loads, exports every symbol
include/stl_b200.h declares, builds handles and plans without a device, and
reports configuration errors the way the reference's bridge does
(crates/stl-bridge/src/lib.rs:75-94: -1 / NULL and stlp_last_error)."""
import ctypes as C
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, PKG

import oracle as O


def header_symbols():
    text = (ROOT / "include" / "stl_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(stlp_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def stl():
    import stl_b200
    return stl_b200


def test_library_exports_every_declared_symbol(stl):
    lib = C.CDLL(str(stl.library_path()))
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert len(header_symbols()) >= 55


def test_symbols_are_dynamic_exports():
    out = subprocess.run(["nm", "-D", "--defined-only", str(PKG / "libstl_b200.so")], capture_output=True, text=True)
    exported = set(re.findall(r"\b(stlp_\w+)\b", out.stdout))
    assert set(header_symbols()) <= exported


@pytest.mark.parametrize("nside,J", [(16, 3), (32, 4), (64, 5), (1024, 9)])
def test_plan_matches_the_reference_plan(stl, nside, J):
    """The plan in stlp_info is the reference's build_plan (plan.rs:80-158)."""
    e = stl.NativeEngine(nside, J)
    ref = O.build_plan(J)
    assert e.ncoeff == len(ref)
    assert [dict(c) for c in e.plan] == ref
    counts = {3: 762, 5: 2522, 7: 5882, 9: 11354, 10: 15042}
    if J in counts:
        assert e.ncoeff == counts[J]
    e.close()


def test_info_reports_sizes_and_dtype(stl):
    e = stl.NativeEngine(32, 4, batch=3, dtype="float32")
    info = e.info()
    assert info["nside"] == 32 and info["batch"] == 3 and info["levels"] == 4
    assert info["dtype"].startswith("float32")
    assert e.native_pixels().tolist() == [12 * (32 >> c["native_dg"]) ** 2 for c in e.plan]


@pytest.mark.parametrize("config,message", [
    ({"nside": 12, "j": 2, "backend": "gpu"}, "power of two"),
    ({"nside": 16, "j": 6, "backend": "gpu"}, "scales"),
    ({"nside": 16, "j": 3, "backend": "cpu"}, "backend"),
    ({"nside": 16, "j": 3, "batch": 0, "backend": "gpu"}, "batch"),
    ({"nside": 16, "j": 3, "dtype": "float16", "backend": "gpu"}, "dtype"),
    ({"nside": 16, "j": 3, "orientations": 2, "backend": "gpu"}, "orientations"),
    ({"nside": 16, "j": 3, "spin": 1}, "spin must be 0 or 2"),
    ({"nside": 16, "j": 3, "spin": 2, "spin_kernel": 4}, "spin_kernel"),
    ({"nside": 16, "j": 3, "spin": 2, "spin_pyramid": "flat"}, "spin_pyramid"),
    ({"nside": 16, "j": 3, "spin": 2, "cross": True, "spin_pyramid": "transported"}, "scalar pyramid"),
    ({"nside": 16, "j": 3, "spin": 2, "cross": True, "spin_a": 1}, "spin_a"),
])
def test_bad_configs_fail_with_a_message(stl, config, message):
    lib = stl.lib()
    assert not lib.stlp_new(json.dumps(config).encode())
    assert message in lib.stlp_last_error().decode()


def test_malformed_json(stl):
    lib = stl.lib()
    assert not lib.stlp_new(b"{nside: 16")
    assert "JSON" in lib.stlp_last_error().decode()


def test_vjp_without_forward_is_refused(stl):
    e = stl.NativeEngine(16, 3)
    with pytest.raises(RuntimeError, match="stale"):
        e.vjp(np.zeros(e.ncoeff, complex))
    lib = stl.lib()
    c = np.zeros(2 * e.ncoeff)
    out = np.zeros(e.npix)
    assert lib.stlp_vjp(e._handle, stl._ptr(c), e.ncoeff, 0, 0, 0, stl._ptr(out)) == -1
    assert "stale" in lib.stlp_last_error().decode()


def test_python_side_checks(stl):
    e = stl.NativeEngine(16, 3)
    with pytest.raises(ValueError, match="expected maps"):
        e.forward(np.zeros(10))
    with pytest.raises(ValueError, match="non-finite"):
        e.forward(np.full(e.npix, np.nan))
    with pytest.raises(ValueError, match="backend"):
        stl.NativeEngine(16, 3, backend="cpu")


def test_spin_handle_shapes(stl):
    """Spin 2: (Q, U) maps, values of chi_E and chi_B; the operators are built
    at the first use, so the handle's description needs no device."""
    e = stl.NativeEngine(16, 3, batch=2, spin=2, spin_pyramid="transported")
    info = e.info()
    assert info["spin"] == 2 and info["spin_pyramid"] == "transported" and info["spin_kernel"] == 5
    assert info["batch"] == 4 and info["spin_batch"] == 2  # the engine's maps: chi_E, chi_B of each
    assert e._map_shape == (2, 2, 3072) and e._shape() == (2, 2, e.ncoeff)
    c = stl.NativeEngine(16, 3, batch=2, spin=2, cross=True, spin_a=0)
    assert c._map_shape == (2, 3, 3072) and c.info()["spin_a"] == 0
    with pytest.raises(ValueError, match="pair"):
        c._input(np.zeros((2, 3, 3072)))


def test_out_of_scope_entry_points_fail_cleanly(stl):
    lib = C.CDLL(str(stl.library_path()))
    lib.stlp_spec_new.restype = C.c_void_p
    lib.stlp_last_error.restype = C.c_char_p
    assert not lib.stlp_spec_new(b"{}")
    assert b"not built" in lib.stlp_last_error()


# the reference checkout (STL_REFERENCE_ROOT, default /root/reference): its
# unmodified Python binding, where the checkout is mounted
REFERENCE_ROOT = Path(os.environ.get("STL_REFERENCE_ROOT", "/root/reference"))
REFERENCE_NATIVE = REFERENCE_ROOT / "python" / "stl_ensemble" / "stl_port" / "native.py"


@pytest.mark.skipif(not REFERENCE_NATIVE.exists(), reason="the reference checkout is not mounted")
def test_reference_native_py_binds_this_library(tmp_path):
    """The reference's unmodified ctypes binding loads libstl_b200.so (all of its
    signature table resolves) and builds a handle whose plan has 762 coefficients."""
    code = f"""
import importlib.util, os, sys
os.environ['STL_NATIVE_LIBRARY'] = {str(PKG / 'libstl_b200.so')!r}
spec = importlib.util.spec_from_file_location('native_ref', {str(REFERENCE_NATIVE)!r})
m = importlib.util.module_from_spec(spec); spec.loader.exec_module(m)
e = m.NativeEngine(16, 3, backend='gpu')
print('NCOEFF', e.ncoeff)
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert "NCOEFF 762" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("config,message", [
    ({"rows": 2, "len": 100, "depth": 2}, "aligned"),
    ({"rows": 1, "len": 64, "depth": 31}, "depth"),
])
def test_terms_configuration_errors(stl, config, message):
    """stlp_terms_new validates its sizes before it touches a device."""
    lib = stl.lib()
    assert not lib.stlp_terms_new(json.dumps(config).encode())
    assert message in lib.stlp_last_error().decode()
