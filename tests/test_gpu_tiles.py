"""Tile heights chosen by the autotuner (rows of the field a thread takes in
the wavelet, adjoint and decimation launches) change no result: an engine that
times them at prepare and one that keeps the defaults give the same
statistics and cotangents bit for bit, on the full sky and on disc batches."""
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


@pytest.mark.parametrize("dtype,batch", [("float32", 4), ("float64", 2)])
def test_tuned_tiles_change_nothing_full_sky(stl, dtype, batch):
    nside, J = 128, 6
    rng = np.random.default_rng(21)
    x = np.exp(rng.standard_normal((batch, 12 * nside * nside)) - 0.5)
    out = {}
    for tune in (True, False):
        e = stl.NativeEngine(nside, J, batch=batch, dtype=dtype, autotune=tune)
        v, var = e.forward(x, moments=True)
        cot = np.random.default_rng(22).standard_normal(v.shape) + 1j
        g = e.vjp(cot)
        out[tune] = (v, var, g, e.info()["tile_heights"])
        e.close()
    th = np.array(out[True][3])
    assert th.shape == (J, 8) and set(th.ravel()) <= {0, 1, 2, 4}
    assert not np.array(out[False][3]).any()
    for a, b in zip(out[True][:3], out[False][:3]):
        np.testing.assert_array_equal(a, b)


def test_tuned_tiles_change_nothing_discs(stl):
    nside, J = 64, 4
    centres = np.array([10, 9000, 30000, 47000], dtype=np.int64)
    radii = np.array([9.0, 25.0, 14.0, 30.0])
    out = {}
    for tune in (True, False):
        pe = stl.PatchEngine(nside, J, dtype="float32", autotune=tune)
        ids = pe.select(centres, radii)
        rng = np.random.default_rng(23)
        patches = [rng.standard_normal(i.size) for i in ids]
        v, var = pe.forward(patches, moments=True, generation=1)
        g = pe.vjp(np.ones_like(v), generation=1)
        out[tune] = (v, var, np.concatenate(g))
        pe.close()
    for a, b in zip(out[True], out[False]):
        np.testing.assert_array_equal(a, b)


def test_tile_cache_file_is_written_and_read(stl, tmp_path):
    """autotune_cache: the heights an engine times are written to the file, and
    a new process takes them from it instead of timing (every height set to 1
    in the file, a valid choice everywhere, comes back as 1; unknown and
    malformed lines are skipped); the statistics stay the same."""
    import json
    import subprocess
    import sys
    nside, J = 64, 4
    path = tmp_path / "tiles.txt"
    x = np.exp(np.random.default_rng(24).standard_normal((2, 12 * nside * nside)) - 0.5)
    e1 = stl.NativeEngine(nside, J, batch=2, dtype="float32", autotune_cache=path)
    v1, _ = e1.forward(x)
    t1 = np.array(e1.info()["tile_heights"])
    e1.close()
    lines = path.read_text().splitlines()
    assert lines and all(line.count("\t") == 1 and line.split("\t")[1] in {"1", "2", "4"} for line in lines)
    path.write_text("".join(line.split("\t")[0] + "\t1\n" for line in lines) + "no such launch\t4\nmalformed\n")
    np.save(tmp_path / "x.npy", x)
    code = f"""
import sys, json, numpy as np
sys.path.insert(0, {str(stl.HERE)!r})
import stl_b200
e = stl_b200.NativeEngine({nside}, {J}, batch=2, dtype="float32", autotune_cache={str(path)!r})
v, _ = e.forward(np.load({str(tmp_path / 'x.npy')!r}))
np.save({str(tmp_path / 'v.npy')!r}, v)
print(json.dumps(e.info()["tile_heights"]))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    t2 = np.array(json.loads(out.stdout.strip().splitlines()[-1]))
    np.testing.assert_array_equal(t2, np.where(t1 > 0, 1, 0))
    np.testing.assert_array_equal(np.load(tmp_path / "v.npy"), v1)
