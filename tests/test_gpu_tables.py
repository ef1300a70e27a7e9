"""The integer tables of the device operators, exactly: the distinct input
cells each pixel's wavelet reads (the bound rotated stencils, the per-row
form of the reference's DIA tables, crates/stl-core/src/conv.rs:73-135 and
dia.rs:213-238) and the fine cells of every coarse pixel's smooth
decimation (the 2-ring coarse neighbourhood's children within the cut,
decimation.rs:108-201, through cdshealpix's kth_neighbourhood restated in
the oracle and pinned to the reference's neighbour fixtures), against the
FP64 oracle as sorted sets with np.array_equal.  FP64 engines hold the
coloured layout, FP32 engines above nside 32 the tensor-core layout: both
are read back."""
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


def padded(rows, width):
    out = np.full((rows.shape[0], width), -1, np.int64)
    out[:, : rows.shape[1]] = rows
    return out


def strong_sets(cells, weights, floor):
    """rows of cells whose weight exceeds floor (the rest -1), sorted, and the
    weak cells' count: a bilinear weight that is exactly zero with one libm
    can be 1e-17 with another, so cells of negligible weight are compared as
    weak, not as members of the set."""
    keep = (cells >= 0) & (weights > floor)
    out = np.where(keep, cells, np.iinfo(np.int64).max)
    out.sort(axis=1)
    out[out == np.iinfo(np.int64).max] = -1
    return out, int(((cells >= 0) & ~keep).sum())


@pytest.mark.parametrize("nside,J,dtype", [(16, 3, "float64"), (64, 3, "float64"), (64, 3, "float32"),
                                           (256, 2, "float32"), (256, 2, "float64")])
def test_wavelet_cells_exact(stl, nside, J, dtype):
    """Every cell of weight above 1e-12 (bound weight in the oracle; largest
    |coefficient| on the device, the bound weight times the f32-rounded
    wavelet) is read by the same pixel on both sides, exactly; cells below
    it are the rounding of exact zeros and are only counted."""
    e = stl.NativeEngine(nside, J, dtype=dtype)
    e.prepare()
    layout = e.info()["operators"]
    for level in range(J):
        ns = nside >> level
        dev, dw = e.operator_rows(level, "wavelet")
        npx = 12 * ns * ns
        assert dev.shape[0] == npx
        # every pixel at nside <= 64; a seeded sample of 40 000 above
        rows = np.arange(npx) if npx <= 49152 else np.sort(np.random.default_rng(ns).choice(npx, 40_000, False))
        ref, rw = O.row_cells(rows, ns)
        a, weak_dev = strong_sets(dev[rows], dw[rows], 1e-12)
        b, weak_ref = strong_sets(ref, rw, 1e-12)
        w = max(a.shape[1], b.shape[1])
        print(f"nside {ns} {dtype} ({layout[level]['layout']}): {a.shape[0]} rows, weak cells device {weak_dev} "
              f"oracle {weak_ref}")
        assert np.array_equal(padded(a, w), padded(b, w)), (level, layout[level]["layout"])
    e.close()


@pytest.mark.parametrize("nside,J", [(16, 3), (64, 3), (256, 3)])
def test_decimation_columns_exact(stl, nside, J):
    for dtype in ("float64", "float32"):
        e = stl.NativeEngine(nside, J, dtype=dtype)
        e.prepare()
        for level in range(J - 1):
            ns = nside >> level
            coarse, indptr, indices, values = O.smooth_decimation(None, ns)
            dev, _ = e.operator_rows(level, "decimation")
            assert dev.shape[0] == coarse.size == 12 * (ns // 2) ** 2
            width = max(dev.shape[1], int(np.diff(indptr).max()))
            ref = np.full((coarse.size, width), -1, np.int64)
            for i in range(coarse.size):
                cols = np.sort(indices[indptr[i]:indptr[i + 1]][values[indptr[i]:indptr[i + 1]] != 0])
                ref[coarse[i], : cols.size] = cols
            assert np.array_equal(padded(dev, width), ref), (dtype, level)
        e.close()
