"""stlp_mean_var_noalloc (fixed device scratch, no allocation) against the mean
and var coefficients of stlp_forward_device, called through the C ABI twice in
a row on the same maps.  Collected last so it also runs after the other GPU
tests have used the device."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(stl):
    f = stl.lib().stlp_mean_var_noalloc
    f.argtypes = [C.c_uint64, C.c_size_t, C.c_size_t, C.c_int, C.c_uint64, C.c_uint64]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("dtype,nside,B", [("float64", 16, 3), ("float32", 16, 3),
                                           # more pixels than one pass of the 296 x 256-thread grid
                                           ("float64", 128, 2), ("float32", 128, 2),
                                           # the largest batch the fixed scratch holds
                                           ("float64", 16, 64)])
def test_mean_var_noalloc_matches_forward(dtype, nside, B):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200 as stl
    f = _entry(stl)
    tdt = torch.float64 if dtype == "float64" else torch.float32
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.exp(torch.randn(B, 12 * nside * nside, device="cuda", dtype=tdt, generator=g) - 0.5)
    e = stl.NativeEngine(nside, 3, batch=B, dtype=dtype)
    values, _ = e.forward_tensor(x)
    fam = [c["family"] for c in e.info()["plan"]]
    i_mean, i_var = fam.index("mean"), fam.index("var")
    want = np.stack([values[:, i_mean].real, values[:, i_var].real], axis=1)
    out = torch.empty(B, 2, device="cuda", dtype=torch.float64)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(float("nan"))
        rc = f(x.data_ptr(), x.shape[1], B, int(tdt == torch.float32), out.data_ptr(), stream)
        assert rc == 0, stl.lib().stlp_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # FP64 sums of the pixel values; the FP32 engine holds its maps as FP32
        # deviations from their FP64 means, so its mean / var carry that rounding
        np.testing.assert_allclose(got, want, rtol=1e-12 if dtype == "float64" else 1e-6, atol=0.0)
    e.close()


def test_mean_var_noalloc_refuses_oversized_batch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    import stl_b200 as stl
    f = _entry(stl)
    x = torch.ones(65, 12, device="cuda", dtype=torch.float64)
    out = torch.empty(65, 2, device="cuda", dtype=torch.float64)
    rc = f(x.data_ptr(), 12, 65, 0, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"exceeds the 64 maps" in stl.lib().stlp_last_error()
