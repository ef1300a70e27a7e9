"""ctypes wrapper of the FP64 CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle is a CPU restatement of the
reference's ScatCov engine (jmdelouis/STL-Dev-MPI, crates/stl-core); only
the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline leg
use it, as the checker.  The CUDA engine never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_lib = None

FAMILIES = ["mean", "var", "S1", "S2", "S3", "S4"]
GAUGES = {"cosmo": 0, "phi": 1}


def build(quiet: bool = True) -> Path:
    """Compile the oracle library (make in oracle/)."""
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{out.stdout}\n{out.stderr}")
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        l = C.CDLL(str(LIB_PATH))
        sig = {
            "or_last_error": ([], C.c_char_p),
            "or_set_threads": ([C.c_int], None),
            "or_get_threads": ([], C.c_int),
            "or_centres": ([C.c_int64, C.c_int64, _I64, _I64, _I64, _I64, _D, _D, _D, _D], None),
            "or_ring2nest": ([C.c_int, C.c_int64, _I64, _I64], None),
            "or_interp_ring": ([C.c_int64, C.c_int64, _D, _D, _I64, _D], None),
            "or_interp_nested": ([C.c_int, C.c_int64, _D, _I64, _D], None),
            "or_rotations": ([C.c_int64, _D, _D, C.c_int, C.c_int, _D], None),
            "or_kernel_grid": ([C.c_int, C.c_int64, _D], None),
            "or_wavelet_weights": ([C.c_int, _D], None),
            "or_bind": ([_I64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, _I64, _D, _U8], C.c_int),
            "or_row_cells": ([_I64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, _I64, _D, C.c_int64, _I64],
                             C.c_int),
            "or_conv_forward": ([_I64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, _D, _D, C.c_int64, _D], C.c_int),
            "or_conv_adjoint": ([_I64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, _D, _D, C.c_int64, _D], C.c_int),
            "or_kth_neighbourhood": ([C.c_int64, C.c_int64, C.c_int, _I64], C.c_int64),
            "or_down_new": ([_I64, C.c_int64, C.c_int64], C.c_void_p),
            "or_down_nrows": ([C.c_void_p], C.c_int64),
            "or_down_nnz": ([C.c_void_p], C.c_int64),
            "or_down_get": ([C.c_void_p, _I64, _I64, _I64, _D], None),
            "or_down_free": ([C.c_void_p], None),
            "or_build_plan": ([C.c_int, C.c_int, C.c_int, C.c_int, _I32, C.c_int64], C.c_int64),
            "or_engine_new": ([C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I32, C.c_int, C.c_double], C.c_void_p),
            "or_engine_free": ([C.c_void_p], None),
            "or_engine_ncoeff": ([C.c_void_p], C.c_int64),
            "or_engine_levels": ([C.c_void_p], C.c_int),
            "or_engine_plan": ([C.c_void_p, _I32], None),
            "or_engine_set_masks": ([C.c_void_p, _D, C.c_int64], C.c_int),
            "or_engine_native_pixels": ([C.c_void_p, _I64], C.c_int64),
            "or_engine_forward": ([C.c_void_p, _D, C.c_int, _D, _D], C.c_int),
            "or_engine_forward_levels": ([C.c_void_p, _D, _D], C.c_int),
            "or_engine_get_map": ([C.c_void_p, C.c_int, _D], C.c_int),
            "or_engine_get_m": ([C.c_void_p, C.c_int, C.c_int, _D], C.c_int),
            "or_engine_get_z": ([C.c_void_p, C.c_int, _D], C.c_int),
            "or_engine_reverse": ([C.c_void_p, _D, _D], C.c_int),
            "or_engine_analysis": ([C.c_void_p, _D, _D], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(l, name)
            f.argtypes, f.restype = args, res
        _lib = l
    return _lib


def _p(a, t=_D):
    return a.ctypes.data_as(t)


def _check(status):
    if status != 0:
        raise RuntimeError(lib().or_last_error().decode())


def set_threads(n: int):
    lib().or_set_threads(int(n))


def threads() -> int:
    return lib().or_get_threads()


# -- geometry primitives ----------------------------------------------------
def centres(nside, ids):
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    n = ids.size
    ix, iy, face = (np.empty(n, np.int64) for _ in range(3))
    th, ph, lo, la = (np.empty(n) for _ in range(4))
    lib().or_centres(nside, n, _p(ids, _I64), _p(ix, _I64), _p(iy, _I64), _p(face, _I64), _p(th), _p(ph), _p(lo), _p(la))
    return ix, iy, face, th, ph, lo, la


def ring2nest(order, ring):
    ring = np.ascontiguousarray(ring, dtype=np.int64)
    out = np.empty_like(ring)
    lib().or_ring2nest(order, ring.size, _p(ring, _I64), _p(out, _I64))
    return out


def interp_ring(nside, theta, phi):
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    pix = np.empty((theta.size, 4), np.int64)
    w = np.empty((theta.size, 4))
    lib().or_interp_ring(nside, theta.size, _p(theta), _p(phi), _p(pix, _I64), _p(w))
    return pix, w


def interp_nested(order, vecs):
    vecs = np.ascontiguousarray(vecs, dtype=np.float64).reshape(-1, 3)
    n = vecs.shape[0]
    pix = np.empty((n, 4), np.int64)
    w = np.empty((n, 4))
    lib().or_interp_nested(order, n, _p(vecs), _p(pix, _I64), _p(w))
    return pix, w


def rotations(theta, phi, G, gauge="cosmo"):
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.empty((theta.size, G, 3, 3))
    lib().or_rotations(theta.size, _p(theta), _p(phi), G, GAUGES[gauge], _p(out))
    return out


def kernel_grid(ksz, nside):
    out = np.empty((ksz * ksz, 3))
    lib().or_kernel_grid(ksz, nside, _p(out))
    return out


def wavelet_weights(ksz):
    out = np.empty(2 * ksz * ksz)
    lib().or_wavelet_weights(ksz, _p(out))
    return out


def bind(grid, nside, ksz, G, gauge="cosmo", eps=0.0):
    """Bound stencils of the rows `grid` on `grid` (reference layout [4, G, K, P])."""
    grid = np.ascontiguousarray(grid, dtype=np.int64)
    K, P = grid.size, ksz * ksz
    pos = np.empty((4, G, K, P), np.int64)
    w = np.empty((4, G, K, P))
    complete = np.empty(K, np.uint8)
    _check(lib().or_bind(_p(grid, _I64), K, nside, ksz, G, GAUGES[gauge], eps, _p(pos, _I64), _p(w), _p(complete, _U8)))
    return pos, w, complete.astype(bool)


def row_cells(rows, nside, ksz=5, G=4, gauge="cosmo", width=128):
    """(cells [len(rows), w] int64 padded with -1, weights [len(rows), w]): the
    sorted distinct cells of nonzero weight each row reads in its bound
    stencils on the whole sky and their largest bound weights."""
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty((rows.size, width), np.int64)
    wmax = np.empty((rows.size, width))
    counts = np.empty(rows.size, np.int64)
    _check(lib().or_row_cells(_p(rows, _I64), rows.size, nside, ksz, G, GAUGES[gauge], _p(out, _I64), _p(wmax),
                              width, _p(counts, _I64)))
    w = max(int(counts.max()) if counts.size else 0, 1)
    return out[:, :w], wmax[:, :w]


def _weights(weights, ksz):
    if weights is None:
        return None, None
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    assert w.size == 2 * ksz * ksz
    return w, _p(w)


def conv_forward(x, nside, ksz=5, G=4, gauge="cosmo", grid=None, eps=0.0, weights=None):
    """Convolution of x [R, n_in] -> [R, G, 2, n_in] on `grid` (None: whole sky) with
    the wavelet, or with the kernel `weights` [2, P] (cast through f32)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    R = x.shape[0] if x.ndim == 2 else 1
    if grid is None:
        gp, n = None, 12 * nside * nside
    else:
        grid = np.ascontiguousarray(grid, dtype=np.int64)
        gp, n = _p(grid, _I64), grid.size
    y = np.empty((R, G, 2, n))
    keep, wp = _weights(weights, ksz)
    _check(lib().or_conv_forward(gp, n, nside, ksz, G, GAUGES[gauge], eps, wp, _p(x), R, _p(y)))
    return y


def conv_adjoint(gy, nside, ksz=5, G=4, gauge="cosmo", grid=None, eps=0.0, weights=None):
    gy = np.ascontiguousarray(gy, dtype=np.float64)
    R = gy.shape[0]
    if grid is None:
        gp, n = None, 12 * nside * nside
    else:
        grid = np.ascontiguousarray(grid, dtype=np.int64)
        gp, n = _p(grid, _I64), grid.size
    gx = np.empty((R, n))
    keep, wp = _weights(weights, ksz)
    _check(lib().or_conv_adjoint(gp, n, nside, ksz, G, GAUGES[gauge], eps, wp, _p(gy), R, _p(gx)))
    return gx


def kth_neighbourhood(pix, nside, k):
    out = np.empty((2 * k + 1) ** 2, np.int64)
    n = lib().or_kth_neighbourhood(int(pix), nside, k, _p(out, _I64))
    return out[:n].copy()


def smooth_decimation(ids, nside):
    """(coarse ids, indptr, indices, values) of the decimation of the sorted `ids` (None: whole sky)."""
    if ids is None:
        h = lib().or_down_new(None, 0, nside)
    else:
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        h = lib().or_down_new(_p(ids, _I64), ids.size, nside)
    if not h:
        raise RuntimeError(lib().or_last_error().decode())
    try:
        nr, nnz = lib().or_down_nrows(h), lib().or_down_nnz(h)
        coarse = np.empty(nr, np.int64)
        indptr = np.empty(nr + 1, np.int64)
        indices = np.empty(nnz, np.int64)
        values = np.empty(nnz)
        lib().or_down_get(h, _p(coarse, _I64), _p(indptr, _I64), _p(indices, _I64), _p(values))
    finally:
        lib().or_down_free(h)
    return coarse, indptr, indices, values


# -- engine -----------------------------------------------------------------
def plan_dicts(plan_rows):
    out = []
    for i, r in enumerate(plan_rows):
        f = lambda v: None if v < 0 else int(v)
        out.append({"index": i, "family": FAMILIES[r[0]], "native_dg": int(r[1]), "c1": int(r[2]), "c2": int(r[3]),
                    "j1": f(r[4]), "j2": f(r[5]), "j3": f(r[6]), "l1": f(r[7]), "l2": f(r[8]), "l3": f(r[9])})
    return out


def build_plan(J, L=4, channels=1, cross_only=False):
    """Plan dicts of dg(j) = j (plan.rs:80-158), as the bridge's stlp_info lists them."""
    n = lib().or_build_plan(J, L, channels, int(cross_only), None, 0)
    rows = np.empty((n, 10), np.int32)
    lib().or_build_plan(J, L, channels, int(cross_only), _p(rows, _I32), n)
    return plan_dicts(rows)


class OracleEngine:
    """Full-sky FP64 ScatCov forward + VJP on the CPU (the reference's LocalEngine semantics)."""

    def __init__(self, nside, J, L=4, kernel=5, batch=1, channels=1, fewer=False, j_to_dg=None,
                 cross_only=False, gauge="cosmo", cache_gb=4.0):
        dg = None
        self._dg = None
        if j_to_dg is not None:
            self._dg = np.ascontiguousarray(j_to_dg, dtype=np.int32)
            dg = _p(self._dg, _I32)
        self._h = lib().or_engine_new(nside, J, L, kernel, GAUGES[gauge], batch, channels, int(fewer), dg,
                                      int(cross_only), float(cache_gb))
        if not self._h:
            raise RuntimeError(lib().or_last_error().decode())
        self.nside, self.J, self.L, self.batch, self.channels = nside, J, L, batch, channels
        self.levels = lib().or_engine_levels(self._h)
        self.ncoeff = lib().or_engine_ncoeff(self._h)
        rows = np.empty((self.ncoeff, 10), np.int32)
        lib().or_engine_plan(self._h, _p(rows, _I32))
        self.plan_rows = rows
        self.nmasks = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().or_engine_free(self._h)
            self._h = None

    __del__ = close

    def npix(self, d):
        return 12 * (self.nside >> d) ** 2

    def plan(self):
        return plan_dicts(self.plan_rows)

    def set_masks(self, w):
        w = np.ascontiguousarray(np.atleast_2d(w), dtype=np.float64) if w is not None else np.zeros((0, 1))
        _check(lib().or_engine_set_masks(self._h, _p(w), w.shape[0] if w.size else 0))
        self.nmasks = w.shape[0] if w.size else 0

    def _shape(self):
        return (self.batch, self.nmasks, self.ncoeff) if self.nmasks else (self.batch, self.ncoeff)

    def forward(self, x, moments=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == self.batch * self.channels * self.npix(0)
        values = np.empty(self._shape(), np.complex128)
        var = np.empty(self._shape()) if moments else np.empty(1)
        _check(lib().or_engine_forward(self._h, _p(x), int(moments), _p(values.view(np.float64)), _p(var)))
        return (values, var) if moments else values

    def forward_levels(self, maps):
        x = np.ascontiguousarray(np.concatenate([np.asarray(m, np.float64).ravel() for m in maps]))
        values = np.empty(self._shape(), np.complex128)
        _check(lib().or_engine_forward_levels(self._h, _p(x), _p(values.view(np.float64))))
        return values

    def native_pixels(self):
        out = np.empty((max(self.nmasks, 1), self.ncoeff), np.int64)
        lib().or_engine_native_pixels(self._h, _p(out, _I64))
        return out if self.nmasks else out[0]

    def map(self, d):
        out = np.empty((self.batch * self.channels, self.npix(d)))
        _check(lib().or_engine_get_map(self._h, d, _p(out)))
        return out

    def m(self, d, n):
        out = np.empty((self.batch * self.channels, self.L, self.npix(n)))
        _check(lib().or_engine_get_m(self._h, d, n, _p(out)))
        return out

    def z(self, n):
        out = np.empty((self.batch * self.channels, self.L, self.npix(n)), np.complex128)
        _check(lib().or_engine_get_z(self._h, n, _p(out.view(np.float64))))
        return out

    def reverse(self, cot):
        """Per-level map cotangents [levels][B*C, N_d] of Re sum(conj(cot) * values)."""
        cot = np.ascontiguousarray(cot, dtype=np.complex128)
        sizes = [self.batch * self.channels * self.npix(d) for d in range(self.levels)]
        out = np.empty(sum(sizes))
        _check(lib().or_engine_reverse(self._h, _p(cot.view(np.float64)), _p(out)))
        res, at = [], 0
        for d, s in enumerate(sizes):
            res.append(out[at:at + s].reshape(self.batch * self.channels, self.npix(d)))
            at += s
        return res

    def analysis(self):
        sizes = [self.batch * self.channels * self.npix(d) for d in range(self.levels)]
        g0 = np.empty(sizes[0])
        bands = np.empty(sum(sizes))
        _check(lib().or_engine_analysis(self._h, _p(g0), _p(bands)))
        res, at = [], 0
        for d, s in enumerate(sizes):
            res.append(bands[at:at + s].reshape(self.batch * self.channels, self.npix(d)))
            at += s
        return g0.reshape(self.batch * self.channels, -1), res

    def vjp(self, cot):
        """Level-0 map cotangent [B*C, N_0]."""
        self.reverse(cot)
        return self.analysis()[0]
