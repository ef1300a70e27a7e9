"""CPU FP64 oracle of the spin-2 front end (crates/stl-core/src/spin.rs and its
use in crates/stl-bridge/src/lib.rs), over oracle/_build/liboracle.so.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker of the engine's
spin-2 path; the CUDA engine never imports it.

- ``SpinOp``: complex sparse rows (spin.rs:88-157), either the operator
  -(d_x - i d_y)^2 of one level (``eth_bar2``, spin.rs:294-338) or the
  transported mean of the four children (``spin_decimation``, spin.rs:193-210).
- ``SpinPyramid``: the operators of every level, the polarisation pyramid, its
  chi fields and their adjoint, and the eroded valid rows (spin.rs:341-433).
- ``SpinOracle``: the statistics of spin-2 maps (scalar or transported
  pyramid; the cross pairs of lib.rs:186-240) on the oracle engine.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

import oracle as O

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_ready = False


def _lib():
    global _ready
    l = O.lib()
    if not _ready:
        sig = {
            "or_spin_last_error": ([], C.c_char_p),
            "or_spin_new": ([C.c_int, C.c_int64, C.c_int], C.c_void_p),
            "or_spin_free": ([C.c_void_p], None),
            "or_spin_shape": ([C.c_void_p, _I64, _I64, _I64], None),
            "or_spin_export": ([C.c_void_p, _I64, _I64, _D], None),
            "or_spin_apply": ([C.c_void_p, _D, C.c_int64, _D, C.c_int], None),
            "or_engine_set_mask_levels": ([C.c_void_p, _D, C.c_int64], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(l, name)
            f.argtypes, f.restype = args, res
        _ready = True
    return l


class SpinOp:
    """out[r] = sum_e w[e] (Q + iU)[col[e]] on [R, 2, n] (Q, U) fields."""

    def __init__(self, kind, nside, kernel=5):
        l = _lib()
        self._h = l.or_spin_new(int(kind), int(nside), int(kernel))
        if not self._h:
            raise ValueError(l.or_spin_last_error().decode())
        r, n, z = C.c_int64(), C.c_int64(), C.c_int64()
        l.or_spin_shape(self._h, C.byref(r), C.byref(n), C.byref(z))
        self.rows, self.n_in, self.nnz = r.value, n.value, z.value

    def __del__(self):
        if getattr(self, "_h", None):
            _lib().or_spin_free(self._h)
            self._h = None

    def export(self):
        """(ptr [rows + 1], col [nnz], w [nnz] complex)."""
        ptr = np.empty(self.rows + 1, np.int64)
        col = np.empty(self.nnz, np.int64)
        w = np.empty(self.nnz, np.complex128)
        _lib().or_spin_export(self._h, ptr.ctypes.data_as(_I64), col.ctypes.data_as(_I64),
                              w.view(np.float64).ctypes.data_as(_D))
        return ptr, col, w

    def _run(self, x, n_in, n_out, adjoint):
        x = np.ascontiguousarray(x, dtype=np.float64)
        R = x.size // (2 * n_in)
        assert x.size == R * 2 * n_in, "field length"
        out = np.empty((R, 2, n_out))
        _lib().or_spin_apply(self._h, x.ctypes.data_as(_D), R, out.ctypes.data_as(_D), int(adjoint))
        return out

    def apply(self, x):
        return self._run(x, self.n_in, self.rows, False)

    def adjoint(self, g):
        return self._run(g, self.rows, self.n_in, True)


def eth_bar2(nside, kernel=5):
    return SpinOp(0, nside, kernel)


def spin_decimation(nside_fine):
    return SpinOp(1, nside_fine)


class SpinPyramid:
    """Operators of `levels` levels from nside0 (spin.rs:341-433)."""

    def __init__(self, nside0, levels, kernel=5):
        assert levels >= 1 and (nside0 >> (levels - 1)) >= 1
        self.nside0, self.kernel = nside0, kernel
        self.down = [spin_decimation(nside0 >> j) for j in range(levels - 1)]
        self.eth = [eth_bar2(nside0 >> j, kernel) for j in range(levels)]

    @property
    def levels(self):
        return len(self.eth)

    def polarisation(self, qu):
        out = [np.ascontiguousarray(qu, dtype=np.float64).reshape(-1, 2, 12 * self.nside0 ** 2)]
        for d in self.down:
            out.append(d.apply(out[-1]))
        return out

    def forward(self, qu):
        return [e.apply(p) for p, e in zip(self.polarisation(qu), self.eth)]

    def adjoint(self, g_chi):
        g = self.eth[-1].adjoint(g_chi[-1])
        for j in range(self.levels - 2, -1, -1):
            g = self.eth[j].adjoint(g_chi[j]) + self.down[j].adjoint(g)
        return g

    def valid_rows(self, valid0):
        data = np.asarray(valid0) != 0
        out = []
        for j, e in enumerate(self.eth):
            if j > 0:
                data = data.reshape(-1, 4).all(axis=1)
            ptr, col, _ = e.export()
            ok = data[col]
            rows = np.array([ok[ptr[r]:ptr[r + 1]].all() for r in range(e.rows)])
            out.append(rows.astype(np.float64))
        return out


def down_rings(nside0, d):
    """Rings of the smooth decimation of level d (local.rs:130-134, radius 3 pixels)."""
    pix_deg = math.sqrt(4.0 * math.pi / (12 * (nside0 >> d) ** 2)) * (180.0 / math.pi)
    radius = 3.0 * pix_deg
    return int(math.ceil(radius / pix_deg)) + 1


def scalar_pyramid_valid(nside0, levels, valid0):
    """Masks of every level of the scalar pyramid from the valid level-0 rows:
    a parent is valid unless a bad pixel lies within the decimation's reach
    (crates/stl-bridge/src/lib.rs:428-441)."""
    out = [np.asarray(valid0, dtype=np.float64)]
    for d in range(levels - 1):
        nside = nside0 >> d
        fine = out[-1]
        bad = np.flatnonzero(fine == 0.0)
        rings = down_rings(nside0, d)
        if rings >= nside:  # the dilation covers the whole level (neighbours.rs:31-35)
            reach = np.arange(12 * nside * nside)
        else:
            reach = np.unique(np.concatenate([O.kth_neighbourhood(p, nside, rings) for p in bad])) if bad.size else bad
        nxt = np.ones(12 * (nside // 2) ** 2)
        nxt[np.unique(reach // 4)] = 0.0
        out.append(nxt)
    return out


def keep_nonempty(levels):
    """A level the erosion emptied gets the parents of the level below
    (crates/stl-bridge/src/lib.rs:447-454)."""
    levels = [np.asarray(v, dtype=np.float64).copy() for v in levels]
    for d in range(1, len(levels)):
        if not (levels[d] != 0).any():
            levels[d] = (levels[d - 1].reshape(-1, 4) != 0).any(axis=1).astype(np.float64)
    return levels


class SpinOracle:
    """Statistics of spin-2 maps through the oracle engine (lib.rs:139-240,
    474-600): maps (Q, U) [batch, 2, npix]; values [batch, 2 (E, B), (K,) ncoeff].

    pyramid="scalar": chi_0 only, decimated by the engine's scalar pyramid;
    "transported": chi_j of every level, no decimation of the maps.
    cross=True (scalar pyramid): pairs (a, b), a [batch, 1 or 2, npix]
    (spin_a 0: T, 2: (Q, U)), b [batch, 2, npix]."""

    def __init__(self, nside, J, batch=1, kernel=5, pyramid="scalar", cross=False, spin_a=2):
        self.nside, self.J, self.batch = nside, J, batch
        self.pyramid, self.cross, self.spin_a = pyramid, cross, spin_a
        self.npix = 12 * nside * nside
        self.engine = O.OracleEngine(nside, J, batch=2 * batch, channels=2 if cross else 1,
                                     cross_only=cross) if cross else O.OracleEngine(nside, J, batch=2 * batch)
        levels = self.engine.levels
        self.spin = SpinPyramid(nside, 1 if pyramid == "scalar" else levels, kernel)
        self.nmasks = 0

    @property
    def plan(self):
        return self.engine.plan()

    def set_masks(self, w):
        """Indicators of the valid data [K, npix], eroded by the stencil (lib.rs:396-422)."""
        w = np.atleast_2d(np.asarray(w, dtype=np.float64))
        levels = self.engine.levels
        per = []
        for m in w:
            if self.pyramid == "scalar":
                lv = keep_nonempty(scalar_pyramid_valid(self.nside, levels, self.spin.valid_rows(m)[0]))
            else:
                lv = keep_nonempty(self.spin.valid_rows(m))
            per.append(np.concatenate(lv))
        flat = np.ascontiguousarray(np.concatenate(per))
        O._check(_lib().or_engine_set_mask_levels(self.engine._h, flat.ctypes.data_as(_D), len(per)))
        self.engine.nmasks = len(per)
        self.nmasks = len(per)

    def native_pixels(self):
        return self.engine.native_pixels()

    def _level0(self, x):
        n, B = self.npix, self.batch
        eth = self.spin.eth[0]
        if not self.cross:
            return eth.apply(np.asarray(x).reshape(B, 2, n)).reshape(2 * B, n)
        a, b = x
        chi_b = eth.apply(np.asarray(b).reshape(B, 2, n))
        if self.spin_a == 2:
            chi_a = eth.apply(np.asarray(a).reshape(B, 2, n))
        else:
            t = np.asarray(a, dtype=np.float64).reshape(B, n)
            chi_a = np.stack([t, t], 1)
        out = np.empty((B, 2, 2, n))
        out[:, :, 0] = chi_a
        out[:, :, 1] = chi_b
        return out.reshape(2 * B, 2 * n)

    def _shape(self, v):
        return v.reshape((self.batch, 2) + v.shape[1:])

    def forward(self, x):
        if self.pyramid == "scalar":
            v = self.engine.forward(self._level0(x))
        else:
            chi = self.spin.forward(np.asarray(x).reshape(self.batch, 2, self.npix))
            v = self.engine.forward_levels([c.reshape(2 * self.batch, -1) for c in chi])
        return self._shape(v)

    def vjp(self, cot):
        cot = np.asarray(cot, dtype=np.complex128).reshape((2 * self.batch,) + np.shape(cot)[2:])
        B, n = self.batch, self.npix
        if self.pyramid == "transported":
            mg = self.engine.reverse(cot)
            return self.spin.adjoint([g.reshape(B, 2, -1) for g in mg])
        g = self.engine.vjp(cot)
        eth = self.spin.eth[0]
        if not self.cross:
            return eth.adjoint(g.reshape(B, 2, n))
        g = g.reshape(B, 2, 2, n)
        gb = eth.adjoint(g[:, :, 1])
        if self.spin_a == 2:
            ga = eth.adjoint(g[:, :, 0])
        else:
            ga = g[:, 0, 0] + g[:, 1, 0]
        return ga, gb

    def fields(self, x, level):
        """((Q, U), (chi_E, chi_B)) of `level`, each [batch, 2, npix_level]."""
        pol = self.spin.polarisation(np.asarray(x).reshape(self.batch, 2, self.npix))
        return pol[level], self.spin.eth[level].apply(pol[level])
