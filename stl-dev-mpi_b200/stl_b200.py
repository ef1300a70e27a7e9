"""Python host side of the B200 ScatCov engine (libstl_b200.so).

``NativeEngine`` mirrors the reference's binding of the same name
(jmdelouis/STL-Dev-MPI, python/stl_ensemble/stl_port/native.py:153-490):
same constructor keywords, the plan from ``info()["plan"]``, ``forward``
returning ``(values, variances)``, ``vjp`` of ``Re sum(conj(cot) values)``,
the (generation, member, objective) identity of a forward state,
``checkpoint`` / ``restore`` and ``native_pixels``.  ``backend`` must be
"gpu": this library has no CPU engine, and fails loudly when the library
or the device is missing.

Additions for PyTorch: ``forward_tensor`` / ``vjp_tensor`` on CUDA tensors
(float32 or float64, no host copy of the maps) and ``scattering(engine, x)``,
a ``torch.autograd.Function`` over them; torch hands the backward of a
complex output the cotangent dL/dRe + i dL/dIm, the engine's convention.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import itertools
import json
import os
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libstl_b200.so"

_D = C.POINTER(C.c_double)
_SIZE = C.POINTER(C.c_size_t)
_VOID = C.c_void_p
_CALLBACK = C.CFUNCTYPE(C.c_double, _D, C.c_size_t, _D, _VOID)
_lib = None
_lock = threading.Lock()


def library_path() -> Path:
    return Path(os.environ.get("STL_B200_LIBRARY", LIBRARY))


def lib():
    """The engine library with its C signatures (include/stl_b200.h)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not path.is_file():
            raise RuntimeError(f"the B200 engine library is missing: {path} (build it with "
                               f"`make -C {HERE}` or __graft_entry__.build()); there is no fallback engine")
        l = C.CDLL(str(path))
        u64, sz, b = C.c_uint64, C.c_size_t, C.c_bool
        sig = {
            "stlp_last_error": ([], C.c_char_p),
            "stlp_string_free": ([_VOID], None),
            "stlp_new": ([C.c_char_p], _VOID),
            "stlp_free": ([_VOID], None),
            "stlp_info": ([_VOID], _VOID),
            "stlp_prepare": ([_VOID], C.c_int),
            "stlp_set_stream": ([_VOID, u64], C.c_int),
            "stlp_profile": ([_VOID, C.c_int, C.c_int], C.c_int),
            "stlp_set_masks": ([_VOID, _D, sz], C.c_int),
            "stlp_synthesize_device": ([_VOID, u64, sz, _D, sz, _D, C.c_char_p, _D, sz], C.c_int64),
            "stlp_native_pixels": ([_VOID, _SIZE], C.c_int),
            "stlp_forward": ([_VOID, _D, sz, u64, u64, u64, b, _D, _D], C.c_int),
            "stlp_vjp": ([_VOID, _D, sz, u64, u64, u64, _D], C.c_int),
            "stlp_forward_device": ([_VOID, u64, sz, C.c_int, u64, u64, u64, b, _D, _D], C.c_int),
            "stlp_vjp_device": ([_VOID, _D, sz, u64, u64, u64, u64, C.c_int], C.c_int),
            "stlp_checkpoint": ([_VOID], _VOID),
            "stlp_checkpoint_free": ([_VOID], None),
            "stlp_checkpoint_bytes": ([_VOID], sz),
            "stlp_restore": ([_VOID, _VOID, u64, u64, u64], C.c_int),
            "stlp_forward_levels": ([_VOID, _D, sz, _D], C.c_int),
            "stlp_lbfgs": ([_D, sz, C.c_char_p, _CALLBACK, _VOID], C.c_int64),
            "stlp_patch_new": ([C.c_char_p], _VOID),
            "stlp_patch_free": ([_VOID], None),
            "stlp_patch_info": ([_VOID], _VOID),
            "stlp_pixel_vectors": ([sz, C.POINTER(C.c_int64), sz, _D], C.c_int),
            "stlp_patch_select": ([_VOID, _D, sz, C.c_double, C.c_double, _SIZE], C.c_int),
            "stlp_patch_select_radii": ([_VOID, _D, sz, _D, _D, _SIZE], C.c_int),
            "stlp_patch_ids": ([_VOID, sz, C.POINTER(C.c_int64)], C.c_int),
            "stlp_patch_core_pixels": ([_VOID, _SIZE], C.c_int),
            "stlp_patch_forward": ([_VOID, _D, sz, u64, b, _D, _D], C.c_int),
            "stlp_patch_vjp": ([_VOID, _D, sz, u64, _D], C.c_int),
            "stlp_patch_forward_device": ([_VOID, u64, sz, u64, b, _D, _D], C.c_int),
            "stlp_patch_vjp_device": ([_VOID, _D, sz, u64, u64], C.c_int),
            "stlp_operator_rows": ([_VOID, sz, C.c_int, C.POINTER(C.c_int64), _D, sz, _SIZE], C.c_int),
            "stlp_memory": ([_SIZE, _SIZE, C.c_int], C.c_int),
            "stlp_spin_fields": ([_VOID, _D, sz, sz, _D, _D], C.c_int),
            "stlp_spin_rows": ([_VOID, sz, C.c_int, C.POINTER(C.c_int64), _D, sz, _SIZE], C.c_int),
            "stlp_terms_new": ([C.c_char_p], _VOID),
            "stlp_terms_free": ([_VOID], None),
            "stlp_terms_set_stream": ([_VOID, u64], C.c_int),
            "stlp_terms_kappa_table": ([_VOID, _D, _D, _D, sz], C.c_int),
            "stlp_terms_kappa": ([_VOID, u64, sz, C.c_double, C.c_double, C.c_double, C.c_double, u64, u64],
                                 C.c_int),
            "stlp_terms_pyramid": ([_VOID, u64], C.c_int),
            "stlp_terms_moments": ([_VOID, u64, _D], C.c_int),
            "stlp_terms_level_power_grad": ([_VOID, u64, _D, sz, u64], C.c_int),
            "stlp_terms_kurtosis_grad": ([_VOID, u64, C.POINTER(C.c_int), sz, _D, u64, u64], C.c_int),
            "stlp_terms_sort": ([_VOID, u64, sz, u64], C.c_int),
            "stlp_terms_marginal": ([_VOID, u64, u64, u64, sz, C.c_double, u64, _D], C.c_int),
            "stlp_terms_add_product": ([_VOID, u64, u64, u64, sz], C.c_int),
            "stlp_map_len": ([C.c_char_p, _SIZE], C.c_int),
            "stlp_npy_shape": ([C.c_char_p, _SIZE, sz, _SIZE], C.c_int),
            "stlp_map_read": ([C.c_char_p, _D, sz], C.c_int),
            "stlp_map_read_range": ([C.c_char_p, sz, sz, _D], C.c_int),
            "stlp_npy_write": ([C.c_char_p, _D, _SIZE, sz], C.c_int),
            "stlp_fits_write": ([C.c_char_p, _D, sz, C.c_char_p, C.c_int], C.c_int),
            "stlp_map_create": ([C.c_char_p, sz, C.c_char_p, C.c_int], C.c_int),
            "stlp_map_write": ([C.c_char_p, sz, _D, sz, C.c_int], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(l, name)
            f.argtypes, f.restype = args, res
        _lib = l
        return l


def device_memory(reset_peak=False):
    """(live, peak) bytes of device memory the library holds (all engines of the
    process); reset_peak first restarts the high-water mark at the live bytes."""
    live, peak = C.c_size_t(0), C.c_size_t(0)
    if lib().stlp_memory(C.byref(live), C.byref(peak), int(bool(reset_peak))):
        raise _error()
    return live.value, peak.value


# ---- map files: NESTED .npy and HEALPix FITS (the library's reader and writer) ----

def _path(path):
    return os.fsencode(os.fspath(path))


def map_len(path):
    """Pixels of the map in a file (.fits / .fit: HEALPix FITS, else .npy),
    read from its header."""
    n = C.c_size_t(0)
    if lib().stlp_map_len(_path(path), C.byref(n)):
        raise _error()
    return n.value


def read_map(path):
    """The whole map as a NESTED float64 vector (a RING FITS map is
    reordered; any float or integer .npy is read as float64)."""
    out = np.empty(map_len(path))
    if lib().stlp_map_read(_path(path), _ptr(out), out.size):
        raise _error()
    return out


def read_npy(path):
    """A .npy array as float64, in its own shape (C order)."""
    shape = (C.c_size_t * 32)()
    ndim = C.c_size_t(0)
    if lib().stlp_npy_shape(_path(path), shape, 32, C.byref(ndim)):
        raise _error()
    return read_map(path).reshape(tuple(shape[i] for i in range(ndim.value)))


def read_map_range(path, start, end):
    """Pixels [start, end) of the NESTED map, read at their offset."""
    start, end = int(start), int(end)
    if end < start:
        raise ValueError("range end before its start")
    out = np.empty(end - start)
    if lib().stlp_map_read_range(_path(path), start, end, _ptr(out)):
        raise _error()
    return out


def write_npy(path, values):
    """values as a little-endian float64 .npy of their shape."""
    v = np.require(values, dtype=np.float64, requirements="C")  # 0-d arrays stay 0-d
    shape = (C.c_size_t * max(1, v.ndim))(*v.shape)
    if lib().stlp_npy_write(_path(path), _ptr(v), shape, v.ndim):
        raise _error()


def write_healpix_fits(path, values, column="VALUE", double=False):
    """A full-sky NESTED map as a HEALPix FITS binary table of one column,
    float32 ('E') or float64 ('D', double=True)."""
    v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    if lib().stlp_fits_write(_path(path), _ptr(v), v.size, str(column).encode(), int(bool(double))):
        raise _error()


class SlicedMap:
    """A map file written in pieces, each at its own offset (every process
    its range): create() writes the headers and sizes the file, write()
    puts one piece.  .npy float64, or HEALPix FITS ('D' when double)."""

    def __init__(self, path, double=False):
        self.path, self.double = path, bool(double)

    def create(self, n, column="VALUE"):
        if lib().stlp_map_create(_path(self.path), int(n), str(column).encode(), int(self.double)):
            raise _error()

    def write(self, start, values):
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if lib().stlp_map_write(_path(self.path), int(start), _ptr(v), v.size, int(self.double)):
            raise _error()


def _all_finite(a, chunk=1 << 20):
    """Every value of a finite, checked a chunk at a time (a check of the
    whole array at once would allocate, and page-fault, a mask of its size
    on every call)."""
    v = np.asarray(a).reshape(-1)
    if np.iscomplexobj(v):
        v = v.view(np.float64) if v.flags.c_contiguous else np.ascontiguousarray(v).view(np.float64)
    for i in range(0, v.size, chunk):
        if not np.isfinite(v[i:i + chunk]).all():
            return False
    return True


def _error():
    msg = lib().stlp_last_error().decode("utf-8", errors="replace")
    # non-finite input maps (the library counts them while it copies the maps) are value errors
    return ValueError(msg) if msg.startswith("input") and "non-finite" in msg else RuntimeError(msg)


def _ptr(a):
    return a.ctypes.data_as(_D)


def _key(generation, member, objective):
    """Identity of a forward state, as native.py:122-129."""
    for name, v in (("generation", generation), ("member", member)):
        if isinstance(v, bool) or not isinstance(v, (int, np.integer)) or v < 0 or v >= 2 ** 64:
            raise ValueError(f"{name} must be an unsigned 64-bit integer")
    if not isinstance(objective, str) or not objective:
        raise ValueError("objective must be a nonempty name")
    return (int(generation), int(member), int.from_bytes(hashlib.sha256(objective.encode()).digest()[:8], "little"))


class Snapshot:
    """Saved forward state (the maps of the forward); ``close()`` frees it."""

    def __init__(self, handle, key, owner):
        self._handle, self.key, self.owner = handle, key, owner

    def close(self):
        if self._handle:
            lib().stlp_checkpoint_free(self._handle)
            self._handle = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *_):
        self.close()


def _mask_weights(masks, npix):
    """[K, npix] float64 indicators of the accepted mask forms (K = 0 for None)."""
    if masks is None:
        return np.zeros((0, npix))
    arr = masks if isinstance(masks, np.ndarray) else None
    if arr is not None and arr.dtype != object and arr.ndim in (1, 2) and arr.shape[-1] == npix:
        w = np.array(arr.reshape(-1, npix), dtype=np.float64, order="C")
    else:
        w = np.zeros((len(masks), npix))
        for k, ids in enumerate(masks):
            ids = np.asarray(ids, dtype=np.int64).ravel()
            if ids.size and not (0 <= ids.min() and ids.max() < npix):
                raise ValueError(f"mask {k}: pixel ids out of range")
            w[k][ids] = 1.0
    if not np.all(np.isfinite(w)):
        raise ValueError("mask weights must be finite")
    return w


class NativeEngine:
    """One persistent B200 workspace with an immutable plan, resolution and batch.

    ``dtype`` is the precision of the fields ("float64": everything FP64;
    "float32": convolutions, moduli and products in FP32, the pixel sums in
    FP64).  Values are complex128 ``[batch, ncoeff]`` in the order of
    ``plan``.

    ``spin=2``: the maps are (Q, U) ``[batch, 2, npix]``; the statistics are
    those of chi_E and chi_B = -(d_x - i d_y)^2 (Q + iU) (a stencil of
    ``spin_kernel`` cells a side), values ``[batch, 2, (K,) ncoeff]``;
    ``spin_pyramid="transported"`` builds chi at every level from the
    children's means turned into the parents' frames.  With ``cross=True``
    the maps are pairs (a, b) (``forward_cross``), a a (Q, U) field
    (``spin_a=2``) or a scalar map (``spin_a=0``).
    """

    def __init__(self, nside, j, batch=1, backend="gpu", kernel=5, orientations=4, device=0, dtype="float64",
                 prepare=False, autotune=True, autotune_cache=None, cross=False, tensor_cores=False, fields="keep",
                 spin=0, spin_kernel=5, spin_pyramid="scalar", spin_a=2, graphs=True, **unused):
        if backend != "gpu":
            raise ValueError("backend must be 'gpu': the B200 engine has no CPU fallback")
        for v in (nside, j, batch, kernel, orientations):
            if isinstance(v, bool) or int(v) != v or int(v) <= 0:
                raise ValueError("engine sizes must be positive integers")
        self.nside, self.j, self.batch = int(nside), int(j), int(batch)
        self.npix = 12 * self.nside ** 2
        # cross: two channels and the plan of their cross terms, maps [batch, 2, npix] (native.py's cross engine)
        self.cross, self.channels = bool(cross), 2 if cross else 1
        # spin 2: (Q, U) maps, statistics of chi_E and chi_B (values [batch, 2, (K,) ncoeff]); with cross,
        # pairs (a, b) of a (Q, U) or scalar field a (spin_a 2 or 0) and a (Q, U) field b
        if spin not in (0, 2) or spin_kernel not in (3, 5, 7, 9):
            raise ValueError("spin is 0 or 2 and spin_kernel 3, 5, 7 or 9")
        if spin_pyramid not in ("scalar", "transported") or spin_a not in (0, 2):
            raise ValueError("spin_pyramid is 'scalar' or 'transported', spin_a 0 or 2")
        if spin and cross and spin_pyramid != "scalar":
            raise ValueError("spin-2 cross statistics run on the scalar pyramid")
        self.spin = int(spin)
        self.spin_a = int(spin_a) if spin and cross else None
        if spin and cross:
            self._map_shape = (self.batch, (2 if spin_a == 2 else 1) + 2, self.npix)
        elif spin or cross:
            self._map_shape = (self.batch, 2, self.npix)
        else:
            self._map_shape = (self.batch, self.npix)
        self.dtype = dtype
        self.device = int(device)
        self.config = dict(nside=self.nside, j=self.j, batch=self.batch, backend="gpu", kernel=int(kernel),
                           orientations=int(orientations), device=self.device, dtype=dtype)
        if not autotune:  # keep the default tile heights (no timing at prepare)
            self.config["autotune"] = False
        if not graphs:  # launch the sweeps kernel by kernel instead of as CUDA graphs
            self.config["graphs"] = False
        # FP32 wavelets: False / "none" (the default: CUDA cores), True / "forward"
        # (forward on the tensor cores, adjoint on the CUDA cores), "all" (both)
        if tensor_cores is not False and tensor_cores != "none":
            self.config["tensor_cores"] = tensor_cores if isinstance(tensor_cores, str) else bool(tensor_cores)
        if fields != "keep":  # "recompute": z and branches recomputed per level in the VJP; "auto"
            self.config["fields"] = fields
        if cross:
            self.config["cross"] = True
        if spin:
            self.config.update(spin=2, spin_kernel=int(spin_kernel), spin_pyramid=spin_pyramid, spin_a=int(spin_a))
        if autotune_cache:  # a file of tile heights timed before (read, then extended)
            self.config["autotune_cache"] = str(autotune_cache)
        self._lib = lib()
        self._handle = self._lib.stlp_new(json.dumps(self.config).encode())
        if not self._handle:
            raise _error()
        self._mutex = threading.RLock()
        info = self.info()
        self.plan = info["plan"]
        self.levels = info["levels"]
        self.ncoeff = len(self.plan)
        self.nmasks = 0
        self._current_key = None
        self._stream = None
        if prepare:
            self.prepare()

    # -- handle plumbing ----------------------------------------------------
    def _open(self):
        if not self._handle:
            raise RuntimeError("engine is closed")

    def prepare(self):
        """Builds the device operators now (otherwise at the first forward)."""
        with self._mutex:
            self._open()
            if self._lib.stlp_prepare(self._handle):
                raise _error()

    def info(self):
        with self._mutex:
            self._open()
            p = self._lib.stlp_info(self._handle)
            if not p:
                raise _error()
            try:
                return json.loads(C.string_at(p))
            finally:
                self._lib.stlp_string_free(p)

    def profile(self, on=True, reset=True):
        """Kernel statistics: reset the counters, and time every launch with CUDA events when on."""
        with self._mutex:
            self._open()
            if self._lib.stlp_profile(self._handle, int(bool(on)), int(bool(reset))):
                raise _error()

    def kernel_stats(self):
        """Per kernel class since the last reset: launches, ms, algorithmic bytes and flops."""
        return {k["name"]: k for k in self.info()["kernels"]}

    def forward_levels(self, levels):
        """Statistics of maps given at every level (no decimation of level 0; for
        validation, no vjp follows): levels[d] [batch, 12 (nside/2^d)^2]
        (native.py:292-303)."""
        with self._mutex:
            self._open()
            x = np.ascontiguousarray(np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in levels]))
            values = np.empty(self._shape(), dtype=np.complex128)
            self._current_key = None
            if self._lib.stlp_forward_levels(self._handle, _ptr(x), x.size, _ptr(values.view(np.float64))):
                raise _error()
            return values

    def operator_rows(self, level, kind="wavelet"):
        """Integer tables of the device operators in pixel order: (cells [pixels,
        width] int64 padded with -1, weights [pixels, width]).  "wavelet": the
        sorted input cells each pixel of `level` reads (weight: the cell's
        largest |coefficient|); "decimation": the fine cells of nonzero weight
        of each coarse pixel of level + 1 (weight: |w|)."""
        k = {"wavelet": 0, "decimation": 1}[kind]
        with self._mutex:
            self._open()
            need = C.c_size_t(0)
            if self._lib.stlp_operator_rows(self._handle, int(level), k, None, None, 0, C.byref(need)):
                raise _error()
            rows = 12 * (self.nside >> (level + k)) ** 2
            out = np.empty((rows, need.value), dtype=np.int64)
            wts = np.empty((rows, need.value))
            if self._lib.stlp_operator_rows(self._handle, int(level), k, out.ctypes.data_as(C.POINTER(C.c_int64)),
                                            _ptr(wts), need.value, C.byref(need)):
                raise _error()
            return out, wts

    def set_masks(self, masks):
        """Averages every coefficient over each of K masks from the next forward
        on; None restores the whole sky.  masks: [npix] or [K, npix] indicators
        (nonzero: in the mask) or a sequence of K arrays of NESTED ids
        (native.py:243-264).  Values, variances and cotangents become
        [batch, K, ncoeff]."""
        w = _mask_weights(masks, self.npix)
        with self._mutex:
            self._open()
            self._current_key = None
            if self._lib.stlp_set_masks(self._handle, _ptr(w), w.shape[0]):
                raise _error()
            self.nmasks = w.shape[0]

    def synthesize(self, x, target, weights=None, options=None):
        """Synthesis on the device: L-BFGS (options of native_lbfgs) of
        sum_i w_i |S_i(x) - T_i|^2 from the CUDA float64 maps x [batch, npix],
        updated in place; the iterate, gradients and curvature pairs stay in
        device memory.  Returns (evaluations, losses per evaluation)."""
        import torch
        if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
            raise ValueError("x must be a contiguous CUDA float64 tensor")
        if x.numel() != self.batch * self.channels * self.npix:
            raise ValueError(f"expected {self.batch * self.channels * self.npix} map values, got {x.numel()}")
        t = np.ascontiguousarray(target, dtype=np.complex128).reshape(-1)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        if w is not None and w.shape != (self.ncoeff,):
            raise ValueError(f"expected {self.ncoeff} weights, got {w.shape}")
        opts = dict(options or {})
        cap = int(opts.get("max_eval") or int(opts.get("max_iter", 20)) * 5 // 4) + 1
        losses = np.zeros(cap)
        with self._mutex:
            self._open()
            self._current_key = None
            torch.cuda.synchronize(x.device)
            n = self._lib.stlp_synthesize_device(self._handle, x.data_ptr(), x.numel(), _ptr(t.view(np.float64)),
                                                 t.size, None if w is None else _ptr(w),
                                                 json.dumps(opts).encode(), _ptr(losses), losses.size)
            if n < 0:
                raise _error()
        return int(n), losses[:min(int(n), losses.size)]

    def _shape(self):
        head = (self.batch, 2) if self.spin else (self.batch,)
        return head + ((self.nmasks, self.ncoeff) if self.nmasks else (self.ncoeff,))

    def spin_fields(self, maps, level=0):
        """Spin 2: ((Q, U), (chi_E, chi_B)) of `level`, each [batch, 2, npix of the
        level] (the scalar pyramid has level 0 only; native.py:305-317)."""
        if not self.spin:
            raise RuntimeError("spin_fields needs NativeEngine(..., spin=2)")
        with self._mutex:
            self._open()
            x = np.ascontiguousarray(maps, dtype=np.float64).reshape(self._map_shape)
            n = 12 * (self.nside >> int(level)) ** 2
            qu = np.empty((self.batch, 2, n))
            chi = np.empty((self.batch, 2, n))
            if self._lib.stlp_spin_fields(self._handle, _ptr(x), x.size, int(level), _ptr(qu), _ptr(chi)):
                raise _error()
            return qu, chi

    def spin_rows(self, level, kind="stencil"):
        """Spin 2: the device-built operator rows (cells [rows, width] int64 padded
        with -1, complex weights [rows, width]): "stencil" the chi operator of
        `level`, "means" the transported means into level + 1."""
        k = {"stencil": 0, "means": 1}[kind]
        with self._mutex:
            self._open()
            need = C.c_size_t(0)
            if self._lib.stlp_spin_rows(self._handle, int(level), k, None, None, 0, C.byref(need)):
                raise _error()
            rows = 12 * (self.nside >> (level + k)) ** 2
            cells = np.empty((rows, need.value), dtype=np.int64)
            w = np.empty((rows, need.value), dtype=np.complex128)
            if self._lib.stlp_spin_rows(self._handle, int(level), k, cells.ctypes.data_as(C.POINTER(C.c_int64)),
                                        _ptr(w.view(np.float64)), need.value, C.byref(need)):
                raise _error()
            return cells, w

    def forward_cross(self, a, b, generation=0, member=0, objective="gaussian", moments=False):
        """Cross statistics of the pairs (a, b) (cross=True): a, b [batch, npix], or
        with spin 2 b [batch, 2, npix] (Q, U) and a [batch, 2, npix] or [batch, npix]."""
        if not self.cross:
            raise RuntimeError("forward_cross needs NativeEngine(..., cross=True)")
        if self.spin:
            return self.forward((a, b), generation, member, objective, moments)
        a = np.asarray(a, dtype=np.float64).reshape(self.batch, self.npix)
        b = np.asarray(b, dtype=np.float64).reshape(self.batch, self.npix)
        return self.forward(np.stack([a, b], 1), generation, member, objective, moments)

    def vjp_cross(self, cotangents, generation=0, member=0, objective="gaussian"):
        """(grad_a, grad_b) in the shapes of a and b, after forward_cross."""
        g = self.vjp(cotangents, generation, member, objective)
        return g if self.spin else (g[:, 0], g[:, 1])

    def _input(self, maps):
        """The library's input array of maps (spin-2 pairs: a then b, flat)."""
        if self.spin and self.cross:
            if not (isinstance(maps, (tuple, list)) and len(maps) == 2):
                raise ValueError("spin-2 cross maps are a pair (a, b)")
            pa = 2 if self.spin_a == 2 else 1
            a = np.asarray(maps[0], dtype=np.float64).reshape(self.batch, pa, self.npix)
            b = np.asarray(maps[1], dtype=np.float64).reshape(self.batch, 2, self.npix)
            return np.concatenate([a.ravel(), b.ravel()])
        x = np.ascontiguousarray(maps, dtype=np.float64)
        if x.shape == self._map_shape[1:] and self.batch == 1:
            x = x[None]
        if x.shape != self._map_shape:
            raise ValueError(f"expected maps {self._map_shape}, got {x.shape}")
        return x

    def native_pixels(self):
        """Pixels each coefficient averages: [K, ncoeff] with masks, else [ncoeff]."""
        with self._mutex:
            self._open()
            out = np.empty((max(self.nmasks, 1), self.ncoeff), dtype=np.uintp)
            if self._lib.stlp_native_pixels(self._handle, out.ctypes.data_as(_SIZE)):
                raise _error()
            out = out.astype(np.int64)
            return out if self.nmasks else out[0]

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.stlp_free(self._handle)
            self._handle = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *_):
        self.close()

    # -- host arrays (the reference's interface) ------------------------------
    def forward(self, maps, generation=0, member=0, objective="gaussian", moments=False):
        """Statistics of maps ``[batch, npix]`` (``[npix]`` when batch = 1), f64 NESTED."""
        with self._mutex:
            self._open()
            key = _key(generation, member, objective)
            x = self._input(maps)
            # non-finite values: the library counts them while it copies the maps (ValueError)
            values = np.empty(self._shape(), dtype=np.complex128)
            var = np.empty(self._shape() if moments else (self.batch, 0))
            self._current_key = None
            if self._lib.stlp_forward(self._handle, _ptr(x), x.size, *key, bool(moments),
                                      _ptr(values.view(np.float64)), _ptr(var)):
                raise _error()
            self._current_key = key
            return values, var

    def _require_state(self, key):
        # a VJP runs on the forward state of its own identity only
        if key != self._current_key:
            raise RuntimeError("no forward state of this identity: it is stale or was never computed")

    def _cotangent(self, cotangents):
        c = np.ascontiguousarray(cotangents, dtype=np.complex128)
        if c.shape == self._shape()[1:] and self.batch == 1:
            c = c[None]
        if c.shape != self._shape():
            raise ValueError(f"expected cotangents {self._shape()}, got {c.shape}")
        if not _all_finite(c):
            raise ValueError("non-finite coefficient cotangent")
        return c

    def vjp(self, cotangents, generation=0, member=0, objective="gaussian", out=None):
        """Gradient ``[batch, npix]`` of ``Re sum(conj(cotangents) * values)``.
        ``out``: a C-contiguous float64 array of the maps' size to write it into
        (returned in the maps' shape), instead of a new array: a caller that
        keeps one spares the page faults of fresh memory on every call."""
        with self._mutex:
            self._open()
            key = _key(generation, member, objective)
            self._require_state(key)
            c = self._cotangent(cotangents)
            size = int(np.prod(self._map_shape))
            if out is None:
                grad = np.empty(size)
            else:
                if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                        and out.size == size):
                    raise ValueError(f"out must be a C-contiguous float64 array of {size} values")
                grad = out.reshape(-1)
            if self._lib.stlp_vjp(self._handle, _ptr(c.view(np.float64)), c.size, *key, _ptr(grad)):
                raise _error()
            if self.spin and self.cross:  # (grad_a, grad_b) in the shapes of a and b
                pa = 2 if self.spin_a == 2 else 1
                ga, gb = np.split(grad, [self.batch * pa * self.npix])
                ga = ga.reshape(self.batch, 2, self.npix) if pa == 2 else ga.reshape(self.batch, self.npix)
                return ga, gb.reshape(self.batch, 2, self.npix)
            return grad.reshape(self._map_shape)

    def checkpoint(self):
        """A copy of the current forward state (the level-0 maps it ran on),
        tagged with that state's identity; restore() brings it back."""
        with self._mutex:
            self._open()
            saved = self._lib.stlp_checkpoint(self._handle)
            if not saved:
                raise _error()
            return Snapshot(saved, self._current_key, self._handle)

    def restore(self, snapshot, generation=0, member=0, objective="gaussian"):
        """Reinstates a Snapshot of this engine as the forward state of the
        identity (generation, member, objective), which must be the one the
        snapshot was taken under."""
        wanted = _key(generation, member, objective)
        live = isinstance(snapshot, Snapshot) and bool(snapshot._handle)
        if not live:
            raise ValueError("restore needs an open Snapshot from checkpoint()")
        with self._mutex:
            self._open()
            if snapshot.owner != self._handle:
                raise ValueError("the snapshot belongs to another engine")
            if snapshot.key != wanted:
                raise RuntimeError("the snapshot holds a stale or different forward identity")
            if self._lib.stlp_restore(self._handle, snapshot._handle, *wanted):
                raise _error()
            self._current_key = wanted

    # -- CUDA tensors -----------------------------------------------------------
    def _bind_stream(self, torch):
        s = torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        if s != self._stream:
            if self._lib.stlp_set_stream(self._handle, s):
                raise _error()
            self._stream = s

    def forward_tensor(self, x, generation=0, member=0, objective="gaussian", moments=False):
        """Statistics of a CUDA tensor ``[batch, npix]`` (float32 or float64), no host copy
        of the maps; runs on torch's current stream.  Returns numpy (values, var)."""
        import torch
        with self._mutex:
            self._open()
            key = _key(generation, member, objective)
            if not x.is_cuda or x.dtype not in (torch.float32, torch.float64):
                raise ValueError("forward_tensor needs a float32/float64 CUDA tensor")
            if x.numel() != int(np.prod(self._map_shape)):
                raise ValueError(f"expected {int(np.prod(self._map_shape))} map values, got {x.numel()}")
            x = x.detach().reshape(-1).contiguous()
            self._bind_stream(torch)
            values = np.empty(self._shape(), dtype=np.complex128)
            var = np.empty(self._shape() if moments else (self.batch, 0))
            self._current_key = None
            if self._lib.stlp_forward_device(self._handle, x.data_ptr(), x.numel(), int(x.dtype == torch.float32),
                                             *key, bool(moments), _ptr(values.view(np.float64)), _ptr(var)):
                raise _error()
            self._current_key = key
            return values, var

    def vjp_tensor(self, cotangents, out, generation=0, member=0, objective="gaussian"):
        """Writes the gradient into the CUDA tensor ``out`` ``[batch, npix]`` (float32/64)."""
        import torch
        with self._mutex:
            self._open()
            key = _key(generation, member, objective)
            self._require_state(key)
            if not (out.is_cuda and out.is_contiguous() and out.numel() == int(np.prod(self._map_shape))
                    and out.dtype in (torch.float32, torch.float64)):
                raise ValueError("out must be a contiguous float32/float64 CUDA tensor [batch, npix]")
            c = self._cotangent(cotangents)
            self._bind_stream(torch)
            if self._lib.stlp_vjp_device(self._handle, _ptr(c.view(np.float64)), c.size, *key, out.data_ptr(),
                                         int(out.dtype == torch.float32)):
                raise _error()
            return out


_generation = itertools.count(1)


def _function():
    import torch

    class ScatCov(torch.autograd.Function):
        """Statistics of a CUDA batch of maps as a differentiable torch op:
        x [batch, npix] -> complex128 [batch, ncoeff] on x's device."""

        @staticmethod
        def forward(ctx, x, engine):
            g = next(_generation)
            values, _ = engine.forward_tensor(x, generation=g)
            ctx.engine, ctx.generation = engine, g
            ctx.shape, ctx.dtype = x.shape, x.dtype
            return torch.from_numpy(values).to(x.device)

        @staticmethod
        def backward(ctx, gy):
            out = torch.empty(ctx.shape, dtype=ctx.dtype, device=gy.device)
            ctx.engine.vjp_tensor(gy.detach().resolve_conj().cpu().numpy(), out, generation=ctx.generation)
            return out, None

    return ScatCov


_ScatCov = None


def scattering(engine, x):
    """Differentiable statistics of the CUDA tensor x [batch, npix] (one forward state
    per engine: run backward before the next forward of the same engine)."""
    global _ScatCov
    if _ScatCov is None:
        _ScatCov = _function()
    return _ScatCov.apply(x, engine)


# options stlp_lbfgs reads (csrc/lbfgs.cpp), with their defaults
_LBFGS_DEFAULTS = {"lr": 1.0, "max_iter": 20, "max_eval": None, "tolerance_grad": 1e-12,
                   "tolerance_change": 1e-15, "history_size": 10}


def _is_count(v):
    """A positive whole number (bool excluded)."""
    if isinstance(v, bool) or not isinstance(v, (int, float, np.integer, np.floating)):
        return False
    return v >= 1 and float(v) == int(v)


def _lbfgs_options(options):
    opts = dict(_LBFGS_DEFAULTS)
    given = dict(options or {})
    extra = sorted(k for k in given if k not in opts)
    if extra:
        raise ValueError(f"unknown native L-BFGS options: {extra}")
    opts.update(given)
    for name in ("max_iter", "history_size"):
        if not _is_count(opts[name]):
            raise ValueError(f"{name} must be a positive integer")
    if opts["max_eval"] is not None and not _is_count(opts["max_eval"]):
        raise ValueError("max_eval must be a positive integer or None")
    return opts


class _LbfgsObjective:
    """The C callback of stlp_lbfgs around a Python callback(x) -> (loss, grad).

    The library owns the trial point and the gradient buffer: the callback
    sees the trial as a read-only array of the caller's shape and the gradient
    is copied into the library's buffer.  A Python exception cannot cross the
    C frames, so the first one is kept here and NaN is returned, which ends
    the library's iteration; native_lbfgs raises it afterwards."""

    def __init__(self, callback, shape):
        self.callback, self.shape = callback, shape
        self.losses, self.failure = [], None
        self.c_function = _CALLBACK(self._call)

    def _call(self, point, n, grad_out, _context):
        if self.failure is not None:
            return float("nan")
        try:
            trial = np.ctypeslib.as_array(point, shape=(n,)).reshape(self.shape)
            trial.flags.writeable = False
            loss, grad = self.callback(trial)
            grad = np.asarray(grad, dtype=np.float64)
            if grad.shape != self.shape:
                raise ValueError(f"callback gradient has shape {grad.shape}, the maps {self.shape}")
            np.copyto(np.ctypeslib.as_array(grad_out, shape=(n,)).reshape(self.shape), grad)
            loss = float(loss)
        except BaseException as exc:  # raised by native_lbfgs once the library returns
            self.failure = exc
            return float("nan")
        self.losses.append(loss)
        return loss


def native_lbfgs(callback, x, options=None):
    """Minimises callback(x) -> (loss, gradient) from x with the library's
    L-BFGS and strong Wolfe line search (stlp_lbfgs, the reference's
    native_lbfgs contract: options lr, max_iter, max_eval, tolerance_grad,
    tolerance_change, history_size).  A float64 C-contiguous x is updated in
    place (other arrays are converted first).  Returns (x, report) with the
    evaluation count and the loss of every evaluation."""
    opts = _lbfgs_options(options)
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.size == 0:
        raise ValueError("native_lbfgs needs a nonempty starting point")
    if not np.isfinite(x).all():
        raise ValueError("native_lbfgs needs a finite starting point")
    objective = _LbfgsObjective(callback, x.shape)
    evaluations = lib().stlp_lbfgs(_ptr(x), x.size, json.dumps(opts).encode(), objective.c_function, None)
    if objective.failure is not None:
        raise objective.failure
    if evaluations < 0:
        raise _error()
    report = {"evaluations": int(evaluations), "loss_history": objective.losses, "options": opts,
              "optimizer": "B200 engine L-BFGS (stlp_lbfgs)", "line_search": "strong_wolfe"}
    return x, report


def synthesis_objective(engine, target, weights=None):
    """Loss sum_k w_k |S_k(x) - T_k|^2 of maps x [batch, npix] and its gradient
    (the synthesis objective of crates/stl-mpi/src/synthesis.rs:207-270):
    a callback for native_lbfgs that evaluates S and the VJP on the engine."""
    target = np.asarray(target, dtype=np.complex128).reshape(engine.batch, engine.ncoeff)
    w = np.ones(engine.ncoeff) if weights is None else np.asarray(weights, dtype=np.float64)
    counter = itertools.count(1)

    def f(x):
        gen = next(counter)
        values, _ = engine.forward(np.asarray(x).reshape(engine.batch, -1), generation=gen)
        r = values - target
        loss = float(np.sum(w * (r.real ** 2 + r.imag ** 2)))
        grad = engine.vjp(2.0 * w * r, generation=gen)
        return loss, grad.reshape(np.shape(x))

    return f


class PatchEngine:
    """Statistics of disc patches and their VJP on the GPU (the reference's
    PatchEngine, native.py:1074-1370, one channel).  Discs are selected by centre
    (NESTED pixel ids at nside, or vectors [B, 3]), radius and optional core
    radius in degrees; the coefficients average the core (else the whole disc)."""

    def __init__(self, nside, j, kernel=5, orientations=4, dtype="float64", device=0, cache=256, threads=0,
                 group_pixels=None, profile=False, autotune=True, graphs=True):
        cfg = dict(nside=int(nside), j=int(j), kernel=int(kernel), orientations=int(orientations), backend="gpu",
                   dtype=dtype, device=int(device), cache=int(cache), threads=int(threads))
        if group_pixels is not None:  # level-0 pixels of the discs one batched engine holds
            cfg["group_pixels"] = int(group_pixels)
        if profile:  # per kernel class device times in info()["kernels"]
            cfg["profile"] = True
        if not autotune:  # keep the default tile heights
            cfg["autotune"] = False
        if not graphs:  # the sweeps kernel by kernel instead of as CUDA graphs
            cfg["graphs"] = False
        self._lib = lib()
        self._mutex = threading.RLock()
        self._handle = self._lib.stlp_patch_new(json.dumps(cfg).encode())
        if not self._handle:
            raise _error()
        self.nside, self.j, self.dtype = int(nside), int(j), dtype
        info = self.info()
        self.plan = info["plan"]
        self.ncoeff = len(self.plan)
        self.levels = info["levels"]
        self._native = np.array([c["native_dg"] for c in self.plan], dtype=np.int64)
        self.ids, self._selection, self._generation, self._dense = [], None, None, False
        self._xbuf = None  # the packed patches of the current selection

    def _open(self):
        if not self._handle:
            raise RuntimeError("patch engine is closed")

    def info(self):
        with self._mutex:
            self._open()
            p = self._lib.stlp_patch_info(self._handle)
            if not p:
                raise _error()
            try:
                return json.loads(C.string_at(p))
            finally:
                self._lib.stlp_string_free(p)

    def centre_vectors(self, centres):
        c = np.asarray(centres)
        if np.issubdtype(c.dtype, np.integer):
            ids = np.ascontiguousarray(c.reshape(-1), dtype=np.int64)
            out = np.empty((ids.size, 3), dtype=np.float64)
            if self._lib.stlp_pixel_vectors(self.nside, ids.ctypes.data_as(C.POINTER(C.c_int64)), ids.size, _ptr(out)):
                raise _error()
            return out
        c = np.ascontiguousarray(c, dtype=np.float64)
        if c.ndim == 1:
            c = c[None]
        if c.ndim != 2 or c.shape[1] != 3:
            raise ValueError("centres must be NESTED pixel indices [B] or vectors [B, 3]")
        return c

    def select(self, centres, radius, core=None):
        """Selects the discs (radius and core radius in degrees, one value for
        all discs or one per disc) and returns each disc's sorted NESTED
        pixels.  Selecting the same discs again costs nothing."""
        vectors = np.ascontiguousarray(self.centre_vectors(centres))
        n = vectors.shape[0]
        uniform = np.ndim(radius) == 0 and (core is None or np.ndim(core) == 0)
        radii = np.ascontiguousarray(np.radians(np.broadcast_to(np.asarray(radius, np.float64), (n,))))
        cores = np.zeros(n) if core is None else np.radians(np.broadcast_to(np.asarray(core, np.float64), (n,)))
        cores = np.ascontiguousarray(cores)
        ident = (vectors.tobytes(), radii.tobytes(), cores.tobytes())
        with self._mutex:
            self._open()
            if ident == self._selection:
                return self.ids
            self._generation = self._selection = None
            counts = np.empty(n, dtype=np.uintp)
            counts_p = counts.ctypes.data_as(_SIZE)
            if uniform:  # the reference's entry point: one radius per call
                status = self._lib.stlp_patch_select(self._handle, _ptr(vectors), n, np.radians(float(radius)),
                                                     0.0 if core is None else np.radians(float(core)), counts_p)
            else:
                status = self._lib.stlp_patch_select_radii(self._handle, _ptr(vectors), n, _ptr(radii),
                                                           _ptr(cores), counts_p)
            if status:
                raise _error()
            self.ids = [self._disc_pixels(i, int(c)) for i, c in enumerate(counts)]
            per_level = np.empty((n, self.levels), dtype=np.uintp)
            if self._lib.stlp_patch_core_pixels(self._handle, per_level.ctypes.data_as(_SIZE)):
                raise _error()
            self.native_pixels = per_level.astype(np.float64)[:, self._native]
            self._selection = ident
            return self.ids

    def _disc_pixels(self, i, count):
        out = np.empty(count, dtype=np.int64)
        if self._lib.stlp_patch_ids(self._handle, i, out.ctypes.data_as(C.POINTER(C.c_int64))):
            raise _error()
        return out

    def gather(self, maps):
        """The patches of the selected discs cut from full-sky maps ([npix]: one
        map for every disc; [B, npix]: map i for disc i)."""
        m = np.asarray(maps)
        if m.ndim == 1:
            return [m[i] for i in self.ids]
        return [m[k][..., i] for k, i in enumerate(self.ids)]

    def _pack(self, maps):
        """One float64 vector of the patches in disc order, checked against the
        selection's pixel counts."""
        if len(maps) != len(self.ids):
            raise ValueError(f"{len(maps)} patches given for {len(self.ids)} selected discs")
        sizes = [i.size for i in self.ids]
        flat = [np.asarray(m, dtype=np.float64) for m in maps]
        for i, (m, size) in enumerate(zip(flat, sizes)):
            if m.shape != (size,):
                raise ValueError(f"patch {i} has shape {m.shape}; its disc holds {size} pixels")
        if not flat:
            return np.zeros(0)
        # one buffer per selection, reused: the library has read it when the
        # call returns, and fresh memory would cost its page faults every call
        total = sum(sizes)
        if self._xbuf is None or self._xbuf.size != total:
            self._xbuf = np.empty(total, dtype=np.float64)
        return np.concatenate(flat, out=self._xbuf)

    def forward(self, maps, centres=None, radius=None, core=None, moments=True, generation=0, out=None):
        """Statistics [B, ncoeff] (and variances, or [B, 0]) of the patches of
        the selected discs (selecting them first when centres are given).
        ``out``: a C-contiguous complex128 array [B, ncoeff] to write the
        statistics into (returned), instead of a new one each call."""
        with self._mutex:
            self._open()
            if centres is not None:
                if radius is None:
                    raise ValueError("selecting discs needs a radius in degrees")
                self.select(centres, radius, core)
            if not self.ids:
                raise RuntimeError("forward before any disc was selected")
            x = self._pack(maps)  # non-finite values are counted by the library's copy (ValueError)
            b = len(self.ids)
            if out is None:
                values = np.empty((b, self.ncoeff), dtype=np.complex128)
            else:
                if not (isinstance(out, np.ndarray) and out.dtype == np.complex128 and out.flags.c_contiguous
                        and out.shape == (b, self.ncoeff)):
                    raise ValueError(f"out must be a C-contiguous complex128 array of shape {(b, self.ncoeff)}")
                values = out
            variance = np.empty((b, self.ncoeff if moments else 0), dtype=np.float64)
            self._generation = None
            self._dense = isinstance(maps, np.ndarray)
            status = self._lib.stlp_patch_forward(self._handle, _ptr(x), x.size, int(generation), bool(moments),
                                                  _ptr(values.view(np.float64)), _ptr(variance) if moments else None)
            if status:
                raise _error()
            self._generation = int(generation)
            return values, variance

    def vjp(self, cotangents, generation=0, out=None):
        """Gradients of Re sum(conj(cotangents) values) with respect to the
        patches of the forward of this generation, shaped like its maps.
        ``out``: a C-contiguous float64 array of the selection's total pixel
        count to write them into (the gradients returned are views of it):
        a caller that keeps one spares the page faults of fresh memory."""
        with self._mutex:
            self._open()
            if self._generation is None or int(generation) != self._generation:
                raise RuntimeError("no forward state of this generation: it is stale or was never computed")
            b = len(self.ids)
            c = np.ascontiguousarray(cotangents, dtype=np.complex128)
            if c.shape != (b, self.ncoeff):
                raise ValueError(f"cotangents have shape {c.shape}, the statistics {(b, self.ncoeff)}")
            if not _all_finite(c):
                raise ValueError("non-finite coefficient cotangent")
            sizes = np.array([i.size for i in self.ids], dtype=np.int64)
            total = int(sizes.sum())
            if out is None:
                grad = np.empty(total, dtype=np.float64)
            else:
                if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                        and out.size == total):
                    raise ValueError(f"out must be a C-contiguous float64 array of {total} values")
                grad = out.reshape(-1)
            if self._lib.stlp_patch_vjp(self._handle, _ptr(c.view(np.float64)), c.size, int(generation),
                                        _ptr(grad)):
                raise _error()
            parts = np.split(grad, np.cumsum(sizes)[:-1])
            return np.stack(parts) if self._dense else parts

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.stlp_patch_free(self._handle)
            self._handle = None

    def __del__(self):
        self.close()


class Terms:
    """The synthesis objective's extra terms on CUDA float64 tensors (the
    reference's device terms, crates/stl-gpu/src/terms.rs): the kappa
    transform of a monotone cubic table, the 4-children pyramid of rows
    [rows, len] with its detail moments and the level-power and kurtosis
    gradients, the stable sort of a row in f64 total order and the pixel
    marginal, and g += a b.  Launches go to torch's current stream; methods
    returning host values wait for it."""

    def __init__(self, rows=1, length=0, depth=0, sort=0, device=0):
        cfg = dict(rows=int(rows), len=int(length), depth=int(depth), sort=int(sort), device=int(device))
        self._lib = lib()
        self._handle = self._lib.stlp_terms_new(json.dumps(cfg).encode())
        if not self._handle:
            raise _error()
        self.rows, self.len, self.depth, self.sort_max, self.device = (cfg["rows"], cfg["len"], cfg["depth"],
                                                                       cfg["sort"], cfg["device"])

    def _call(self, name, *args):
        import torch
        if not self._handle:
            raise RuntimeError("terms handle is closed")
        s = torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        if self._lib.stlp_terms_set_stream(self._handle, s) or getattr(self._lib, name)(self._handle, *args):
            raise _error()

    @staticmethod
    def _dev(t, n=None, dtype=None):
        import torch
        want = dtype or torch.float64
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == want and t.is_contiguous()):
            raise ValueError(f"expected a contiguous CUDA {want} tensor")
        if n is not None and t.numel() != n:
            raise ValueError(f"expected {n} values, got {t.numel()}")
        return t.data_ptr()

    def kappa_table(self, x, y, d):
        kx, ky, kd = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, d))
        if not (kx.shape == ky.shape == kd.shape and kx.ndim == 1):
            raise ValueError("knots, values and slopes must be 1-d arrays of one length")
        self._call("stlp_terms_kappa_table", _ptr(kx), _ptr(ky), _ptr(kd), kx.size)

    def kappa(self, x, gm, gs, km, ks):
        """(k, dk) of the values x: k = (f(x gs + gm) - km) / ks, dk its derivative."""
        import torch
        k, dk = torch.empty_like(x), torch.empty_like(x)
        self._call("stlp_terms_kappa", self._dev(x), x.numel(), float(gm), float(gs), float(km), float(ks),
                   k.data_ptr(), dk.data_ptr())
        return k, dk

    def pyramid(self, x):
        self._call("stlp_terms_pyramid", self._dev(x, self.rows * self.len))

    def moments(self, x):
        """[rows, depth, 2]: (sum d^2, sum d^4) of the details of every level."""
        out = np.empty((self.rows, self.depth, 2))
        self._call("stlp_terms_moments", self._dev(x, self.rows * self.len), _ptr(out))
        return out

    def level_power_grad(self, x, coef, g):
        c = np.ascontiguousarray(coef, dtype=np.float64).reshape(self.rows, -1)
        self._call("stlp_terms_level_power_grad", self._dev(x, self.rows * self.len), _ptr(c), c.shape[1],
                   self._dev(g, self.rows * self.len))

    def kurtosis_grad(self, x, levels, cf, g, dk=None):
        lev = np.ascontiguousarray(levels, dtype=np.int32)
        c = np.ascontiguousarray(cf, dtype=np.float64).reshape(self.rows, lev.size, 3)
        self._call("stlp_terms_kurtosis_grad", self._dev(x, self.rows * self.len),
                   lev.ctypes.data_as(C.POINTER(C.c_int)), lev.size, _ptr(c),
                   0 if dk is None else self._dev(dk, self.rows * self.len), self._dev(g, self.rows * self.len))

    def sort(self, x):
        """int32 CUDA tensor of the positions of x in increasing f64 total order (ties by position)."""
        import torch
        perm = torch.empty(x.numel(), dtype=torch.int32, device=x.device)
        self._call("stlp_terms_sort", self._dev(x), x.numel(), perm.data_ptr())
        return perm

    def marginal(self, x, perm, t_sorted, coef, g):
        import torch
        out = np.zeros(1)
        self._call("stlp_terms_marginal", self._dev(x), self._dev(perm, x.numel(), torch.int32),
                   self._dev(t_sorted, x.numel()), x.numel(), float(coef), self._dev(g, x.numel()), _ptr(out))
        return float(out[0])

    def add_product(self, g, a, b=None):
        n = g.numel()
        self._call("stlp_terms_add_product", self._dev(g), self._dev(a, n), 0 if b is None else self._dev(b, n), n)

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.stlp_terms_free(self._handle)
            self._handle = None

    __del__ = close
