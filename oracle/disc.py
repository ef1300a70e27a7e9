"""FP64 disc-patch statistics on the CPU: the oracle of the patch engine.

TEST INFRASTRUCTURE ONLY (the checker of the CUDA patch engine; nothing in the
product imports it).  A numpy restatement of the reference's disc model
(crates/stl-core/src/disc.rs): the support of level 0 is every NESTED pixel
whose centre lies within the angle R of the disc centre (disc.rs:70-93), level
d + 1 holds the parents of level d; the pyramid is the smooth decimation
restricted to the support, the wavelet is bound to the support of its level
with the binding threshold BIND_EPS (disc.rs:38-44,163-168); the coefficients
are pixel means over the core of their native level (disc.rs:17-21), with the
term formulas and cotangents of the full-sky engine (engine.rs:1194-1277).
The wavelet and the decimation come from the C++ oracle (oracle.py).  Pixel
loops are vectorised over numpy arrays; meant for nside <= 64.
"""
from __future__ import annotations

import numpy as np

import oracle as O

BIND_EPS = 1e-9
L = 4


def pixel_vectors(nside, ids):
    """Unit vectors of the NESTED pixel centres (disc.rs:46-51)."""
    th, ph = O.centres(nside, np.asarray(ids, np.int64))[3:5]
    s = np.sin(th)
    return np.stack([s * np.cos(ph), s * np.sin(ph), np.cos(th)], axis=-1)


def angles(u, v):
    """atan2(|u x v|, u . v) of unit vectors (disc.rs:53-59)."""
    cr = np.cross(u, v)
    return np.arctan2(np.sqrt(np.sum(cr * cr, axis=-1)), np.sum(u * v, axis=-1))


def unit(v):
    v = np.asarray(v, np.float64)
    return v / np.sqrt(np.sum(v * v))


def disc_pixels(nside, centre, radius):
    """Sorted NESTED pixels whose centre is within `radius` of `centre` (every
    pixel from pi on); a scan of all pixels (the reference descends the
    hierarchy to the same set)."""
    ids = np.arange(12 * nside * nside, dtype=np.int64)
    if radius >= np.pi:
        return ids
    return ids[angles(unit(centre)[None, :], pixel_vectors(nside, ids)) <= radius]


class Disc:
    """Support, core and operators of one disc (DiscSupport + DiscGeometry)."""

    def __init__(self, nside, levels, centre, radius, core=None):
        self.nside, self.levels = nside, levels
        c = unit(centre)
        ids0 = disc_pixels(nside, c, radius)
        assert ids0.size > 0, "empty disc support"
        core0 = None
        if core is not None and 0 < core < radius:
            core0 = ids0[angles(c[None, :], pixel_vectors(nside, ids0)) <= core]
            assert core0.size > 0, "the core holds no pixel centre"
        self.ids = [ids0]
        self.down = []
        for d in range(levels - 1):
            coarse, indptr, indices, values = O.smooth_decimation(self.ids[d], nside >> d)
            assert np.array_equal(coarse, np.unique(self.ids[d] >> 2))
            self.ids.append(coarse)
            self.down.append((indptr, indices, values))
        self.core = []
        cc = core0
        for n in range(levels):
            self.core.append(np.arange(self.ids[n].size) if cc is None else np.searchsorted(self.ids[n], cc))
            cc = None if cc is None else np.unique(cc >> 2)

    def core_pixels(self):
        return [int(c.size) for c in self.core]

    def dec(self, d, x):
        """Decimation d -> d + 1 of rows x [..., n_d]."""
        indptr, indices, values = self.down[d]
        rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
        out = np.zeros(x.shape[:-1] + (indptr.size - 1,))
        np.add.at(out, (..., rows), x[..., indices] * values)
        return out

    def dec_t(self, d, g):
        """Transpose of dec: cotangents [..., n_{d+1}] -> [..., n_d]."""
        indptr, indices, values = self.down[d]
        rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
        out = np.zeros(g.shape[:-1] + (self.ids[d].size,))
        np.add.at(out, (..., indices), g[..., rows] * values)
        return out

    def conv(self, n, x):
        """Wavelet of rows x [R, n_n] on the support: complex [R, L, n_n]."""
        y = O.conv_forward(x, self.nside >> n, grid=self.ids[n], eps=BIND_EPS)
        return y[:, :, 0, :] + 1j * y[:, :, 1, :]

    def conv_t(self, n, gz):
        """Adjoint of conv: complex cotangents [R, L, n_n] -> [R, n_n]."""
        gy = np.stack([gz.real, gz.imag], axis=2)
        return O.conv_adjoint(gy, self.nside >> n, grid=self.ids[n], eps=BIND_EPS)


def _rn(z):
    return z / np.sqrt(np.abs(z) + 1e-8)


def _modvjp(z, g):
    m = np.abs(z)
    return np.where(m > 0, g * z / np.where(m > 0, m, 1.0), 0.0)


class DiscModel:
    """Statistics of one channel on a disc and their VJP (disc.rs:183-445)."""

    def __init__(self, J, L=4):
        self.J, self.L = J, L
        self.plan = O.build_plan(J, L)

    def forward(self, disc, x, moments=False):
        lv = disc.levels
        maps = [np.asarray(x, np.float64)]
        for d in range(lv - 1):
            maps.append(disc.dec(d, maps[d]))
        z, mods = [], {}
        for n in range(lv):
            zn = disc.conv(n, maps[n][None, :])[0]  # [L, n_n]
            mods[(n, n)] = np.abs(zn)
            for d in range(n):
                mods[(d, n)] = disc.dec(n - 1, mods[(d, n - 1)])
            z.append(zn)
        branch = {}
        for c in self.plan:
            if c["family"] in ("S3", "S4"):
                branch.setdefault((c["j1"], c["native_dg"]), None)
                if c["family"] == "S4":
                    branch.setdefault((c["j2"], c["native_dg"]), None)
        for (d, n) in list(branch):
            branch[(d, n)] = disc.conv(n, mods[(d, n)])[:, :, disc.core[n]]  # [L(l1), L(l3), core]
        self.state = dict(maps=maps, z=z, mods=mods, branch=branch)
        values = np.empty(len(self.plan), np.complex128)
        var = np.empty(len(self.plan))
        for i, c in enumerate(self.plan):
            a, b = self._operands(disc, c)
            t = self._term(c, a, b)
            values[i] = t.mean()
            if moments:
                var[i] = max(np.mean(np.abs(t) ** 2) - abs(values[i]) ** 2, 0.0)
        return (values, var) if moments else values

    def _operands(self, disc, c):
        s, n = self.state, c["native_dg"]
        core = disc.core[n]
        f = c["family"]
        if f in ("mean", "var"):
            return s["maps"][0][disc.core[0]].astype(np.complex128), None
        if f in ("S1", "S2"):
            v = s["z"][n][c["l1"], core]
            return v, v
        if f == "S3":
            return s["branch"][(c["j1"], n)][c["l1"], c["l3"]], s["z"][n][c["l3"], core]
        return s["branch"][(c["j1"], n)][c["l1"], c["l3"]], s["branch"][(c["j2"], n)][c["l2"], c["l3"]]

    @staticmethod
    def _term(c, a, b):
        f = c["family"]
        if f == "mean":
            return a
        if f in ("var", "S2"):
            return np.abs(a) ** 2 + 0j
        if f == "S1":
            return np.abs(a) + 0j
        return a * np.conj(b)

    def reverse(self, disc, cot):
        """Patch cotangent of the coefficient cotangents (gradient of Re sum conj(cot) S)."""
        s, lv = self.state, disc.levels
        gmaps = [np.zeros(disc.ids[n].size) for n in range(lv)]
        gz = [np.zeros((self.L, disc.ids[n].size), np.complex128) for n in range(lv)]
        gbranch, gmod = {}, {}
        for n in range(lv - 1, -1, -1):
            core = disc.core[n]
            nc = core.size
            for i, c in enumerate(self.plan):
                g = cot[i]
                if c["native_dg"] != n or g == 0:
                    continue
                a, b = self._operands(disc, c)
                f = c["family"]
                if f == "mean":
                    gmaps[0][disc.core[0]] += g.real / nc
                elif f == "var":
                    gmaps[0][disc.core[0]] += 2.0 * g.real * a.real / nc
                elif f == "S1":
                    gz[n][c["l1"], core] += _modvjp(a, g.real / nc)
                elif f == "S2":
                    gz[n][c["l1"], core] += 2.0 * g.real * a / nc
                elif f == "S3":
                    key = (c["j1"], n)
                    gbranch.setdefault(key, np.zeros((self.L, self.L, nc), np.complex128))
                    gbranch[key][c["l1"], c["l3"]] += g * b / nc
                    gz[n][c["l3"], core] += np.conj(g) * a / nc
                else:
                    for key, l1, v in (((c["j1"], n), c["l1"], g * b / nc), ((c["j2"], n), c["l2"], np.conj(g) * a / nc)):
                        gbranch.setdefault(key, np.zeros((self.L, self.L, nc), np.complex128))
                        gbranch[key][l1, c["l3"]] += v
            for key in [k for k in gbranch if k[1] == n]:
                full = np.zeros((self.L, self.L, disc.ids[n].size), np.complex128)
                full[:, :, core] = gbranch.pop(key)
                gmod[key] = gmod.get(key, 0.0) + disc.conv_t(n, full)
            for d in range(n):
                if (d, n) in gmod:
                    gmod[(d, n - 1)] = gmod.get((d, n - 1), 0.0) + disc.dec_t(n - 1, gmod.pop((d, n)))
            if (n, n) in gmod:
                gz[n] += _modvjp(s["z"][n], gmod.pop((n, n)))
            if np.any(gz[n] != 0):
                gmaps[n] += disc.conv_t(n, gz[n][None, :, :])[0]
        for n in range(lv - 1, 0, -1):
            gmaps[n - 1] += disc.dec_t(n - 1, gmaps[n])
        return gmaps[0]
