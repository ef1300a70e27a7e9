"""Map files through the library (stlp_map_*, stlp_npy_*, stlp_fits_write):
the behaviour of the reference's io.rs (crates/stl-mpi/src/io.rs, its test
fits_and_npy_roundtrip at :519-568) -- .npy of every float and integer
dtype in either byte order read as float64, written as '<f8' that numpy
reads back; HEALPix FITS tables ('E' / 'D', rows of several pixels, other
HDUs before the table, RING maps reordered to NESTED with the oracle's
ring2nest); pixel ranges read at their offset; files written in pieces."""
import numpy as np
import pytest

import oracle as O

S = pytest.importorskip("stl_b200")

BLOCK = 2880


def card(key, value=None):
    c = key.ljust(8)
    if value is not None:
        c += "= " + value.rjust(20)
    return c.ljust(80)


def quoted(s):
    return ("'" + s.ljust(8) + "'").ljust(20)


def fits_bytes(values, form, ordering="NESTED", extra_hdu=False):
    """A HEALPix FITS file built here, field by field from the FITS rules:
    the values big-endian, `form` 'E', 'D' or 'nE' / 'nD' (n pixels a row)."""
    code = form[-1]
    repeat = int(form[:-1]) if len(form) > 1 else 1
    dt = ">f4" if code == "E" else ">f8"
    v = np.asarray(values, dtype=dt)
    rows = v.size // repeat
    out = b""
    prim = card("SIMPLE", "T") + card("BITPIX", "8") + card("NAXIS", "0") + card("EXTEND", "T") + card("END")
    out += prim.encode().ljust(BLOCK, b" ")
    if extra_hdu:  # an image extension of 3 x 5 int16 before the table
        img = (card("XTENSION", quoted("IMAGE")) + card("BITPIX", "16") + card("NAXIS", "2") + card("NAXIS1", "3")
               + card("NAXIS2", "5") + card("PCOUNT", "0") + card("GCOUNT", "1") + card("END"))
        out += img.encode().ljust(BLOCK, b" ")
        out += np.arange(15, dtype=">i2").tobytes().ljust(BLOCK, b"\0")
    hdr = (card("XTENSION", quoted("BINTABLE")) + card("BITPIX", "8") + card("NAXIS", "2")
           + card("NAXIS1", str(repeat * v.itemsize)) + card("NAXIS2", str(rows)) + card("PCOUNT", "0")
           + card("GCOUNT", "1") + card("TFIELDS", "1") + card("TTYPE1", quoted("TEMPERATURE"))
           + card("TFORM1", quoted(form)) + card("ORDERING", quoted(ordering)) + card("END"))
    out += hdr.encode().ljust(BLOCK, b" ")
    data = v.tobytes()
    return out + data + b"\0" * ((-len(data)) % BLOCK)


@pytest.mark.parametrize("dtype", ["<f8", ">f8", "<f4", ">f4", "<i8", ">i8", "<i4", ">i4"])
def test_npy_dtypes_read_as_float64(tmp_path, dtype):
    rng = np.random.default_rng(1)
    a = (rng.standard_normal(12 * 16 * 16) * 1000).astype(dtype)
    p = tmp_path / "m.npy"
    np.save(p, a)
    np.testing.assert_array_equal(S.read_map(p), a.astype(np.float64))
    assert S.map_len(p) == a.size
    np.testing.assert_array_equal(S.read_map_range(p, 37, 1001), a[37:1001].astype(np.float64))
    np.testing.assert_array_equal(S.read_map_range(p, 5, 5), np.zeros(0))


def test_npy_shapes_and_writer(tmp_path):
    rng = np.random.default_rng(2)
    for shape in [(7,), (3, 4), (2, 3, 5), ()]:
        a = rng.standard_normal(shape)
        p = tmp_path / "w.npy"
        S.write_npy(p, a)
        b = np.load(p)
        assert b.dtype == np.float64 and b.shape == a.shape
        np.testing.assert_array_equal(b, a)
        r = S.read_npy(p)
        assert r.shape == a.shape
        np.testing.assert_array_equal(r, a)
        with open(p, "rb") as f:
            head = f.read(10)
        assert head[:8] == b"\x93NUMPY\x01\x00" and (10 + int.from_bytes(head[8:10], "little")) % 64 == 0
    q = tmp_path / "v2.npy"  # a version 2.0 header
    np.lib.format.write_array(open(q, "wb"), np.arange(48.0).reshape(4, 12), version=(2, 0))
    np.testing.assert_array_equal(S.read_npy(q), np.arange(48.0).reshape(4, 12))


def test_npy_refusals(tmp_path):
    p = tmp_path / "f.npy"
    np.save(p, np.asfortranarray(np.ones((3, 4))))
    with pytest.raises(RuntimeError, match="Fortran"):
        S.read_map(p)
    np.save(p, np.zeros(4, dtype=[("a", "<f8"), ("b", "<i4")]))
    with pytest.raises(RuntimeError, match="structured"):
        S.read_map(p)
    np.save(p, np.zeros(4, dtype=np.complex128))
    with pytest.raises(RuntimeError, match="dtype"):
        S.read_map(p)
    (tmp_path / "x.npy").write_bytes(b"not a numpy file at all")
    with pytest.raises(RuntimeError, match="not a .npy"):
        S.read_map(tmp_path / "x.npy")
    np.save(p, np.arange(10.0))
    with pytest.raises(RuntimeError, match="beyond"):
        S.read_map_range(p, 5, 11)
    with pytest.raises(RuntimeError):
        S.read_map(tmp_path / "missing.npy")


@pytest.mark.parametrize("double", [False, True])
def test_fits_writer_round_trip_and_layout(tmp_path, double):
    rng = np.random.default_rng(3)
    nside = 16
    v = rng.standard_normal(12 * nside * nside)
    p = tmp_path / "m.fits"
    S.write_healpix_fits(p, v, column="VALUE", double=double)
    expect = v if double else v.astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(S.read_map(p), expect)
    assert S.map_len(p) == v.size
    np.testing.assert_array_equal(S.read_map_range(p, 37, 101), expect[37:101])
    raw = p.read_bytes()
    assert len(raw) % BLOCK == 0
    header = raw[BLOCK:2 * BLOCK].decode("ascii")
    cards = [header[i:i + 80] for i in range(0, BLOCK, 80)]
    assert cards[0] == card("XTENSION", quoted("BINTABLE"))
    assert card("TFORM1", quoted("D" if double else "E")) in cards
    assert card("TTYPE1", quoted("VALUE")) in cards
    assert card("ORDERING", quoted("NESTED")) in cards
    assert card("NSIDE", str(nside)) in cards
    assert card("NAXIS2", str(v.size)) in cards
    assert card("END") in cards
    data = np.frombuffer(raw[2 * BLOCK:2 * BLOCK + v.size * (8 if double else 4)], dtype=">f8" if double else ">f4")
    np.testing.assert_array_equal(data.astype(np.float64), expect)
    with pytest.raises(RuntimeError, match="full-sky"):
        S.write_healpix_fits(tmp_path / "bad.fits", np.ones(100))


@pytest.mark.parametrize("form", ["E", "D", "64E", "1024D"])
def test_fits_tables_of_other_writers(tmp_path, form):
    """Rows of several pixels (as healpy writes them) and an image HDU before
    the table: the map is the first column, pixel after pixel."""
    rng = np.random.default_rng(4)
    v = rng.standard_normal(12 * 32 * 32)
    p = tmp_path / "o.fits"
    p.write_bytes(fits_bytes(v, form, extra_hdu=True))
    expect = v.astype(np.float32).astype(np.float64) if form.endswith("E") else v
    np.testing.assert_array_equal(S.read_map(p), expect)
    assert S.map_len(p) == v.size
    for a, b in [(0, 1), (63, 65), (1000, 5000), (v.size - 3, v.size)]:
        np.testing.assert_array_equal(S.read_map_range(p, a, b), expect[a:b])


def test_ring_fits_is_reordered_to_nested(tmp_path):
    nside = 8
    order = 3
    rng = np.random.default_rng(5)
    nest = rng.standard_normal(12 * nside * nside)
    ring_ids = np.arange(nest.size, dtype=np.int64)
    nest_of_ring = O.ring2nest(order, ring_ids)  # NESTED id of every RING pixel
    ring = nest[nest_of_ring]  # the map in RING order
    p = tmp_path / "r.fits"
    p.write_bytes(fits_bytes(ring, "D", ordering="RING"))
    np.testing.assert_array_equal(S.read_map(p), nest)
    np.testing.assert_array_equal(S.read_map_range(p, 100, 300), nest[100:300])
    q = tmp_path / "u.fits"
    q.write_bytes(fits_bytes(ring, "D", ordering="GALACTIC"))
    with pytest.raises(RuntimeError, match="ORDERING"):
        S.read_map(q)


@pytest.mark.parametrize("name,double", [("s.npy", False), ("s.fits", False), ("d.fits", True)])
def test_maps_written_in_pieces(tmp_path, name, double):
    """io.rs SlicedMap: the headers and the size first, then every piece at
    its offset, in any order."""
    rng = np.random.default_rng(6)
    v = rng.standard_normal(12 * 16 * 16)
    p = tmp_path / name
    out = S.SlicedMap(p, double=double)
    out.create(v.size, column="VALUE")
    starts = list(range(0, v.size, 50))
    for s in reversed(starts):
        out.write(s, v[s:s + 50])
    expect = v.astype(np.float32).astype(np.float64) if name == "s.fits" else v
    np.testing.assert_array_equal(S.read_map(p), expect)
    np.testing.assert_array_equal(S.read_map_range(p, 60, 130), expect[60:130])
    if name.endswith(".fits"):
        assert p.stat().st_size % BLOCK == 0
        np.testing.assert_array_equal(S.read_map(p), S.read_map(_whole(tmp_path, v, double)))
    else:
        np.testing.assert_array_equal(np.load(p), v)
    with pytest.raises(RuntimeError, match="beyond"):
        out.write(v.size - 10, np.ones(20))


def _whole(tmp_path, v, double):
    q = tmp_path / "whole.fits"
    S.write_healpix_fits(q, v, column="VALUE", double=double)
    return q
