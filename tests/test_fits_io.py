"""FITS image layers through the C ABI (reference src/io.cpp:79-178 behind
_core.read_fits / write_fits, src/bindings.cpp:128-166): round trips, the
written file checked against the FITS standard by an independent parser here,
and hand-built files of other BITPIX / layouts read back. Host only."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import _core


def _card(key, value=None, comment=""):
    if value is None:
        return f"{key:<80}"[:80]
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, str):
        v = f"{chr(39) + value.ljust(8) + chr(39):<20}"
    else:
        v = f"{value:>20}"
    return f"{key:<8}= {v} / {comment}".ljust(80)[:80]


def _hdu(cards, data: bytes = b""):
    head = "".join(cards) + _card("END")
    head += " " * (-len(head) % 2880)
    return head.encode("ascii") + data + b"\0" * (-len(data) % 2880)


def _image(primary, bitpix, arr, extra=()):
    h, w = arr.shape
    cards = [_card("SIMPLE", True)] if primary else [_card("XTENSION", "IMAGE")]
    cards += [_card("BITPIX", bitpix), _card("NAXIS", 2), _card("NAXIS1", w), _card("NAXIS2", h)]
    cards += [_card("EXTEND", True)] if primary else [_card("PCOUNT", 0), _card("GCOUNT", 1)]
    cards += list(extra)
    return _hdu(cards, arr.tobytes())


def _parse(raw: bytes):
    """Independent reader of the written file: (cards, data bytes) per HDU."""
    out, pos = [], 0
    while pos < len(raw):
        cards = []
        while True:
            block = raw[pos : pos + 2880]
            assert len(block) == 2880
            pos += 2880
            cs = [block[i : i + 80].decode("ascii") for i in range(0, 2880, 80)]
            cards += cs
            if any(c.startswith("END ") for c in cs):
                break
        kw = {}
        for c in cards:
            if c[8:10] == "= ":
                val = c[10:].split("/")[0].strip().strip("'").strip()
                kw[c[:8].strip()] = val
        n = abs(int(kw["BITPIX"])) // 8
        for i in range(1, int(kw["NAXIS"]) + 1):
            n *= int(kw[f"NAXIS{i}"])
        out.append((cards, kw, raw[pos : pos + n]))
        pos += n + (-n % 2880)
    return out


def test_round_trip_and_standard_layout(tmp_path):
    rng = np.random.default_rng(0)
    data = rng.normal(size=(37, 53)).astype(np.float32)
    var = rng.uniform(1, 2, size=data.shape).astype(np.float32)
    mask = (rng.uniform(size=data.shape) < 0.1).astype(np.uint8) * 5
    path = tmp_path / "frame.fits"
    _core.write_fits(str(path), data, var, mask)
    got = _core.read_fits(str(path))
    assert got["data"].dtype == np.float32 and got["mask"].dtype == np.uint8
    np.testing.assert_array_equal(got["data"], data)
    np.testing.assert_array_equal(got["variance"], var)
    np.testing.assert_array_equal(got["mask"], mask)

    raw = path.read_bytes()
    assert len(raw) % 2880 == 0
    hdus = _parse(raw)
    assert [kw.get("EXTNAME") for _, kw, _ in hdus] == [None, "VARIANCE", "MASK"]
    cards0, kw0, d0 = hdus[0]
    assert cards0[0].startswith("SIMPLE  =") and cards0[0][29] == "T"
    assert [c[:8].strip() for c in cards0[:5]] == ["SIMPLE", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2"]
    assert kw0["BITPIX"] == "-32" and kw0["NAXIS1"] == "53" and kw0["NAXIS2"] == "37"
    assert d0 == data.astype(">f4").tobytes()
    cards1, kw1, d1 = hdus[1]
    assert cards1[0].startswith("XTENSION= 'IMAGE   '") and kw1["PCOUNT"] == "0" and kw1["GCOUNT"] == "1"
    assert d1 == var.astype(">f4").tobytes()
    assert hdus[2][1]["BITPIX"] == "8" and hdus[2][2] == mask.tobytes()


def test_optional_layers_and_overwrite(tmp_path):
    data = np.arange(12, dtype=np.float32).reshape(3, 4)
    path = str(tmp_path / "d.fits")
    _core.write_fits(path, data)
    got = _core.read_fits(path)
    assert got["variance"] is None and got["mask"] is None
    with pytest.raises(RuntimeError, match="exists"):
        _core.write_fits(path, data)
    _core.write_fits(path, data * 2, overwrite=True)
    np.testing.assert_array_equal(_core.read_fits(path)["data"], data * 2)
    with pytest.raises(RuntimeError, match="variance shape"):
        _core.write_fits(path, data, np.zeros((2, 2), np.float32), overwrite=True)
    with pytest.raises(RuntimeError, match="mask shape"):
        _core.write_fits(path, data, None, np.zeros((2, 2), np.uint8), overwrite=True)


def test_reads_scaled_integers_and_difference_extension(tmp_path):
    rng = np.random.default_rng(1)
    # unsigned 16-bit convention: stored int16 = value - 32768 (BZERO 32768)
    u = rng.integers(0, 65535, size=(5, 7)).astype(np.int64)
    path = tmp_path / "u16.fits"
    path.write_bytes(_image(True, 16, (u - 32768).astype(">i2"), [_card("BZERO", 32768), _card("BSCALE", 1)]))
    np.testing.assert_array_equal(_core.read_fits(str(path))["data"], u.astype(np.float32))

    # dataless primary, an unrelated binary table (with a heap), then the
    # DIFFERENCE (float64), VARIANCE (scaled int32) and MASK (int16) images
    d = rng.normal(size=(4, 6))
    v = rng.integers(0, 1000, size=d.shape)
    m = rng.integers(0, 4, size=d.shape)
    table = _hdu([_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2), _card("NAXIS1", 4),
                  _card("NAXIS2", 3), _card("PCOUNT", 10), _card("GCOUNT", 1), _card("TFIELDS", 1),
                  _card("TFORM1", "1J"), _card("EXTNAME", "CATALOG")], bytes(22))
    raw = _hdu([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)])
    raw += table
    raw += _image(False, -64, d.astype(">f8"), [_card("EXTNAME", "DIFFERENCE")])
    raw += _image(False, 32, v.astype(">i4"), [_card("BSCALE", 0.5), _card("EXTNAME", "variance")])
    raw += _image(False, 16, m.astype(">i2"), [_card("EXTNAME", "MASK")])
    path = tmp_path / "diff.fits"
    path.write_bytes(raw)
    got = _core.read_fits(str(path))
    np.testing.assert_array_equal(got["data"], d.astype(np.float32))
    np.testing.assert_array_equal(got["variance"], (0.5 * v).astype(np.float32))
    np.testing.assert_array_equal(got["mask"], m.astype(np.uint8))


def test_read_errors(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        _core.read_fits(str(tmp_path / "missing.fits"))
    empty = tmp_path / "empty.fits"
    empty.write_bytes(_hdu([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0)]))
    with pytest.raises(RuntimeError, match="no DIFFERENCE extension"):
        _core.read_fits(str(empty))
    comp = tmp_path / "comp.fits"
    comp.write_bytes(
        _hdu([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)])
        + _hdu([_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2), _card("NAXIS1", 8),
                _card("NAXIS2", 1), _card("PCOUNT", 0), _card("GCOUNT", 1), _card("TFIELDS", 1),
                _card("TFORM1", "1PB(0)"), _card("ZIMAGE", True), _card("EXTNAME", "DIFFERENCE")], bytes(8)))
    with pytest.raises(RuntimeError, match="tile-compressed"):
        _core.read_fits(str(comp))
    bad = tmp_path / "badmask.fits"
    a = np.zeros((2, 3), np.float32)
    bad.write_bytes(_image(True, -32, a.astype(">f4")) + _image(False, 16, np.full((2, 3), 300, ">i2"),
                                                                  [_card("EXTNAME", "MASK")]))
    with pytest.raises(RuntimeError, match="MASK value"):
        _core.read_fits(str(bad))
    notfits = tmp_path / "x.fits"
    notfits.write_bytes(b"hello" * 600)
    with pytest.raises(RuntimeError, match="SIMPLE"):
        _core.read_fits(str(notfits))


@pytest.mark.parametrize("card,value,match", [("NAXIS1", -5760, "negative NAXISn"), ("PCOUNT", -2880, "PCOUNT"),
                                              ("GCOUNT", 0, "GCOUNT"), ("NAXIS2", 2**62, "overflows")])
def test_hostile_sizes_are_refused_not_looped(tmp_path, card, value, match):
    """Header sizes are untrusted: a negative axis or count would move the next
    HDU offset backwards onto an earlier header (parsed again forever), and a
    huge one would overflow the byte count. Each must fail at once."""
    a = np.zeros((2, 3), np.float32)
    ext_cards = [_card("XTENSION", "IMAGE"), _card("BITPIX", -32), _card("NAXIS", 2), _card("NAXIS1", 3),
                 _card("NAXIS2", 2), _card("PCOUNT", 0), _card("GCOUNT", 1), _card("EXTNAME", "VARIANCE")]
    ext_cards = [_card(card, value) if c.startswith(card.ljust(8)) else c for c in ext_cards]
    path = tmp_path / "hostile.fits"
    path.write_bytes(_image(True, -32, a.astype(">f4")) + _hdu(ext_cards, bytes(24)))
    with pytest.raises(RuntimeError, match=match):
        _core.read_fits(str(path))


def test_read_refuses_a_data_layer_of_another_shape(tmp_path):
    """dgpu_fits_read takes the caller's buffer shape and writes nothing when
    the file's data layer differs from it (e.g. the file changed after the probe)."""
    import ctypes

    from delta_b200 import _lib

    path = tmp_path / "a.fits"
    _core.write_fits(str(path), np.ones((4, 5), np.float32))
    buf = np.zeros((3, 5), np.float32)
    rc = _lib.lib().dgpu_fits_read(str(path).encode(), ctypes.c_int64(5), ctypes.c_int64(3),
                                   buf.ctypes.data_as(ctypes.c_void_p), None, None)
    assert rc == _lib.DGPU_ERR_INVALID
    assert b"4" in _lib.lib().dgpu_last_error(None)
    assert not buf.any()


def test_pinned_style_allocator(tmp_path):
    data = np.arange(20, dtype=np.float32).reshape(4, 5)
    path = str(tmp_path / "a.fits")
    _core.write_fits(path, data, data + 1)
    seen = []

    def alloc(shape, dtype):
        seen.append((shape, np.dtype(dtype)))
        return np.zeros(shape, dtype)

    got = _core.read_fits(path, alloc=alloc)
    assert seen == [((4, 5), np.dtype(np.float32)), ((4, 5), np.dtype(np.float32))]
    np.testing.assert_array_equal(got["variance"], data + 1)


def _solution():
    from delta_b200.solution import KernelSolution

    return KernelSolution(beta=1.25, n_max=2, radius=4, knots=np.zeros((9, 2)), theta=np.ones(63), n_components=6,
                          n_spatial=9, lam=1e-6, gcv=0.5, effective_dof=12.5, rss=3.0, component_sums=np.ones(6),
                          direction="reference", shape=(3, 4), reduced_chi2=1.01, n_stamps_used=10,
                          n_stamps_rejected=2)


def test_diffresult_write_uncompressed_without_astropy(tmp_path):
    """DiffResult.write(compress=False) without astropy: the reference's
    uncompressed layout (difference + provenance cards in the primary, VARIANCE,
    MASK, SCORE images, CATALOG table), checked by the independent parser."""
    try:
        import astropy  # noqa: F401
    except ImportError:
        pass
    else:
        pytest.skip("astropy present: DiffResult.write goes through it, as in the reference")
    from delta_b200.catalog import CATALOG_DTYPE
    from delta_b200.pipeline import DiffResult

    rng = np.random.default_rng(3)
    d = rng.normal(size=(3, 4)).astype(np.float32)
    cat = np.zeros(2, dtype=CATALOG_DTYPE)
    cat["x"], cat["peak_x"], cat["quality"] = [1.5, 2.25], [1, 2], [0, 3]
    cat["is_dipole"] = [False, True]
    res = DiffResult(difference=d, variance=d * d, mask=np.eye(3, 4, dtype=np.uint8), score=d * 2,
                     solution=_solution(), source_catalog=cat, config={"DLTPREC": "mixed"}, elapsed=0.25)
    path = tmp_path / "prod.fits"
    res.write(str(path), compress=False)
    with pytest.raises(OSError):
        res.write(str(path), compress=False)
    res.write(str(path), compress=False, overwrite=True, extra_cards={"DLTNOTE": "x"})
    with pytest.raises(ImportError, match="compress"):
        res.write(str(path), overwrite=True)

    raw = path.read_bytes()
    pos, hdus = 0, []
    while pos < len(raw):
        cards = []
        while True:
            block = raw[pos : pos + 2880]
            pos += 2880
            cs = [block[i : i + 80].decode("ascii") for i in range(0, 2880, 80)]
            cards += cs
            if any(c.startswith("END ") for c in cs):
                break
        kw = {c[:8].strip(): c[10:].split("/")[0].strip().strip("'").strip() for c in cards if c[8:10] == "= "}
        n = abs(int(kw["BITPIX"])) // 8 * int(kw["NAXIS1"]) * int(kw["NAXIS2"])
        hdus.append((kw, raw[pos : pos + n]))
        pos += n + (-n % 2880)
    assert [kw.get("EXTNAME") for kw, _ in hdus] == [None, "VARIANCE", "MASK", "SCORE", "CATALOG"]
    kw0, d0 = hdus[0]
    assert d0 == d.astype(">f4").tobytes()
    assert kw0["DLTBETA"] == "1.25" and kw0["DLTCONV"] == "reference" and kw0["DLTNOTE"] == "x"
    assert kw0["DLTPREC"] == "mixed" and kw0["DLTNSTU"] == "10" and kw0["DLTELAP"] == "0.25"
    np.testing.assert_array_equal(_core.read_fits(str(path))["data"], d)
    kwt, rows = hdus[4]
    assert kwt["XTENSION"] == "BINTABLE" and int(kwt["TFIELDS"]) == len(CATALOG_DTYPE.names)
    names = [kwt[f"TTYPE{i}"] for i in range(1, len(CATALOG_DTYPE.names) + 1)]
    assert names == list(CATALOG_DTYPE.names)
    assert kwt["TFORM1"] == "D" and kwt["TFORM3"] == "J"
    be = np.dtype([("x", ">f8"), ("y", ">f8"), ("peak_x", ">i4")])
    first = np.frombuffer(rows, dtype=np.uint8).reshape(2, -1)[:, : be.itemsize].copy().view(be).ravel()
    np.testing.assert_array_equal(first["x"], cat["x"])
    np.testing.assert_array_equal(first["peak_x"], cat["peak_x"])


def test_product_header_cards_follow_the_fixed_format():
    from delta_b200._fits_products import card

    c = card("DLTLAM", 1e-06, "lambda")
    assert len(c) == 80 and c[:10] == "DLTLAM  = " and c[10:30].strip() == "1E-06" and c[30:33] == " / "
    assert card("DLTDECOR", True)[29] == "T" and card("DLTNMAX", 6)[10:30] == f"{6:>20}"
    s = card("DLTCONV", "it's")
    assert s[10] == "'" and "'it''s" in s
    assert card("END") == "END".ljust(80)
    with pytest.raises(ValueError):
        card("TOOLONGKEY", 1)
    with pytest.raises(ValueError):
        card("DLTCHI2", float("nan"))
    with pytest.raises(ValueError):
        card("DLTNOTE", "x" * 69)


def test_subtract_files_validates_before_any_work(tmp_path):
    import delta_b200 as delta

    with pytest.raises(ValueError, match="one path per pair"):
        delta.subtract_files([("a.fits", "b.fits")], [], device_resident=False)
    assert delta.subtract_files([], device_resident=False) == []
