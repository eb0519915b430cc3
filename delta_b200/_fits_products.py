"""Uncompressed multi-extension FITS product of DiffResult.write without astropy.

The reference writes its products through astropy (python/delta/pipeline.py:150-194).
When astropy is not installed, ``DiffResult.write(..., compress=False)`` uses
this writer for the same layout: the difference in the primary HDU with the
provenance cards, then VARIANCE, MASK and SCORE image extensions and the
CATALOG binary table. It follows the FITS standard (version 4.0): 2880-byte
records, 80-character cards, big-endian data. Tile compression needs astropy.
"""

from __future__ import annotations

import math
import os

import numpy as np

_RECORD = 2880

# numpy kind/size -> (TFORM letter, big-endian dtype, TZERO for unsigned storage)
_TFORM = {
    ("f", 8): ("D", ">f8", None), ("f", 4): ("E", ">f4", None),
    ("i", 8): ("K", ">i8", None), ("i", 4): ("J", ">i4", None), ("i", 2): ("I", ">i2", None),
    ("i", 1): ("I", ">i2", None), ("u", 1): ("B", "u1", None), ("u", 2): ("I", ">i2", 32768),
    ("u", 4): ("J", ">i4", 2147483648), ("b", 1): ("L", "S1", None),
}


def _value(v) -> str:
    if isinstance(v, (bool, np.bool_)):
        return f"{'T' if v else 'F':>20}"
    if isinstance(v, (int, np.integer)):
        return f"{int(v):>20}"
    if isinstance(v, (float, np.floating)):
        x = float(v)
        if not math.isfinite(x):
            raise ValueError("non-finite values are not allowed in FITS headers")
        text = repr(x).upper()
        if "." not in text and "E" not in text:
            text += ".0"
        return f"{text:>20}"
    s = str(v).replace("'", "''")
    if len(s) > 68:
        raise ValueError("string header values longer than 68 characters need the CONTINUE convention")
    return f"{chr(39) + s.ljust(8) + chr(39):<20}"


def card(key: str, value=None, comment: str = "") -> str:
    key = key.upper()
    if len(key) > 8:
        raise ValueError(f"header keyword {key!r} is longer than 8 characters")
    if value is None:
        return f"{key:<80}"[:80]
    text = f"{key:<8}= {_value(value)}"
    if comment:
        text += f" / {comment}"
    if len(text) > 80:
        text = text[:80]
    return text.ljust(80)


def _header(cards) -> bytes:
    text = "".join(cards) + card("END")
    text += " " * (-len(text) % _RECORD)
    return text.encode("ascii")


def _pad(data: bytes) -> bytes:
    return data + b"\0" * (-len(data) % _RECORD)


def _image(arr, *, primary: bool, extra=()) -> bytes:
    a = np.ascontiguousarray(arr)
    if a.dtype == np.uint8:
        bitpix, raw = 8, a.tobytes()
    elif a.dtype.kind == "f" and a.dtype.itemsize == 4:
        bitpix, raw = -32, a.astype(">f4").tobytes()
    elif a.dtype.kind == "f":
        bitpix, raw = -64, a.astype(">f8").tobytes()
    else:
        bitpix, raw = 32, a.astype(">i4").tobytes()
    h, w = a.shape
    cards = [card("SIMPLE", True, "conforms to the FITS standard")] if primary else [card("XTENSION", "IMAGE")]
    cards += [card("BITPIX", bitpix), card("NAXIS", 2), card("NAXIS1", w), card("NAXIS2", h)]
    cards += [card("EXTEND", True)] if primary else [card("PCOUNT", 0), card("GCOUNT", 1)]
    cards += list(extra)
    return _header(cards) + _pad(raw)


def _table(rec, name: str) -> bytes:
    fields = rec.dtype.names
    cols, forms, tzero = [], [], {}
    for i, f in enumerate(fields, start=1):
        dt = rec.dtype[f]
        key = (dt.kind, dt.itemsize)
        if key not in _TFORM:
            raise ValueError(f"column {f!r}: unsupported dtype {dt}")
        letter, be, zero = _TFORM[key]
        col = np.asarray(rec[f])
        if dt.kind == "b":
            col = np.where(col, b"T", b"F").astype("S1")
        elif zero is not None:
            col = (col.astype(np.int64) - zero).astype(be)
            tzero[i] = zero
        else:
            col = col.astype(be)
        cols.append(col)
        forms.append(letter)
    out = np.empty(len(rec), dtype=[(f, c.dtype) for f, c in zip(fields, cols, strict=True)])
    for f, c in zip(fields, cols, strict=True):
        out[f] = c
    raw = out.tobytes()
    cards = [card("XTENSION", "BINTABLE", "binary table extension"), card("BITPIX", 8), card("NAXIS", 2),
             card("NAXIS1", out.dtype.itemsize), card("NAXIS2", len(rec)), card("PCOUNT", 0), card("GCOUNT", 1),
             card("TFIELDS", len(fields))]
    for i, (f, letter) in enumerate(zip(fields, forms, strict=True), start=1):
        cards.append(card(f"TTYPE{i}", f))
        cards.append(card(f"TFORM{i}", letter))
        if i in tzero:
            cards.append(card(f"TZERO{i}", tzero[i]))
    cards.append(card("EXTNAME", name))
    return _header(cards) + _pad(raw)


def write_products(path: str, difference, layers, catalog, cards: dict, overwrite: bool = False) -> None:
    """The uncompressed product: difference + provenance cards in the primary,
    the given (name, array) image layers, then the CATALOG table when given."""
    if os.path.exists(path) and not overwrite:
        raise OSError(f"File {path!r} already exists.")
    parts = [_image(difference, primary=True, extra=[card(k, v) for k, v in cards.items()])]
    for name, arr in layers:
        if arr is not None:
            parts.append(_image(arr, primary=False, extra=[card("EXTNAME", name)]))
    if catalog is not None:
        parts.append(_table(np.asarray(catalog), "CATALOG"))
    with open(path, "wb") as f:
        for p in parts:
            f.write(p)
