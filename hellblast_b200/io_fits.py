"""FITS I/O of maps and alm with the names and layouts of hellblast's io_fits.py and
io_fits_multi.py (read_map_fits, write_map_fits, read_alm_fits, write_alm_fits, write_tqu_fits,
read_tqu_fits), written against the FITS standard (version 4.0) itself: the reference goes
through astropy (io_fits.py:4-9), which is not a dependency of this library.

What is written (all data big-endian, every header and data unit padded to 2880-byte blocks,
headers of 80-character cards ending with END):
  * maps: the primary HDU holds the map as a 1-D (or [nmaps, npix]) image, BITPIX -64 or -32
    (io_fits.py:20-31);
  * alm: an empty primary HDU, then a BINTABLE with float64 columns REAL and IMAG, one row per
    entry of the alm array as given (io_fits.py:46-63); ``index=True`` adds healpy's INDEX column
    (l^2 + l + m + 1, int32) before them, for healpy-layout input;
  * T, Q, U: an empty primary HDU, then one IMAGE extension per map named T, Q, U with NSIDE,
    ORDERING and COORDSYS cards (io_fits_multi.py:24-41).
Readers accept what the writers produce, images of BITPIX 8/16/32/64/-32/-64 (with BSCALE/BZERO),
and BINTABLEs whose REAL/IMAG (and INDEX) columns are of types D, E, J or K.  Arrays come back as
CUDA tensors (``to_gpu=True``, the reference's default) or numpy arrays.
"""
from __future__ import annotations

import numpy as np
import torch

BLOCK = 2880
_BITPIX = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
_TFORM = {"D": (">f8", 8), "E": (">f4", 4), "J": (">i4", 4), "K": (">i8", 8), "I": (">i2", 2), "B": (">u1", 1)}


# ----------------------------------------------------------------------------- header cards
def _card(key: str, value=None, comment: str = "") -> bytes:
    key = key.upper()
    if value is None:
        s = key.ljust(80)
    else:
        if isinstance(value, bool):
            v = ("T" if value else "F").rjust(20)
        elif isinstance(value, (int, np.integer)):
            v = str(int(value)).rjust(20)
        elif isinstance(value, (float, np.floating)):
            v = repr(float(value)).upper().rjust(20)
        else:
            v = "'" + str(value).replace("'", "''").ljust(8) + "'"
        s = f"{key:<8}= {v}"
        if comment:
            s += " / " + comment
    if len(s) > 80:
        raise ValueError(f"FITS card too long: {s!r}")
    return s.ljust(80).encode("ascii")


def _header(cards) -> bytes:
    h = b"".join(cards) + b"END".ljust(80)
    return h + b" " * ((-len(h)) % BLOCK)


def _pad(data: bytes) -> bytes:
    return data + b"\0" * ((-len(data)) % BLOCK)


def _parse_value(v: str):
    v = v.strip()
    if v.startswith("'"):
        end = v.find("'", 1)
        while end != -1 and end + 1 < len(v) and v[end + 1] == "'":
            end = v.find("'", end + 2)
        return v[1:end].replace("''", "'").rstrip()
    if "/" in v:
        v = v.split("/", 1)[0].strip()
    if v in ("T", "F"):
        return v == "T"
    try:
        return int(v)
    except ValueError:
        try:
            return float(v.replace("D", "E"))
        except ValueError:
            return v


def _read_hdus(path: str):
    """[(header dict, data bytes)] of every HDU in the file."""
    raw = open(path, "rb").read()
    out, pos = [], 0
    while pos + BLOCK <= len(raw):
        hdr, done = {}, False
        while not done:
            if pos + BLOCK > len(raw):
                raise ValueError(f"{path}: truncated FITS header")
            blk = raw[pos:pos + BLOCK]
            pos += BLOCK
            for i in range(0, BLOCK, 80):
                card = blk[i:i + 80].decode("ascii", "replace")
                key = card[:8].strip()
                if key == "END":
                    done = True
                    break
                if card[8:10] == "= " and key:
                    hdr[key] = _parse_value(card[10:])
        naxis = int(hdr.get("NAXIS", 0))
        n = 1 if naxis else 0
        for k in range(1, naxis + 1):
            n *= int(hdr[f"NAXIS{k}"])
        nbytes = abs(int(hdr.get("BITPIX", 8))) // 8 * int(hdr.get("GCOUNT", 1)) * (int(hdr.get("PCOUNT", 0)) + n)
        out.append((hdr, raw[pos:pos + nbytes]))
        pos += nbytes + ((-nbytes) % BLOCK)
    if not out:
        raise ValueError(f"{path}: not a FITS file")
    return out


def _image(hdr, data) -> np.ndarray:
    naxis = int(hdr.get("NAXIS", 0))
    if naxis == 0:
        return np.zeros(0)
    shape = tuple(int(hdr[f"NAXIS{k}"]) for k in range(naxis, 0, -1))
    a = np.frombuffer(data, dtype=_BITPIX[int(hdr["BITPIX"])], count=int(np.prod(shape))).reshape(shape)
    bscale, bzero = float(hdr.get("BSCALE", 1.0)), float(hdr.get("BZERO", 0.0))
    a = a.astype(a.dtype.newbyteorder("="))
    return a * bscale + bzero if (bscale != 1.0 or bzero != 0.0) else a


def _table(hdr, data) -> dict:
    if hdr.get("XTENSION", "").strip() != "BINTABLE":
        raise ValueError("expected a BINTABLE extension")
    nrow, rowb, nf = int(hdr["NAXIS2"]), int(hdr["NAXIS1"]), int(hdr["TFIELDS"])
    fields, off = [], 0
    for k in range(1, nf + 1):
        form = str(hdr[f"TFORM{k}"]).strip()
        rep = int(form[:-1]) if len(form) > 1 and form[:-1].isdigit() else 1
        code = form[-1]
        if code not in _TFORM:
            raise ValueError(f"unsupported BINTABLE column type {form}")
        dt, size = _TFORM[code]
        fields.append((str(hdr.get(f"TTYPE{k}", f"COL{k}")).strip().upper(), off, np.dtype(dt), rep))
        off += size * rep
    if off != rowb:
        raise ValueError("BINTABLE row size does not match its columns")
    rec = np.frombuffer(data, dtype=np.uint8, count=nrow * rowb).reshape(nrow, rowb)
    cols = {}
    for name, o, dt, rep in fields:
        b = np.ascontiguousarray(rec[:, o:o + dt.itemsize * rep])
        cols[name] = b.view(dt).reshape(nrow * rep).astype(dt.newbyteorder("="))
    return cols


def _host(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    try:
        import cupy  # noqa: F401
        if hasattr(x, "__cuda_array_interface__"):
            return cupy.asnumpy(x)
    except ImportError:
        pass
    return np.asarray(x)


def _out(a: np.ndarray, to_gpu: bool, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return torch.from_numpy(a).cuda() if to_gpu else a


def _write(path: str, blobs, overwrite: bool):
    import os
    if os.path.exists(path) and not overwrite:
        raise FileExistsError(path)
    with open(path, "wb") as f:
        for b in blobs:
            f.write(b)
    return path


def _extra(header):
    return [_card(k, v) for k, v in (header or {}).items()]


# ----------------------------------------------------------------------------- maps
def write_map_fits(path, m, header=None, overwrite=True):
    """Map(s) as the primary image (io_fits.py:20-31); float32 input stays float32."""
    a = _host(m)
    a = a.astype(">f4" if a.dtype == np.float32 else ">f8")
    bitpix = -32 if a.dtype.itemsize == 4 else -64
    cards = [_card("SIMPLE", True), _card("BITPIX", bitpix), _card("NAXIS", a.ndim)]
    cards += [_card(f"NAXIS{k + 1}", n) for k, n in enumerate(reversed(a.shape))]
    cards += [_card("EXTEND", True)] + _extra(header)
    return _write(path, [_header(cards), _pad(a.tobytes())], overwrite)


def read_map_fits(path, hdu=1, to_gpu=True, dtype=np.float64):
    """The image of HDU ``hdu`` (io_fits.py:11-18; an index past the last HDU is an IndexError,
    as in the reference, whose writer puts the map in HDU 0)."""
    hdr, data = _read_hdus(path)[hdu]
    return _out(_image(hdr, data), to_gpu, dtype)


# ----------------------------------------------------------------------------- alm
def write_alm_fits(path, alm, header=None, overwrite=True, index=False, lmax=None, mmax=None):
    """REAL, IMAG float64 columns (io_fits.py:46-63), one row per alm entry as given; with
    ``index`` the input is healpy-layout alm and an INDEX column l^2 + l + m + 1 precedes them."""
    a = _host(alm).astype(np.complex128).reshape(-1)
    cols = []
    if index:
        from .alm_ops import getlmax
        L = getlmax(a.size, mmax) if lmax is None else int(lmax)
        M = L if mmax is None else int(mmax)
        ls = np.concatenate([np.arange(m, L + 1) for m in range(M + 1)])
        ms = np.concatenate([np.full(L + 1 - m, m) for m in range(M + 1)])
        cols.append(("INDEX", "J", (ls * ls + ls + ms + 1).astype(">i4")))
    cols += [("REAL", "D", a.real.astype(">f8")), ("IMAG", "D", a.imag.astype(">f8"))]
    rowb = sum(c[2].dtype.itemsize for c in cols)
    rec = np.empty((a.size, rowb), dtype=np.uint8)
    off = 0
    for _, _, v in cols:
        w = v.dtype.itemsize
        rec[:, off:off + w] = v.reshape(-1, 1).view(np.uint8).reshape(a.size, w)
        off += w
    prim = _header([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)])
    cards = [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2), _card("NAXIS1", rowb),
             _card("NAXIS2", a.size), _card("PCOUNT", 0), _card("GCOUNT", 1), _card("TFIELDS", len(cols))]
    for k, (name, form, _) in enumerate(cols, 1):
        cards += [_card(f"TTYPE{k}", name), _card(f"TFORM{k}", form)]
    cards += _extra(header)
    return _write(path, [prim, _header(cards), _pad(rec.tobytes())], overwrite)


def read_alm_fits(path, hdu=1, to_gpu=True, dtype=np.complex128, lmax=None, mmax=None):
    """REAL + i IMAG of HDU ``hdu`` (io_fits.py:33-44).  When the table has an INDEX column the
    entries are placed in healpy layout (lmax, mmax from the largest index unless given)."""
    hdr, data = _read_hdus(path)[hdu]
    cols = _table(hdr, data)
    if "REAL" not in cols or "IMAG" not in cols:
        raise ValueError(f"{path}: HDU {hdu} has no REAL/IMAG columns")
    a = cols["REAL"].astype(np.float64) + 1j * cols["IMAG"].astype(np.float64)
    if "INDEX" in cols:
        idx = cols["INDEX"].astype(np.int64) - 1
        l = np.floor(np.sqrt(idx)).astype(np.int64)
        m = idx - l * l - l
        L = int(l.max()) if lmax is None else int(lmax)
        M = int(m.max()) if mmax is None else int(mmax)
        out = np.zeros(M * (2 * L + 1 - M) // 2 + L + 1, dtype=np.complex128)
        keep = (l <= L) & (m <= M) & (m >= 0)
        out[m[keep] * (2 * L + 1 - m[keep]) // 2 + l[keep]] = a[keep]
        a = out
    return _out(a, to_gpu, dtype)


# ----------------------------------------------------------------------------- T, Q, U
def write_tqu_fits(path, T=None, Q=None, U=None, nside=None, ordering="RING", coordsys="G", overwrite=True,
                   extra_header=None):
    """Empty primary HDU, then IMAGE extensions T, Q, U (io_fits_multi.py:24-41)."""
    blobs = [_header([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)])]
    for arr, name in ((T, "T"), (Q, "Q"), (U, "U")):
        if arr is None:
            continue
        a = _host(arr)
        a = a.astype(">f4" if a.dtype == np.float32 else ">f8")
        cards = [_card("XTENSION", "IMAGE"), _card("BITPIX", -32 if a.dtype.itemsize == 4 else -64),
                 _card("NAXIS", a.ndim)]
        cards += [_card(f"NAXIS{k + 1}", n) for k, n in enumerate(reversed(a.shape))]
        cards += [_card("PCOUNT", 0), _card("GCOUNT", 1), _card("EXTNAME", name)]
        if nside is not None:
            cards.append(_card("NSIDE", int(nside)))
        cards += [_card("ORDERING", str(ordering).upper()), _card("COORDSYS", coordsys)] + _extra(extra_header)
        blobs += [_header(cards), _pad(a.tobytes())]
    return _write(path, blobs, overwrite)


def read_tqu_fits(path, to_gpu=True):
    """((T, Q, U), meta) from the extensions named T, Q, U (io_fits_multi.py:43-63)."""
    maps = {"T": None, "Q": None, "U": None}
    meta = {}
    for hdr, data in _read_hdus(path)[1:]:
        name = str(hdr.get("EXTNAME", "")).strip().upper()
        if name in maps:
            a = _image(hdr, data)
            maps[name] = torch.from_numpy(np.ascontiguousarray(a)).cuda() if to_gpu else a
        for k in ("NSIDE", "ORDERING", "COORDSYS"):
            if k in hdr:
                meta[k] = hdr[k]
    return (maps["T"], maps["Q"], maps["U"]), meta
