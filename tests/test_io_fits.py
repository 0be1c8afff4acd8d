"""FITS I/O (hellblast_b200.io_fits; the reference's io_fits.py / io_fits_multi.py, which need
astropy): round trips, and the bytes on disk checked against the FITS standard (2880-byte
blocks, 80-character cards, mandatory keyword order, big-endian data)."""
import numpy as np
import pytest

from hellblast_b200 import io_fits as F


def cards(raw, start=0):
    out = []
    for i in range(start, len(raw), 80):
        c = raw[i:i + 80].decode("ascii")
        out.append(c)
        if c.startswith("END     ") or c.rstrip() == "END":
            break
    return out


def test_map_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(0)
    m = rng.standard_normal(12 * 16 * 16)
    p = str(tmp_path / "m.fits")
    F.write_map_fits(p, m, header={"NSIDE": 16, "ORDERING": "RING"})
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0
    c = cards(raw)
    assert c[0] == "SIMPLE  =                    T".ljust(80)
    assert c[1] == "BITPIX  =                  -64".ljust(80)
    assert c[2] == "NAXIS   =                    1".ljust(80)
    assert c[3] == f"NAXIS1  = {m.size:>20}".ljust(80)
    assert "NSIDE   =                   16".ljust(80) in c and "ORDERING= 'RING    '".ljust(80) in c
    data_at = 2880 * ((len(c) * 80 + 2879) // 2880)
    assert np.array_equal(np.frombuffer(raw[data_at:data_at + 8 * m.size], dtype=">f8"), m)
    back = F.read_map_fits(p, hdu=0, to_gpu=False)
    assert np.array_equal(back, m)
    with pytest.raises(IndexError):  # the reference's default hdu=1 does not exist in its own output
        F.read_map_fits(p, to_gpu=False)
    m32 = m.astype(np.float32).reshape(3, -1)
    F.write_map_fits(p, m32)
    assert np.array_equal(F.read_map_fits(p, hdu=0, to_gpu=False, dtype=np.float32), m32)


def test_alm_round_trip_and_bintable_layout(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    p = str(tmp_path / "a.fits")
    F.write_alm_fits(p, a)
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0
    ext = cards(raw, 2880)
    assert ext[0] == "XTENSION= 'BINTABLE'".ljust(80)
    want = ["BITPIX  =                    8", "NAXIS   =                    2", "NAXIS1  =                   16",
            "NAXIS2  =                   50", "PCOUNT  =                    0", "GCOUNT  =                    1",
            "TFIELDS =                    2", "TTYPE1  = 'REAL    '", "TFORM1  = 'D       '", "TTYPE2  = 'IMAG    '",
            "TFORM2  = 'D       '"]
    assert ext[1:12] == [w.ljust(80) for w in want]
    rows = np.frombuffer(raw[5760:5760 + 800], dtype=">f8").reshape(50, 2)
    assert np.array_equal(rows[:, 0], a.real) and np.array_equal(rows[:, 1], a.imag)
    assert np.array_equal(F.read_alm_fits(p, to_gpu=False), a)


def test_alm_with_healpy_index_column(tmp_path):
    lmax, mmax = 6, 4
    n = mmax * (2 * lmax + 1 - mmax) // 2 + lmax + 1
    a = np.arange(n) * (1 + 0.5j)
    p = str(tmp_path / "ai.fits")
    F.write_alm_fits(p, a, index=True, lmax=lmax, mmax=mmax)
    assert np.array_equal(F.read_alm_fits(p, to_gpu=False), a)
    raw = open(p, "rb").read()
    rec = np.frombuffer(raw[5760:5760 + 20 * n], dtype=np.uint8).reshape(n, 20)
    idx = rec[:, :4].copy().view(">i4").reshape(-1)
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(mmax + 1)])
    ms = np.concatenate([np.full(lmax + 1 - m, m) for m in range(mmax + 1)])
    assert np.array_equal(idx, ls * ls + ls + ms + 1)


def test_tqu_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    T, Q, U = (rng.standard_normal(48).astype(np.float32) for _ in range(3))
    p = str(tmp_path / "tqu.fits")
    F.write_tqu_fits(p, T, Q, U, nside=2, ordering="ring", coordsys="G", extra_header={"OBJECT": "sim"})
    (t, q, u), meta = F.read_tqu_fits(p, to_gpu=False)
    assert np.array_equal(t, T) and np.array_equal(q, Q) and np.array_equal(u, U)
    assert meta == {"NSIDE": 2, "ORDERING": "RING", "COORDSYS": "G"}
    (t, q, u), _ = F.read_tqu_fits(F.write_tqu_fits(p, T=T), to_gpu=False)
    assert q is None and u is None and np.array_equal(t, T)


def test_reads_scaled_integer_image(tmp_path):
    """A hand-built primary image of BITPIX 16 with BSCALE/BZERO (standard FITS, not written by
    this module) reads back as the scaled physical values."""
    vals = np.array([-3, 0, 7, 32767, -32768], dtype=">i2")
    hdr = b"".join(F._card(k, v) for k, v in [("SIMPLE", True), ("BITPIX", 16), ("NAXIS", 1), ("NAXIS1", 5),
                                              ("BSCALE", 0.5), ("BZERO", 10.0)])
    p = str(tmp_path / "i16.fits")
    open(p, "wb").write(F._header([hdr]) + F._pad(vals.tobytes()))
    assert np.array_equal(F.read_map_fits(p, hdu=0, to_gpu=False), vals.astype(np.float64) * 0.5 + 10.0)


@pytest.mark.gpu
def test_gpu_tensors_in_and_out(tmp_path):
    import torch
    m = torch.randn(192, dtype=torch.float64, device="cuda")
    p = str(tmp_path / "g.fits")
    F.write_map_fits(p, m)
    back = F.read_map_fits(p, hdu=0)
    assert back.is_cuda and torch.equal(back, m)
    a = torch.randn(21, dtype=torch.complex128, device="cuda")
    F.write_alm_fits(p, a)
    assert torch.equal(F.read_alm_fits(p), a)
