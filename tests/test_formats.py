"""DRFT / KRNL file formats, the GRF table generator and set-up error paths
of the host library (no GPU needed: these run before any device call)."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

from conftest import dup
from libirl_b200 import api, workloads as W


def _swap_file(src, dst, float_fields_from=None):
    """Byte-swap every 4-byte word after the signature/title/name header."""
    b = bytearray(open(src, "rb").read())
    hdr_words = [(4, 8)]  # version
    out = bytearray(b)

    def swap(off):
        out[off:off + 4] = b[off:off + 4][::-1]

    swap(4)
    start = 8 + 80 + 20
    for off in range(start, len(b), 4):
        swap(off)
    open(dst, "wb").write(bytes(out))


def test_drft_roundtrip_native_and_swapped(product, tmp_path):
    psfs = W.gaussian_drf_table(0.4, 5.0, 0.4, 7)
    f = str(tmp_path / "t.drft")
    W.write_drft(f, psfs, 0.4, 0.4, 5.0, title="table", colname="LEHR")
    title, col = C.c_char_p(), C.c_char_p()
    t = product.sReadDrfTab(f.encode(), C.byref(title), C.byref(col))
    assert t.iNumDistances == 7 and abs(t.fPixSize - 0.4) < 1e-7 and abs(t.fStartDistance - 5.0) < 1e-7
    assert title.value == b"table" and col.value == b"LEHR"
    # fields libirl's reader leaves unset (drftabio.c:168-174) come back zeroed
    assert t.bFFTconvolve == 0 and not t.psBckDrfTab
    for i, p in enumerate(psfs):
        d = t.psDrfs[i]
        assert (2 * d.MaxOffsY - 1, 2 * d.MaxOffsX - 1) == p.shape
        got = np.ctypeslib.as_array(d.Psf, shape=(p.size,)).reshape(p.shape)
        assert np.array_equal(got, p)
    g = str(tmp_path / "s.drft")
    _swap_file(f, g)
    t2 = product.sReadDrfTab(g.encode(), C.byref(title), C.byref(col))
    assert t2.iNumDistances == 7 and abs(t2.fStartDistance - 5.0) < 1e-7
    d = t2.psDrfs[3]
    got = np.ctypeslib.as_array(d.Psf, shape=(psfs[3].size,)).reshape(psfs[3].shape)
    assert np.array_equal(got, psfs[3])


def test_write_drft_byte_identical_to_reference_layout(product, orc, tmp_path):
    psfs = W.gaussian_drf_table(0.3, 2.0, 0.3, 4)
    a = str(tmp_path / "py.drft")
    W.write_drft(a, psfs, 0.3, 0.3, 2.0, title="x", colname="y")
    title, col = C.c_char_p(), C.c_char_p()
    t = product.sReadDrfTab(a.encode(), C.byref(title), C.byref(col))
    b = str(tmp_path / "c.drft")
    product.vWriteDrfTab(C.byref(t), b.encode(), b"x", b"y")
    assert open(a, "rb").read() == open(b, "rb").read()
    if os.path.exists(orc.REF_SO):
        # the reference reads what the product wrote
        ref = orc.ref()
        t3 = ref.sReadDrfTab(b.encode(), C.byref(title), C.byref(col))
        assert t3.iNumDistances == 4


def test_krnl_swapped_reads_numxyoffs(product, tmp_path):
    k, kmu = W.esse_kernel(6, 12, 0.8)
    f = str(tmp_path / "k.krnl")
    W.write_krnl(f, k, kmu, 0.15, 0.8)
    product.psReadKrnlFile.restype = C.c_void_p
    product.psReadKrnlFile.argtypes = [C.c_char_p, C.c_int]

    class Krnl(C.Structure):
        _fields_ = [("title", C.c_char_p), ("iso", C.c_char_p), ("nxy", C.c_int), ("nd", C.c_int),
                    ("mu0", C.c_float), ("pix", C.c_float), ("hi", C.c_float), ("lo", C.c_float),
                    ("pri", C.c_float), ("scat", C.c_float), ("cntr", C.c_float),
                    ("k", api.FLOAT_P), ("kmu", api.FLOAT_P)]

    for path in (f, str(tmp_path / "ks.krnl")):
        if path != f:
            _swap_file(f, path)
        p = C.cast(product.psReadKrnlFile(path.encode(), 1), C.POINTER(Krnl)).contents
        assert (p.nxy, p.nd) == (6, 12)
        assert abs(p.mu0 - 0.15) < 1e-7 and abs(p.pix - 0.8) < 1e-7
        got = np.ctypeslib.as_array(p.k, shape=(k.size,)).reshape(k.shape)
        assert np.array_equal(got, k)


# (col thick, hole diam, gap, intrinsic FWHM, max error, bin, spacing, first distance), distances, NOffs
GENDRF_CASES = [
    ((2.405, 0.111, 0.64, 0.38, 0.05, 0.4, 0.4, 3.0), 6, 16),
    ((2.405, 0.111, 0.64, 0.38, 0.0, 0.3125, 0.3125, -1.0), 10, 64),   # no truncation; distances <= 0
    ((3.5, 0.15, 1.0, 0.3, 0.01, 0.1, 0.2, 0.5), 8, 32),
    ((2.0, 0.2, 0.5, 0.5, 0.002, 0.05, 0.6, 10.0), 5, 40),             # oversampled (ratio > 1), wide
    ((2.405, 0.111, 0.64, 0.38, 0.02, 0.2, 1.0, 1.0), 40, 128),
]


@pytest.mark.parametrize("args,nd,noffs", GENDRF_CASES)
def test_gendrf_matches_reference_and_is_normalised(product, orc, args, nd, noffs):
    tab = (api.Drf * nd)()
    product.irl_gendrf(*args, nd, noffs, tab)
    for i in range(nd):
        d = tab[i]
        p = np.ctypeslib.as_array(d.Psf, shape=((2 * d.MaxOffsY - 1) * (2 * d.MaxOffsX - 1),))
        assert abs(float(p.astype(np.float64).sum()) - 1.0) < 1e-5  # gendrf.c:339-375
    if os.path.exists(orc.REF_SO):
        ref = orc.ref()
        ref.gendrf.argtypes = [C.c_int, C.c_float] + [C.c_float] * 8 + [C.c_int, C.c_int, C.POINTER(api.Drf)]
        ref.gendrf.restype = None
        rt = (api.Drf * nd)()
        ref.gendrf(0, 0.0, *args, nd, noffs, rt)
        for i in range(nd):
            assert (tab[i].MaxOffsX, tab[i].MaxOffsY) == (rt[i].MaxOffsX, rt[i].MaxOffsY)
            cnt = (2 * rt[i].MaxOffsY - 1) * (2 * rt[i].MaxOffsX - 1)
            a = np.ctypeslib.as_array(tab[i].Psf, shape=(cnt,))
            b = np.ctypeslib.as_array(rt[i].Psf, shape=(cnt,))
            assert np.allclose(a, b, rtol=1e-6, atol=1e-9)


def _genprj(lib, case, drf_name, krnl_name=None):
    p, o, v = case.parms(), case.options(), case.views()
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    rc = lib.IrlGenprj(C.byref(p), C.byref(o), v, dup(drf_name), dup(krnl_name), None, None, api.fptr(act),
                       api.fptr(atn), api.fptr(prj), 1.0, None, None)
    return rc, lib.pchIrlErrorString()


@pytest.mark.parametrize("kind", ["truncated", "signature", "version"])
def test_bad_drf_table_is_a_clean_error(product, tmp_path, kind):
    case = W.plain64(n=16, nviews=4)
    files = case.write_tables(str(tmp_path))
    b = bytearray(open(files["drf"], "rb").read())
    if kind == "truncated":
        b = b[: len(b) // 2]
    elif kind == "signature":
        b[0:4] = b"XXXX"
    else:
        b[4:8] = struct.pack("=i", 7)
    bad = str(tmp_path / "bad.drft")
    open(bad, "wb").write(bytes(b))
    rc, msg = _genprj(product, case, bad)
    assert rc != 0
    assert {"truncated": b"truncated", "signature": b"signature", "version": b"version"}[kind] in msg


def test_pixel_size_mismatch_is_fatal(product, tmp_path):
    case = W.plain64(n=16, nviews=4)
    f = str(tmp_path / "p.drft")
    W.write_drft(f, case.drf_psfs, case.pix * 1.5, case.drf_spacing, case.drf_start)
    rc, msg = _genprj(product, case, f)
    assert rc != 0 and b"pixel size" in msg
