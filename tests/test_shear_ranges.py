"""The needed-range trimming of the column-walk shear kernel, on the CPU.

k_shear_cw computes the three-shear intermediates X (pass 1) and Y (pass 2)
only where the output reads them: per column, the rows that pass 3 reads
(RotTabs::col_rng), and per row, the columns of X that pass 2 reads
(row_rng); k_shear_ranges derives both from the shift tables.  This test
restates those range rules and the three passes in numpy, with every
skipped entry left NaN, and checks for each angle that no NaN is read and
that the result equals the oracle's vShearsRotate bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from libirl_b200 import api

F32 = np.float32


class ShearTab(C.Structure):
    """irl_shear_tab (libirl_b200/csrc/host/irl_geom.h)."""

    _fields_ = [("b90", C.c_int), ("b180", C.c_int), ("iadd", C.c_int), ("mdim", C.c_int),
                ("row_sh", C.POINTER(C.c_int)), ("row_f1", C.POINTER(C.c_float)), ("row_f2", C.POINTER(C.c_float)),
                ("col_sh", C.POINTER(C.c_int)), ("col_f1", C.POINTER(C.c_float)), ("col_f2", C.POINTER(C.c_float))]


def _lerp(f1, a, f2, b):
    return F32(F32(f1) * F32(a)) + F32(F32(f2) * F32(b))


def _tables(lib, angle, n):
    ip, fp = C.POINTER(C.c_int), C.POINTER(C.c_float)
    rsh, csh = np.zeros(n, np.int32), np.zeros(2 * n, np.int32)
    rf1, rf2 = np.zeros(n, np.float32), np.zeros(n, np.float32)
    cf1, cf2 = np.zeros(2 * n, np.float32), np.zeros(2 * n, np.float32)
    t = ShearTab(0, 0, 0, 0, rsh.ctypes.data_as(ip), rf1.ctypes.data_as(fp), rf2.ctypes.data_as(fp),
                 csh.ctypes.data_as(ip), cf1.ctypes.data_as(fp), cf2.ctypes.data_as(fp))
    lib.irl_shear_table(C.c_float(angle), n, C.byref(t))
    st, en = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib.irl_shear_support(n, st.ctypes.data_as(ip), en.ctypes.data_as(ip))
    return t, rsh, rf1, rf2, csh, cf1, cf2, st, en


def _ranges(t, n, rsh, csh, st, en):
    """k_shear_ranges: column -> rows of Y read by pass 3; row -> columns of
    X read by pass 2 (hulls; None when empty)."""
    col = [None] * t.mdim
    for j in range(n):
        xa, xb = st[j] + 1, en[j] - 1
        if xa >= xb:
            continue
        off = rsh[j] + t.iadd
        for c in range(max(0, xa + off), min(t.mdim - 1, xb + off) + 1):
            col[c] = (j, j) if col[c] is None else (col[c][0], j)
    row = [None] * n
    for c, rg in enumerate(col):
        if rg is None:
            continue
        for r in range(max(0, rg[0] + csh[c]), min(n - 1, rg[1] + csh[c] + 1) + 1):
            row[r] = (c, c) if row[r] is None else (row[r][0], c)
    return col, row


def _rotate(lib, angle, sl):
    n = sl.shape[0]
    t, rsh, rf1, rf2, csh, cf1, cf2, st, en = _tables(lib, angle, n)
    col, row = _ranges(t, n, rsh, csh, st, en)
    m, iadd = t.mdim, t.iadd

    def src(y, x):
        return sl[y, x] if 0 <= y < n and 0 <= x < n else F32(0)

    X = np.full((n, m), np.nan, np.float32)  # NaN: never computed
    for j in range(n):
        if row[j] is None:
            continue
        sh = rsh[j]
        lo, vb = st[j] - sh + iadd, min(en[j] - sh - 1 + iadd, m)
        for i in range(row[j][0], row[j][1] + 1):
            if not lo <= i < vb:
                X[j, i] = 0
                continue
            if not t.b180:
                p = i + sh - iadd
                a, b = (src(j, p), src(j, p + 1)) if not t.b90 else (src(p, n - j - 1), src(p + 1, n - j - 1))
            else:
                p = n - i - (sh - iadd + 1)
                a, b = (src(n - j - 1, p), src(n - j - 1, p - 1)) if not t.b90 else (src(p, j), src(p - 1, j))
            X[j, i] = _lerp(rf1[j], a, rf2[j], b)
    Y = X.copy()
    for c in range(m):
        if col[c] is None:
            continue
        jt = csh[c]
        vlo, vhi = max(0, -jt) - iadd, min(m, m - jt - 1) - iadd
        for j in range(col[c][0], col[c][1] + 1):
            if not vlo <= j < vhi:
                Y[j, c] = 0
                continue
            x0 = X[j + jt, c] if 0 <= j + jt < n else F32(0)
            x1 = X[j + jt + 1, c] if 0 <= j + jt + 1 < n else F32(0)
            assert not (np.isnan(x0) or np.isnan(x1)), ("pass 2 read a skipped X", c, j)
            Y[j, c] = _lerp(cf1[c], x0, cf2[c], x1)
    out = np.zeros((n, n), np.float32)
    for j in range(n):
        off = rsh[j] + iadd
        for x in range(st[j] + 1, en[j] - 1):
            y0 = Y[j, x + off] if 0 <= x + off < m else F32(0)
            y1 = Y[j, x + off + 1] if 0 <= x + off + 1 < m else F32(0)
            assert not (np.isnan(y0) or np.isnan(y1)), ("pass 3 read a skipped Y", j, x)
            out[j, x] = _lerp(rf1[j], y0, rf2[j], y1)
    return out


@pytest.mark.parametrize("n", [16, 33, 48])
def test_trimmed_shear_passes_match_oracle(orc, n):
    import libirl_b200 as L
    if not __import__("os").path.exists(L.SO):
        pytest.skip("libirl_b200.so not built")
    lib = L.load()
    rng = np.random.default_rng(40 + n)
    angles = list(rng.uniform(-7, 7, 5)) + [0.0, np.pi / 4, np.pi / 2, -np.pi / 2, np.pi, 2.5]
    for a in angles:
        a = float(np.float32(a))
        vol = rng.random((n, 1, n), dtype=np.float32)
        want = np.zeros_like(vol)
        orc.orc().or_shears_rotate(a, api.fptr(vol), api.fptr(want), n, 1)
        assert np.array_equal(_rotate(lib, a, vol[:, 0, :]), want[:, 0, :]), (n, a)
