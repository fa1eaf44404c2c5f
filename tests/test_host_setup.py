"""IrlOsemBegin's host set-up against the oracle, bit for bit.

Before its first device call IrlOsemBegin:
* puts the caller's attenuation map in libirl's internal layout, scales and
  clamps it, all in place;
* computes the initial estimate from the unclamped projections, then
  clamps the projections in place;
* hands the initial estimate to the iteration callback as iteration 0.

The element-wise passes run on several host threads (irl_par.c), and the
results must not depend on that. Without a device, IrlOsemBegin stops at its
first device call, after all of this. With one it completes, and the session
is ended.
"""
import ctypes as C

import numpy as np

from conftest import dup
from libirl_b200 import api, workloads as W


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_host_setup_matches_oracle_bit_for_bit(product, orc, tmp_path):
    cases = [W.full128(seed=2000),
             W.full128(seed=7, n=33, nviews=8, subsets=2, iterations=1, collapse=1, drf_max_offs=6),
             W.plain64(seed=5, n=48, nviews=12, subsets=4, iterations=1)]
    rng = np.random.default_rng(3)
    for i, case in enumerate(cases):
        files = case.write_tables(str(tmp_path / f"c{i}"))
        p, o, v = case.parms(), case.options(), case.views()
        atn, rec = case.atn.copy(), np.zeros_like(case.act)
        meas = (rng.random((case.nviews, case.nz, case.n)) - 0.1).astype(np.float32)  # some negative bins
        m = meas.copy()
        got = []
        cb = api.ITER_CB(lambda it, q: got.append(np.ctypeslib.as_array(q, shape=(case.act.size,)).copy()))
        rc = product.IrlOsemBegin(C.byref(p), C.byref(o), v, dup(files["drf"]), dup(files.get("krnl")), cb,
                                  None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        if rc == 0:
            product.IrlOsemEnd(None)
        # attenuation: internal layout, scaled (C float products), clamped at 0
        want = orc.to_internal(case.atn)
        if p.fAtnScaleFac > 0 and p.fAtnScaleFac != 1.0:
            want = want * np.float32(p.fAtnScaleFac)
        want = np.where(want < 0, np.float32(0), want)
        assert np.array_equal(_bits(atn), _bits(want)), i
        # projections clamped at 0 in place
        assert np.array_equal(_bits(m), _bits(np.where(meas < 0, np.float32(0), meas))), i
        # the initial estimate (from the unclamped projections), clamped, in
        # the external layout
        est = np.zeros((case.n, case.nz, case.n), np.float32)
        orc.orc().or_initial_estimate(case.n, case.nz, case.nviews, api.fptr(meas), api.fptr(est))
        est = np.where(est < 0, np.float32(0), est)
        assert got, "no iteration-0 callback"
        assert np.array_equal(_bits(got[0]), _bits(orc.to_external(est)).ravel()), i


class EsseHost(C.Structure):
    """irl_esse_host (libirl_b200/csrc/host/irl_host.h)."""

    _fields_ = [("on", C.c_int), ("kx", C.c_int), ("ky", C.c_int), ("kz", C.c_int), ("collapse", C.c_int),
                ("nterms", C.c_int), ("mu0", C.c_float), ("mu_avg", C.c_float), ("pix", C.c_float),
                ("cntr_pix_fac", C.c_float), ("krnl", C.POINTER(C.c_float)), ("kmu", C.POINTER(C.c_float)),
                ("kmu2", C.POINTER(C.c_float))]


class HostParms(C.Structure):
    """irl_parms (libirl_b200/csrc/host/irl_host.h)."""

    _fields_ = [("n", C.c_int), ("nz", C.c_int), ("nviews", C.c_int), ("nbins", C.c_int), ("pix", C.c_float),
                ("atn_scale", C.c_float), ("scatest_fac", C.c_float), ("srf_iters", C.c_int),
                ("prj_model", C.c_int), ("bck_model", C.c_int), ("model", C.c_int), ("norm_base", C.c_char_p),
                ("ang_per_subset", C.c_int), ("iterations", C.c_int), ("start_iteration", C.c_int),
                ("pad_len", C.c_int), ("avg_len", C.c_int), ("hole_diam", C.c_float), ("hole_len", C.c_float),
                ("back_to_det", C.c_float), ("intrinsic_fwhm", C.c_float), ("max_frac_err", C.c_float)]


def test_esse_kernel_grids_match_oracle_bit_for_bit(product, orc, tmp_path):
    """The ESSE kernel grids and their weighted mean mu (krnlprj3d.c:403-547):
    the library sums only the kernel's support, the oracle the whole grid in
    index order; the grids, K (mu - mu_avg) and mu_avg must be identical."""
    for case in (W.full128(seed=2000), W.full128(seed=8, n=48, nviews=8, subsets=2, iterations=1, collapse=3),
                 W.full128(seed=9, n=32, nviews=8, subsets=2, iterations=1, collapse=1)):
        files = case.write_tables(str(tmp_path / case.name / str(case.n)))
        hp = HostParms()
        hp.n, hp.nz, hp.nviews, hp.pix = case.n, case.nz, case.nviews, case.pix
        e = EsseHost()
        product.irl_esse_prepare(files["krnl"].encode(), C.byref(hp), case.collapse, C.byref(e))
        pr = orc.Problem(case)
        cnt = e.kx * e.ky * e.kz
        assert (e.kx, e.ky, e.kz) == (pr.P.kx, pr.P.ky, pr.P.kz)
        got_k = np.ctypeslib.as_array(e.krnl, shape=(cnt,)).copy()
        got_km = np.ctypeslib.as_array(e.kmu, shape=(cnt,)).copy()
        want_k = np.ctypeslib.as_array(pr.P.krnl, shape=(cnt,))
        want_km = np.ctypeslib.as_array(pr.P.kmu, shape=(cnt,))
        assert np.float32(e.mu_avg).view(np.uint32) == np.float32(pr.P.mu_avg).view(np.uint32)
        assert np.array_equal(_bits(got_k), _bits(want_k))
        assert np.array_equal(_bits(got_km), _bits(want_km))
        product.irl_esse_free(C.byref(e))
