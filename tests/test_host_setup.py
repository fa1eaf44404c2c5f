"""IrlOsemBegin's host set-up against the oracle, bit for bit.

IrlOsemBegin (irlosem.c:150-243):
* puts the caller's attenuation map in libirl's internal layout, scales and
  clamps it, all in place;
* computes the initial estimate from the unclamped projections, then
  clamps the projections in place;
* hands the initial estimate to the iteration callback as iteration 0.

These host passes run on helper threads and split over the host's cores
(irl_par.c) while the device builds its tables, and the results must not
depend on that.  The whole call needs a device; the host functions it uses
(the projection sum, the one-pass initial estimate, the reorder) are also
checked on their own without one.
"""
import ctypes as C

import numpy as np
import pytest

import libirl_b200 as L
from conftest import dup, rel_l2
from libirl_b200 import api, workloads as W


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.gpu
def test_host_setup_matches_oracle_bit_for_bit(product, orc, tmp_path):
    cases = [W.full128(seed=2000),
             W.full128(seed=7, n=40, nviews=8, subsets=2, iterations=1, collapse=1, drf_max_offs=6),
             W.plain64(seed=5, n=48, nviews=12, subsets=4, iterations=1),
             W.plain64(seed=6, n=33, nviews=8, subsets=2, iterations=1)]
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
        assert rc == 0, product.pchIrlErrorString()
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
                ("cntr_pix_fac", C.c_float), ("noffs", C.c_int), ("ndepths", C.c_int),
                ("krnl_file", C.POINTER(C.c_float)), ("mu_file", C.POINTER(C.c_float)),
                ("kmu_outside", C.c_float)]


class IrlcuEsse(C.Structure):
    """irlcu_esse (include/irlcu.h)."""

    _fields_ = [("kx", C.c_int), ("ky", C.c_int), ("kz", C.c_int), ("collapse", C.c_int), ("nterms", C.c_int),
                ("mu0", C.c_float), ("mu_avg", C.c_float), ("pix", C.c_float), ("cntr_pix_fac", C.c_float),
                ("noffs", C.c_int), ("ndepths", C.c_int), ("krnl", C.POINTER(C.c_float)),
                ("mu", C.POINTER(C.c_float)), ("kmu_outside", C.c_float)]


class HostParms(C.Structure):
    """irl_parms (libirl_b200/csrc/host/irl_host.h)."""

    _fields_ = [("n", C.c_int), ("nz", C.c_int), ("nviews", C.c_int), ("nbins", C.c_int), ("pix", C.c_float),
                ("atn_scale", C.c_float), ("scatest_fac", C.c_float), ("srf_iters", C.c_int),
                ("prj_model", C.c_int), ("bck_model", C.c_int), ("model", C.c_int), ("norm_base", C.c_char_p),
                ("ang_per_subset", C.c_int), ("iterations", C.c_int), ("start_iteration", C.c_int),
                ("pad_len", C.c_int), ("avg_len", C.c_int), ("hole_diam", C.c_float), ("hole_len", C.c_float),
                ("back_to_det", C.c_float), ("intrinsic_fwhm", C.c_float), ("max_frac_err", C.c_float)]


ESSE_GRID_CASES = [dict(seed=2000), dict(seed=8, n=48, nviews=8, subsets=2, iterations=1, collapse=3),
                   dict(seed=9, n=32, nviews=8, subsets=2, iterations=1, collapse=1)]


def _esse_host(product, case, files):
    hp = HostParms()
    hp.n, hp.nz, hp.nviews, hp.pix = case.n, case.nz, case.nviews, case.pix
    e = EsseHost()
    product.irl_esse_prepare(files["krnl"].encode(), C.byref(hp), case.collapse, C.byref(e))
    return e


def test_esse_kernel_mean_matches_oracle_bit_for_bit(product, orc, tmp_path):
    """The weighted mean mu of the ESSE kernel (krnlprj3d.c:495-510): the
    library sums the kernel's support in grid order straight from the
    file's arrays, the oracle the whole reordered grid in index order; the
    bits must agree, and so must the grid size."""
    for kw in ESSE_GRID_CASES:
        case = W.full128(**kw)
        files = case.write_tables(str(tmp_path / case.name / str(case.n)))
        e = _esse_host(product, case, files)
        pr = orc.Problem(case)
        assert (e.kx, e.ky, e.kz) == (pr.P.kx, pr.P.ky, pr.P.kz)
        assert np.float32(e.mu_avg).view(np.uint32) == np.float32(pr.P.mu_avg).view(np.uint32)
        outside = np.float32(np.float32(0.0) - np.float32(e.mu_avg)) * np.float32(0.0)
        assert np.float32(e.kmu_outside).view(np.uint32) == outside.view(np.uint32)
        product.irl_esse_free(C.byref(e))


@pytest.mark.gpu
def test_esse_kernel_grids_match_oracle_bit_for_bit(product, orc, tmp_path):
    """The ESSE grids K and K (mu - mu_avg) that the device expands from the
    file form (pfReorder3dKrnl, krnlprj3d.c:43-128, and
    krnlprj3d.c:512-547) equal the oracle's host-built grids bit for bit."""
    product.irlcu_esse_expand.restype = C.c_int
    product.irlcu_esse_expand.argtypes = [C.c_void_p, C.c_int, api.FLOAT_P]
    for kw in ESSE_GRID_CASES:
        case = W.full128(**kw)
        files = case.write_tables(str(tmp_path / case.name / str(case.n)))
        e = _esse_host(product, case, files)
        g = L.IrlcuGeom(case.n, case.nz, case.nviews, 1, 4)
        assert product.irlcu_init(C.byref(g)) == 0, product.irlcu_error_string()
        d = IrlcuEsse(e.kx, e.ky, e.kz, e.collapse, e.nterms, e.mu0, e.mu_avg, e.pix, e.cntr_pix_fac, e.noffs,
                      e.ndepths, e.krnl_file, e.mu_file, e.kmu_outside)
        pr = orc.Problem(case)
        cnt = e.kx * e.ky * e.kz
        want = (np.ctypeslib.as_array(pr.P.krnl, shape=(cnt,)), np.ctypeslib.as_array(pr.P.kmu, shape=(cnt,)))
        for term in (0, 1):
            got = np.full(cnt, np.nan, np.float32)
            assert product.irlcu_esse_expand(C.byref(d), term, api.fptr(got)) == 0, product.irlcu_error_string()
            assert np.array_equal(_bits(got), _bits(want[term])), (kw, term)
        product.irlcu_shutdown()
        product.irl_esse_free(C.byref(e))


def test_initial_estimate_and_reorder_bit_for_bit(product, orc):
    """The host functions of the set-up on their own: libirl's serial float
    sum of the projections, the one-pass initial estimate (mean, circle,
    attenuation-map threshold; initial_est.c:29-158) and the layout reorder
    (irlosem.c:170-176), against the oracle and numpy."""
    product.irl_projection_sum.restype = C.c_float
    product.irl_projection_sum.argtypes = [api.FLOAT_P, C.c_size_t]
    product.irl_initial_estimate_sum.restype = api.FLOAT_P
    product.irl_initial_estimate_sum.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_float,
                                                 api.FLOAT_P, api.FLOAT_P]
    product.irl_reorder.restype = None
    product.irl_reorder.argtypes = [C.c_int, C.c_int, C.c_int, api.FLOAT_P, api.FLOAT_P]
    rng = np.random.default_rng(11)
    for n, nz, na in ((128, 128, 120), (33, 33, 8), (48, 40, 12), (7, 5, 3)):
        hp = HostParms()
        hp.n, hp.nz, hp.nviews, hp.pix = n, nz, na, np.float32(0.3125)
        meas = (rng.random((na, nz, n)) - 0.1).astype(np.float32)
        fsum = product.irl_projection_sum(api.fptr(meas), meas.size)
        want = np.zeros((n, nz, n), np.float32)
        orc.orc().or_initial_estimate(n, nz, na, api.fptr(meas), api.fptr(want))
        got = np.full((n, nz, n), np.float32(np.nan), np.float32)
        product.irl_initial_estimate_sum(C.byref(hp), 0, 0.0, None, fsum, None, api.fptr(got))
        assert np.array_equal(_bits(got), _bits(want)), (n, nz)
        # attenuation-map support: voxels whose (internal-layout) map value is
        # below thresh * pixel size are 0 as well
        atn = (rng.random((n, nz, n)) * 0.2).astype(np.float32)
        thresh = np.float32(0.3)
        got_m = np.empty_like(got)
        product.irl_initial_estimate_sum(C.byref(hp), 0, float(thresh), None, fsum, api.fptr(atn), api.fptr(got_m))
        cut = np.float32(thresh * hp.pix)
        want_m = np.where(atn < cut, np.float32(0), want)
        assert np.array_equal(_bits(got_m), _bits(want_m)), (n, nz)
        assert 0 < int((want_m != want).sum()) < want.size
        ext = rng.random((nz, n, n)).astype(np.float32)
        out = np.empty((n, nz, n), np.float32)
        product.irl_reorder(nz, n, n, api.fptr(ext), api.fptr(out))
        assert np.array_equal(out, orc.to_internal(ext)), (n, nz)


@pytest.mark.gpu
@pytest.mark.parametrize("contour,thresh", [(1, 0.0), (0, 0.5), (1, 0.5)])
def test_initial_estimate_support_matches_reference(product, orc, tmp_path, contour, thresh):
    """bUseContourSupport (everything behind each view's detector face is 0)
    and fAtnMapThresh (attenuation below thresh x pixel size is 0): the
    iteration-0 image of IrlOsem equals the compiled reference's bit for bit,
    and the reconstruction after one iteration is within the image
    tolerance."""
    if not orc.have_ref():
        pytest.skip("compiled reference not available")
    ref = orc.ref()
    from test_gpu_parity import IMAGE_TOL
    case = W.plain64(seed=1700 + 3 * contour + int(10 * thresh), n=32, nviews=8, subsets=2, iterations=1)
    files = case.write_tables(str(tmp_path))
    meas = W.poisson_counts(np.abs(np.random.default_rng(5).random((case.nviews, case.nz, case.n))
                                   .astype(np.float32)), 2e5, 1700)
    out = {}
    for name, lib in (("product", product), ("reference", ref)):
        p, o, v = case.parms(), case.options(), case.views()
        o.bUseContourSupport = contour
        o.fAtnMapThresh = thresh
        atn, m, rec = case.atn.copy(), meas.copy(), np.zeros_like(case.act)
        first = []
        cb = api.ITER_CB(lambda it, q: first.append(np.ctypeslib.as_array(q, shape=(case.act.size,)).copy())
                         if it == 0 else None)
        rc = lib.IrlOsem(C.byref(p), C.byref(o), v, dup(files["drf"]), None, cb, None, api.fptr(atn),
                         api.fptr(m), api.fptr(rec), None, None)
        assert rc == 0, lib.pchIrlErrorString()
        out[name] = (first[0], rec, atn)
    assert np.array_equal(_bits(out["product"][0]), _bits(out["reference"][0]))
    assert np.array_equal(_bits(out["product"][2]), _bits(out["reference"][2]))
    zeros = int((out["reference"][0] == 0).sum())
    assert zeros > (case.act.size * 0.2)  # the support mattered
    assert rel_l2(out["product"][1], out["reference"][1]) <= IMAGE_TOL
