"""GPU tests against the compiled reference (oracle/_ref) for the set-up
paths that run device code:

* ComputeOrbit (computeorbit.c:21-150): body-contour orbits (types 1 and 2)
  come from the device edge search (k_orbit.cu); the CFCRs must equal the
  reference's bit for bit.
* Computed GRF tables (gendrf.c, IrlSetup.c:243-334, 514-588): IrlGenprj
  with no DRF file, and IrlOsem with bUseGrfInBck (the backprojector uses
  the GRF, prjbck.c:308-310), within the projection and image tolerances.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import dup, rel_l2
from libirl_b200 import api, workloads as W
from test_gpu_parity import IMAGE_TOL, VIEW_TOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(orc):
    if not orc.have_ref():
        pytest.skip("compiled reference not available")
    return orc.ref()


def _body(n, seed, off=(0.0, 0.0)):
    """An off-centre elliptical body with some structure, n x n."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:n, 0:n].astype(np.float32)
    c = (n - 1) / 2
    img = np.zeros((n, n), np.float32)
    body = ((x - c - off[0] * n) / (0.33 * n)) ** 2 + ((y - c - off[1] * n) / (0.24 * n)) ** 2 <= 1
    img[body] = 1.0 + rng.random(int(body.sum()), dtype=np.float32)
    img += 0.02 * rng.random((n, n), dtype=np.float32)  # low background, removed by the threshold
    return img


def _orbit(lib, img, n, nviews, margin, margins, thresh, otype):
    p = api.IrlParms()
    p.NumPixels, p.NumSlices, p.NumViews, p.BinWidth = n, n, nviews, 0.3125
    angles = (2 * np.pi * np.arange(nviews) / nviews).astype(np.float32)
    v = api.make_views(angles, np.zeros(nviews, np.float32), 0.0, float(n))
    im = img.copy()
    mg = None if margins is None else np.ascontiguousarray(margins, np.float32)
    rc = lib.ComputeOrbit(api.fptr(im), C.byref(p), margin, api.fptr(mg), thresh, otype, v)
    return rc, np.array([v[i].CFCR for i in range(nviews)], np.float32), im


@pytest.mark.parametrize("n,nviews,off,thresh", [
    (64, 60, (0.0, 0.0), 0.1),
    (64, 64, (0.12, -0.08), 0.05),
    (33, 36, (-0.1, 0.1), -0.5),      # odd size, absolute threshold
    (128, 120, (0.05, 0.02), 0.2),
])
@pytest.mark.parametrize("otype", [1, 2])
def test_compute_orbit_contour_matches_reference(product, ref, n, nviews, off, thresh, otype):
    img = _body(n, 40 + n, off)
    for margins in (None, np.linspace(0.5, 3.0, nviews)):
        rc_p, cf_p, im_p = _orbit(product, img, n, nviews, 2.0, margins, thresh, otype)
        rc_r, cf_r, im_r = _orbit(ref, img, n, nviews, 2.0, margins, thresh, otype)
        assert rc_p == rc_r == 0
        assert np.array_equal(im_p, im_r)  # the threshold is applied to the caller's image
        assert np.array_equal(cf_p, cf_r), np.abs(cf_p - cf_r).max()


def test_compute_orbit_circular_and_bad_type(product, ref):
    img = _body(32, 7)
    for lib in (product, ref):
        rc, cf, _ = _orbit(lib, img, 32, 8, 21.5, None, 0.1, 0)
        assert rc == 0 and np.all(cf == np.float32(21.5))
        rc, _, _ = _orbit(lib, img, 32, 8, 21.5, None, 0.1, 3)
        assert rc == 2


def _genprj(lib, case, drf, opts=None):
    p, o, v = case.parms(), case.options(), case.views()
    for k, val in (opts or {}).items():
        setattr(o, k, val)
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    rc = lib.IrlGenprj(C.byref(p), C.byref(o), v, dup(drf), None, None, None, api.fptr(act), api.fptr(atn),
                       api.fptr(prj), 1.0, None, None)
    assert rc == 0, lib.pchIrlErrorString()
    return prj


def _osem(lib, case, drf, meas, opts=None):
    p, o, v = case.parms(), case.options(), case.views()
    for k, val in (opts or {}).items():
        setattr(o, k, val)
    atn, m, rec = case.atn.copy(), meas.copy(), np.zeros_like(case.act)
    rc = lib.IrlOsem(C.byref(p), C.byref(o), v, dup(drf), None, api.ITER_CB(lambda i, q: None), None,
                     api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    assert rc == 0, lib.pchIrlErrorString()
    return rec


def test_genprj_with_computed_grf_matches_reference(product, ref, tmp_path):
    """No DRF file: both libraries compute the collimator's GRF table from
    the IrlParms hole geometry and project with it."""
    case = W.plain64(seed=1600, n=32, nviews=8, subsets=2, iterations=2)
    got = _genprj(product, case, None)
    want = _genprj(ref, case, None)
    for v in range(case.nviews):
        assert rel_l2(got[v], want[v]) <= VIEW_TOL, (v, rel_l2(got[v], want[v]))
    plain = _genprj(product, case, None, {"bModelDrf": 0})
    assert rel_l2(got, plain) > 1e-3  # the GRF blur mattered


def test_osem_with_grf_in_backprojector_matches_reference(product, ref, tmp_path):
    """bUseGrfInBck: the projector uses the DRF file, the backprojector the
    computed GRF."""
    case = W.plain64(seed=1601, n=32, nviews=8, subsets=2, iterations=2)
    files = case.write_tables(str(tmp_path))
    meas = W.poisson_counts(_genprj(ref, case, files["drf"]), 2e5, 1601)
    got = _osem(product, case, files["drf"], meas, {"bUseGrfInBck": 1})
    want = _osem(ref, case, files["drf"], meas, {"bUseGrfInBck": 1})
    assert rel_l2(got, want) <= IMAGE_TOL
    same = _osem(product, case, files["drf"], meas)
    assert rel_l2(got, same) > 1e-4  # the backprojector's table mattered
    got_nofile = _osem(product, case, None, meas)
    want_nofile = _osem(ref, case, None, meas)
    assert rel_l2(got_nofile, want_nofile) <= IMAGE_TOL
