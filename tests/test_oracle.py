"""The CPU oracle (oracle/src/irl_oracle.c) pinned against the reference.

Golden fixtures come from the unmodified reference C compiled with the MIP
shim (tests/golden/make_golden.py).  Where the compiled reference is
present (oracle/_ref), further seeded cases are compared live.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN, dup, golden_case, rel_l2
from libirl_b200 import api, workloads as W


def _rot(orc, fn, angle, vol):
    out = np.zeros_like(vol)
    n, nz, _ = vol.shape
    getattr(orc.orc(), fn)(float(angle), api.fptr(vol), api.fptr(out), n, nz)
    return out


def test_rotations_match_golden_bit_for_bit(orc):
    d = np.load(os.path.join(GOLDEN, "rotate.npz"))
    vol = d["vol"]
    for i, a in enumerate(d["angles"]):
        assert np.array_equal(_rot(orc, "or_shears_rotate", a, vol), d["shears"][i])
        assert np.array_equal(_rot(orc, "or_rot3dpar", a, vol), d["rot3dpar"][i])


def test_shear_rotation_reads_nothing_past_the_volume(orc):
    """For odd n the middle row's last second tap lies one past the row, with
    weight 0 (for the last row of the last slice: past the volume). The
    oracle reads 0 there, so NaN in the memory after the volume (and before
    it, for the flipped taps) must not reach the output."""
    rng = np.random.default_rng(9)
    for n, nz in [(33, 2), (17, 3), (65, 1)]:
        pad = n * nz * n
        buf = np.full(3 * pad, np.nan, np.float32)
        vol = buf[pad:2 * pad].reshape(n, nz, n)  # NaN on both sides of the volume
        vol[...] = rng.random((n, nz, n), dtype=np.float32)
        angles = np.concatenate([rng.uniform(-7, 7, 24), np.pi / 2 * np.arange(-4, 5)]).astype(np.float32)
        for a in angles:
            out = np.zeros_like(vol)
            orc.orc().or_shears_rotate(float(a), api.fptr(vol), api.fptr(out), n, nz)
            assert np.isfinite(out).all(), (n, nz, float(a))


def test_conv2d_ypad_matches_golden_bit_for_bit(orc):
    d = np.load(os.path.join(GOLDEN, "conv2d_ypad.npz"))
    plane, psf = d["plane"], d["psf"]
    ny, nx = plane.shape
    for i, (pad, avg) in enumerate(d["pads"]):
        out = np.zeros_like(plane)
        orc.orc().or_conv2d_ypad(api.fptr(plane), nx, ny, api.fptr(psf), (psf.shape[1] - 1) // 2,
                                 (psf.shape[0] - 1) // 2, int(pad), int(avg), api.fptr(out))
        assert np.array_equal(out, d["out"][i])


def test_genprj_osem_plain_match_golden_bit_for_bit(orc):
    case, d = golden_case("plain16")
    pr = orc.Problem(case)
    assert np.array_equal(pr.genprj(), d["prj"])
    est = pr.osem(d["meas"], case.iterations, case.nviews // case.subsets)
    assert np.array_equal(orc.to_external(est), d["recon"])


def test_genprj_osem_scatter_match_golden(orc):
    # ESSE uses an FFT: the shim rounds each transform to float, the oracle
    # convolves in double, so agreement is to float rounding
    case, d = golden_case("srf16")
    pr = orc.Problem(case)
    prj = pr.genprj()
    for v in range(case.nviews):
        assert rel_l2(prj[v], d["prj"][v]) < 1e-6
    est = pr.osem(d["meas"], case.iterations, case.nviews // case.subsets)
    assert rel_l2(orc.to_external(est), d["recon"]) < 1e-5


def test_subset_scheme_known_answer(orc):
    # osemrecon.c:433-450: subset s starts at s/2 + (s%2)*S/2, stride S
    import libirl_b200 as L
    lib = L.load() if os.path.exists(L.SO) else None
    if lib is None:
        pytest.skip("libirl_b200.so not built")
    p = C.POINTER(C.c_int)()
    ns = lib.irl_compute_subsets(120, 15, C.byref(p))
    assert ns == 8
    got = np.ctypeslib.as_array(p, shape=(120,)).reshape(8, 15)
    for s in range(8):
        start = s // 2 + (s % 2) * 8 // 2
        assert list(got[s]) == [start + 8 * m for m in range(15)]
    assert sorted(got.ravel().tolist()) == list(range(120))


def _have_ref(orc):
    return os.path.exists(orc.REF_SO)


@pytest.mark.parametrize("fast", [1, 0])
def test_oracle_vs_reference_live_rotations(orc, fast):
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    rng = np.random.default_rng(11 + fast)
    for n, nz in [(17, 2), (32, 3), (64, 2)]:
        vol = rng.random((n, nz, n), dtype=np.float32)
        for a in rng.uniform(-8, 8, 6).astype(np.float32):
            if fast:
                assert np.array_equal(_rot(orc, "or_shears_rotate", a, vol), orc.ref_shears_rotate(float(a), vol))
            else:
                assert np.array_equal(_rot(orc, "or_rot3dpar", a, vol), orc.ref_rot3dpar(float(a), vol))


def test_oracle_vs_reference_live_osem_padding(orc):
    """Axial padding and a non-default rotator, full IrlOsem chain."""
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    case = W.plain64(seed=1077, n=24, nviews=8, subsets=2, iterations=2)
    files = case.write_tables("/tmp/irl_oracle_pad")
    ref = orc.ref()
    p, o, v = case.parms(), case.options(), case.views()
    o.iAxialPadLength, o.iAxialAvgLength = 3, 2
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    assert ref.IrlGenprj(C.byref(p), C.byref(o), v, dup(files["drf"]), None, None, None, api.fptr(act),
                         api.fptr(atn), api.fptr(prj), 1.0, None, None) == 0
    pr = orc.Problem(case, pad_len=3, avg_len=2)
    assert np.array_equal(pr.genprj(), prj)


def test_oracle_backproject_single_view_matches_reference(orc, tmp_path):
    """BackProject of one view on a constant projection (prjbck.c:254-427,
    attenuation + DRF, three-shear unrotation): the per-view term of a norm
    image (osemrecon.c:282-320), which the GPU single-view backprojection
    test compares with or_backproject.  Here or_backproject is compared
    with the reference's own BackProject for every view of the same
    elliptical-orbit case, bit for bit."""
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    case = W.full128(seed=2060, n=32, nviews=8, subsets=8, iterations=1, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    ref = orc.ref()
    F, I, FL = api.FLOAT_P, C.c_int, C.c_float
    ref.BackProject.restype = None
    ref.BackProject.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.c_void_p, F, F, F, FL, FL,
                                I, I, I, I]
    title, col = C.c_char_p(), C.c_char_p()
    tab = ref.sReadDrfTab(files["drf"].encode(), C.byref(title), C.byref(col))
    tab.psBckDrfTab = None
    tab.bFFTconvolve = 0  # sReadDrfTab leaves it unset; IrlSetup.c:577 sets it from the options
    n, nz = case.n, case.nz
    pr = orc.Problem(case)
    ones = np.ones((nz, n), np.float32)
    model = pr.model(srf=False)
    assert model == 3
    ref.InitPrj(nz, n, n, 7)  # every work image, as IrlOsem with a scatter model sets up
    try:
        for v in range(case.nviews):
            want = np.zeros((n, nz, n), np.float32)
            atn, ratio = pr.atn.copy(), ones.copy()
            ref.BackProject(nz, n, n, model, case.pix, v, float(case.angles[v]), float(case.cfcr[v]), C.byref(tab),
                            None, api.fptr(atn), api.fptr(ratio), api.fptr(want), 1.0, 1.0, 0, 0, 0, 1)
            got = np.zeros_like(want)
            orc.orc().or_backproject(C.byref(pr.P), model, v, api.fptr(pr.atn), api.fptr(ones), api.fptr(got))
            assert want.max() > 0.5
            assert np.array_equal(got, want), f"view {v}: relL2 {rel_l2(got, want):.3e}"
    finally:
        ref.FreePrj()


def test_oracle_project_single_view_matches_reference(orc, tmp_path):
    """Project of one view (prjbck.c:68-252, attenuation + DRF, three-shear
    rotation of activity and attenuation) from or_project against the
    reference's own Project, every view of the elliptical-orbit case, bit
    for bit."""
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    case = W.full128(seed=2061, n=32, nviews=8, subsets=8, iterations=1, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    ref = orc.ref()
    F, I, FL = api.FLOAT_P, C.c_int, C.c_float
    ref.Project.restype = None
    ref.Project.argtypes = [I, I, I, I, FL, I, FL, FL, C.POINTER(api.DrfTab), C.c_void_p, F, F, F, FL, FL,
                            I, I, I, I, I]
    title, col = C.c_char_p(), C.c_char_p()
    tab = ref.sReadDrfTab(files["drf"].encode(), C.byref(title), C.byref(col))
    tab.psBckDrfTab = None
    tab.bFFTconvolve = 0  # sReadDrfTab leaves it unset; IrlSetup.c:577 sets it from the options
    n, nz = case.n, case.nz
    pr = orc.Problem(case)
    model = pr.model(srf=False)
    ref.InitPrj(nz, n, n, 7)
    try:
        for v in range(case.nviews):
            want = np.zeros((nz, n), np.float32)
            atn, act = pr.atn.copy(), pr.act.copy()
            ref.Project(nz, n, n, model, case.pix, v, float(case.angles[v]), float(case.cfcr[v]), C.byref(tab),
                        None, api.fptr(atn), api.fptr(act), api.fptr(want), 1.0, 1.0, 0, 0, 0, 0, 1)
            got = np.zeros_like(want)
            orc.orc().or_project(C.byref(pr.P), model, v, api.fptr(pr.act), api.fptr(pr.atn), 1.0, api.fptr(got))
            assert want.max() > 0
            assert np.array_equal(got, want), f"view {v}: relL2 {rel_l2(got, want):.3e}"
    finally:
        ref.FreePrj()


def test_reference_fft_convolution_is_zero_padded_direct(orc):
    """libirl's FFT convolution branch (PadSwap + realft3d + conv2dPsfFFT on a
    2N x 2Nz grid) equals the direct "same" convolution with no axial
    padding: the axial pad is ignored and, for h <= N, the circular
    convolution never wraps onto the cropped output."""
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    rng = np.random.default_rng(31)
    for ny, nx, h in [(12, 16, 3), (17, 20, 6), (32, 32, 16), (9, 40, 8)]:
        plane = rng.random((ny, nx), dtype=np.float32)
        psf = rng.random((2 * h + 1, 2 * h + 1)).astype(np.float32)
        psf /= psf.sum()
        fft = orc.ref_conv2d_fft(plane, psf)
        direct = orc.ref_conv2d_ypad(plane, psf, pad=0, avg=0)
        assert rel_l2(fft, direct) <= 1e-6, (ny, nx, h, rel_l2(fft, direct))
        padded = orc.ref_conv2d_ypad(plane, psf, pad=min(3, h), avg=2)
        assert rel_l2(padded, direct) > 1e-4  # the pad would have mattered


def test_reference_fft_table_genprj_matches_oracle_without_pad(orc):
    """Full IrlGenprj chain with bFFTConvolve: the reference's projections
    equal the oracle's direct convolution with the axial pad switched off."""
    if not _have_ref(orc):
        pytest.skip("compiled reference not available")
    case = W.plain64(seed=1078, n=24, nviews=6, subsets=2, iterations=1)
    files = case.write_tables("/tmp/irl_oracle_fft")
    ref = orc.ref()
    p, o, v = case.parms(), case.options(), case.views()
    o.iAxialPadLength, o.iAxialAvgLength, o.bFFTConvolve = 3, 2, 1
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    assert ref.IrlGenprj(C.byref(p), C.byref(o), v, dup(files["drf"]), None, None, None, api.fptr(act),
                         api.fptr(atn), api.fptr(prj), 1.0, None, None) == 0
    want = orc.Problem(case, pad_len=0, avg_len=0).genprj()
    for vi in range(case.nviews):
        assert rel_l2(prj[vi], want[vi]) <= 1e-6, (vi, rel_l2(prj[vi], want[vi]))


def test_oracle_threads_do_not_change_results(orc):
    """The restatement runs the views of IrlGenprj and of each OSEM subset on
    host threads and adds the backprojections in view order afterwards, so
    one thread and several give the same bits."""
    case = W.full128(seed=2300, n=24, nviews=8, subsets=2, iterations=2, drf_max_offs=5)
    out = {}
    for t in (1, 4):
        orc.orc().or_set_threads(t)
        try:
            pr = orc.Problem(case)
            prj = pr.genprj()
            est = pr.osem(W.poisson_counts(prj, 1e5, 2300), 2, 4)
        finally:
            orc.orc().or_set_threads(orc._threads())
        out[t] = (prj, est)
    assert np.array_equal(out[1][0], out[4][0])
    assert np.array_equal(out[1][1], out[4][1])
