"""GPU parity: libirl_b200.so (CUDA) against the CPU oracle.

Tolerances are the ones the path is specified to: relative L2 <= 1e-4 per
projection view and <= 1e-3 on the image after the stated iterations.
Rotations, being pure interpolation with exact rounding, must match bit for
bit.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import dup, golden_case, rel_l2
from libirl_b200 import api, workloads as W

pytestmark = pytest.mark.gpu

VIEW_TOL = 1e-4
IMAGE_TOL = 1e-3

_libc = C.CDLL(None)
_libc.malloc.restype = C.c_void_p
_libc.malloc.argtypes = [C.c_size_t]


def malloc_array(values, ctype):
    p = _libc.malloc(C.sizeof(ctype) * len(values))
    arr = (ctype * len(values)).from_address(p)
    for i, v in enumerate(values):
        arr[i] = v
    return p


def gpu_genprj(lib, case, files, primary=1.0, opts=None, scatest=None, model_drf=True, krnl=True, cb=None):
    p, o, v = case.parms(), case.options(model_drf=model_drf), case.views()
    if opts:
        for k, val in opts.items():
            setattr(o, k, val)
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    se = None if scatest is None else scatest.copy()
    rc = lib.IrlGenprj(C.byref(p), C.byref(o), v, dup(files.get("drf")) if model_drf else None,
                       dup(files.get("krnl")) if krnl else None, cb, api.fptr(se), api.fptr(act), api.fptr(atn),
                       api.fptr(prj), primary, None, None)
    assert rc == 0, lib.pchIrlErrorString()
    return prj


def gpu_osem(lib, case, files, meas, iterations=None, opts=None, parms=None, krnl=True, cb=None, scatest=None):
    p, o, v = case.parms(), case.options(), case.views()
    if iterations is not None:
        p.NumIterations = iterations
    for k, val in (parms or {}).items():
        setattr(p, k, val)
    for k, val in (opts or {}).items():
        setattr(o, k, val)
    atn = case.atn.copy()
    rec = np.zeros_like(case.act)
    m = meas.copy()
    se = None if scatest is None else scatest.copy()
    cbf = cb if cb is not None else api.ITER_CB(lambda i, q: None)
    rc = lib.IrlOsem(C.byref(p), C.byref(o), v, dup(files.get("drf")), dup(files.get("krnl")) if krnl else None,
                     cbf, api.fptr(se), api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    assert rc == 0, lib.pchIrlErrorString()
    return rec


# ------------------------------------------------------------- rotations

@pytest.mark.parametrize("n,nz", [(16, 3), (33, 2), (64, 4), (128, 2), (128, 5), (200, 1), (256, 2)])
@pytest.mark.parametrize("fast", [1, 0, "fused", "single", "pair", "split", "global"])
def test_rotation_bit_exact(product, orc, monkeypatch, n, nz, fast):
    """Both rotators bit for bit against the oracle; the three-shear one in
    its two-slice and one-slice column-walk forms, its fused-pass form, and
    for slices beyond one SM's shared memory (n = 256) its two-CTA cluster
    form (default), its column-split form and its global-memory form."""
    import libirl_b200 as L
    if fast == "fused":
        monkeypatch.setenv("IRLCU_SHEAR_STAGE", "0")
        fast = 1
    if fast in ("single", "pair"):
        monkeypatch.setenv("IRLCU_SHEAR_PAIR", "0" if fast == "single" else "1")
        fast = 1
    if fast in ("split", "global"):  # slices beyond shared memory: not the cluster form
        monkeypatch.setenv("IRLCU_SHEAR_CLUSTER", "0")
        if fast == "global":  # the two global-memory kernels, not the column split
            monkeypatch.setenv("IRLCU_SHEAR_SPLIT", "0")
        fast = 1
    rng = np.random.default_rng(n * 7 + nz)
    vol = rng.random((n, nz, n), dtype=np.float32)
    g = L.IrlcuGeom(n, nz, 1, fast, 1)
    L.check(product, product.irlcu_init(C.byref(g)))
    try:
        angles = np.concatenate([rng.uniform(-7, 7, 9), [np.pi / 2, -np.pi / 2, np.pi, 0.0]]).astype(np.float32)
        for a in angles:
            out = np.zeros_like(vol)
            L.check(product, product.irlcu_rotate_volume(float(a), api.fptr(vol), api.fptr(out), 0, 0))
            ref = np.zeros_like(vol)
            fn = orc.orc().or_shears_rotate if fast else orc.orc().or_rot3dpar
            fn(float(a), api.fptr(vol), api.fptr(ref), n, nz)
            assert np.array_equal(out, ref), f"angle {a}: {int((out != ref).sum())} voxels differ"
    finally:
        product.irlcu_shutdown()


# -------------------------------------------------------------- projection

@pytest.mark.parametrize("variant", ["atn", "atn_drf", "drf_pad", "fft_table", "srf_c2", "srf_c1", "srf_primary0"])
def test_genprj_per_view(product, orc, tmp_path, variant):
    if variant.startswith("srf"):
        c = 1 if variant == "srf_c1" else 2
        case = W.full128(seed=2100, n=32, nviews=12, subsets=2, iterations=2, collapse=c, drf_max_offs=6)
    else:
        case = W.plain64(seed=1100, n=48, nviews=12, subsets=2, iterations=2)
    files = case.write_tables(str(tmp_path))
    pad = (3, 2) if variant in ("drf_pad", "fft_table") else (0, 0)
    opts = {"iAxialPadLength": pad[0], "iAxialAvgLength": pad[1]}
    if variant == "fft_table":
        # libirl's FFT convolution path ignores the axial pad
        # (convolve_ypad.c:63-94): the oracle runs without it
        opts["bFFTConvolve"] = 1
        pad = (0, 0)
    prim = 0.0 if variant == "srf_primary0" else 1.0
    use_drf = variant != "atn"
    got = gpu_genprj(product, case, files, primary=prim, opts=opts, model_drf=use_drf)
    pr = orc.Problem(case, with_drf=use_drf, pad_len=pad[0], avg_len=pad[1])
    want = pr.genprj(primary=prim)
    for vi in range(case.nviews):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL, (variant, vi, rel_l2(got[vi], want[vi]))


@pytest.mark.parametrize("engine", ["direct", "fft", "fft_lines"])
def test_genprj_drf_engines(product, orc, tmp_path, monkeypatch, engine):
    """The DRF engines (direct convolution kernels; the Fourier-domain
    engine with one CTA per plane, and in its row/column-pass form) against
    the oracle on a 33 x 33 DRF with axial padding."""
    monkeypatch.setenv("IRLCU_DRF_ENGINE", "fft" if engine.startswith("fft") else engine)
    monkeypatch.setenv("IRLCU_DRF_PLANE", "0" if engine == "fft_lines" else "1")
    case = W.full128(seed=2150, n=48, nviews=6, subsets=2, iterations=1, drf_max_offs=17, with_srf=False)
    files = case.write_tables(str(tmp_path))
    opts = {"iAxialPadLength": 4, "iAxialAvgLength": 3}
    got = gpu_genprj(product, case, files, opts=opts, krnl=False)
    want = orc.Problem(case, with_srf=False, pad_len=4, avg_len=3).genprj()
    for vi in range(case.nviews):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL, (engine, vi, rel_l2(got[vi], want[vi]))


def test_drf_half_width_beyond_direct_limit(product, orc, tmp_path, monkeypatch):
    """A 73 x 73 DRF (half-width 36) runs on the Fourier-domain engine only;
    the direct engine refuses it."""
    case = W.full128(seed=2160, n=40, nviews=3, subsets=1, iterations=1, drf_max_offs=37, with_srf=False)
    files = case.write_tables(str(tmp_path))
    monkeypatch.setenv("IRLCU_DRF_ENGINE", "direct")
    p, o, v = case.parms(), case.options(), case.views()
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
    rc = product.IrlGenprj(C.byref(p), C.byref(o), v, dup(files["drf"]), None, None, None, api.fptr(act),
                           api.fptr(atn), api.fptr(prj), 1.0, None, None)
    assert rc != 0 and b"limit" in product.pchIrlErrorString()
    monkeypatch.setenv("IRLCU_DRF_ENGINE", "auto")
    got = gpu_genprj(product, case, files, krnl=False)
    want = orc.Problem(case, with_srf=False).genprj()
    for vi in range(case.nviews):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL, (vi, rel_l2(got[vi], want[vi]))


@pytest.mark.parametrize("form", ["reg", "pass"])
def test_genprj_esse_yz_forms(product, orc, tmp_path, monkeypatch, form):
    """The y-z part of ESSE in its register-transform form and its
    Stockham-pass form, on a 64^3 grid with both Taylor terms."""
    monkeypatch.setenv("IRLCU_ESSE_YZ", form)
    case = W.full128(seed=2180, n=64, nviews=6, subsets=2, iterations=1, collapse=2, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    got = gpu_genprj(product, case, files)
    want = orc.Problem(case).genprj()
    for vi in range(case.nviews):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL, (form, vi, rel_l2(got[vi], want[vi]))


@pytest.mark.parametrize("n,collapse", [(40, 2), (48, 2), (24, 1)])
def test_genprj_esse_mixed_radix_grid(product, orc, tmp_path, n, collapse):
    """ESSE grids of ceil(2 N / c) that are not powers of two (40 = 8*5,
    48 = 16*3) run on the mixed-radix transforms."""
    case = W.full128(seed=2170 + n, n=n, nviews=6, subsets=2, iterations=1, collapse=collapse, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    got = gpu_genprj(product, case, files)
    want = orc.Problem(case).genprj()
    for vi in range(case.nviews):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL, (n, collapse, vi, rel_l2(got[vi], want[vi]))


def test_genprj_golden_fixture(product, tmp_path):
    """The GPU path against the reference's own outputs."""
    for name in ("plain16", "srf16"):
        case, d = golden_case(name)
        files = case.write_tables(str(tmp_path / name))
        got = gpu_genprj(product, case, files)
        for vi in range(case.nviews):
            assert rel_l2(got[vi], d["prj"][vi]) <= VIEW_TOL


def test_genprj_scatter_estimate_view_times_and_detectors(product, orc, tmp_path):
    """IrlGenprj adds the scaled scatter estimate and applies per-view times
    and per-detector sensitivities (irlgenprj.c:245-257)."""
    case = W.plain64(seed=1200, n=32, nviews=8, subsets=2, iterations=1)
    files = case.write_tables(str(tmp_path))
    base = gpu_genprj(product, case, files)
    se = np.abs(np.random.default_rng(3).random(base.shape, dtype=np.float32)) * 0.01
    times = [0.5 + 0.1 * i for i in range(case.nviews)]
    dets = [0 if i % 2 == 0 else 1 for i in range(case.nviews)]
    assert product.iSetupExtraPrjViewData(case.nviews, malloc_array(times, C.c_float),
                                          malloc_array(dets, C.c_int)) == 0
    d0 = product.pvStoreDetectorData(0.1, 2.4, 0.6, 0.38, 1.0, 0, 0, dup(files["drf"]))
    d1 = product.pvStoreDetectorData(0.1, 2.4, 0.6, 0.38, 2.0, 0, 0, dup(files["drf"]))
    arr = _libc.malloc(2 * C.sizeof(C.c_void_p))
    (C.c_void_p * 2).from_address(arr)[:] = [d0, d1]
    assert product.iSetupDetectors(2, arr) == 0
    got = gpu_genprj(product, case, files, scatest=se)
    for vi in range(case.nviews):
        want = (base[vi] * case.nviews + se[vi]) * np.float32(times[vi]) * np.float32(1.0 + dets[vi])
        want /= case.nviews
        assert rel_l2(got[vi], want) <= VIEW_TOL


# ------------------------------------------------------------------- OSEM

def test_osem_plain_config_full_size(product, orc, tmp_path):
    """The CPU-runnable case at its stated size: 64^3, 60 views, 4 subsets,
    5 iterations, attenuation + Gaussian DRF."""
    case = W.plain64()
    files = case.write_tables(str(tmp_path))
    pr = orc.Problem(case)
    meas = W.poisson_counts(pr.genprj(), case.counts, 1000)
    got = gpu_osem(product, case, files, meas)
    want = orc.to_external(pr.osem(meas, case.iterations, case.nviews // case.subsets))
    assert rel_l2(got, want) <= IMAGE_TOL


def test_osem_golden_fixture(product, tmp_path):
    for name in ("plain16", "srf16"):
        case, d = golden_case(name)
        files = case.write_tables(str(tmp_path / name))
        got = gpu_osem(product, case, files, d["meas"])
        assert rel_l2(got, d["recon"]) <= IMAGE_TOL


@pytest.mark.parametrize("srf_iters", [3, 1, 0])
def test_osem_scatter_modelling(product, orc, tmp_path, srf_iters):
    """ESSE in the projector; with fewer scatter iterations than iterations
    the stored scatter projection is reused (osemrecon.c:734-788)."""
    case = W.full128(seed=2200, n=32, nviews=8, subsets=2, iterations=3, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    pr = orc.Problem(case)
    meas = W.poisson_counts(pr.genprj(), 2e5, 2200)
    got = gpu_osem(product, case, files, meas, parms={"iNumSrfIterations": srf_iters})
    want = orc.to_external(pr.osem(meas, 3, 4, srf_iters=srf_iters))
    assert rel_l2(got, want) <= IMAGE_TOL


@pytest.mark.parametrize("pair", ["0", "1"])
def test_osem_shear_forms(product, orc, tmp_path, monkeypatch, pair):
    """The one-slice and two-slice shear kernels in both of their uses, the
    rotation of the shared estimate and the unrotation of the per-view
    backprojections, through a whole reconstruction."""
    monkeypatch.setenv("IRLCU_SHEAR_PAIR", pair)
    case = W.full128(seed=2210, n=48, nz=33, nviews=8, subsets=2, iterations=2, drf_max_offs=6, with_srf=False)
    files = case.write_tables(str(tmp_path))
    pr = orc.Problem(case)
    meas = W.poisson_counts(pr.genprj(), 2e5, 2210)
    got = gpu_osem(product, case, files, meas)
    want = orc.to_external(pr.osem(meas, 2, 4))
    assert rel_l2(got, want) <= IMAGE_TOL


def test_esse_collapse_in_two_slice_shear_is_bit_exact(product, tmp_path, monkeypatch):
    """With ESSE at collapse 2 the two-slice shear also writes the collapsed
    rotated volumes (CollapseByFac, krnlprj3d.c:559-592); the one-slice
    shear leaves that to the separate collapse pass.  Projections and a
    reconstruction must be the same bits either way."""
    case = W.full128(seed=2230, n=64, nviews=8, subsets=2, iterations=2, collapse=2, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    out = {}
    for pair in ("0", "1"):
        monkeypatch.setenv("IRLCU_SHEAR_PAIR", pair)
        prj = gpu_genprj(product, case, files)
        meas = W.poisson_counts(prj, 2e5, 2230)
        out[pair] = (prj, gpu_osem(product, case, files, meas))
    assert np.array_equal(out["0"][0], out["1"][0])
    assert np.array_equal(out["0"][1], out["1"][1])


def test_osem_bilinear_rotator_and_callbacks(product, orc, tmp_path):
    case = W.plain64(seed=1300, n=32, nviews=8, subsets=2, iterations=3)
    files = case.write_tables(str(tmp_path))
    pr = orc.Problem(case, fast_rotate=False)
    meas = W.poisson_counts(pr.genprj(), 1e5, 1300)
    adv = api.AdvOptions(0, 0)
    product.OsemSetAdvOptions(C.byref(adv))
    seen = []

    @api.ITER_CB
    def cb(i, ptr):
        seen.append((i, float(np.ctypeslib.as_array(ptr, shape=(case.n ** 2 * case.nz,)).sum())))

    try:
        got = gpu_osem(product, case, files, meas, cb=cb)
    finally:
        adv = api.AdvOptions(1, 0)
        product.OsemSetAdvOptions(C.byref(adv))
    assert [s[0] for s in seen] == [0, 1, 2, 3]  # iteration 0 then every iteration
    assert abs(seen[-1][1] - float(got.sum())) <= 1e-4 * abs(float(got.sum()))
    want = orc.to_external(pr.osem(meas, 3, 4))
    assert rel_l2(got, want) <= IMAGE_TOL


def test_osem_hooks_see_and_modify_state(product, tmp_path):
    case = W.plain64(seed=1400, n=24, nviews=8, subsets=2, iterations=2)
    files = case.write_tables(str(tmp_path))
    meas = np.abs(np.random.default_rng(1).random((8, 24, 24), dtype=np.float32)) * 10
    calls = {"it": 0, "sub": 0, "ang": 0}

    @api.HOOK_CB
    def post_subset(d, ctx):
        calls["sub"] += 1

    @api.HOOK_CB
    def post_angle(d, ctx):
        calls["ang"] += 1

    @api.HOOK_CB
    def prev_iter(d, ctx):
        calls["it"] += 1
        if d.contents.iIterationIdx == 2:  # zero the estimate before the last iteration
            est = np.ctypeslib.as_array(d.contents.pfEst, shape=(24 * 24 * 24,))
            est[:] = 0

    product.OsemSetPostSubsetHook(C.cast(post_subset, C.c_void_p), None)
    product.OsemSetPostAngleHook(C.cast(post_angle, C.c_void_p), None)
    product.OsemSetPrevIterHook(C.cast(prev_iter, C.c_void_p), None)
    try:
        got = gpu_osem(product, case, files, meas)
    finally:
        for fn in ("OsemSetPostSubsetHook", "OsemSetPostAngleHook", "OsemSetPrevIterHook"):
            getattr(product, fn)(None, None)
    assert calls == {"it": 2, "sub": 4, "ang": 16}
    assert float(np.abs(got).max()) == 0.0


def test_osem_norm_files_and_errors(product, tmp_path):
    import glob
    case = W.plain64(seed=1500, n=16, nviews=8, subsets=2, iterations=1)
    files = case.write_tables(str(tmp_path))
    meas = np.ones((8, 16, 16), np.float32)
    base = str(tmp_path / "nrm")
    gpu_osem(product, case, files, meas, parms={"pchNormImageBase": base.encode()})
    assert glob.glob(base + "*") == []  # written during the run, deleted at the end
    # views per subset must divide the views (osemrecon.c:416-420) and the
    # subset count must be 1 or even (osemrecon.c:422-425)
    for per, msg in ((3, b"multiple"), (8 // 1, None), (2, None)):
        p, o, v = case.parms(), case.options(), case.views()
        p.NumAngPerSubset = per
        atn, rec, m = case.atn.copy(), np.zeros_like(case.act), meas.copy()
        rc = product.IrlOsem(C.byref(p), C.byref(o), v, dup(files["drf"]), None, api.ITER_CB(lambda i, q: None),
                             None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        if msg is None:
            assert rc == 0, product.pchIrlErrorString()
        else:
            assert rc != 0 and msg in product.pchIrlErrorString()
    case6 = W.plain64(seed=1501, n=16, nviews=6, subsets=3, iterations=1)
    files6 = case6.write_tables(str(tmp_path / "six"))
    p, o, v = case6.parms(), case6.options(), case6.views()
    atn, rec, m = case6.atn.copy(), np.zeros_like(case6.act), np.ones((6, 16, 16), np.float32)
    rc = product.IrlOsem(C.byref(p), C.byref(o), v, dup(files6["drf"]), None, api.ITER_CB(lambda i, q: None), None,
                         api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    assert rc != 0 and b"not even" in product.pchIrlErrorString()


def test_backprojection_per_view_through_norm_images(product, orc, tmp_path):
    """BackProject of one view (prjbck.c:254-427) on its own: with one view
    per subset, each subset's norm image is the inverted backprojection of
    that view's measured-bin mask times its ViewTime (osemrecon.c:282-320),
    here all bins (positive data, the detector spanning the slice).  The
    norm files written during IrlOsem are read at the iteration-0 callback
    and inverted back; every view's backprojection (attenuation + DRF, the
    backprojector model) is compared with the oracle's or_backproject,
    within the per-view tolerance on the voxels both keep (the 1e-6 floor of
    the inversion may fall either way on a voxel at the threshold)."""
    case = W.full128(seed=2060, n=32, nviews=8, subsets=8, iterations=1, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    base = str(tmp_path / "nrm")
    ns = case.nviews
    got = {}

    def cb(it, _img):
        if it == 0:
            for s in range(ns):
                got[s] = np.fromfile(f"{base}.norm.{s}.dat", dtype=np.float32).reshape(case.n, case.nz, case.n)

    meas = np.ones((case.nviews, case.nz, case.n), np.float32)
    gpu_osem(product, case, files, meas, parms={"pchNormImageBase": base.encode()}, cb=api.ITER_CB(cb))
    assert len(got) == ns
    order = C.POINTER(C.c_int)()
    assert product.irl_compute_subsets(case.nviews, 1, C.byref(order)) == ns
    views = [order[s] for s in range(ns)]
    assert sorted(views) == list(range(ns))
    pr = orc.Problem(case)
    bck_model = pr.model(srf=False)
    ones = np.ones((case.nz, case.n), np.float32)
    for s, v in enumerate(views):
        ref = np.zeros((case.n, case.nz, case.n), np.float32)
        orc.orc().or_backproject(C.byref(pr.P), bck_model, v, api.fptr(pr.atn), api.fptr(ones), api.fptr(ref))
        norm = got[s]
        both = (norm > 0) & (ref >= np.float32(1e-6))
        assert both.sum() > 0.5 * (ref >= np.float32(1e-6)).sum(), f"view {v}: backprojection support lost"
        flips = int(((norm > 0) != (ref >= np.float32(1e-6))).sum())
        assert flips <= max(2, int(1e-3 * both.sum())), f"view {v}: {flips} voxels on opposite sides of the floor"
        bp = np.zeros_like(ref)
        bp[both] = 1.0 / norm[both].astype(np.float64)
        err = rel_l2(bp[both], ref[both])
        assert err <= VIEW_TOL, f"view {v}: backprojection relL2 {err:.3e}"


# --------------------------------------------------------- full-size checks

@pytest.mark.parametrize("engine", ["direct", "fft"])
def test_full_size_views_against_oracle(product, orc, tmp_path, monkeypatch, engine):
    """Two views of the full-physics 128^3 case (DRF 33x33 + ESSE c=2)
    against the oracle, with each DRF engine (the Fourier-domain one on its
    160 x 160 one-CTA-per-plane grid)."""
    monkeypatch.setenv("IRLCU_DRF_ENGINE", engine)
    full = W.full128(seed=2000)
    sel = [0, 37]
    case = W.Case(full.name, full.n, full.nz, full.pix, len(sel), 1, 1, full.counts, full.act, full.atn,
                  full.angles[sel], full.cfcr[sel], full.atn_scale, full.drf_psfs, full.drf_start,
                  full.drf_spacing, full.krnl, full.collapse, 1)
    files = case.write_tables(str(tmp_path))
    got = gpu_genprj(product, case, files)
    want = orc.Problem(case).genprj()
    for vi in range(len(sel)):
        assert rel_l2(got[vi], want[vi]) <= VIEW_TOL
