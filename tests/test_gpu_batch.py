"""IrlOsemBatch and whole-iteration CUDA graphs.

Each problem of a batch runs exactly the kernels IrlOsem runs for it alone,
on its own device context and stream, so the reconstructions must be
bit-identical to separate IrlOsem calls; likewise an iteration replayed from
its captured CUDA graph must equal the eagerly launched one.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import dup
from libirl_b200 import api, workloads as W
from test_gpu_parity import gpu_osem

pytestmark = pytest.mark.gpu

_libc = C.CDLL(None)
_libc.strdup.restype = C.c_void_p
_libc.strdup.argtypes = [C.c_char_p]


def _cases():
    return [
        W.plain64(seed=3100, n=32, nviews=12, subsets=4, iterations=3),
        W.full128(seed=3200, n=32, nviews=12, subsets=2, iterations=3, collapse=2, drf_max_offs=6),
        W.plain64(seed=3300, n=48, nviews=16, subsets=4, iterations=2),
    ]


def _meas(case):
    return W.poisson_counts(np.abs(np.random.default_rng(case.n).random((case.nviews, case.nz, case.n))).astype(np.float32) * 20,
                            1e5, case.n)


def _batch(product, cases, files, meas):
    keep = []
    probs = (api.OsemProblem * len(cases))()
    for i, (c, f, m) in enumerate(zip(cases, files, meas)):
        p, o, v = c.parms(), c.options(), c.views()
        atn, prj, rec = c.atn.copy(), m.copy(), np.zeros_like(c.act)
        keep.append((p, o, v, atn, prj, rec))
        q = probs[i]
        q.psIrlParms, q.psOptions = C.pointer(p), C.pointer(o)
        q.psViews = C.cast(v, C.POINTER(api.PrjView))
        q.pchDrfTabFname = _libc.strdup(f["drf"].encode())
        q.pchScatKrnlFname = _libc.strdup(f["krnl"].encode()) if "krnl" in f else None
        q.pfAtnMap, q.pfPrjImage, q.pfReconImage = api.fptr(atn), api.fptr(prj), api.fptr(rec)
    rc = product.IrlOsemBatch(len(cases), probs)
    assert rc == 0, product.pchIrlErrorString()
    for i in range(len(cases)):
        assert probs[i].iStatus == 0
    return [k[5] for k in keep]


def _check_batch(product, cases, tmp_path):
    files = [c.write_tables(str(tmp_path / f"c{i}")) for i, c in enumerate(cases)]
    meas = [_meas(c) for c in cases]
    alone = [gpu_osem(product, c, f, m) for c, f, m in zip(cases, files, meas)]
    got = _batch(product, cases, files, meas)
    for i, (rec, ref) in enumerate(zip(got, alone)):
        assert np.array_equal(rec, ref), f"problem {i}: {int((rec != ref).sum())} voxels differ"


@pytest.mark.parametrize("depth", ["1", "2", "4", "8"])
def test_batch_equals_separate_calls(product, tmp_path, monkeypatch, depth):
    """Any number of problems in flight (IRL_BATCH_DEPTH) gives the separate
    calls' results."""
    monkeypatch.setenv("IRL_BATCH_DEPTH", depth)
    _check_batch(product, _cases() + _cases()[:2], tmp_path)


def test_mem_info(product):
    fr, tot = C.c_size_t(), C.c_size_t()
    assert product.irlcu_mem_info(C.byref(fr), C.byref(tot)) == 0
    assert 0 < fr.value <= tot.value


def test_batch_small_problems_behind_a_large_one(product, tmp_path):
    # 64^3 problems are set up while the 112^3 problem before them still
    # runs: their set-up copies and memsets must be ordered on their own
    # streams, or their first kernels read buffers not yet written
    cases = [W.full128(seed=3700, n=112, nviews=60, subsets=12, iterations=3)]
    cases += [W.full128(seed=3710 + k, n=64, nviews=nv, subsets=ns, iterations=3)
              for k, (nv, ns) in enumerate([(90, 6), (120, 8), (60, 12)])]
    _check_batch(product, cases, tmp_path)


def test_graph_replay_equals_eager(product, tmp_path, monkeypatch):
    case = W.full128(seed=3400, n=32, nviews=12, subsets=4, iterations=4, collapse=2, drf_max_offs=6)
    files = case.write_tables(str(tmp_path))
    m = _meas(case)
    monkeypatch.setenv("IRLCU_GRAPHS", "0")
    eager = gpu_osem(product, case, files, m)
    monkeypatch.setenv("IRLCU_GRAPHS", "1")
    graphed = gpu_osem(product, case, files, m)
    assert np.array_equal(eager, graphed)


def test_batch_rejects_hooks(product, tmp_path):
    case = W.plain64(seed=3500, n=24, nviews=8, subsets=2, iterations=1)
    files = case.write_tables(str(tmp_path))
    p, o, v = case.parms(), case.options(), case.views()
    atn, prj, rec = case.atn.copy(), np.ones((case.nviews, case.nz, case.n), np.float32), np.zeros_like(case.act)
    probs = (api.OsemProblem * 1)()
    q = probs[0]
    q.psIrlParms, q.psOptions = C.pointer(p), C.pointer(o)
    q.psViews = C.cast(v, C.POINTER(api.PrjView))
    q.pfAtnMap, q.pfPrjImage, q.pfReconImage = api.fptr(atn), api.fptr(prj), api.fptr(rec)
    hook = api.HOOK_CB(lambda d, ctx: None)
    product.OsemSetPostIterHook(hook, None)
    try:
        q.pchDrfTabFname = _libc.strdup(files["drf"].encode())
        assert product.IrlOsemBatch(1, probs) != 0
        assert b"hooks" in product.pchIrlErrorString()
    finally:
        product.OsemSetPostIterHook(None, None)


def test_drf_autotuner_keeps_the_faster_engine(product, tmp_path, monkeypatch):
    monkeypatch.delenv("IRLCU_DRF_ENGINE", raising=False)
    # a geometry no other test uses, so the decision is measured here
    case = W.full128(seed=3600, n=56, nviews=8, subsets=2, iterations=1, drf_max_offs=17, with_srf=False)
    files = case.write_tables(str(tmp_path))
    p, o, v = case.parms(), case.options(), case.views()
    atn, prj, rec = case.atn.copy(), np.ones((case.nviews, case.nz, case.n), np.float32), np.zeros_like(case.act)
    rc = product.IrlOsemBegin(C.byref(p), C.byref(o), v, dup(files["drf"]), None, api.ITER_CB(), None,
                              api.fptr(atn), api.fptr(prj), api.fptr(rec), None, None)
    assert rc == 0, product.pchIrlErrorString()
    try:
        grids = (C.c_int * 5)()
        ms = (C.c_float * 2)()
        assert product.irlcu_grids(grids) == 0
        assert product.irlcu_drf_tuning(ms) == 0
    finally:
        product.IrlOsemEnd(None)
    assert ms[0] > 0 and ms[1] > 0
    assert (grids[0] > 0) == (ms[1] < ms[0]), (list(grids), list(ms))


def test_shear_autotuner_keeps_the_faster_kernel(product, orc, tmp_path, monkeypatch):
    """The shape autotuner runs a context's first two whole iterations with
    the one- and then the two-slice shear kernel, timing every rotation
    launch per source kind, keeps the faster kernel of each kind from the
    third iteration on, and the reconstruction (trial iterations included)
    still matches the oracle."""
    monkeypatch.delenv("IRLCU_SHEAR_PAIR", raising=False)
    # a geometry no other test uses, so the decision is measured here
    case = W.full128(seed=3601, n=72, nz=40, nviews=8, subsets=2, iterations=4, drf_max_offs=5, with_srf=False)
    files = case.write_tables(str(tmp_path))
    pr = orc.Problem(case)
    meas = W.poisson_counts(pr.genprj(), 1e5, 3601)
    p, o, v = case.parms(), case.options(), case.views()
    atn, prj, rec = case.atn.copy(), meas.copy(), np.zeros_like(case.act)
    rc = product.IrlOsemBegin(C.byref(p), C.byref(o), v, dup(files["drf"]), None, api.ITER_CB(), None,
                              api.fptr(atn), api.fptr(prj), api.fptr(rec), None, None)
    assert rc == 0, product.pchIrlErrorString()
    try:
        assert product.IrlOsemIterate(case.iterations) == 0, product.pchIrlErrorString()
        ms, form = (C.c_float * 4)(), (C.c_int * 2)()
        assert product.irlcu_shear_tuning(ms, form) == 0
    finally:
        assert product.IrlOsemEnd(api.fptr(rec)) == 0
    assert all(m > 0 for m in ms), list(ms)
    for k in range(2):
        assert form[k] == (1 if ms[2 * k + 1] < ms[2 * k] else 0), (list(ms), list(form))
    want = orc.to_external(pr.osem(meas, case.iterations, case.nviews // case.subsets))
    assert float(np.linalg.norm(rec - want) / np.linalg.norm(want)) <= 1e-3
