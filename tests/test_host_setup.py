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
