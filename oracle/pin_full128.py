"""Pins the oracle's restatement against the compiled reference on the
full-physics 128^3 case (TEST INFRASTRUCTURE ONLY).

Runs libirl's own IrlOsem (oracle/_ref, the unmodified reference C with the
MIP shim) on the seeded 128^3 / 120-view / 8 x 10 case with attenuation,
the 33x33 DRF and ESSE in every iteration, and the restatement (threaded
over the views of each subset) on the same inputs, and prints the relative
L2 differences of the noise-free projections and of the reconstruction.
The reference is single-threaded: about 40 minutes on one core.

    python -m oracle.pin_full128 [--iterations 10] [--out summary.json]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from libirl_b200 import api, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

_libc = C.CDLL(None)
_libc.strdup.restype = C.c_void_p
_libc.strdup.argtypes = [C.c_char_p]


def _dup(s):
    return C.cast(_libc.strdup(s.encode()), C.c_char_p)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=10)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    case = W.full128(seed=2000, iterations=a.iterations)
    files = case.write_tables(tempfile.mkdtemp(prefix="irlpin_"))
    ref = O.ref()
    pr = O.Problem(case)
    t = time.time()
    clean = pr.genprj()
    t_or_prj = time.time() - t
    p, o, v = case.parms(), case.options(), case.views()
    act, atn = case.act.copy(), case.atn.copy()
    prj = np.zeros_like(clean)
    t = time.time()
    rc = ref.IrlGenprj(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]), None, None,
                       api.fptr(act), api.fptr(atn), api.fptr(prj), 1.0, None, None)
    t_ref_prj = time.time() - t
    assert rc == 0, ref.pchIrlErrorString()
    view_err = [_rel(prj[i], clean[i]) for i in range(case.nviews)]
    meas = W.poisson_counts(clean, case.counts, 2000)
    t = time.time()
    want = O.to_external(pr.osem(meas, case.iterations, case.nviews // case.subsets))
    t_or_osem = time.time() - t
    p, o, v = case.parms(), case.options(), case.views()
    atn, m, rec = case.atn.copy(), meas.copy(), np.zeros_like(case.act)
    t = time.time()
    rc = ref.IrlOsem(C.byref(p), C.byref(o), v, _dup(files["drf"]), _dup(files["krnl"]),
                     api.ITER_CB(lambda i, q: None), None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
    t_ref_osem = time.time() - t
    assert rc == 0, ref.pchIrlErrorString()
    out = {"case": "full128 seed 2000: 128^3, 120 views, 8 subsets x %d iterations, DRF 33x33, ESSE c=2 in every "
                   "iteration" % case.iterations,
           "views_max_rel_l2": max(view_err), "views_mean_rel_l2": float(np.mean(view_err)),
           "image_rel_l2": _rel(want, rec),
           "seconds": {"oracle_genprj": round(t_or_prj, 1), "reference_genprj": round(t_ref_prj, 1),
                       "oracle_osem": round(t_or_osem, 1), "reference_osem": round(t_ref_osem, 1)},
           "oracle_threads": O._threads()}
    print(json.dumps(out))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
