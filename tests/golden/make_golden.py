"""Generates tests/golden/*.npz from the reference library compiled here.

The reference C sources (libirl) are compiled unmodified with the
project-written MIP shim into oracle/_ref/libirl_ref.so (make -C oracle
ref).  This script runs its own entry points on small seeded inputs and
stores inputs and outputs, so that the CPU restatement in oracle/ can be
pinned against the reference's own results on machines without the
reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from libirl_b200 import api, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def _dup(libc, s):
    return C.cast(libc.strdup(s.encode()), C.c_char_p) if s else None


def main():
    O.build(ref=True)
    ref = O.ref()
    libc = C.CDLL(None)
    libc.strdup.restype = C.c_void_p
    libc.strdup.argtypes = [C.c_char_p]
    rng = np.random.default_rng(424242)

    # rotations: vShearsRotate and rot3dpar on a 16 x 3 x 16 volume
    vol = rng.random((16, 3, 16), dtype=np.float32)
    angles = np.array([-2.9, -0.7, 0.0, 0.3, 1.2, 2.1, 3.9, 5.5], np.float32)
    shears = np.stack([O.ref_shears_rotate(float(a), vol) for a in angles])
    bilin = np.stack([O.ref_rot3dpar(float(a), vol) for a in angles])
    np.savez_compressed(os.path.join(HERE, "rotate.npz"), vol=vol, angles=angles, shears=shears, rot3dpar=bilin)

    # conv2d_ypad with and without axial padding
    plane = rng.random((12, 10), dtype=np.float32)
    psf = rng.random((7, 5), dtype=np.float32)
    cases = [(0, 0), (2, 1), (3, 4)]
    outs = np.stack([O.ref_conv2d_ypad(plane, psf, p, a) for p, a in cases])
    np.savez_compressed(os.path.join(HERE, "conv2d_ypad.npz"), plane=plane, psf=psf, pads=np.array(cases), out=outs)

    # IrlGenprj / IrlOsem, plain (atn + Gaussian DRF) and full physics (ESSE c=2)
    tmp = tempfile.mkdtemp()
    for name, case in [("plain16", W.plain64(seed=1001, n=16, nviews=8, subsets=2, iterations=2)),
                       ("srf16", W.full128(seed=2001, n=16, nviews=8, subsets=2, iterations=2, drf_max_offs=4))]:
        files = case.write_tables(os.path.join(tmp, name))
        p, o, v = case.parms(), case.options(), case.views()
        act, atn = case.act.copy(), case.atn.copy()
        prj = np.zeros((case.nviews, case.nz, case.n), np.float32)
        rc = ref.IrlGenprj(C.byref(p), C.byref(o), v, _dup(libc, files["drf"]), _dup(libc, files.get("krnl")),
                           None, None, api.fptr(act), api.fptr(atn), api.fptr(prj), 1.0, None, None)
        assert rc == 0, ref.pchIrlErrorString()
        meas = W.poisson_counts(prj, 2e4, 7)
        p, o, v = case.parms(), case.options(), case.views()
        atn = case.atn.copy()
        rec = np.zeros_like(case.act)
        m = meas.copy()
        rc = ref.IrlOsem(C.byref(p), C.byref(o), v, _dup(libc, files["drf"]), _dup(libc, files.get("krnl")),
                         api.ITER_CB(lambda i, q: None), None, api.fptr(atn), api.fptr(m), api.fptr(rec), None, None)
        assert rc == 0, ref.pchIrlErrorString()
        extra = {}
        if case.krnl is not None:
            extra = dict(krnl=case.krnl[0], krnl_mu=case.krnl[1], mu0=case.krnl[2], krnl_pix=case.krnl[3],
                         collapse=case.collapse)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), act=case.act, atn=case.atn, angles=case.angles, cfcr=case.cfcr,
            pix=case.pix, atn_scale=case.atn_scale, subsets=case.subsets, iterations=case.iterations,
            drf_start=case.drf_start, drf_spacing=case.drf_spacing,
            psf_flat=np.concatenate([q.ravel() for q in case.drf_psfs]),
            psf_shapes=np.array([q.shape for q in case.drf_psfs], np.int32),
            prj=prj, meas=meas, recon=rec, **extra)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
