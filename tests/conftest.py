"""Shared fixtures for the libirl_b200 tests.

CPU tests (no marker) check the oracle against the golden fixtures and the
compiled reference, the host-side logic, the file formats and the C ABI.
GPU tests (@pytest.mark.gpu) compare the CUDA path, called through
libirl_b200.so's C entry points, with the CPU oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


_libc = C.CDLL(None)
_libc.strdup.restype = C.c_void_p
_libc.strdup.argtypes = [C.c_char_p]


def dup(s):
    """malloc'd copy of a file name: libirl frees the DRF file name it is given."""
    return C.cast(_libc.strdup(s.encode()), C.c_char_p) if s else None


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


@pytest.fixture(scope="session")
def product():
    import libirl_b200 as L
    L.build()
    return L.load()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.build(ref=True)
    return O


def golden_case(name):
    """Rebuild a workloads.Case from a golden fixture."""
    from libirl_b200 import workloads as W
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    shapes = d["psf_shapes"]
    flat = d["psf_flat"]
    psfs, off = [], 0
    for sh in shapes:
        cnt = int(sh[0] * sh[1])
        psfs.append(flat[off:off + cnt].reshape(sh).astype(np.float32))
        off += cnt
    act = d["act"]
    nz, n = act.shape[0], act.shape[1]
    nv = len(d["angles"])
    krnl = None
    collapse = 1
    if "krnl" in d:
        krnl = (d["krnl"], d["krnl_mu"], float(d["mu0"]), float(d["krnl_pix"]))
        collapse = int(d["collapse"])
    case = W.Case(name, n, nz, float(d["pix"]), nv, int(d["subsets"]), int(d["iterations"]), 2e4,
                  act, d["atn"], d["angles"], d["cfcr"], float(d["atn_scale"]), psfs, float(d["drf_start"]),
                  float(d["drf_spacing"]), krnl, collapse, int(d["iterations"]) if krnl is not None else 0)
    return case, d
