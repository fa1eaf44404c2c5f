"""The C ABI of libirl_b200.so: every function declared in include/*.h is
exported, the library loads without a GPU, and there is no CPU fallback."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, dup
from libirl_b200 import api, workloads as W

DECL = re.compile(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith("#"))
        txt = txt.replace('extern "C" {', "")
        txt = re.sub(r"typedef\s+struct[^{]*\{.*?\}[^;]*;", "", txt, flags=re.S)
        for stmt in txt.split(";"):
            stmt = " ".join(stmt.replace("}", " ").split())
            m = re.match(r"^(?:[A-Za-z_]\w*[\s\*]+)+([A-Za-z_]\w*)\s*\(", stmt)
            if m and not stmt.startswith("typedef"):
                names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(product):
    names = declared_functions()
    # the public libirl API and the device ABI must both be there
    for must in ("IrlOsem", "IrlGenprj", "ComputeOrbit", "pchIrlErrorString", "OsemSetAdvOptions",
                 "OsemSetPrevIterHook", "iSetupExtraPrjViewData", "iSetupDetectors", "pvStoreDetectorData",
                 "vWriteDrfTab", "sReadDrfTab", "vWriteKrnlFile", "psReadKrnlFile", "psFreeKrnlData",
                 "irlcu_init", "irlcu_osem_subset", "irlcu_project"):
        assert must in names, must
    missing = [n for n in sorted(names) if not hasattr(product, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_no_cpu_fallback_without_a_device(product):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    case = W.plain64(n=16, nviews=4, subsets=2, iterations=1)
    files = case.write_tables("/tmp/irl_abi_nodev")
    p, o, v = case.parms(), case.options(), case.views()
    atn = case.atn.copy()
    meas = np.ones((4, 16, 16), np.float32)
    rec = np.zeros_like(case.act)
    rc = product.IrlOsem(C.byref(p), C.byref(o), v, dup(files["drf"]), None, api.ITER_CB(lambda i, q: None), None,
                         api.fptr(atn), api.fptr(meas), api.fptr(rec), None, None)
    assert rc != 0
    assert b"CUDA" in product.pchIrlErrorString()


def test_device_copies_and_memsets_are_stream_ordered():
    """Every copy and memset of the CUDA sources is issued on a stream
    (the *Async forms). A context's kernels run on a non-blocking stream,
    which legacy-stream copies and memsets do not order against. A batch of
    reconstructions, set up while the previous one still ran, raced on
    exactly that."""
    legacy = re.compile(r"\bcudaMem(?:cpy|set|cpy2D|cpy3D|cpyToSymbol|cpyFromSymbol)\s*\(")
    bad = []
    for f in sorted(glob.glob(os.path.join(ROOT, "libirl_b200", "csrc", "**", "*.cu*"), recursive=True)):
        for i, line in enumerate(open(f), 1):
            if legacy.search(line):
                bad.append(f"{os.path.relpath(f, ROOT)}:{i}: {line.strip()}")
    assert not bad, "\n".join(bad)
