"""irlcu_rotate_volume_noalloc: the three-shear rotation whose tables and
intermediate live in a static device array, called through the C ABI.

Checked against irlcu_rotate_volume (the allocating entry point) on two
calls in a row, for a slice that irlcu_rotate_volume rotates in shared
memory (n = 128) and one it rotates through its lazily allocated global
intermediate (n = 200).  The file is named to be collected last, so it runs
both after the other GPU tests and alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IRLCU_EARG = 102  # include/irlcu.h


def _ctx(product, n, nz):
    import libirl_b200 as L
    g = L.IrlcuGeom(n, nz, 1, 1, 1)
    L.check(product, product.irlcu_init(C.byref(g)))


@pytest.mark.parametrize("n,nz", [(128, 6), (200, 2)])
def test_noalloc_matches_rotate_volume(product, n, nz):
    import torch
    import libirl_b200 as L
    _ctx(product, n, nz)
    try:
        rng = np.random.default_rng(9000 + n)
        vol = torch.from_numpy(rng.random((n, nz, n), dtype=np.float32)).cuda()
        want = torch.empty_like(vol)
        got = torch.empty_like(vol)
        torch.cuda.synchronize()
        free = []
        # two calls in a row, each against the allocating entry point
        fp = lambda t: C.cast(t.data_ptr(), L.api.FLOAT_P)  # noqa: E731
        for angle in rng.uniform(-7, 7, 2).astype(np.float32):
            L.check(product, product.irlcu_rotate_volume(float(angle), fp(vol), fp(want), 0, 1))
            got.fill_(-1.0)
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
            L.check(product, product.irlcu_rotate_volume_noalloc(float(angle), vol.data_ptr(), got.data_ptr(), n, nz))
            free.append(torch.cuda.mem_get_info()[0])
            diff = int((got != want).sum())
            assert diff == 0, f"angle {angle}: {diff} voxels differ from irlcu_rotate_volume"
        # no device memory taken by either call
        assert free[1] == free[0] and free[3] == free[2], free
    finally:
        product.irlcu_shutdown()


def test_noalloc_rejects_oversize(product):
    import torch
    import libirl_b200 as L
    n = nz = 256  # nz*n*mdim > the static intermediate for every angle
    _ctx(product, 16, 1)
    try:
        src = torch.zeros((n, nz, n), dtype=torch.float32, device="cuda")
        dst = torch.zeros_like(src)
        torch.cuda.synchronize()
        rc = product.irlcu_rotate_volume_noalloc(0.3, src.data_ptr(), dst.data_ptr(), n, nz)
        assert rc == IRLCU_EARG
        assert b"static scratch" in product.irlcu_error_string()
        assert float(dst.abs().sum()) == 0.0
        rc = product.irlcu_rotate_volume_noalloc(0.3, src.data_ptr(), dst.data_ptr(), 2048, 1)
        assert rc == IRLCU_EARG
    finally:
        product.irlcu_shutdown()
