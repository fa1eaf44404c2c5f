"""ctypes access to the CPU oracles.  TEST INFRASTRUCTURE ONLY.

Two libraries, both built by oracle/Makefile:
  _build/liboracle.so : the project's C restatement of libirl's hot path
                        (oracle/src/irl_oracle.c), always buildable from this
                        repository;
  _ref/libirl_ref.so  : the unmodified reference C sources linked with the
                        project-written MIP shim (built only where the
                        reference tree is present; travels as a prebuilt file).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this
module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from libirl_b200 import api

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libirl_ref.so")
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REFDIR = os.environ.get("IRL_REFERENCE_DIR", "/root/reference")

_F = api.FLOAT_P
_I = C.c_int
_FL = C.c_float


def build(ref: bool = True) -> None:
    """Compile the restatement and, when the reference tree exists, _ref."""
    subprocess.run(["make", "-s", "-C", HERE, "restate"], check=True)
    if ref and os.path.isdir(REFDIR):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFDIR={REFDIR}"], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_SO)


_ref = None
_orc = None


def ref() -> C.CDLL:
    """The reference library compiled here (libirl's own C)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        lib = api.declare_irl(C.CDLL(REF_SO))
        lib.vShearsRotate.argtypes = [_FL, _F, _F, _I, _I, _I]
        lib.vShearsRotate.restype = None
        lib.vInitFastRotate.argtypes = [_I]
        lib.vInitFastRotate.restype = None
        lib.rot3dpar.argtypes = [_FL, _F, _F, _I, _I, _I, _I]
        lib.rot3dpar.restype = None
        lib.conv2d_ypad.argtypes = [_F, _I, _I, _F, _I, _I, _I, _I, _F]
        lib.conv2d_ypad.restype = None
        lib.conv2dPsfFFT.argtypes = [_F, _I, _I, _F, _I, _I, _F]
        lib.conv2dPsfFFT.restype = None
        lib.PadSwap.argtypes = [_F, _I, _I, _F, _I, _I]
        lib.PadSwap.restype = None
        lib.realft3d.argtypes = [_F, _I, _I, _I]
        lib.realft3d.restype = None
        lib.realinvft3d.argtypes = [_F, _I, _I, _I]
        lib.realinvft3d.restype = None
        lib.multrealft3d.argtypes = [_I, _I, _I, _F, _F, _F]
        lib.multrealft3d.restype = None
        lib.pfSwapQuadrants.argtypes = [_F, _I, _I]
        lib.pfSwapQuadrants.restype = _F
        lib.InitPrj.argtypes = [_I, _I, _I, _I]
        lib.InitPrj.restype = None
        lib.FreePrj.argtypes = []
        lib.FreePrj.restype = None
        _ref = lib
    return _ref


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def ref_shears_rotate(angle, vol, pb_flag=0):
    """vShearsRotate on an internal-layout volume [y][z][x] (N x Nz x N)."""
    lib = ref()
    n, nz, n2 = vol.shape
    assert n == n2
    src = _arr(vol)
    out = np.zeros_like(src)
    lib.vInitFastRotate(n)
    lib.vShearsRotate(angle, api.fptr(src), api.fptr(out), pb_flag, nz, n)
    return out


def ref_rot3dpar(angle, vol, pb_flag=0):
    lib = ref()
    n, nz, _ = vol.shape
    src = _arr(vol)
    out = np.zeros_like(src)
    lib.rot3dpar(angle, api.fptr(src), api.fptr(out), pb_flag, nz, n, n)
    return out


def ref_conv2d_ypad(plane, psf, pad=0, avg=0):
    lib = ref()
    plane = _arr(plane)
    psf = _arr(psf)
    ny, nx = plane.shape
    py, px = psf.shape
    out = np.zeros_like(plane)
    lib.conv2d_ypad(api.fptr(plane), nx, ny, api.fptr(psf), (px - 1) // 2, (py - 1) // 2,
                    pad, avg, api.fptr(out))
    return out
