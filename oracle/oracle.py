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


def ref_conv2d_fft(plane, psf):
    """The reference's FFT convolution branch as ConvolveDrfYpad runs it
    (convolve_ypad.c:63-94): PadSwap the PSF into a 2N x 2Nz grid, realft3d,
    conv2dPsfFFT."""
    lib = ref()
    plane = _arr(plane)
    psf = _arr(psf)
    ny, nx = plane.shape
    py, px = psf.shape
    grid = np.zeros((2 * ny, 2 * nx), np.float32)
    lib.PadSwap(api.fptr(psf), px, py, api.fptr(grid), 2 * nx, 2 * ny)
    lib.realft3d(api.fptr(grid), 2 * nx, 2 * ny, 1)
    out = np.zeros_like(plane)
    lib.conv2dPsfFFT(api.fptr(plane), nx, ny, api.fptr(grid), 2 * nx, 2 * ny, api.fptr(out))
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


# ------------------------------------------------------------ restatement

class OrProblem(C.Structure):
    """or_problem (oracle/src/irl_oracle.h)."""

    _fields_ = [
        ("n", C.c_int), ("nz", C.c_int), ("nviews", C.c_int), ("pix", C.c_float),
        ("fast_rotate", C.c_int),
        ("angle", _F), ("cfcr", _F), ("left", _F), ("right", _F), ("view_time", _F), ("sens", _F),
        ("ndist", C.c_int), ("drf_start", C.c_float), ("drf_spacing", C.c_float),
        ("mx", C.POINTER(C.c_int)), ("my", C.POINTER(C.c_int)), ("psf", _F), ("psf_off", C.POINTER(C.c_long)),
        ("bck_ndist", C.c_int), ("bck_start", C.c_float), ("bck_spacing", C.c_float),
        ("bck_mx", C.POINTER(C.c_int)), ("bck_my", C.POINTER(C.c_int)), ("bck_psf", _F),
        ("bck_off", C.POINTER(C.c_long)),
        ("pad_len", C.c_int), ("avg_len", C.c_int),
        ("esse_on", C.c_int), ("kx", C.c_int), ("ky", C.c_int), ("kz", C.c_int), ("collapse", C.c_int),
        ("nterms", C.c_int), ("mu0", C.c_float), ("mu_avg", C.c_float), ("esse_pix", C.c_float),
        ("cntr", C.c_float), ("krnl", _F), ("kmu", _F),
    ]


def _threads() -> int:
    """Host threads for the restatement's view loops: IRL_ORACLE_THREADS,
    else every core this process may run on."""
    env = os.environ.get("IRL_ORACLE_THREADS")
    if env:
        return max(1, int(env))
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def orc() -> C.CDLL:
    """The restatement library (oracle/src/irl_oracle.c)."""
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        lib = C.CDLL(ORACLE_SO)
        P = C.POINTER(OrProblem)
        lib.or_shears_rotate.argtypes = [_FL, _F, _F, _I, _I]
        lib.or_rot3dpar.argtypes = [_FL, _F, _F, _I, _I]
        lib.or_conv2d_ypad.argtypes = [_F, _I, _I, _F, _I, _I, _I, _I, _F]
        lib.or_esse_prepare.argtypes = [_F, _F, _I, _I, _I, _I, _I, _F, _F, _F]
        lib.or_esse_source.argtypes = [P, _F, _F, _F]
        lib.or_project.argtypes = [P, _I, _I, _F, _F, _FL, _F]
        lib.or_backproject.argtypes = [P, _I, _I, _F, _F, _F]
        lib.or_genprj.argtypes = [P, _I, _F, _F, _F, _FL, _F]
        lib.or_osem.argtypes = [P, _I, _I, _I, _I, _I, _F, _F, _F, _F]
        lib.or_osem.restype = _I
        lib.or_initial_estimate.argtypes = [_I, _I, _I, _F, _F]
        lib.or_set_threads.argtypes = [_I]
        lib.or_set_threads(_threads())
        for f in ("or_shears_rotate", "or_rot3dpar", "or_conv2d_ypad", "or_esse_prepare", "or_esse_source",
                  "or_project", "or_backproject", "or_genprj", "or_initial_estimate", "or_set_threads"):
            getattr(lib, f).restype = None
        _orc = lib
    return _orc


def to_internal(vol):
    """external [z][y][x] -> internal [y][z][x]"""
    return np.ascontiguousarray(np.transpose(vol, (1, 0, 2)), dtype=np.float32)


def to_external(vol):
    return np.ascontiguousarray(np.transpose(vol, (1, 0, 2)), dtype=np.float32)


class Problem:
    """An or_problem built from a libirl_b200.workloads.Case; keeps its
    arrays alive.  atn_scale is applied to the attenuation map."""

    def __init__(self, case, fast_rotate=True, with_drf=True, with_srf=None, pad_len=0, avg_len=0):
        self.case = case
        self.keep = []
        P = OrProblem()
        P.n, P.nz, P.nviews, P.pix = case.n, case.nz, case.nviews, case.pix
        P.fast_rotate = int(fast_rotate)
        nv = case.nviews

        def farr(a):
            a = np.ascontiguousarray(a, dtype=np.float32)
            self.keep.append(a)
            return api.fptr(a)

        P.angle = farr(case.angles)
        P.cfcr = farr(case.cfcr)
        P.left = farr(np.zeros(nv))
        P.right = farr(np.full(nv, case.n))
        P.view_time = farr(np.ones(nv))
        P.sens = farr(np.ones(nv))
        if with_drf and case.drf_psfs is not None:
            psfs = case.drf_psfs
            mx = np.array([(p.shape[1] + 1) // 2 for p in psfs], np.int32)
            my = np.array([(p.shape[0] + 1) // 2 for p in psfs], np.int32)
            off = np.cumsum([0] + [p.size for p in psfs[:-1]]).astype(np.int64)
            flat = np.concatenate([np.ascontiguousarray(p, np.float32).ravel() for p in psfs])
            self.keep += [mx, my, off, flat]
            P.ndist, P.drf_start, P.drf_spacing = len(psfs), case.drf_start, case.drf_spacing
            P.mx = mx.ctypes.data_as(C.POINTER(C.c_int))
            P.my = my.ctypes.data_as(C.POINTER(C.c_int))
            P.psf = api.fptr(flat)
            P.psf_off = off.ctypes.data_as(C.POINTER(C.c_long))
        P.pad_len, P.avg_len = pad_len, avg_len
        if with_srf is None:
            with_srf = case.krnl is not None
        self.srf = bool(with_srf and case.krnl is not None)
        if self.srf:
            k, kmu, mu0, kpix = case.krnl
            c = case.collapse
            kx = int(np.ceil(np.float32(2.0) * np.float32(case.n // c)))
            kz = int(np.ceil(np.float32(2.0) * np.float32(case.nz // c)))
            gk = np.zeros(kx * kx * kz, np.float32)
            gkm = np.zeros_like(gk)
            mavg = C.c_float()
            kk = np.ascontiguousarray(k, np.float32)
            km = np.ascontiguousarray(kmu, np.float32)
            orc().or_esse_prepare(api.fptr(kk), api.fptr(km), k.shape[2], k.shape[0], case.n, case.nz, c,
                                  api.fptr(gk), api.fptr(gkm), C.byref(mavg))
            self.keep += [gk, gkm]
            P.esse_on, P.kx, P.ky, P.kz, P.collapse, P.nterms = 1, kx, kx, kz, c, 2
            P.mu0, P.mu_avg, P.esse_pix, P.cntr = mu0, mavg.value, case.pix, 0.0
            P.krnl, P.kmu = api.fptr(gk), api.fptr(gkm)
        self.P = P
        self.atn = to_internal(case.atn * np.float32(case.atn_scale))
        self.act = to_internal(case.act)

    def model(self, drf=True, srf=None):
        m = 1
        if drf and self.P.ndist > 0:
            m |= 2
        if (self.srf if srf is None else srf):
            m |= 4
        return m

    def genprj(self, model=None, primary=1.0):
        nv, nz, n = self.case.nviews, self.case.nz, self.case.n
        out = np.zeros((nv, nz, n), np.float32)
        orc().or_genprj(C.byref(self.P), self.model() if model is None else model, api.fptr(self.act),
                        api.fptr(self.atn), None, primary, api.fptr(out))
        return out

    def osem(self, meas, iterations, per_subset, prj_model=None, bck_model=None, srf_iters=None, est=None):
        n, nz = self.case.n, self.case.nz
        meas = np.ascontiguousarray(meas, np.float32)
        if est is None:
            est = np.zeros((n, nz, n), np.float32)
            orc().or_initial_estimate(n, nz, self.case.nviews, api.fptr(meas), api.fptr(est))
        pm = self.model() if prj_model is None else prj_model
        bm = (pm & 3) if bck_model is None else bck_model
        si = iterations if srf_iters is None else srf_iters
        rc = orc().or_osem(C.byref(self.P), pm, bm, si, iterations, per_subset, api.fptr(meas),
                           api.fptr(self.atn), None, api.fptr(est))
        if rc:
            raise ValueError(f"or_osem failed ({rc})")
        return est
