"""ctypes mirror of the libirl C API (include/irl.h, include/osemhooks.h).

The struct layouts follow libirl's irl.h:39-143 and osemhooks.h:18-33 field
for field, so the same Python objects can be handed to libirl_b200.so or to
any library exporting the libirl ABI.  This module holds types and argument
marshalling only; it loads nothing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

MODEL_ATN, MODEL_DRF, MODEL_SRF = 1, 2, 4


class IrlParms(C.Structure):
    """libirl IrlParms_t (irl.h:39-79)."""

    _fields_ = [
        ("NumPixels", C.c_int),
        ("NumSlices", C.c_int),
        ("NumViews", C.c_int),
        ("BinWidth", C.c_float),
        ("fAtnScaleFac", C.c_float),
        ("iNumSrfIterations", C.c_int),
        ("fScatEstFac", C.c_float),
        ("NumAngPerSubset", C.c_int),
        ("NumIterations", C.c_int),
        ("pchNormImageBase", C.c_char_p),
        ("SrfCollapseFac", C.c_int),
        ("fHoleDiam", C.c_float),
        ("fHoleLen", C.c_float),
        ("fBackToDet", C.c_float),
        ("fIntrinsicFWHM", C.c_float),
    ]


class Options(C.Structure):
    """libirl Options_t (irl.h:81-124)."""

    _fields_ = [
        ("bModelDrf", C.c_int),
        ("bReconIsInitEst", C.c_int),
        ("bUseGrfInBck", C.c_int),
        ("bFFTConvolve", C.c_int),
        ("bUseContourSupport", C.c_int),
        ("fAtnMapThresh", C.c_float),
        ("iMsgLevel", C.c_int),
        ("iAxialPadLength", C.c_int),
        ("iAxialAvgLength", C.c_int),
    ]


class PrjView(C.Structure):
    """libirl PrjView_t (irl.h:127-143)."""

    _fields_ = [
        ("Angle", C.c_float),
        ("Left", C.c_float),
        ("Right", C.c_float),
        ("CFCR", C.c_float),
    ]


class OsemData(C.Structure):
    """libirl sOsemData (osemhooks.h:18-27)."""

    _fields_ = [
        ("iIterationIdx", C.c_int),
        ("iSubsetIdx", C.c_int),
        ("iAngleIdx", C.c_int),
        ("pfEst", C.POINTER(C.c_float)),
        ("pfSct", C.POINTER(C.c_float)),
        ("pfNorm", C.POINTER(C.c_float)),
        ("pfUpdate", C.POINTER(C.c_float)),
    ]


class AdvOptions(C.Structure):
    """libirl sAdvOptions (osemhooks.h:29-33)."""

    _fields_ = [("bFastRotate", C.c_int), ("iStartIteration", C.c_int)]


class Drf(C.Structure):
    """libirl Drf_t (drftabio.h:7-12)."""

    _fields_ = [
        ("MaxOffsX", C.c_int),
        ("MaxOffsY", C.c_int),
        ("bFFTdone", C.c_int),
        ("Psf", C.POINTER(C.c_float)),
    ]


class DrfTab(C.Structure):
    """libirl DrfTab_t (drftabio.h:14-28)."""


DrfTab._fields_ = [
    ("iNumDistances", C.c_int),
    ("fStartDistance", C.c_float),
    ("fDrfSpacing", C.c_float),
    ("fPixSize", C.c_float),
    ("bIncKrnl", C.c_int),
    ("bDrfFromFile", C.c_int),
    ("psBckDrfTab", C.POINTER(DrfTab)),
    ("fGap", C.c_float),
    ("fHoleDiam", C.c_float),
    ("fColThick", C.c_float),
    ("fIntrinsicFWHM", C.c_float),
    ("fMaxFracErr", C.c_float),
    ("psDrfs", C.POINTER(Drf)),
    ("bFFTconvolve", C.c_int),
]

ITER_CB = C.CFUNCTYPE(None, C.c_int, C.POINTER(C.c_float))
HOOK_CB = C.CFUNCTYPE(None, C.POINTER(OsemData), C.c_void_p)

FLOAT_P = C.POINTER(C.c_float)


def fptr(a: np.ndarray | None):
    """float* of a C-contiguous float32 array (NULL for None)."""
    if a is None:
        return None
    if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float32 array")
    return a.ctypes.data_as(FLOAT_P)


def bstr(s):
    return None if s is None else (s.encode() if isinstance(s, str) else s)


class OsemProblem(C.Structure):
    """IrlOsemProblem_t (include/irl_b200.h): one reconstruction of a batch."""
    _fields_ = [
        ("psIrlParms", C.POINTER(IrlParms)),
        ("psOptions", C.POINTER(Options)),
        ("psViews", C.POINTER(PrjView)),
        ("pchDrfTabFname", C.c_void_p),     # malloc'd (the library frees it)
        ("pchScatKrnlFname", C.c_void_p),
        ("pfScatterEstimate", FLOAT_P),
        ("pfAtnMap", FLOAT_P),
        ("pfPrjImage", FLOAT_P),
        ("pfReconImage", FLOAT_P),
        ("iStatus", C.c_int),
    ]


def declare_irl(lib: C.CDLL) -> C.CDLL:
    """Declare the libirl entry points (irl.h, osemhooks.h) on a CDLL."""
    lib.IrlOsem.restype = C.c_int
    lib.IrlOsem.argtypes = [
        C.POINTER(IrlParms), C.POINTER(Options), C.POINTER(PrjView),
        C.c_char_p, C.c_char_p, ITER_CB, FLOAT_P, FLOAT_P, FLOAT_P, FLOAT_P,
        C.c_char_p, C.c_char_p,
    ]
    lib.IrlGenprj.restype = C.c_int
    lib.IrlGenprj.argtypes = [
        C.POINTER(IrlParms), C.POINTER(Options), C.POINTER(PrjView),
        C.c_char_p, C.c_char_p, C.c_void_p, FLOAT_P, FLOAT_P, FLOAT_P, FLOAT_P,
        C.c_float, C.c_char_p, C.c_char_p,
    ]
    lib.ComputeOrbit.restype = C.c_int
    lib.ComputeOrbit.argtypes = [
        FLOAT_P, C.POINTER(IrlParms), C.c_float, FLOAT_P, C.c_float, C.c_int,
        C.POINTER(PrjView),
    ]
    lib.pchIrlErrorString.restype = C.c_char_p
    lib.pchIrlErrorString.argtypes = []
    lib.OsemSetAdvOptions.restype = C.c_int
    lib.OsemSetAdvOptions.argtypes = [C.POINTER(AdvOptions)]
    for name in ("PrevIter", "PostIter", "PrevSubset", "PostSubset", "PrevAngle", "PostAngle"):
        fn = getattr(lib, f"OsemSet{name}Hook")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_void_p]
    lib.iSetupExtraPrjViewData.restype = C.c_int
    lib.iSetupExtraPrjViewData.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    lib.iSetupDetectors.restype = C.c_int
    lib.iSetupDetectors.argtypes = [C.c_int, C.c_void_p]
    lib.pvStoreDetectorData.restype = C.c_void_p
    lib.pvStoreDetectorData.argtypes = [
        C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
        C.c_char_p,
    ]
    lib.sReadDrfTab.restype = DrfTab
    lib.sReadDrfTab.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p)]
    lib.vWriteDrfTab.restype = None
    lib.vWriteDrfTab.argtypes = [C.POINTER(DrfTab), C.c_char_p, C.c_char_p, C.c_char_p]
    return lib


def make_views(angles, cfcr, left=0.0, right=None, n=None):
    arr = (PrjView * len(angles))()
    for i, (a, r) in enumerate(zip(angles, cfcr)):
        arr[i].Angle = float(a)
        arr[i].CFCR = float(r)
        arr[i].Left = float(left)
        arr[i].Right = float(right if right is not None else n)
    return arr
