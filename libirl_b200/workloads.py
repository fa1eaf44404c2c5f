"""Seeded synthetic SPECT workloads with the shapes of libirl's use cases.

There is no public dataset for this path; every case is generated from a
seed (case k, problem j -> seed 1000*k + j, numpy default_rng):

  plain64  : 64^3 volume, 0.4 cm voxels, 6 random ellipsoids on background
             0.5, water-ellipsoid attenuation (0.15/cm), 60 views on a 20 cm
             circular orbit, Gaussian DRF with FWHM = 0.3 + 0.03 d cm,
             no scatter, 1e6 counts, 4 subsets x 5 iterations.
  full128  : 128^3 volume, 0.3125 cm voxels, 12 ellipsoids (lesions 2-20
             voxels across), body ellipse 0.15/cm with lungs 0.04/cm and a
             spine cylinder 0.25/cm, 120 views on an elliptical 22 x 18 cm
             orbit, 33x33-tap DRF at every depth, ESSE scatter with a
             two-exponential kernel, collapse factor 2, 5e6 counts,
             8 subsets x 10 iterations.

DRFT and KRNL tables are written in libirl's binary formats
(drftabio.c:26-48, krnlio.c:31-63) by the writers below.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field

import numpy as np

from . import api


# ----------------------------------------------------------------- formats

def write_drft(path, psfs, pix, spacing, start, title="synthetic", colname="synthetic", inc_krnl=0):
    """Write a DRFT file.  psfs: list of 2D float arrays of odd shape
    (2*MaxOffsY-1, 2*MaxOffsX-1), x fastest."""
    with open(path, "wb") as f:
        f.write(b"DRFT")
        f.write(struct.pack("=i", 1))
        f.write(title.encode()[:79].ljust(80, b"\0"))
        f.write(colname.encode()[:19].ljust(20, b"\0"))
        f.write(struct.pack("=fffii", pix, spacing, start, len(psfs), inc_krnl))
        for p in psfs:
            p = np.ascontiguousarray(p, dtype=np.float32)
            ny, nx = p.shape
            f.write(struct.pack("=ii", (nx + 1) // 2, (ny + 1) // 2))
            f.write(p.tobytes())


def read_drft(path):
    """Parse a DRFT file (native order) into a dict; used for checks."""
    with open(path, "rb") as f:
        b = f.read()
    assert b[:4] == b"DRFT"
    (ver,) = struct.unpack_from("=i", b, 4)
    assert ver == 1
    off = 8 + 80 + 20
    pix, spacing, start, n, inc = struct.unpack_from("=fffii", b, off)
    off += 20
    psfs = []
    for _ in range(n):
        mx, my = struct.unpack_from("=ii", b, off)
        off += 8
        cnt = (2 * mx - 1) * (2 * my - 1)
        psfs.append(np.frombuffer(b, np.float32, cnt, off).reshape(2 * my - 1, 2 * mx - 1).copy())
        off += 4 * cnt
    return dict(pix=pix, spacing=spacing, start=start, psfs=psfs, inc=inc)


def write_krnl(path, krnl, krnl_mu, mu0, pix, prifac=1.0, scatfac=1.0, cntrpixfac=0.0,
               title="synthetic two-exponential ESSE kernel", isotope="Tc99m",
               high=154.0, low=126.0):
    """Write a KRNL file.  krnl, krnl_mu: float arrays [NumDists][NumXYoffs][NumXYoffs]."""
    krnl = np.ascontiguousarray(krnl, dtype=np.float32)
    krnl_mu = np.ascontiguousarray(krnl_mu, dtype=np.float32)
    nd, ny, nx = krnl.shape
    assert nx == ny and krnl_mu.shape == krnl.shape
    with open(path, "wb") as f:
        f.write(b"KRNL")
        f.write(struct.pack("=i", 1))
        f.write(title.encode()[:79].ljust(80, b"\0"))
        f.write(isotope.encode()[:19].ljust(20, b"\0"))
        f.write(struct.pack("=fffffff", mu0, high, low, pix, prifac, scatfac, cntrpixfac))
        f.write(struct.pack("=ii", nx, nd))
        f.write(krnl.tobytes())
        f.write(krnl_mu.tobytes())


# ------------------------------------------------------------------ tables

def gaussian_drf_table(pix, start, spacing, count, fwhm0=0.3, slope=0.03):
    """Gaussian PSFs, FWHM = fwhm0 + slope*d cm, MaxOffs = ceil(3.5 sigma)+1."""
    psfs = []
    for i in range(count):
        d = start + i * spacing
        sig = max(fwhm0 + slope * d, 1e-3) / (2.0 * np.sqrt(2.0 * np.log(2.0))) / pix
        m = int(np.ceil(3.5 * sig)) + 1
        o = np.arange(-(m - 1), m, dtype=np.float64)
        g = np.exp(-(o[None, :] ** 2 + o[:, None] ** 2) / (2 * sig * sig))
        psfs.append((g / g.sum()).astype(np.float32))
    return psfs


def tailed_drf_table(pix, start, spacing, count, max_offs=17, fwhm0=0.25, slope=0.025,
                     tail=0.03, tail_len=1.2):
    """Radially symmetric, non-separable PSFs on a fixed (2*max_offs-1)^2 grid:
    a Gaussian core (FWHM = fwhm0 + slope*d cm) plus an exponential tail that
    grows with distance, normalised to unit sum."""
    psfs = []
    o = np.arange(-(max_offs - 1), max_offs, dtype=np.float64) * pix
    r = np.sqrt(o[None, :] ** 2 + o[:, None] ** 2)
    for i in range(count):
        d = max(start + i * spacing, 0.0)
        sig = (fwhm0 + slope * d) / (2.0 * np.sqrt(2.0 * np.log(2.0)))
        core = np.exp(-(r ** 2) / (2 * sig * sig))
        lam = tail_len * (1.0 + d / 20.0)
        t = np.exp(-r / lam)
        p = core / core.sum() + tail * t / t.sum()
        psfs.append((p / p.sum()).astype(np.float32))
    return psfs


def esse_kernel(noffs, ndists, pix, mu0=0.15, amps=(0.25, 0.08), lens=(0.9, 4.0)):
    """Two-exponential ESSE kernel in libirl's one-quadrant layout
    [depth][y offset][x offset]; the depth centre is ndists/2-1
    (krnlprj3d.c:43-62).  The mu kernel varies with offset so that the
    first-order Taylor term of ESSE is exercised."""
    iz = np.arange(ndists, dtype=np.float64) - (ndists // 2 - 1)
    o = np.arange(noffs, dtype=np.float64)
    dd, yy, xx = np.meshgrid(iz, o, o, indexing="ij")
    r = np.sqrt(xx ** 2 + yy ** 2 + dd ** 2) * pix
    k = sum(a * np.exp(-r / l) for a, l in zip(amps, lens))
    # make the full (mirrored) kernel sum to ~0.35 scatter per primary
    w = np.where(xx > 0, 2.0, 1.0) * np.where(yy > 0, 2.0, 1.0)
    k *= 0.35 / float((k * w).sum())
    kmu = mu0 * (0.82 + 0.3 * np.exp(-r / 3.0) + 0.04 * np.tanh(dd / 8.0))
    return k.astype(np.float32), kmu.astype(np.float32)


# ----------------------------------------------------------------- phantoms

def _grid(n, nz, pix):
    c = (n - 1) / 2.0
    cz = (nz - 1) / 2.0
    x = (np.arange(n) - c) * pix
    z = (np.arange(nz) - cz) * pix
    Z, Y, X = np.meshgrid(z, x, x, indexing="ij")  # external [z][y][x]
    return X, Y, Z


def _ellipsoid(X, Y, Z, c, ax, rot=0.0):
    cr, sr = np.cos(rot), np.sin(rot)
    dx, dy, dz = X - c[0], Y - c[1], Z - c[2]
    u = cr * dx + sr * dy
    v = -sr * dx + cr * dy
    return (u / ax[0]) ** 2 + (v / ax[1]) ** 2 + (dz / ax[2]) ** 2 <= 1.0


@dataclass
class Case:
    name: str
    n: int
    nz: int
    pix: float
    nviews: int
    subsets: int
    iterations: int
    counts: float
    act: np.ndarray          # external layout [z][y][x], float32
    atn: np.ndarray          # per cm, external layout
    angles: np.ndarray
    cfcr: np.ndarray
    atn_scale: float         # cm -> per pixel
    drf_psfs: list | None = None
    drf_start: float = 0.0
    drf_spacing: float = 0.0
    krnl: tuple | None = None   # (krnl, krnl_mu, mu0, pix)
    collapse: int = 1
    srf_iters: int = 0
    files: dict = field(default_factory=dict)

    def views(self):
        return api.make_views(self.angles, self.cfcr, 0.0, float(self.n))

    def parms(self):
        p = api.IrlParms()
        p.NumPixels, p.NumSlices, p.NumViews = self.n, self.nz, self.nviews
        p.BinWidth = self.pix
        p.fAtnScaleFac = self.atn_scale
        p.iNumSrfIterations = self.srf_iters
        p.fScatEstFac = 1.0
        p.NumAngPerSubset = self.nviews // self.subsets
        p.NumIterations = self.iterations
        p.pchNormImageBase = None
        p.SrfCollapseFac = self.collapse
        p.fHoleDiam, p.fHoleLen, p.fBackToDet, p.fIntrinsicFWHM = 0.111, 2.405, 0.64, 0.38
        return p

    def options(self, model_drf=None):
        o = api.Options()
        o.bModelDrf = int(self.drf_psfs is not None if model_drf is None else model_drf)
        o.bReconIsInitEst = 0
        o.bUseGrfInBck = 0
        o.bFFTConvolve = 0
        o.bUseContourSupport = 0
        o.fAtnMapThresh = 0.0
        o.iMsgLevel = 1
        o.iAxialPadLength = 0
        o.iAxialAvgLength = 0
        return o

    def write_tables(self, directory):
        """Write the DRFT/KRNL files of this case into directory."""
        os.makedirs(directory, exist_ok=True)
        if self.drf_psfs is not None:
            p = os.path.join(directory, f"{self.name}.drft")
            write_drft(p, self.drf_psfs, self.pix, self.drf_spacing, self.drf_start)
            self.files["drf"] = p
        if self.krnl is not None:
            k, kmu, mu0, kpix = self.krnl
            p = os.path.join(directory, f"{self.name}.krnl")
            write_krnl(p, k, kmu, mu0, kpix)
            self.files["krnl"] = p
        return self.files


def plain64(seed=1000, n=64, nviews=60, subsets=4, iterations=5):
    """The CPU-runnable plain OSEM case (64^3, no scatter)."""
    rng = np.random.default_rng(seed)
    pix = 0.4 * 64 / n
    nz = n
    X, Y, Z = _grid(n, nz, pix)
    fov = n * pix
    act = np.zeros(X.shape, np.float32)
    cyl = X ** 2 + Y ** 2 <= (fov / 2) ** 2
    act[cyl] = 0.5
    for _ in range(6):
        rr = 0.3 * fov * np.sqrt(rng.uniform())
        th = rng.uniform(0, 2 * np.pi)
        c = (rr * np.cos(th), rr * np.sin(th), rng.uniform(-0.3, 0.3) * fov)
        ax = rng.uniform(1.0, 5.0, 3) * (fov / 25.6)
        act[_ellipsoid(X, Y, Z, c, ax, rng.uniform(0, np.pi))] = rng.uniform(1, 10)
    atn = np.zeros(X.shape, np.float32)
    atn[_ellipsoid(X, Y, Z, (0, 0, 0), (0.42 * fov, 0.32 * fov, 0.45 * fov))] = 0.15
    angles = 2 * np.pi * np.arange(nviews) / nviews
    cfcr = np.full(nviews, 20.0 * fov / 25.6)
    r0 = float(cfcr[0])
    start = r0 - fov / 2
    count = int(round(fov / pix)) + 1
    psfs = gaussian_drf_table(pix, start, pix, count)
    return Case("plain64", n, nz, pix, nviews, subsets, iterations, 1e6, act, atn,
                angles.astype(np.float32), cfcr.astype(np.float32), pix,
                psfs, start, pix)


def full128(seed=2000, n=128, nz=None, nviews=120, subsets=8, iterations=10, collapse=2,
            drf_max_offs=17, with_srf=True, pix=None, body_scale=None, orbit_radius=None, counts=5e6,
            krnl_lens=(0.9, 4.0), name="full128"):
    """The full-physics case (DRF + ESSE); n/nz/nviews may be reduced for tests.

    Defaults give config 2: 0.3125 cm voxels at 128, the body scaled to a
    40 cm field of view, the 22 x 18 cm elliptical orbit.  pix, body_scale
    (cm per body unit), orbit_radius (a circular orbit) and krnl_lens (the
    two scatter-kernel decay lengths) override them."""
    rng = np.random.default_rng(seed)
    pix = 0.3125 * 128 / n if pix is None else pix
    nz = n if nz is None else nz
    X, Y, Z = _grid(n, nz, pix)
    fov = n * pix
    s = fov / 40.0 if body_scale is None else body_scale
    body = _ellipsoid(X, Y, Z, (0, 0, 0), (17 * s, 12.5 * s, 0.6 * fov))
    act = np.zeros(X.shape, np.float32)
    act[body] = 0.5
    for i in range(12):
        lesion = i >= 8
        rr = 8 * s * np.sqrt(rng.uniform())
        th = rng.uniform(0, 2 * np.pi)
        c = (rr * np.cos(th), 0.75 * rr * np.sin(th), rng.uniform(-0.3, 0.3) * fov)
        if lesion:
            d = rng.uniform(2, 20) * pix / 2
            ax = np.array([d, d, d]) * rng.uniform(0.8, 1.2, 3)
        else:
            ax = rng.uniform(1.5, 6.0, 3) * s
        act[_ellipsoid(X, Y, Z, c, ax, rng.uniform(0, np.pi)) & body] = rng.uniform(1, 10)
    atn = np.zeros(X.shape, np.float32)
    atn[body] = 0.15
    for sx in (-1, 1):
        atn[_ellipsoid(X, Y, Z, (sx * 6.5 * s, -1.0 * s, 0.0), (4.0 * s, 6.0 * s, 0.45 * fov)) & body] = 0.04
    atn[((X - 0.0) ** 2 + (Y - 8.0 * s) ** 2 <= (1.8 * s) ** 2) & body] = 0.25
    angles = 2 * np.pi * np.arange(nviews) / nviews
    if orbit_radius is None:
        cfcr = np.sqrt((22 * s * np.cos(angles)) ** 2 + (18 * s * np.sin(angles)) ** 2)
    else:
        cfcr = np.full(nviews, float(orbit_radius))
    # distance range as libirl's psDrfSetup computes it (IrlSetup.c:538-540)
    dmin = float(cfcr.min()) - n // 2 * pix + pix / 2
    if dmin < 0:
        dmin = pix / 2
    dmax = float(cfcr.max()) + n // 2 * pix - pix / 2
    count = int(np.ceil((dmax - dmin) / pix)) + 2
    psfs = tailed_drf_table(pix, dmin, pix, count, max_offs=drf_max_offs)
    krnl = None
    if with_srf:
        kpix = pix * collapse
        noffs = max(8, int(round(10.0 / kpix)))
        ndists = 2 * noffs
        k, kmu = esse_kernel(noffs, ndists, kpix, lens=krnl_lens)
        krnl = (k, kmu, 0.15, kpix)
    return Case(name, n, nz, pix, nviews, subsets, iterations, counts, act, atn,
                angles.astype(np.float32), cfcr.astype(np.float32), pix,
                psfs, dmin, pix, krnl, collapse, iterations if with_srf else 0)


def large256(seed=5000, window="photopeak", n=256, nviews=128, subsets=16, iterations=8):
    """Config 5: 256^3 at 0.2 cm (51.2 cm field of view), 128 views on a
    28 cm circular orbit, a 65 x 65 DRF (the FFT convolution path), ESSE
    with c = 2, 2e7 counts.  window: "photopeak", or "lower" (a scatter
    window with a broader kernel, projected with fPrimaryFac = 0)."""
    lens = (0.9, 4.0) if window == "photopeak" else (1.6, 7.0)
    return full128(seed=seed, n=n, nviews=nviews, subsets=subsets, iterations=iterations, collapse=2,
                   drf_max_offs=33, pix=0.2, body_scale=1.0, orbit_radius=28.0, counts=2e7, krnl_lens=lens,
                   name="large256_" + window)


def batch32(seed0=3000, count=32, iterations=5):
    """Config 3: independent problems of uneven size, each drawn from its own
    seed: N in {64, 80, 96, 112, 128}, views in {60, 72, 90, 96, 120}, an
    even number of subsets (4..12) that divides the views, DRF and ESSE on.
    N is restricted to sides whose ESSE grid (N at c = 2) has factors 2, 3,
    5, 7 only."""
    rng = np.random.default_rng(seed0)
    cases = []
    for j in range(count):
        n = int(rng.choice([64, 80, 96, 112, 128]))
        nv = int(rng.choice([60, 72, 90, 96, 120]))
        subs = [k for k in (4, 6, 8, 10, 12) if nv % k == 0]
        ns = int(rng.choice(subs))
        cases.append(full128(seed=seed0 + 1 + j, n=n, nviews=nv, subsets=ns, iterations=iterations,
                             name=f"batch{j}"))
    return cases


def poisson_counts(prj, counts, seed):
    """Scale noise-free projections to `counts` total and Poisson-sample."""
    rng = np.random.default_rng(seed)
    tot = float(prj.sum())
    lam = np.clip(prj, 0, None) * (counts / tot if tot > 0 else 0.0)
    return rng.poisson(lam).astype(np.float32)
