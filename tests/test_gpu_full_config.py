"""GPU parity at the benchmarked sizes, against the CPU oracle.

* The full-physics 128^3 case (128^3, 0.3125 cm voxels, 120 views on the
  22 x 18 cm elliptical orbit, 33x33 DRF at every depth, ESSE with c = 2,
  5e6 counts): every one of the 120 IrlGenprj views within 1e-4 relative
  L2, and IrlOsem over 8 subsets x 10 iterations, with the ESSE scatter
  model in all 10 (iNumSrfIterations = 10, osemrecon.c:637-852), within
  1e-3 relative L2 on the image.
* The 256^3 FFT-DRF case (0.2 cm voxels, 28 cm orbit, 65x65 DRF through
  the FFT convolution branch, ESSE with c = 2): a few views of each energy
  window, the lower one projected with fPrimaryFac = 0 (irl.h:281), within
  1e-4 per view.

The oracle's view loops run on every host core (or_set_threads); the 128^3
reconstruction is about 2000 core-seconds of oracle work.
"""
import numpy as np
import pytest

from conftest import rel_l2
from libirl_b200 import workloads as W
from test_gpu_parity import IMAGE_TOL, VIEW_TOL, gpu_genprj, gpu_osem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full128(orc, tmp_path_factory):
    """The 128^3 case, its oracle projections and its Poisson data."""
    case = W.full128(seed=2000)
    files = case.write_tables(str(tmp_path_factory.mktemp("full128")))
    pr = orc.Problem(case)
    clean = pr.genprj()
    meas = W.poisson_counts(clean, case.counts, 2000)
    return case, files, pr, clean, meas


def test_full128_every_view_against_oracle(product, full128):
    case, files, _, clean, _ = full128
    got = gpu_genprj(product, case, files)
    errs = [rel_l2(got[v], clean[v]) for v in range(case.nviews)]
    worst = int(np.argmax(errs))
    assert errs[worst] <= VIEW_TOL, f"view {worst}: relative L2 {errs[worst]:.3e}"


def test_full128_osem_8x10_with_esse_against_oracle(product, orc, full128):
    case, files, pr, _, meas = full128
    assert (case.subsets, case.iterations, case.srf_iters) == (8, 10, 10)
    got = gpu_osem(product, case, files, meas)
    want = orc.to_external(pr.osem(meas, case.iterations, case.nviews // case.subsets))
    err = rel_l2(got, want)
    assert err <= IMAGE_TOL, f"image relative L2 {err:.3e}"


@pytest.mark.parametrize("window,primary", [("photopeak", 1.0), ("lower", 0.0)])
def test_large256_fft_drf_views_against_oracle(product, orc, tmp_path, window, primary):
    """Three views of each window of the 256^3 case through IrlGenprj with
    bFFTConvolve = 1: the 65x65 DRF runs in the row/column Fourier form on
    its 320 x 320 grid, ESSE on the 256^3 grid."""
    full = W.large256(window=window)
    sel = [0, 45, 101]
    case = W.Case(full.name, full.n, full.nz, full.pix, len(sel), 1, 1, full.counts, full.act, full.atn,
                  full.angles[sel], full.cfcr[sel], full.atn_scale, full.drf_psfs, full.drf_start,
                  full.drf_spacing, full.krnl, full.collapse, 1)
    files = case.write_tables(str(tmp_path))
    got = gpu_genprj(product, case, files, primary=primary, opts={"bFFTConvolve": 1})
    want = orc.Problem(case).genprj(primary=primary)
    for vi in range(len(sel)):
        err = rel_l2(got[vi], want[vi])
        assert err <= VIEW_TOL, f"view {sel[vi]}: relative L2 {err:.3e}"
