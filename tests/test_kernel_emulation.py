"""Host emulation of the register-transform CUDA kernels (no GPU).

Each phase of the one-CTA-per-plane DRF kernels (drf_plane.cuh) and of the
ESSE x and y-z kernels (esse_rows.cuh, esse_yz.cuh) is a function of the
thread index, and the ESSE expansion's line walk (esse_walk.cuh) a function
of one line.  The C++ programs under tests/emulation run every phase for
all threads of a CTA, once in increasing and once in decreasing thread order
(a phase that read another thread's result of the same phase would differ),
under AddressSanitizer (any index outside the shared-memory buffers or the
global arrays aborts), and compare with direct transforms in double; the
line walk at coarse resolution is compared bit for bit with the
full-resolution expansion and in-place smoothing.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_SRC = os.path.join(ROOT, "libirl_b200", "csrc", "cuda")
CUDA_INC = "/usr/local/cuda/include"


def _build_and_run(name, tmp_path):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path / name)
    src = os.path.join(ROOT, "tests", "emulation", name + ".cpp")
    flags = ["-std=c++17", "-O1", "-g", "-w", f"-I{CUDA_SRC}", f"-I{CUDA_INC}"]
    asan = ["-fsanitize=address", "-fno-omit-frame-pointer"]
    r = subprocess.run(["g++"] + flags + asan + [src, "-o", exe], capture_output=True, text=True)
    if r.returncode != 0:  # no sanitizer runtime: plain build
        r = subprocess.run(["g++"] + flags + [src, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, (run.stdout[-3000:], run.stderr[-3000:])
    return run.stdout


@pytest.mark.parametrize("name", ["dplane_host_test", "esse_yz_host_test", "esse_rows_host_test", "esse_walk_host_test"])
def test_kernel_phases_match_direct_transforms(name, tmp_path):
    out = _build_and_run(name, tmp_path)
    assert "worst" in out
