"""The tcgen05 operand conventions of warpsph_b200/csrc/sph_tcgen05.cuh checked on the
host against CuTe's own descriptor construction (a CUTLASS header tree is needed; the
test is skipped without one).  No GPU: the check program only builds descriptors."""
import glob
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cutlass_include():
    cands = []
    for base in sys.path:
        cands += glob.glob(os.path.join(base, "flashinfer", "data", "cutlass", "include"))
        cands += glob.glob(os.path.join(base, "tilelang", "3rdparty", "cutlass", "include"))
    for c in cands:
        if os.path.exists(os.path.join(c, "cute", "atom", "mma_traits_sm100.hpp")):
            return c
    return None


def test_umma_layout_matches_cute(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    inc = _cutlass_include()
    if not os.path.exists(nvcc) or inc is None:
        pytest.skip("nvcc or a CUTLASS header tree with the sm100 UMMA traits is not available")
    exe = tmp_path / "umma_layout_check"
    src = os.path.join(ROOT, "tests", "native", "umma_layout_check.cu")
    r = subprocess.run([nvcc, "-std=c++17", "-w", "-I", inc, "-I", os.path.join(ROOT, "warpsph_b200", "csrc"), "-I",
                        os.path.join(ROOT, "include"), "-o", str(exe), src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stdout + out.stderr
