"""Builds libwarpsph_b200.so in-tree with nvcc for sm_100a.

Usage: python -m warpsph_b200.build [--force] [--checked]

The shared library is written next to this file so that it travels with the
source tree; there is no JIT cache and no fallback path.  ``--checked`` adds
``-DSPH_CHECKED`` (device-side index checks that set a status word instead of
trapping) and writes ``libwarpsph_b200_checked.so``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
LIB_NAME = "libwarpsph_b200.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                "-Xptxas", "-O3"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build libwarpsph_b200")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def lib_path(checked: bool = False) -> Path:
    return HERE / (LIB_NAME.replace(".so", "_checked.so") if checked else LIB_NAME)


def needs_build(checked: bool = False) -> bool:
    out = lib_path(checked)
    if not out.exists():
        return True
    t = out.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, checked: bool = False, verbose: bool = False) -> Path:
    out = lib_path(checked)
    if not force and not needs_build(checked):
        return out
    objdir = HERE / "_build" / ("checked" if checked else "release")
    objdir.mkdir(parents=True, exist_ok=True)
    extra = ["-DSPH_CHECKED"] if checked else []
    cc = nvcc()

    def compile_one(src: Path) -> Path:
        obj = objdir / (src.stem + ".o")
        cmd = [cc, *ARCH_FLAGS, *COMMON_FLAGS, *extra, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = out.with_suffix(".so.tmp")
    cmd = [cc, *ARCH_FLAGS, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--checked", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    p = build(force=a.force, checked=a.checked, verbose=a.verbose)
    print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
