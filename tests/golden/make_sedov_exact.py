"""Generates tests/golden/sedov_exact.npz from the reference's Sedov similarity solution
(caseUtils/compressible/sedov/sedovSolution.py:86-190, SedovSolution.shockState and
.solution), read from the reference checkout at generation time only; the module needs
nothing beyond the standard library.

The fixture holds the shock state (shock speed, radius, post-shock velocity, density and
pressure) and the radial density, velocity and pressure profiles of the 2D blast
(gamma 5/3, rho0 1, E0 1) at t = 0.1 and t = 0.05, on 201 radii up to 1.2 shock radii.
tests/test_gpu_sedov_exact.py checks the GPU's Sedov 2D CRKSPH run against it.

Usage:  python tests/golden/make_sedov_exact.py --reference <reference checkout>
"""
from __future__ import annotations

import argparse
import importlib.util
from pathlib import Path

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout (wi-re/warpSPH)")
    a = ap.parse_args()
    path = Path(a.reference) / "src" / "warpSPH" / "caseUtils" / "compressible" / "sedov" / "sedovSolution.py"
    spec = importlib.util.spec_from_file_location("ref_sedovSolution", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for tag, t in (("t010", 0.1), ("t005", 0.05)):
        sol = mod.SedovSolution(nDim=2, gamma=5 / 3, rho0=1.0, E0=1.0)
        vs, r2, v2, rho2, P2 = sol.shockState(t)
        r = [1.2 * r2 * i / 200 for i in range(201)]
        _, v, u, rho, P, A, h = sol.solution(t, r)
        out[f"{tag}_shock"] = np.array([vs, r2, v2, rho2, P2])
        out[f"{tag}_r"] = np.asarray(r)
        out[f"{tag}_rho"] = np.asarray(rho)
        out[f"{tag}_v"] = np.asarray(v)
        out[f"{tag}_P"] = np.asarray(P)
    dst = Path(__file__).parent / "sedov_exact.npz"
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v for k, v in out.items() if k.endswith("shock")})


if __name__ == "__main__":
    main()
