"""Generates tests/golden/sod_exact.npz from the reference's exact Sod solver
(caseUtils/compressible/sod/sodSolution.py:200, solve), read from the reference checkout
at generation time only.  The module needs numpy and scipy and nothing of Warp, so it is
loaded from its file directly.

The fixture holds the reference's (x, rho, u, p) profile and wave positions for the Sod
states (left rho=1, p=1, v=0; right rho=0.125, p=0.1, v=0; gamma=1.4) at t = 0.2 on
[-0.5, 0.5] with the interface at 0.  tests/test_sod.py checks oracle/riemann.py against it.

Usage:  python tests/golden/make_sod_exact.py --reference <reference checkout>
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
    path = Path(a.reference) / "src" / "warpSPH" / "caseUtils" / "compressible" / "sod" / "sodSolution.py"
    spec = importlib.util.spec_from_file_location("ref_sodSolution", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    t, gamma = 0.2, 1.4
    positions, regions, values = mod.solve(left_state=(1.0, 1.0, 0.0), right_state=(0.1, 0.125, 0.0), geometry=(-0.5, 0.5, 0.0),
                                           t=t, gamma=gamma, npts=2001)
    out = Path(__file__).parent / "sod_exact.npz"
    np.savez_compressed(out, x=np.asarray(values["x"], np.float64), rho=np.asarray(values["rho"], np.float64),
                        u=np.asarray(values["u"], np.float64), p=np.asarray(values["p"], np.float64),
                        t=np.array([t]), gamma=np.array([gamma]),
                        head=np.array([positions["Head of Rarefaction"]]), tail=np.array([positions["Foot of Rarefaction"]]),
                        contact=np.array([positions["Contact Discontinuity"]]), shock=np.array([positions["Shock"]]),
                        p_star=np.array([regions["Region 3"][0]]), u_star=np.array([regions["Region 3"][2]]))
    print("wrote", out)


if __name__ == "__main__":
    main()
