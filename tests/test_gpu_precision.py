"""Precision of the FP32 GPU path against an all-FP64 oracle run.

The GPU path computes in FP32, except:
  * the CRK moment-matrix inversion, which is FP64 (sph_crk_factors);
  * the conservation sums, which are FP64 (sph_conservation_sums);
  * optionally, compensated (Neumaier) accumulation of the momentum and energy
    right-hand sides (SphParams.kahan).
The oracle runs the same Sedov steps entirely in FP64.  For every state field, the test
states the error after 20 RK2 steps, relative to the field's scale.  It also states the
total-energy drift of both runs (the compatible-energy scheme conserves energy up to
round-off).  Run with -s to print the table."""
import numpy as np
import pytest

import warpsph_b200 as ws
from oracle.steps import CRKSPHOracle, SWITCH_CULLEN, state_to_numpy
from tests.test_gpu_step import sedov

pytestmark = pytest.mark.gpu
FIELDS = ("positions", "velocities", "internalEnergies", "densities", "supports", "alphas")


def energy(m, v, u):
    m, v, u = (np.asarray(a, np.float64) for a in (m, v, u))
    return float(np.sum(m * (u + 0.5 * np.sum(v * v, 1))))


@pytest.mark.parametrize("kahan", [False, True])
def test_fp32_path_against_fp64_oracle(cuda, kahan):
    nx, steps, dt = 48, 20, 2e-4
    cfg, sch, integ, step, system = sedov(nx, cuda, kahan=kahan)
    from warpsph_b200 import ops
    p = ws.make_params(cfg, sch)
    st = {k: v.astype(np.float64) for k, v in state_to_numpy(system.state).items()}
    orc = CRKSPHOracle(ws.make_params(cfg, sch), "f64", switch=SWITCH_CULLEN)
    S = system.state
    e0_gpu = float(ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies)[3].item())
    e0_orc = energy(st["masses"], st["velocities"], st["internalEnergies"])
    for _ in range(steps):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        st, _, _ = orc.step(st, dt, "rungeKutta2")
    S = system.state
    rows = []
    for name in FIELDS:
        g = getattr(S, name).detach().cpu().numpy().astype(np.float64)
        r = np.asarray(st[name], np.float64)
        if name == "positions":   # minimum image in the unit periodic box
            d = g - r
            d = d - np.round(d)
            scale = 1.0
        else:
            d = g - r
            scale = np.abs(r).max()
        rows.append((name, np.abs(d).max() / scale, np.sqrt(np.mean(d * d)) / scale))
    e1_gpu = float(ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies)[3].item())
    e1_orc = energy(st["masses"], st["velocities"], st["internalEnergies"])
    drift_gpu, drift_orc = abs(e1_gpu - e0_gpu) / e0_gpu, abs(e1_orc - e0_orc) / e0_orc
    print(f"\nSedov 2D {nx}^2, {steps} RK2 steps, dt {dt}, kahan={kahan}: FP32 GPU vs FP64 oracle")
    for name, mx, rms in rows:
        print(f"  {name:18s} max {mx:.3e}  rms {rms:.3e}   (relative to the field's max |value|)")
    print(f"  total-energy drift: GPU {drift_gpu:.3e}, FP64 oracle {drift_orc:.3e}")
    bounds = {"positions": 1e-6, "velocities": 5e-3, "internalEnergies": 5e-3, "densities": 1e-4, "supports": 1e-4, "alphas": 5e-2}
    for name, mx, rms in rows:
        assert mx <= bounds[name], (name, mx)
    assert drift_gpu <= 1e-6 + drift_orc, (drift_gpu, drift_orc)
