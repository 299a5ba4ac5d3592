"""The Sod shock tube (CRKSPH, 1D, RK4, CFL 0.3, Balsara) on the GPU: the case builder
against the oracle's restatement, the first steps against the oracle's steps, and the
full run to t = 0.2 against the exact Riemann solution and the CPU oracle's run."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle.steps import SWITCH_BALSARA, CRKSPHOracle, state_to_numpy
from tests import sod_case as S
from tests.cases import assert_close

pytestmark = pytest.mark.gpu


def build(cuda):
    cfg, sch, integ = S.config(cuda)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    system = ws.buildSod1D(System, State, S.RATIO, S.LEFT, S.RIGHT, S.GAMMA, cfg, smoothIC=True,
                           smoothingSpacings=S.SMOOTH_SPACINGS)
    return cfg, sch, integ, step, system


def test_sod_builder_matches_oracle_restatement(cuda):
    cfg, sch, integ, step, system = build(cuda)
    st = S.oracle_initial_state(ws.make_params(cfg, sch))
    g = state_to_numpy(system.state)
    assert g["positions"].shape == (1998, 1)
    assert_close(g["positions"], st["positions"], 1e-6, 1e-7, "x")
    assert_close(g["masses"], st["masses"], 1e-6, 1e-7, "m")
    assert_close(g["supports"], st["supports"], 1e-4, 1e-5, "H after 16 Newton iterations")
    assert_close(g["densities"], st["densities"], 1e-4, 1e-5, "rho")
    assert_close(g["internalEnergies"], st["internalEnergies"], 1e-5, 1e-6, "u")
    assert_close(g["pressures"], st["pressures"], 1e-4, 1e-5, "P")
    assert cfg.dt is not None and cfg.dt > 0


def test_sod_first_steps_match_oracle(cuda):
    cfg, sch, integ, step, system = build(cuda)
    p = ws.make_params(cfg, sch)
    st = state_to_numpy(system.state)
    orc = CRKSPHOracle(p, "f32", switch=SWITCH_BALSARA)
    dt = float(cfg.dt)
    for k in range(3):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        st, _, _ = orc.step(st, dt, "rungeKutta4")
        S_ = system.state
        tol = 2e-4 * (k + 1)
        assert_close(S_.positions.cpu().numpy(), st["positions"], 1e-6, 1e-6, f"x step {k}")
        assert_close(S_.velocities.cpu().numpy(), st["velocities"], tol, tol, f"v step {k}")
        assert_close(S_.internalEnergies.cpu().numpy(), st["internalEnergies"], tol, tol, f"u step {k}")
        assert_close(S_.densities.cpu().numpy(), st["densities"], 1e-5, 1e-5, f"rho step {k}")
        # alpha = |div v| / (|div v| + 1e-4 c) is ill-conditioned where div v is at rounding
        # level (the flat states, where v is zero analytically): compare it where the flow is
        # actually compressing or expanding
        a, ra = S_.alphas.cpu().numpy(), st["alphas"]
        sel = ra > 0.9
        assert sel.sum() > 20
        assert_close(a[sel], ra[sel], 1e-2, 1e-2, f"Balsara alpha step {k}")


def test_sod_full_run_accuracy(cuda):
    cfg, sch, integ, step, system = build(cuda)
    t, steps = 0.0, 0
    while t < 0.2 - 1e-12:
        dt = float(ws.computeTimestep(system, cfg, sch, dt=cfg.dt))
        dt = min(dt, 0.2 - t)
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        cfg.dt = dt
        t += dt
        steps += 1
    S_ = state_to_numpy(system.state)
    P = (S.GAMMA - 1) * S_["densities"].astype(np.float64) * S_["internalEnergies"]
    e = S.right_half_errors(S_["positions"], S_["densities"], S_["velocities"], P, t)
    print(f"\nSod GPU: {steps} RK4 steps to t={t:.3f}; L1 errors against the exact solution: {e}")
    assert 300 < steps < 1000
    assert e["rho"] < 5e-3 and e["v"] < 1e-2 and e["p"] < 5e-3, e
    # mirror symmetry of the two halves (x -> -x, v -> -v)
    x = S_["positions"][:, 0].astype(np.float64)
    o = np.argsort(x)
    r = S_["densities"][o]
    assert np.max(np.abs(r - r[::-1])) < 2e-2 * r.max()
