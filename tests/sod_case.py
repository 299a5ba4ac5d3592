"""The Sod shock-tube case (CRKSPH, 1D) shared by the CPU and GPU tests.

Configuration: the mirrored periodic layout of caseUtils/compressible/sod/sod.py on
[-1, 1], 1,776 dense particles on |x| < 1/2 and 222 coarse ones outside (8:1 spacing,
equal masses), so each half is a 999-particle tube with reflecting walls at its ends.
Left state rho=1, p=1, v=0; right state rho=0.125, p=0.1, v=0; gamma=1.4; Wendland C2
with n_h = 5 (10 neighbours); the Balsara switch; RK4 with the CFL time step (0.3)
recomputed every step; the internal energy ramped over two dense spacings.  Errors are
taken on the half 0 < x < 1, shifted to [-1/2, 1/2] with the interface at 0, against the
exact solution at t (oracle/riemann.py)."""
from __future__ import annotations

import numpy as np

from oracle import riemann
from oracle.steps import SWITCH_BALSARA, CRKSPHOracle
import warpsph_b200 as ws
from warpsph_b200 import configurations as cf
from warpsph_b200 import core

NX, RATIO, GAMMA = 1776, 8, 1.4
LEFT = ws.sodInitialState(p=1.0, rho=1.0, v=0.0)
RIGHT = ws.sodInitialState(p=0.1, rho=0.125, v=0.0)
SMOOTH_SPACINGS = 2.0


def config(device):
    cfg, integrator = ws.buildConfig(dim=1, domain=core.buildDomainDescription(2.0, 1, True, device), kernel=ws.KernelFunctions.Wendland2,
                                     targetNeighbors=core.n_h_to_nH(5, 1), integrationScheme=ws.IntegrationSchemeType.rungeKutta4,
                                     cflFactor=0.3, device=device)
    cfg.nx = NX
    sch = cf.CRKSPHConfig()
    sch.gamma = GAMMA
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.Balsara1995
    return cfg, sch, integrator


def exact(x_half, t):
    return riemann.sample(x_half, t, (LEFT.rho, LEFT.v, LEFT.p), (RIGHT.rho, RIGHT.v, RIGHT.p), 0.0, GAMMA)


def right_half_errors(x, rho, v, p, t):
    """L1 errors (mean absolute) of rho, v and p over the particles of 0 < x < 1."""
    x = np.asarray(x, np.float64).reshape(-1)
    sel = (x > 0.0) & (x < 1.0)
    xs = x[sel] - 0.5
    er, eu, ep = exact(xs, t)
    return {"rho": float(np.mean(np.abs(np.asarray(rho, np.float64)[sel] - er))),
            "v": float(np.mean(np.abs(np.asarray(v, np.float64).reshape(-1)[sel] - eu))),
            "p": float(np.mean(np.abs(np.asarray(p, np.float64)[sel] - ep))),
            "particles": int(sel.sum())}


def oracle_initial_state(params):
    """buildSod1D's initial state restated on numpy arrays and the C oracle."""
    f = np.float32
    dxl, nr = 1.0 / NX, NX // RATIO
    dxr = 1.0 / nr
    xl = np.linspace(-0.5 + dxl / 2, 0.5 - dxl / 2, NX)
    xr = np.linspace(-0.5 + dxr / 2, 0.5 - dxr / 2, nr)
    xr = np.where(xr < 0, xr - 0.5, xr + 0.5)
    x = np.concatenate([xl, xr]).astype(f)[:, None]
    left = np.arange(NX + nr) < NX
    nH = core.n_h_to_nH(5, 1)
    m = np.where(left, dxl * LEFT.rho, dxl * RIGHT.rho * (NX / nr)).astype(f)
    H = np.where(left, nH * dxl / 2, nH * dxr / 2).astype(f)
    rho0 = np.where(left, LEFT.rho, RIGHT.rho).astype(f)
    st = dict(positions=x, velocities=np.zeros_like(x), supports=H, masses=m, densities=rho0.copy(),
              divergence=np.zeros_like(m), alpha0s=np.ones_like(m), alphas=np.ones_like(m))
    orc = CRKSPHOracle(params, "f32", adaptive_iterations=16, adaptive_threshold=1e-3)
    rho_opt, H_opt = orc.optimal_support(st)
    st["supports"] = H_opt.astype(f)
    dx = dxl * SMOOTH_SPACINGS
    ul, ur = LEFT.p / ((GAMMA - 1) * LEFT.rho), RIGHT.p / ((GAMMA - 1) * RIGHT.rho)
    xx = x[:, 0].astype(np.float64)
    with np.errstate(over="ignore"):
        u = np.where(xx > 0, (ul - ur) / (np.exp((xx - 0.5) / dx) + 1) + ur, 0.0)
        u = np.where(xx < 0, (ur - ul) / (np.exp((xx + 0.5) / dx) + 1) + ul, u)
    st["densities"] = rho_opt.astype(f)
    st["internalEnergies"] = u.astype(f)
    st["entropies"], st["pressures"], st["soundspeeds"] = orc.o.eos(params, st["internalEnergies"], st["densities"])
    return st


def run_oracle(params, st, t_end, max_steps=5000):
    """RK4 steps with the CFL time step (growth-limited by the previous dt) to t_end."""
    orc = CRKSPHOracle(params, "f32", switch=SWITCH_BALSARA)
    o = orc.o
    t, dt_prev, steps = 0.0, None, 0
    while t < t_end - 1e-12 and steps < max_steps:
        dt = float(o.cfl_dt(params, st["supports"], st["internalEnergies"], dt_prev))
        dt = min(dt, t_end - t)
        st, _, _ = orc.step(st, dt, "rungeKutta4")
        t += dt
        dt_prev = dt
        steps += 1
    return st, t, steps
