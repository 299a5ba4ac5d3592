"""The Sedov 2D CRKSPH blast on the GPU against the reference's Sedov similarity solution
(caseUtils/compressible/sedov/sedovSolution.py, SedovSolution.shockState and .solution;
fixture tests/golden/sedov_exact.npz made by make_sedov_exact.py): 128^2 particles on the
periodic unit square, E0 = 1 deposited kernel-weighted at the centre, gamma 5/3, Wendland4
with 32 neighbours, Cullen-Dehnen switch, RK2 with the CFL step, compatible energy, run to
t = 0.1 (the benchmark's configuration at a quarter of its resolution per axis).

Checks, on the azimuthal average of the density in radial bins of width 0.01:
- the density peak lies between 0.85 and 1.03 shock radii (the smoothing length here is
  about 0.07 shock radii and the peak sits just behind the front);
- the peak density lies between half and 1.05 times the analytic jump 4;
- the mean absolute density error over 0.1 to 1.2 shock radii is below 0.25 of the jump;
- the total energy is conserved to 1e-4 (compatible energy update)."""
from pathlib import Path

import numpy as np
import pytest
import torch

import warpsph_b200 as ws

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "sedov_exact.npz"


def energy(S):
    return float((S.masses.double() * (S.internalEnergies.double() + 0.5 * (S.velocities.double() ** 2).sum(-1))).sum())


def test_sedov_2d_against_similarity_solution(cuda):
    g = dict(np.load(GOLD))
    cfg, integ = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, cuda), kernel=ws.KernelFunctions.Wendland4,
                                targetNeighbors=32, device=cuda)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    system = ws.buildSedov(System, State, cfg, nx=128, dim=2, domainExtent=1.0, gamma=5 / 3, kernel=ws.KernelFunctions.Wendland4,
                           targetNeighbors=32, device=cuda)
    e0 = energy(system.state)
    t_end, t, steps = 0.1, 0.0, 0
    while t < t_end - 1e-12 and steps < 20000:
        dt = min(float(cfg.dt), t_end - t)
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        t += dt
        steps += 1
        cfg.dt = ws.computeTimestep(system, cfg, sch, dt=cfg.dt)
    assert abs(t - t_end) < 1e-9, f"stopped at t = {t} after {steps} steps"
    S = system.state
    assert abs(energy(S) / e0 - 1) < 1e-4
    x = S.positions.double().cpu().numpy()
    rho = S.densities.double().cpu().numpy()
    r = np.linalg.norm(x, axis=1)
    vs, r2, v2, rho2, P2 = g["t010_shock"]
    edges = np.arange(0.0, 1.3 * r2, 0.01)
    idx = np.digitize(r, edges) - 1
    centres = 0.5 * (edges[1:] + edges[:-1])
    prof = np.array([rho[idx == k].mean() if np.any(idx == k) else np.nan for k in range(len(centres))])
    k_peak = int(np.nanargmax(prof))
    assert 0.85 * r2 <= centres[k_peak] <= 1.03 * r2, (centres[k_peak], r2)
    assert 0.5 * rho2 <= prof[k_peak] <= 1.05 * rho2, prof[k_peak]
    exact = np.interp(centres, g["t010_r"], g["t010_rho"])
    sel = (centres > 0.1 * r2) & (centres < 1.2 * r2) & np.isfinite(prof)
    l1 = np.mean(np.abs(prof[sel] - exact[sel]))
    assert l1 < 0.25 * rho2, l1
