"""3D Sedov-Taylor blast (CRKSPH): the FP32 GPU path against the all-FP64 oracle, and
energy and momentum conservation with compensated sums (the 3D case of the precision
design: FP64 only for the 4x4 CRK moment inversion and the conservation reductions).
Run with -s for the error table."""
import numpy as np
import pytest

import warpsph_b200 as ws
from oracle.steps import CRKSPHOracle, SWITCH_CULLEN, state_to_numpy

pytestmark = pytest.mark.gpu
NEIGHBOURS_3D = 128


def sedov3d(nx, dev, kahan=True):
    cfg, integrator = ws.buildConfig(dim=3, domain=ws.buildDomainDescription(1.0, 3, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                     targetNeighbors=NEIGHBOURS_3D, integrationScheme=ws.IntegrationSchemeType.rungeKutta2, device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    sch.compensatedSums = kahan
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=3, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=NEIGHBOURS_3D, device=dev)
    return cfg, sch, integrator, step, system


def test_sedov3d_fp32_against_fp64_oracle(cuda):
    nx, steps = 16, 4
    cfg, sch, integ, step, system = sedov3d(nx, cuda)
    dt = float(cfg.dt)
    p = ws.make_params(cfg, sch)
    st = {k: v.astype(np.float64) for k, v in state_to_numpy(system.state).items()}
    orc = CRKSPHOracle(p, "f64", switch=SWITCH_CULLEN)
    for _ in range(steps):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        st, _, _ = orc.step(st, dt, "rungeKutta2")
    S = system.state
    print(f"\nSedov 3D {nx}^3, {steps} RK2 steps, dt {dt:.3g}: FP32 GPU (Kahan) vs FP64 oracle")
    bounds = {"positions": 1e-6, "velocities": 5e-3, "internalEnergies": 5e-3, "densities": 1e-4, "supports": 1e-4}
    for name, b in bounds.items():
        g = getattr(S, name).detach().cpu().numpy().astype(np.float64)
        r = np.asarray(st[name], np.float64)
        d = g - r
        scale = 1.0 if name == "positions" else np.abs(r).max()
        if name == "positions":
            d = d - np.round(d)
        mx, rms = np.abs(d).max() / scale, np.sqrt(np.mean(d * d)) / scale
        print(f"  {name:18s} max {mx:.3e}  rms {rms:.3e}")
        assert mx <= b, (name, mx)
    assert np.abs(st["velocities"]).max() > 0.05


def test_sedov3d_conservation(cuda):
    cfg, sch, integ, step, system = sedov3d(40, cuda)
    p = ws.make_params(cfg, sch)
    from warpsph_b200 import ops
    S = system.state
    c0 = ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    dt = ws.computeTimestep(system, cfg, sch, dt=None)
    for _ in range(5):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
    S = system.state
    c1 = ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    drift = abs(c1[3] - c0[3]) / c0[3]
    print(f"\nSedov 3D 40^3: total-energy drift over 5 RK2 steps {drift:.3e}, kinetic fraction {c1[1] / c1[3]:.3e}")
    assert drift < 1e-6, (c0[3], c1[3])
    assert c1[1] > 1e-4 * c1[3]
    assert np.max(np.abs(c1[4:7])) < 1e-6 * np.sqrt(2 * c1[1] * c1[0]) + 1e-12
