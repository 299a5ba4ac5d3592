"""Full CRKSPH integrator steps on the GPU against the CPU oracle's step, plus the
size-independent properties of the step at the benchmark size (conservation,
symmetry of the Sedov blast)."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle.steps import CRKSPHOracle, SWITCH_BALSARA, SWITCH_CULLEN, SWITCH_NONE, state_to_numpy
from tests.cases import assert_close

pytestmark = pytest.mark.gpu


def sedov(nx, dev, switch=ws.ViscositySwitch.CullenDehnen2010, scheme=ws.IntegrationSchemeType.rungeKutta2, kahan=False):
    cfg, integrator = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                     targetNeighbors=32, integrationScheme=scheme, device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = switch
    sch.compensatedSums = kahan
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=2, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=32, device=dev)
    return cfg, sch, integrator, step, system


SWITCHES = {ws.ViscositySwitch.CullenDehnen2010: SWITCH_CULLEN, ws.ViscositySwitch.Balsara1995: SWITCH_BALSARA,
            ws.ViscositySwitch.NoneSwitch: SWITCH_NONE}


@pytest.mark.parametrize("switch", list(SWITCHES))
def test_step_matches_oracle(cuda, switch):
    cfg, sch, integ, step, system = sedov(32, cuda, switch=switch)
    dt = 2e-4
    st = state_to_numpy(system.state)
    orc = CRKSPHOracle(ws.make_params(cfg, sch), "f32", switch=SWITCHES[switch])
    for k in range(3):
        res = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
        system = res.state
        st, _, _ = orc.step(st, dt, "rungeKutta2")
        S = system.state
        tol = 2e-4 * (k + 1)
        assert_close(S.positions.cpu().numpy(), st["positions"], 1e-6, 1e-6, f"x step {k}")
        assert_close(S.velocities.cpu().numpy(), st["velocities"], tol, tol, f"v step {k}")
        assert_close(S.internalEnergies.cpu().numpy(), st["internalEnergies"], tol, tol, f"u step {k}")
        assert_close(S.densities.cpu().numpy(), st["densities"], 1e-5, 1e-5, f"rho step {k}")
        assert_close(S.supports.cpu().numpy(), st["supports"], 1e-5, 1e-5, f"H step {k}")
        assert_close(S.alphas.cpu().numpy(), st["alphas"], 1e-3, 1e-3, f"alpha step {k}")


def test_rk4_step_matches_oracle(cuda):
    cfg, sch, integ, step, system = sedov(24, cuda, scheme=ws.IntegrationSchemeType.rungeKutta4)
    st = state_to_numpy(system.state)
    orc = CRKSPHOracle(ws.make_params(cfg, sch), "f32", switch=SWITCH_CULLEN)
    res = integ.function(state=system, f=step, dt=2e-4, config=cfg, compParams=sch)
    st, _, _ = orc.step(st, 2e-4, "rungeKutta4")
    assert len(res.stages) == 4
    assert_close(res.state.state.velocities.cpu().numpy(), st["velocities"], 2e-4, 2e-4, "v")
    assert_close(res.state.state.internalEnergies.cpu().numpy(), st["internalEnergies"], 2e-4, 2e-4, "u")


def test_step_vs_fp64_oracle_error(cuda):
    """FP32 GPU against the all-FP64 oracle after 5 steps (the stated field error)."""
    cfg, sch, integ, step, system = sedov(32, cuda)
    st = {k: v.astype(np.float64) for k, v in state_to_numpy(system.state).items()}
    orc = CRKSPHOracle(ws.make_params(cfg, sch), "f64", switch=SWITCH_CULLEN)
    for _ in range(5):
        system = integ.function(state=system, f=step, dt=2e-4, config=cfg, compParams=sch).state
        st, _, _ = orc.step(st, 2e-4, "rungeKutta2")
    S = system.state
    for name, tol in (("densities", 1e-5), ("velocities", 1e-3), ("internalEnergies", 1e-3)):
        assert_close(getattr(S, name).cpu().numpy(), st[name], tol, tol, name)


@pytest.mark.parametrize("nx", [128, 512])
def test_energy_momentum_conservation_and_symmetry(cuda, nx):
    cfg, sch, integ, step, system = sedov(nx, cuda, kahan=True)
    p = ws.make_params(cfg, sch)
    from warpsph_b200 import ops
    S = system.state
    c0 = ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    dt = ws.computeTimestep(system, cfg, sch, dt=None)
    for _ in range(5):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
    S = system.state
    c1 = ops.conservation_sums(p, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    assert abs(c1[3] - c0[3]) / c0[3] < 2e-6, ("total energy drift", c0[3], c1[3])
    assert np.max(np.abs(c1[4:6])) < 1e-6 * np.sqrt(2 * c1[1] * c1[0]) + 1e-12
    assert abs(c1[0] - c0[0]) == 0.0
    # the blast is symmetric under x -> -x: compare the kinetic energy of the two half planes
    x = S.positions.cpu().numpy().astype(np.float64)
    ke = 0.5 * S.masses.cpu().numpy() * np.sum(S.velocities.cpu().numpy().astype(np.float64) ** 2, 1)
    left, right = ke[x[:, 0] < 0].sum(), ke[x[:, 0] > 0].sum()
    assert abs(left - right) / (left + right) < 1e-3


def test_fused_entries_equal_separate_calls(cuda):
    """The launch-saving entries give the separate calls' results bit for bit:
    sph_crk_factors_eos against sph_crk_factors + sph_eos_ideal_gas, and
    sph_rk_combine_fields against one sph_rk_combine per field."""
    from warpsph_b200 import ops
    cfg, sch, integ, step, system = sedov(48, cuda)
    params = ws.make_params(cfg, sch)
    S = system.state
    adj = ops.buildVerletList(S.positions, S.supports, params, cfg.verletScale, None)
    V = ops.crk_volume(params, S.positions, S.supports, adj)
    crk1, rho1 = ops.crk_factors(params, S.positions, S.supports, S.masses, V, adj)
    A1, P1, c1 = ops.eos_ideal_gas(params, S.internalEnergies, rho1)
    crk2, rho2, A2, P2, c2 = ops.crk_factors_eos(params, S.positions, S.supports, S.masses, V, adj, S.internalEnergies)
    for a, b in ((crk1.A, crk2.A), (crk1.B, crk2.B), (crk1.gradA, crk2.gradA), (crk1.gradB, crk2.gradB), (rho1, rho2),
                 (A1, A2), (P1, P2), (c1, c2)):
        assert torch.equal(a, b)
    g = torch.Generator(device=cuda).manual_seed(11)
    n, d = S.positions.shape
    ks = [[torch.randn(S.positions.shape, generator=g, device=cuda) for _ in range(2)],
          [torch.randn(S.velocities.shape, generator=g, device=cuda) for _ in range(2)],
          [torch.randn(S.internalEnergies.shape, generator=g, device=cuda) for _ in range(2)]]
    fields = [(S.positions, ks[0], d), (S.velocities, ks[1], 0), (S.internalEnergies, ks[2], 0)]
    w, dt = [0.5, 0.5], torch.tensor([3e-3], device=cuda)
    fused = ops.rk_combine_fields(params, fields, w, dt)
    for (y0, kf, wrap), y in zip(fields, fused):
        assert torch.equal(ops.rk_combine(params, y0, kf, w, dt, wrap), y)
