"""dfsph_step with mDBC walls on the GPU against the oracle's restatement of the same step
(oracle/steps.py DFSPHWallOracle): a small 2D dam break (a fluid column in an open tank
with three wall layers and one mirrored ghost point per wall particle, the layout of the
reference's addBoundaryGhostParticles), gravity on, fixed Jacobi iteration counts.

Tolerances: 2e-4 of each field's scale after one step (the Verlet rows of the GPU and the
oracle are in different orders, so the sums differ by FP32 rounding; the fixed iteration
counts keep the comparison away from the stopping rule).  Walls and ghosts must not move."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle.steps import DFSPHWallOracle
from tests.cases import assert_close
from warpsph_b200 import core
from warpsph_b200.cases import buildDamBreak
from warpsph_b200.configurations import RelaxedJacobiSolverConfig, jacobi_config, wc_params
from warpsph_b200.integrators import getIntegrator

pytestmark = pytest.mark.gpu


def fixed(n):
    return RelaxedJacobiSolverConfig(minIterations=n, maxIterations=n, tolerance=0.0, relaxationFactor=0.3)


@pytest.mark.parametrize("scheme", ["explicitEuler", "rungeKutta2"])
def test_dfsph_step_with_walls_matches_oracle(cuda, scheme):
    cfg, _ = ws.buildConfig(device=cuda, dim=2, kernel=core.KernelFunctions.Wendland2, targetNeighbors=20.0)
    System, State, Config, Update, step, *_ = ws.buildScheme("divergenceFree")
    sch = Config()
    sch.gravityConfig.active = True
    sch.solverConfig.divergenceFreeSolver = fixed(10)
    sch.solverConfig.pressureSolver = fixed(8)
    system = buildDamBreak(System, State, cfg, dx=0.04, column=(0.4, 0.8), tank=(1.2, 1.0), jitter=0.05, seed=3, device=cuda)
    S = system.state
    k = S.kinds.cpu().numpy()
    nf, nw = int((k == 0).sum()), int((k == 1).sum())
    # a little motion so that every term of the step is exercised
    gen = torch.Generator(device="cpu").manual_seed(1)
    v = (0.2 * torch.randn(S.velocities.shape, generator=gen)).to(cuda)
    S.velocities = torch.where(S.kinds[:, None] == 0, v, torch.zeros_like(v))
    st0 = {name: getattr(S, name).cpu().numpy() for name in ("positions", "velocities", "supports", "masses")}
    st0["densities"] = None
    st0["pressures"] = None
    walls = dict(kinds=k, ghost_indices=S.ghostIndices.cpu().numpy().astype(np.int32), ghost_offsets=S.ghostOffsets.cpu().numpy(),
                 nfw=nf + nw, rho0=1.0, c_s=float(sch.fluid.fixedSoundSpeed))
    S.densities = None
    dt = 1e-3
    res = getIntegrator(getattr(core.IntegrationSchemeType, scheme)).function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
    p = ws.make_params(cfg)
    orc = DFSPHWallOracle(p, wc_params(sch), jacobi_config(sch.solverConfig.divergenceFreeSolver, 1.0),
                          jacobi_config(sch.solverConfig.pressureSolver, 1.0), walls, gravity=[0.0, -9.81])
    want, _, rvs = orc.step(st0, dt, scheme)
    G = res.state.state
    x = G.positions.cpu().numpy()
    assert np.array_equal(x[nf:], st0["positions"][nf:]), "walls and ghosts moved"
    assert np.abs(x[:nf] - want["positions"][:nf]).max() < 2e-6
    for name in ("velocities", "densities", "pressures"):
        g_, w_ = getattr(G, name).cpu().numpy()[:nf + nw], want[name][:nf + nw]
        assert_close(g_, w_, 2e-4, 2e-4, f"dam break {scheme} {name}")
    assert np.all(G.velocities.cpu().numpy()[nf:] == 0)
    # the last stage's state: the mDBC wall densities and the divergence-free pressures
    Sl, Wl = res.stages[-1].aux[1], rvs[-1][1]
    assert_close(Sl.densities.cpu().numpy()[:nf + nw], Wl["densities"][:nf + nw], 2e-4, 2e-4, f"stage densities {scheme}")
    assert not np.allclose(Wl["densities"][nf:nf + nw], 1.0)
