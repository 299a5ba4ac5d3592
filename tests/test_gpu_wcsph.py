"""dfsph_step and deltaSPH_step through the reference's integrator interface on the GPU,
against the CPU oracle's restatement of the same steps (oracle/steps.py DFSPHOracle,
DeltaSPHOracle) on a periodic fluid box with gravity.

The GPU keeps valid Verlet lists between stages, so its rows can be ordered differently
from the oracle's fresh lists: sums differ by FP32 rounding.  Tolerances are 2e-4 of
each field's scale for one step (the Jacobi solves run a fixed number of iterations,
which keeps the comparison away from the stopping rule)."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle.steps import DeltaSPHOracle, DFSPHOracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core
from warpsph_b200.configurations import (IncompressibleSPHConfig, NormalSource, RelaxedJacobiSolverConfig,
                                         SurfaceDetectionScheme, WeaklyCompressibleSPHConfig, jacobi_config, wc_params)
from warpsph_b200.integrators import getIntegrator

pytestmark = pytest.mark.gpu


def fluid_box(n_side=24, seed=4, kernel=core.KernelFunctions.Wendland2):
    cfg, _, p = make_params(2, kernel=kernel)
    rng = np.random.default_rng(seed)
    dx = 1.0 / n_side
    g = (np.arange(n_side) + 0.5) * dx - 0.5
    X, Y = np.meshgrid(g, g, indexing="xy")
    x = np.stack([X.ravel(), Y.ravel()], 1)
    x = ((x + 0.2 * dx * (rng.random(x.shape) - 0.5) + 0.5) % 1.0 - 0.5).astype(np.float32)
    n = len(x)
    H = np.full(n, core.volumeToSupportHelper(dx * dx, cfg.targetNeighbors, 2), np.float32)
    m = np.full(n, dx * dx, np.float32)
    v = (0.2 * np.stack([np.sin(2 * np.pi * x[:, 1]), np.cos(2 * np.pi * x[:, 0])], 1) + 0.05 * rng.standard_normal(x.shape)).astype(np.float32)
    return cfg, p, dict(positions=x, supports=H, masses=m, velocities=v)


def gpu_system(System, State, st, cuda, densities=None):
    t = {k: torch.from_numpy(v).to(cuda) for k, v in st.items()}
    S = State(positions=t["positions"], velocities=t["velocities"], supports=t["supports"], masses=t["masses"],
              densities=None if densities is None else torch.from_numpy(densities).to(cuda),
              kinds=torch.zeros(len(st["masses"]), dtype=torch.int32, device=cuda))
    return System(state=S)


def fixed(n):
    return RelaxedJacobiSolverConfig(minIterations=n, maxIterations=n, tolerance=0.0, relaxationFactor=0.3)


@pytest.mark.parametrize("scheme", ["explicitEuler", "rungeKutta2"])
def test_dfsph_step_matches_oracle(cuda, scheme):
    cfg, p, st = fluid_box()
    System, State, Config, Update, step, *_ = ws.buildScheme("divergenceFree")
    sch = Config()
    sch.solverConfig.divergenceFreeSolver = fixed(8)
    sch.solverConfig.pressureSolver = fixed(6)
    sch.gravityConfig.active = True
    dt = 2e-3
    system = gpu_system(System, State, st, cuda)
    res = getIntegrator(getattr(core.IntegrationSchemeType, scheme)).function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
    rho0 = sch.fluid.restDensity
    orc = DFSPHOracle(p, wc_params(sch), jacobi_config(sch.solverConfig.divergenceFreeSolver, rho0),
                      jacobi_config(sch.solverConfig.pressureSolver, rho0), gravity=[0.0, -9.81])
    want, _, rvs = orc.step(dict(st, densities=None, pressures=None), dt, scheme)
    S = res.state.state
    for name in ("positions", "velocities", "densities", "pressures"):
        got = getattr(S, name).cpu().numpy()
        if name == "positions":
            d = got - want[name]
            d = d - np.round(d)          # periodic unit box
            assert np.abs(d).max() < 2e-6, f"positions differ by {np.abs(d).max():.3g}"
        else:
            assert_close(got, want[name], 2e-4, 2e-4, f"DFSPH {scheme} {name}")
    # the solve history of the last stage and the density solve of the finalize
    errs, _ = res.stages[-1].aux[2]
    assert len(errs) == 8 and np.allclose(errs, rvs[-1][2]["errors"], rtol=2e-3, atol=1e-7)
    assert len(res.stages[-1].aux[3][0]) == 6


def test_deltasph_step_matches_oracle(cuda):
    cfg, p, st = fluid_box(seed=6, kernel=core.KernelFunctions.Wendland4)
    System, State, Config, Update, step, *_ = ws.buildScheme("deltaSPH")
    sch = Config()
    sch.gravityConfig.active = True
    assert sch.shiftProperties.active            # the reference's default: shifting on
    dt = 1e-3
    rng = np.random.default_rng(2)
    rho = (1.0 + 0.01 * rng.standard_normal(len(st["masses"]))).astype(np.float32)
    system = gpu_system(System, State, st, cuda, densities=rho)
    res = getIntegrator(core.IntegrationSchemeType.rungeKutta2).function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
    orc = DeltaSPHOracle(p, wc_params(sch), gravity=[0.0, -9.81],
                         shift=dict(cfl=sch.shiftProperties.CFL, c0=sch.fluid.fixedSoundSpeed, iterations=sch.shiftProperties.iterations))
    want, _, _ = orc.step(dict(st, densities=rho, pressures=None), dt, "rungeKutta2")
    S = res.state.state
    d = S.positions.cpu().numpy() - want["positions"]
    d = d - np.round(d)
    assert np.abs(d).max() < 2e-6, f"positions differ by {np.abs(d).max():.3g}"
    for name in ("velocities", "densities", "pressures"):
        assert_close(getattr(S, name).cpu().numpy(), want[name], 2e-4, 2e-4, f"delta-SPH {name}")
    # the shift moved the particles: compare with the run without it
    sch2 = Config()
    sch2.gravityConfig.active = True
    sch2.shiftProperties.active = False
    res2 = getIntegrator(core.IntegrationSchemeType.rungeKutta2).function(state=gpu_system(System, State, st, cuda, densities=rho),
                                                                          f=step, dt=dt, config=cfg, compParams=sch2)
    dd = (res.state.state.positions - res2.state.state.positions).abs().max().item()
    assert 0 < dd < 1e-3


def test_visc_continuity_and_shift_match_oracle(cuda):
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    cfg, p, st = fluid_box(n_side=40, seed=8, kernel=core.KernelFunctions.Wendland4)
    o = oracle.get("f32")
    x, H, m, v = st["positions"], st["supports"], st["masses"], st["velocities"]
    nb = o.neighbors(p, x, H, cell_capacity_for(len(H), 2))
    rho = o.density(p, 0, x, H, m, nb)
    t = {k: torch.from_numpy(a).to(cuda) for k, a in dict(x=x, H=H, m=m, v=v, rho=rho).items()}
    adj = ws.ops.buildVerletList(t["x"], t["H"], p, cfg.verletScale)
    sch = IncompressibleSPHConfig()
    sch.diffusionParams.inviscid = False
    dv, dr = ws.ops.wc_visc_continuity(p, wc_params(sch), t["x"], t["H"], t["m"], t["rho"], t["v"], adj)
    rdv, rdr = o.visc_continuity(p, wc_params(sch), x, H, m, rho, v, nb)
    assert_close(dv.cpu().numpy(), rdv, 1e-5, 1e-5, "velocity diffusion")
    assert_close(dr.cpu().numpy(), rdr, 1e-5, 1e-5, "continuity")
    kinds = torch.zeros(len(H), dtype=torch.int32, device=cuda)
    kinds[::5] = 1
    s = ws.ops.delta_shift(p, t["x"], t["H"], t["m"], t["rho"], t["v"], kinds, adj, 0.3, 10.0)
    rs = o.delta_shift(p, x, H, m, rho, v, nb, 0.3, 10.0, kinds=kinds.cpu().numpy())
    assert_close(s.cpu().numpy(), rs, 1e-5, 1e-5, "delta-plus shift")
    assert bool((s[::5] == 0).all())


def test_deltasph_rhs_surface_mask_matches_reference(cuda):
    """The Antuono pressure force with free-surface particles on the GPU against the
    reference's own pair body (golden vectors), divided by rho_i as the reference's
    kernel wrapper does (wp_surfaceAware.py:207-218)."""
    from pathlib import Path
    g = dict(np.load(Path(__file__).resolve().parent / "golden" / "deltasph_golden.npz"))
    cfg, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    sch = WeaklyCompressibleSPHConfig()
    sch.diffusionParams.inviscid = True
    sch.diffusionParams.inviscidAlpha = 0.0
    sch.pressureForceTerm = "Antuono"
    t = {k: torch.from_numpy(np.ascontiguousarray(g[k])).to(cuda) for k in ("x", "H", "m", "rho", "v", "offsets", "counts", "list",
                                                                              "surface_mask")}
    n = len(g["H"])
    adj = core.AdjacencyList(neighborOffsets=t["offsets"], numNeighbors=t["counts"], neighborList=t["list"], numRows=n, numCols=n,
                             nnz=int(g["list"].shape[0]))
    dv, _, _, P = ws.ops.deltasph_rhs(p, wc_params(sch), t["x"], t["H"], t["m"], t["rho"], t["v"], adj, t["surface_mask"])
    assert_close(P.cpu().numpy(), g["P"], 1e-5, 1e-5, "stiff Tait pressure")
    assert_close(dv.cpu().numpy(), -g["pf_antuono_mask"] / g["rho"][:, None], 1e-4, 1e-4, "Antuono force with surface mask")
    dv0, _, _, _ = ws.ops.deltasph_rhs(p, wc_params(sch), t["x"], t["H"], t["m"], t["rho"], t["v"], adj)
    assert_close(dv0.cpu().numpy(), -g["pf"][2] / g["rho"][:, None], 1e-4, 1e-4, "Antuono force without surface mask")


def test_deltasph_step_free_surface_matches_oracle(cuda):
    """deltaSPH_step with colour-field surface detection active on a block of fluid with
    free edges: the dilated indicators switch the Antuono term of the surface particles."""
    cfg, p, st = fluid_box(n_side=20, seed=7, kernel=core.KernelFunctions.Wendland4)
    # squeeze the lattice into the middle of the periodic box: free surfaces on all sides
    st = dict(st, positions=(st["positions"] * 0.5).astype(np.float32), masses=(st["masses"] * 0.25).astype(np.float32),
              supports=(st["supports"] * 0.5).astype(np.float32))
    System, State, Config, Update, step, *_ = ws.buildScheme("deltaSPH")
    sch = Config()
    sch.shiftProperties.active = False
    sch.surfaceDetectionConfig.active = True
    sch.surfaceDetectionConfig.scheme = SurfaceDetectionScheme.ColorField
    sch.surfaceDetectionConfig.normalSource = NormalSource.ColorFieldGrad
    sch.pressureForceTerm = "Antuono"
    dt = 5e-4
    rng = np.random.default_rng(5)
    rho = (1.0 + 0.01 * rng.standard_normal(len(st["masses"]))).astype(np.float32)
    system = gpu_system(System, State, st, cuda, densities=rho)
    res = getIntegrator(core.IntegrationSchemeType.rungeKutta2).function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
    sd = sch.surfaceDetectionConfig
    orc = DeltaSPHOracle(p, wc_params(sch), surface=dict(limit=float(cfg.targetNeighbors) * float(sd.colorFieldThreshold),
                                                         iterations=int(sd.expansionIterations)))
    want, _, rvs = orc.step(dict(st, densities=rho, pressures=None), dt, "rungeKutta2")
    S = res.state.state
    mask = S.surfaceIndicators.cpu().numpy()
    assert 0 < mask.sum() < len(mask)
    assert np.array_equal(mask, rvs[-1][1]["surfaceIndicators"])
    d = S.positions.cpu().numpy() - want["positions"]
    d = d - np.round(d)
    assert np.abs(d).max() < 2e-6, f"positions differ by {np.abs(d).max():.3g}"
    for name in ("velocities", "densities", "pressures"):
        assert_close(getattr(S, name).cpu().numpy(), want[name], 2e-4, 2e-4, f"delta-SPH free surface {name}")
