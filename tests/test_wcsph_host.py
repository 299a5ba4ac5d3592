"""Host-side logic of the DFSPH and delta-SPH step functions (no GPU): the scheme
builder entries, configuration round trips, the enum forms the reference passes, gravity,
the wall-particle layout check and boundary velocities, and the cases the GPU path
refuses (walls in deltaSPH_step or without ghost points, boundary conditions, rigid
bodies, unknown surface detection schemes and normal sources), which raise before any
device work."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from warpsph_b200 import configurations as cf
from warpsph_b200.configurations import NormalSource, SurfaceDetectionScheme
from warpsph_b200.enumTypes import IncompressibleSPHScheme, WeaklyCompressibleSPHScheme
from warpsph_b200.systems import IncompressibleState, IncompressibleSystem, WeaklyCompressibleSystem
from warpsph_b200.wcsph import computeGravity, deltaSPH_step, dfsph_step


@pytest.mark.parametrize("name,system,step", [("deltaSPH", WeaklyCompressibleSystem, deltaSPH_step),
                                              (WeaklyCompressibleSPHScheme.deltaSPH, WeaklyCompressibleSystem, deltaSPH_step),
                                              ("divergenceFree", IncompressibleSystem, dfsph_step),
                                              ("dfsph", IncompressibleSystem, dfsph_step),
                                              (IncompressibleSPHScheme.divergenceFree, IncompressibleSystem, dfsph_step)])
def test_build_scheme_entries(name, system, step):
    t = ws.buildScheme(name)
    assert len(t) == 7 and t[0] is system and t[4] is step
    # builder.py:26-29 pairs deltaSPH with CompressibleSystemUpdate
    if step is deltaSPH_step:
        from warpsph_b200.systems import CompressibleSystemUpdate
        assert t[3] is CompressibleSystemUpdate
    cfg = t[2]()
    assert t[6](t[5](cfg)) == cfg


def test_defaults_follow_the_reference():
    i, w = cf.IncompressibleSPHConfig(), cf.WeaklyCompressibleSPHConfig()
    for c in (i, w):
        assert c.shiftProperties.active and c.shiftProperties.iterations == 1 and c.shiftProperties.CFL == 0.3
        assert not c.gravityConfig.active and c.gravityConfig.magnitude == 9.81
        assert not c.surfaceDetectionConfig.active
        assert c.diffusionParams.inviscid and c.diffusionParams.inviscidAlpha == 0.01
    assert i.solverConfig.divergenceFreeSolver.maxIterations == 32 and i.solverConfig.pressureSolver.maxIterations == 64


def test_wc_params_accepts_reference_enums():
    from enum import Enum

    class PressureForceScheme(Enum):
        conservative = 0
        Antuono = 2

    class DensityDiffusionScheme(Enum):
        densityOnly = 2

    class EquationOfState(Enum):
        Tait = "Tait"

    c = cf.WeaklyCompressibleSPHConfig()
    c.pressureForceTerm = PressureForceScheme.conservative
    c.diffusionParams.densityDiffusionTerm = DensityDiffusionScheme.densityOnly
    c.fluid.eosType = EquationOfState.Tait
    w = cf.wc_params(c)
    assert (w.pressure_term, w.density_scheme, w.eos) == (0, 2, 1)


def cpu_state(n=16, kinds=None):
    x = torch.rand(n, 2) - 0.5
    return IncompressibleState(positions=x, velocities=torch.zeros(n, 2), supports=torch.full((n,), 0.2), masses=torch.ones(n),
                               kinds=torch.zeros(n, dtype=torch.int32) if kinds is None else kinds)


@pytest.mark.parametrize("step,cfgcls", [(dfsph_step, cf.IncompressibleSPHConfig), (deltaSPH_step, cf.WeaklyCompressibleSPHConfig)])
def test_unsupported_inputs_raise(step, cfgcls):
    config = cf.SimulationConfig()
    k = torch.zeros(16, dtype=torch.int32)
    k[3] = 1
    # a wall particle without a ghost point after the fluid and walls
    with pytest.raises(NotImplementedError, match="ghost point" if step is dfsph_step else "wall"):
        step(IncompressibleSystem(state=cpu_state(kinds=k)), 1e-3, config, cfgcls())
    k[14], k[15] = 1, 2
    k[3] = 0
    st = cpu_state(kinds=k)
    if step is dfsph_step:      # walls with ghosts are accepted, but need their ghost fields
        with pytest.raises(ValueError, match="ghostIndices"):
            step(IncompressibleSystem(state=st), 1e-3, config, cfgcls())
    else:
        with pytest.raises(NotImplementedError, match="dfsph_step only"):
            step(IncompressibleSystem(state=st), 1e-3, config, cfgcls())
    for attr, val, msg in (("boundaryConditions", [object()], "boundary conditions"), ("rigidBodies", [object()], "rigid bodies")):
        c = cfgcls()
        setattr(c, attr, val)
        with pytest.raises(NotImplementedError, match=msg):
            step(IncompressibleSystem(state=cpu_state()), 1e-3, config, c)
    # every scheme and normal source of the reference is built; unknown ones raise before any pass runs
    from warpsph_b200 import surface
    st = cpu_state()
    for scheme, normals in (("NoSuchScheme", NormalSource.ColorFieldGrad), (SurfaceDetectionScheme.Barecasco, "NoSuchSource")):
        sd = ws.configurations.SurfaceDetectionConfig(scheme=scheme, normalSource=normals)
        with pytest.raises(ValueError, match="Unknown"):
            surface.detectFreeSurface(st, config, cfgcls(), sd, None)
    fsm, fs, n, _, _ = surface.detectFreeSurface(st, config, cfgcls(), ws.configurations.buildDefaultSurfaceDetectionConfig(), None)
    assert not fsm.any() and not fs.any() and not n.any()


def test_gravity_forms():
    S = cpu_state()
    c = cf.IncompressibleSPHConfig()
    assert torch.equal(computeGravity(S, None, c), torch.zeros(16, 2))
    c.gravityConfig.active = True
    g = computeGravity(S, None, c)
    assert g.shape == (16, 2) and torch.allclose(g, torch.tensor([0.0, -9.81]).expand(16, 2))
    c.gravityConfig.type = cf.GravityType.PointSource
    c.gravityConfig.origin = [0.1, 0.2]
    g = computeGravity(S, None, c)
    d = torch.tensor([0.1, 0.2]) - S.positions
    assert g.shape == (16, 2)
    assert torch.allclose(g, d / (d.norm(dim=1, keepdim=True) + 1e-8) * 9.81)
    c.gravityConfig.type = cf.GravityType.PotentialField
    with pytest.raises(NotImplementedError):
        computeGravity(S, None, c)


def test_boundary_velocities_and_wall_layout():
    from warpsph_b200.wcsph import _wall_layout, computeBoundaryVelocities
    k = torch.tensor([0, 0, 0, 1, 1, 2, 2], dtype=torch.int32)
    st = cpu_state(7, kinds=k)
    st.velocities = torch.ones(7, 2)
    st.ghostIndices = torch.tensor([-1, -1, -1, 5, 6, 3, 4], dtype=torch.int32)
    st.ghostOffsets = torch.zeros(7, 2)
    assert _wall_layout(st, True) == 5 and _wall_layout(cpu_state(7), True) is None
    v = computeBoundaryVelocities(st, cf.SimulationConfig(), cf.IncompressibleSPHConfig())
    assert torch.equal(v[3:5], torch.zeros(2, 2)) and torch.equal(v[:3], torch.ones(3, 2)) and torch.equal(v[5:], torch.ones(2, 2))
    # per-region types: material 0 a zeros wall, material 1 a constant wall
    import types
    Z, Cn, B = (types.SimpleNamespace(name=s_) for s_ in ("zeros", "constant", "Boundary"))
    config = cf.SimulationConfig()
    config.regions = [types.SimpleNamespace(type=B, kind=Z), types.SimpleNamespace(type=B, kind=Cn)]
    st.materials = torch.tensor([0, 0, 0, 0, 1, 0, 1], dtype=torch.int32)
    v = computeBoundaryVelocities(st, config, cf.IncompressibleSPHConfig())
    assert torch.equal(v[3], torch.zeros(2)) and torch.equal(v[4], torch.ones(2))
    config.regions[1].kind = types.SimpleNamespace(name="noSlip")
    with pytest.raises(NotImplementedError, match="noSlip"):
        computeBoundaryVelocities(st, config, cf.IncompressibleSPHConfig())


def test_weakly_compressible_step_limit():
    """The weakly compressible time-step rule (timestep/weaklyCompressible.py:13-88) as the
    ensemble applies it per box: the smallest enabled limit."""
    from warpsph_b200.wcsph import weaklyCompressibleStepLimit
    c = cf.WeaklyCompressibleSPHConfig()
    H, c0, nu, k = 0.05, 10.0, 1e-3, 1.9
    v, a = 0.125 * H * H / nu / k, 0.3 * H / c0 / k
    assert weaklyCompressibleStepLimit(H, c0, nu, k, 0.3, c) == min(v, a)
    acc = 0.25 * (H / (1e4 + 1e-7)) ** 0.5 / k
    assert weaklyCompressibleStepLimit(H, c0, nu, k, 0.3, c, max_accel=1e4) == min(v, a, acc)
    c.dt_acousticConstraint = False
    assert weaklyCompressibleStepLimit(H, 1.0, 1.0, k, 0.3, c) == 0.125 * H * H / 1.0 / k
