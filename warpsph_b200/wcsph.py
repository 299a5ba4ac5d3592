"""DFSPH and delta-SPH step functions on the GPU, with the finalize steps of their systems.

``dfsph_step`` follows src/warpSPH/schemes/dfsph.py:13-218 and ``deltaSPH_step``
follows schemes/deltaSPH.py:11-208, call for call, for fluid-only systems:

  Verlet list (super-symmetric rows)      dfsph.py:27     -> sph_neighbors_build / refresh
  gather density                          dfsph.py:36-40  -> sph_density_gather
  mDBC density, boundary velocities,      dfsph.py:48-59, -> sph_mdbc_density, computeBoundaryVelocities,
  no-penetration shift                    :120-126           sph_mdbc_nopen_shift (identities without walls,
                                                             the reference's own early returns)
  Dirichlet conditions, forcing           :57, :110-113     -> none (no boundary conditions on this path)
  free-surface detection                  dfsph.py:72-77  -> surface.detectFreeSurface (colour-field scheme)
  velocity diffusion + continuity         dfsph.py:100-109 -> sph_wc_visc_continuity (one pass)
  gravity                                 dfsph.py:117-120 -> computeGravity (elementwise)
  divergence-free solve                   dfsph.py:132-140 -> sph_dfsph_div_solve (persistent kernel)

  delta-SPH right-hand side               deltaSPH.py:52-98 -> sph_deltasph_rhs (EOS, renormalised
                                                               density gradient, density and
                                                               velocity diffusion, continuity,
                                                               pressure force in two passes; the
                                                               surface indicators enter the
                                                               Antuono pressure term)

dfsph_step also runs systems with wall particles (kind 1) and their ghost points (kind 2):
the mDBC wall density (sph_mdbc_density), the wall velocities and the no-penetration
shift (sph_mdbc_nopen_shift), see _dfsph_step_walls.  Boundary conditions, rigid bodies,
walls in deltaSPH_step and the surface-aware shift raise NotImplementedError.
"""
from __future__ import annotations

import math

import dataclasses
from typing import Any, Optional

import torch

from . import ops
from .configurations import GravityType, make_params, wc_params
from .core import SupportScheme, sphKernelScale, volumeToSupportHelper
from .incompressible import solveDivergenceFree, solveIncompressible
from .surface import detectFreeSurface
from .systems import _LAST_STAGE_FIELDS, IncompressibleSystemUpdate, WeaklyCompressibleSystemUpdate

_KINDS_CHECKED: dict = {}
# the last list over every particle (ghost points included) per (device, particle count):
# the prior that the next mDBC density pass's list build validates and keeps or rebuilds
_GHOST_LISTS: dict = {}


def _wall_layout(state, allow_walls: bool) -> Optional[int]:
    """None for a fluid-only system.  With wall particles (kind 1) and their ghost points
    (kind 2): the number of fluid and wall particles, which come first, followed by the
    ghosts, as addBoundaryGhostParticles lays them out (rigidBody/ghostParticles.py:61-79).
    One host read each time the kinds tensor changes."""
    k = state.kinds
    if k is None:
        return None
    key = (id(k), k._version, k.data_ptr(), tuple(k.shape))
    hit = _KINDS_CHECKED.get(id(k))
    if hit is not None and hit[0] == key:
        nfw = hit[1]
    else:
        n = int(k.shape[0])
        nf, nw, ng = (int(c) for c in torch.stack([(k == 0).sum(), (k == 1).sum(), (k == 2).sum()]).tolist())
        if nw == 0 and ng == 0 and nf == n:
            nfw = None
        else:
            if nf + nw + ng != n:
                raise ValueError("particle kinds must be 0 (fluid), 1 (wall) or 2 (ghost)")
            if ng != nw or not bool((k[nf + nw:] == 2).all()):
                raise NotImplementedError("wall particles need one ghost point each, the ghosts after every fluid and wall particle "
                                          "(the layout of addBoundaryGhostParticles)")
            nfw = nf + nw
        _KINDS_CHECKED.clear()
        _KINDS_CHECKED[id(k)] = (key, nfw)
    if nfw is not None:
        if not allow_walls:
            raise NotImplementedError("wall and ghost particles are on the GPU path of dfsph_step only")
        if state.ghostIndices is None or state.ghostOffsets is None:
            raise ValueError("wall particles need the state's ghostIndices and ghostOffsets")
    return nfw


def _check_supported(state, schemeConfig, allow_walls: bool = False) -> Optional[int]:
    """Raises for what the GPU path does not cover; returns the wall layout (_wall_layout)."""
    if getattr(schemeConfig, "boundaryConditions", None):
        raise NotImplementedError("boundary conditions are not on the GPU path")
    if getattr(schemeConfig, "rigidBodies", None):
        raise NotImplementedError("rigid bodies are not on the GPU path")
    return _wall_layout(state, allow_walls)


def _head(state, n: int):
    """The first n particles of every per-particle field (views, no copies)."""
    N = state.positions.shape[0]
    kw = {}
    for f in dataclasses.fields(state):
        v = getattr(state, f.name)
        kw[f.name] = v[:n] if isinstance(v, torch.Tensor) and v.dim() >= 1 and v.shape[0] == N else v
    return type(state)(**kw)


def _pad(t: Optional[torch.Tensor], n: int) -> Optional[torch.Tensor]:
    """t with zero rows appended up to n rows (the ghost points' rows)."""
    if t is None or t.shape[0] == n:
        return t
    return torch.cat([t, t.new_zeros((n - t.shape[0],) + tuple(t.shape[1:]))])


def _gravity_vector(schemeConfig, dim: int):
    g = schemeConfig.gravityConfig
    if not g.active or g.type != GravityType.Directional:
        return None
    return [float(a) * float(g.magnitude) for a in list(g.direction)[:dim]]


def computeBoundaryVelocities(currentState: Any, config: Any, schemeConfig: Any, adjacency=None) -> torch.Tensor:
    """modules/mdbc/velocity.py:167-268 for walls with the zeros and constant boundary
    types (BCType, moduleConfigurations/boundaryConditions.py:8-13): a wall particle of a
    zeros region gets zero velocity, a constant region keeps its own.  The wall regions are
    config.regions' boundary regions in order (a wall particle's material indexes them);
    without regions every wall is a zeros wall.  The interpolated types (noSlip, freeSlip,
    extended) raise NotImplementedError."""
    k, v = currentState.kinds, currentState.velocities
    if k is None:
        return v
    regions = [r for r in (getattr(config, "regions", None) or []) if getattr(getattr(r, "type", None), "name", "") == "Boundary"]
    kinds_bc = [getattr(getattr(r, "kind", None), "name", "zeros") for r in regions]
    bad = sorted(set(kinds_bc) - {"zeros", "constant"})
    if bad:
        raise NotImplementedError(f"boundary velocity types {bad} are not on the GPU path")
    wall = k == 1
    if regions:
        zero_of_material = torch.tensor([b == "zeros" for b in kinds_bc], device=v.device)
        mat = currentState.materials.long().clamp(0, len(kinds_bc) - 1)
        wall = wall & zero_of_material[mat]
    return torch.where(wall[:, None], torch.zeros_like(v), v)


def computeGravity(currentState: Any, config: Any, schemeConfig: Any, adjacency=None) -> torch.Tensor:
    """modules/gravity/wrapper.py:20-34.  Directional (directional.py:12-22): the constant
    magnitude * direction.  Point source (pointGravity.py:13-29): magnitude times the unit
    vector towards the origin, per particle (the reference's trailing .repeat(n, 1) turns
    that [n, d] field into an [n^2, d] tensor, which no caller can use; the per-particle
    field is returned here)."""
    g = schemeConfig.gravityConfig
    v = currentState.velocities
    if not g.active:
        return torch.zeros_like(v)
    d = v.shape[1]
    if g.type == GravityType.Directional:
        direction = torch.as_tensor(g.direction, dtype=v.dtype, device=v.device)[:d]
        return (direction * g.magnitude).expand(v.shape[0], d).contiguous()
    if g.type == GravityType.PointSource:
        origin = torch.as_tensor(g.origin, dtype=v.dtype, device=v.device)[:d]
        direction = origin - currentState.positions
        norm = torch.linalg.vector_norm(direction, dim=1, keepdim=True)
        return direction / (norm + 1e-8) * g.magnitude
    raise NotImplementedError(f"gravity type {g.type} is not on the GPU path")


def _zero_surface(S) -> None:
    """detectFreeSurface with an inactive configuration (surfaceDetection/wrapper.py:93-96)."""
    S.surfaceIndicators = torch.zeros(S.positions.shape[0], dtype=torch.int32, device=S.positions.device)
    S.surfaceNormals = torch.zeros_like(S.positions)
    S.surfaceLambdas = None


def _surface(S, config, schemeConfig, adjacency) -> None:
    """Step 8 of dfsph.py:72-77 / deltaSPH.py:86-91: indicators = (dilated mask > 0.5)."""
    sd = getattr(schemeConfig, "surfaceDetectionConfig", None)
    if sd is None or not sd.active:
        _zero_surface(S)
        return
    fsm, fs, n, _, lmin = detectFreeSurface(S, config, schemeConfig, sd, adjacency, returnNormals=True)
    S.surfaceIndicators = (fs > 0.5).to(torch.int32)
    S.surfaceNormals = n
    S.surfaceLambdas = lmin


def _passive(S) -> torch.Tensor:
    return torch.zeros(S.densities.shape, device=S.densities.device, dtype=torch.bool)


def dfsph_step(system, dt, config, schemeConfig, verbose: bool = False):
    """schemes/dfsph.py:13-218 on the GPU.  Returns (update, adjacency, state, (errors, pressures))."""
    S = system.state
    nfw = _check_supported(S, schemeConfig, allow_walls=True)
    if nfw is not None:
        return _dfsph_step_walls(system, dt, config, schemeConfig, nfw)
    params = make_params(config)
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, system.adjacency)
    system.adjacency = adjacency
    if S.densities is None or not schemeConfig.solverConfig.integrateRho:
        S.densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
    _surface(S, config, schemeConfig, adjacency)
    dvdt_diss, drhodt = ops.wc_visc_continuity(params, wc_params(schemeConfig), S.positions, S.supports, S.masses, S.densities,
                                               S.velocities, adjacency)
    dvdt = computeGravity(S, config, schemeConfig, adjacency)
    if S.pressures is None:
        S.pressures = torch.zeros_like(S.densities)
    dvdt_pressure, pressure, errors, pressures = solveDivergenceFree(S, config, schemeConfig, adjacency, dvdt + dvdt_diss, dt)
    S.pressures = pressure
    update = IncompressibleSystemUpdate(dxdt=S.velocities.clone(), dvdt=dvdt + dvdt_diss + dvdt_pressure, drhodt=drhodt,
                                        passive=_passive(S))
    return update, adjacency, S, (errors, pressures)


def _dfsph_step_walls(system, dt, config, schemeConfig, nfw: int):
    """dfsph_step with wall particles and their ghost points (dfsph.py:27-126, 170-186).

    The fluid and wall particles (the first nfw) form the particle set of every pass
    that the reference runs over fluid and walls; the ghost points take part only in the
    mDBC density, whose Liu-Liu sums run over a second list built over every particle.
    Steps: gather density; mDBC wall density (density2025.py); wall velocities
    (mdbc/velocity.py); surface detection; velocity diffusion and continuity; gravity; the
    no-penetration shift over dt (wp_nopenshift.py); the divergence-free solve, in which
    the walls take part with their mDBC densities and zero velocities; and the update,
    zero for walls and ghosts (dfsph.py:183-186)."""
    S = system.state
    n = int(S.positions.shape[0])
    params = make_params(config)
    vs = config.verletScale
    adjacency = ops.buildVerletList(S.positions[:nfw], S.supports[:nfw], params, vs, system.adjacency)
    key = (S.positions.device.index, n)
    full = ops.buildVerletList(S.positions, S.supports, params, vs, _GHOST_LISTS.get(key))
    _GHOST_LISTS.clear()
    _GHOST_LISTS[key] = full
    system.adjacency = adjacency
    rho0 = float(schemeConfig.fluid.restDensity)
    if S.densities is None or not schemeConfig.solverConfig.integrateRho:
        rho = ops.density(params, S.positions[:nfw], S.supports[:nfw], S.masses[:nfw], adjacency, SupportScheme.Gather)
        tail = S.densities[nfw:] if S.densities is not None else torch.full((n - nfw,), rho0, device=rho.device, dtype=rho.dtype)
        S.densities = torch.cat([rho, tail])
    S.densities = ops.mdbc_density(params, S.positions, S.supports, S.masses, S.densities, S.kinds, S.ghostIndices, S.ghostOffsets,
                                   full, rho0, float(schemeConfig.fluid.fixedSoundSpeed), _gravity_vector(schemeConfig, int(config.dim)))
    S.velocities = computeBoundaryVelocities(S, config, schemeConfig, adjacency)
    Hd = _head(S, nfw)
    _surface(Hd, config, schemeConfig, adjacency)
    S.surfaceIndicators, S.surfaceNormals = _pad(Hd.surfaceIndicators, n), _pad(Hd.surfaceNormals, n)
    S.surfaceLambdas = _pad(Hd.surfaceLambdas, n)
    dvdt_diss, drhodt = ops.wc_visc_continuity(params, wc_params(schemeConfig), Hd.positions, Hd.supports, Hd.masses, Hd.densities,
                                               Hd.velocities, adjacency)
    dvdt = computeGravity(Hd, config, schemeConfig, adjacency)
    nopen = ops.mdbc_nopen_shift(params, Hd.positions, Hd.supports, Hd.masses, Hd.velocities, Hd.kinds, Hd.ghostOffsets, adjacency)
    dvdt = dvdt + nopen / dt
    if S.pressures is None:
        S.pressures = torch.zeros_like(S.densities)
    Hd.pressures = S.pressures[:nfw]
    dvdt_pressure, pressure, errors, pressures = solveDivergenceFree(Hd, config, schemeConfig, adjacency, dvdt + dvdt_diss, dt)
    S.pressures = _pad(pressure, n)
    fluid = (Hd.kinds == 0)[:, None]
    zero_v = torch.zeros_like(Hd.velocities)
    update = IncompressibleSystemUpdate(dxdt=_pad(torch.where(fluid, Hd.velocities, zero_v), n),
                                        dvdt=_pad(torch.where(fluid, dvdt + dvdt_diss + dvdt_pressure, zero_v), n),
                                        drhodt=_pad(torch.where(fluid[:, 0], drhodt, torch.zeros_like(drhodt)), n),
                                        passive=_passive(S))
    return update, adjacency, S, (errors, pressures)


def deltaSPH_step(system, dt, config, schemeConfig, verbose: bool = False):
    """schemes/deltaSPH.py:11-208 on the GPU.  Returns (update, adjacency, state)."""
    S = system.state
    _check_supported(S, schemeConfig)
    params = make_params(config)
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, system.adjacency)
    system.adjacency = adjacency
    if S.densities is None:
        S.densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
    _surface(S, config, schemeConfig, adjacency)
    dvdt_rhs, drhodt, _, P = ops.deltasph_rhs(params, wc_params(schemeConfig), S.positions, S.supports, S.masses, S.densities,
                                              S.velocities, adjacency, S.surfaceIndicators)
    S.pressures = P
    update = WeaklyCompressibleSystemUpdate(dxdt=S.velocities.clone(), dvdt=dvdt_rhs + computeGravity(S, config, schemeConfig, adjacency),
                                            drhodt=drhodt, passive=_passive(S))
    return update, adjacency, S


def weaklyCompressibleStepLimit(H: float, c_s: float, nu: float, kernel_scale: float, cfl: float, compParams,
                                max_accel: Optional[float] = None, max_dt: float = float("inf")) -> float:
    """The limit of modules/timestep/weaklyCompressible.py:13-88 for one simulation as host
    floats: min over the enabled constraints of 0.125 H^2 / nu / k (viscous), cfl H / c_s / k
    (acoustic) and, when max_accel is given, 0.25 sqrt(H / (max_accel + 1e-7)) / k, with H
    the smallest support and k the kernel scale (computeTimestep's rule before its clamps)."""
    new_dt = max_dt
    if compParams.dt_viscosityConstraint:
        new_dt = 0.125 * H * H / nu / kernel_scale
    if compParams.dt_accelerationConstraint and max_accel is not None:
        new_dt = min(new_dt, 0.25 * math.sqrt(H / (max_accel + 1e-7)) / kernel_scale)
    if compParams.dt_acousticConstraint:
        new_dt = min(new_dt, cfl * H / c_s / kernel_scale)
    return new_dt


def computeTimestep(system, config, compParams, dt=None, systemUpdate=None):
    """modules/timestep/weaklyCompressible.py:13-88 (Sun et al., the delta-SPH time step):
    the viscous limit 0.125 H^2 / nu / k, the acoustic limit CFL H / c0 / k and the
    acceleration limit 0.25 sqrt(H / (max|dv/dt| + 1e-7)) / k, with H the smallest
    support and k the kernel scale, each applied when its flag is set; then clamped to
    [minDt, maxDt] and to dtGrowthFactor * dt when it would grow.  nu is
    alpha c0 H / (2 (d + 2)) for the inviscid form.  Returns a 0-d device tensor, as the
    reference does."""
    if not config.adaptiveDt:
        return dt
    S = system.state
    dev, dtype = S.supports.device, S.supports.dtype
    H = ops.minmax(S.supports)[0]
    scale = float(sphKernelScale(config.kernel, int(config.dim)))
    d = compParams.diffusionParams
    c_s = float(compParams.fluid.fixedSoundSpeed)
    dim = int(S.positions.shape[1])
    nu = d.inviscidAlpha * c_s * H / (2 * (dim + 2)) if d.inviscid else torch.tensor(float(d.viscidNu), dtype=dtype, device=dev)
    dt_v = 0.125 * H * H / nu / scale
    dt_c = float(config.cflFactor) * H / c_s / scale
    vel = getattr(systemUpdate, "velocities", None) if systemUpdate is not None else None
    if vel is not None:
        # the reference drops NaN components before taking the largest norm
        finite = vel[~torch.isnan(vel)]
        max_accel = torch.max(torch.linalg.norm(finite, dim=-1))
        dt_a = 0.25 * torch.sqrt(H / (max_accel + 1e-7)) / scale
    else:
        dt_a = torch.tensor(float(config.maxDt), dtype=dtype, device=dev)
    prev = torch.tensor(float(config.maxDt) if dt is None else float(dt), dtype=dtype, device=dev)
    new_dt = prev
    if compParams.dt_viscosityConstraint:
        new_dt = dt_v
    if compParams.dt_accelerationConstraint:
        new_dt = torch.minimum(new_dt, dt_a)
    if compParams.dt_acousticConstraint:
        new_dt = torch.minimum(new_dt, dt_c)
    new_dt = torch.clamp(new_dt, min=float(config.minDt), max=float(config.maxDt))
    if bool(new_dt > prev):
        new_dt = torch.clamp(new_dt, max=float(config.dtGrowthFactor) * prev)
    return new_dt


def setupWeaklyCompressibleTimestep(config, schemeConfig, compressibleSystem, targetDt, verbose: bool = True):
    """modules/timestep/weaklyCompressible.py:90-116: the sound speed c0 for which the
    acoustic limit at the 2D support of spacing config.dx equals targetDt,
    c0 = 0.3 H2(dx) / k2 / targetDt (H2 and k2 evaluated in two dimensions, as the reference
    does for every dimension); sets schemeConfig.fluid.fixedSoundSpeed and config.dt =
    targetDt.  Returns (c0, dt)."""
    dx = float(config.dx)
    c0 = 0.3 * float(volumeToSupportHelper(dx ** 2, config.targetNeighbors, 2)) / float(sphKernelScale(config.kernel, 2)) / targetDt
    if verbose:
        print(f"Computed c0: {c0}, target c0: {schemeConfig.fluid.fixedSoundSpeed}, diff: {abs(c0 - schemeConfig.fluid.fixedSoundSpeed)}")
    schemeConfig.fluid.fixedSoundSpeed = c0
    dt = targetDt
    uMax = torch.max(torch.linalg.norm(compressibleSystem.state.velocities, dim=1))
    if verbose:
        print(f"Computed dt: {dt}, target dt: {targetDt}, diff: {abs(dt - targetDt)}")
        print(f"Max velocity: {uMax}, CFL: {uMax * dt / dx}, Max Mach: {uMax / c0}")
    if uMax / c0 > 0.1:
        print(f"Warning: Max Mach number ({uMax / c0:.2f}) is greater than 0.1, which may lead to instability in the simulation. "
              "Consider changing the relevant parameters.")
    config.dt = dt
    return c0, dt


def _add_positions(params, x, dx, dim) -> torch.Tensor:
    """x + dx, wrapped into the periodic axes of the domain."""
    return ops.rk_combine(params, x, [dx.contiguous()], [1.0], 1.0, dim)


def solveShifting(state, config, schemeConfig, adjacency, dt):
    """modules/shifting/wrapper.py:20-135 for a domain without free surface: per iteration
    the Verlet list at the shifted positions and one delta-plus shift
    (modules/shifting/delta.py), zero for kinds != 0.  Returns (dx, adjacency): the summed
    shift, the state itself left unchanged."""
    sp = schemeConfig.shiftProperties
    sd = getattr(schemeConfig, "surfaceDetectionConfig", None)
    if sd is not None and sd.active:
        raise NotImplementedError("the free-surface treatment of the shift (shifting/wrapper.py:71-120) is not on the GPU path")
    params = make_params(config)
    dim = int(config.dim)
    c0 = schemeConfig.fluid.fixedSoundSpeed if schemeConfig.fluid.fixedSoundSpeed is not None else 1.0
    x = state.positions
    dx = torch.zeros_like(x)
    for _ in range(int(sp.iterations)):
        adjacency = ops.buildVerletList(x, state.supports, params, config.verletScale, adjacency)
        rho = (ops.density(params, x, state.supports, state.masses, adjacency, SupportScheme.Gather) if sp.summationDensity
               else state.densities)
        upd = ops.delta_shift(params, x, state.supports, state.masses, rho, state.velocities, state.kinds, adjacency, sp.CFL, c0)
        dx = dx + upd
        x = _add_positions(params, x, upd, dim)
    return dx, adjacency


def finalize_incompressible(system, initialState, dt, returnValues, updateValues, config, schemeConfig):
    """systems/incompressible.py:71-277.  The delta-plus shift the reference computes when
    shiftProperties.active (:134-209) is not applied anywhere (the lines that would apply
    it, :262-267, are commented out), so it is not evaluated here.  With wall particles the
    density solve runs over the fluid and wall particles and only fluid particles move:
    the reference moves every particle by dt^2 a_p (:250-255), walls included, which would
    carry the tank's walls along with the solve."""
    last = returnValues[-1][1]
    S = system.state
    for name in _LAST_STAGE_FIELDS + ("densities",):
        setattr(S, name, getattr(last, name))
    params = make_params(config)
    nfw = _wall_layout(S, True)
    if nfw is not None:
        n = int(S.positions.shape[0])
        adjacency = ops.buildVerletList(S.positions[:nfw], S.supports[:nfw], params, config.verletScale, returnValues[-1][0])
        rho = ops.density(params, S.positions[:nfw], S.supports[:nfw], S.masses[:nfw], adjacency, SupportScheme.Gather)
        S.densities = torch.cat([rho, S.densities[nfw:]])
        Hd = _head(S, nfw)
        zero = torch.zeros_like(Hd.velocities)
        dvdt_incomp, _, errors_incomp, pressures_incomp = solveIncompressible(Hd, config, schemeConfig, adjacency, zero, dt)
        shift = torch.where((Hd.kinds == 0)[:, None], (dt * dt) * dvdt_incomp, zero)
        S.positions = torch.cat([_add_positions(params, Hd.positions, shift, int(config.dim)), S.positions[nfw:]])
        system.adjacency = adjacency
        returnValues[-1] = tuple(returnValues[-1][:3]) + ((errors_incomp, pressures_incomp),)
        return system
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, returnValues[-1][0])
    S.densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
    zero = torch.zeros_like(S.velocities)
    dvdt_incomp, _, errors_incomp, pressures_incomp = solveIncompressible(S, config, schemeConfig, adjacency, zero, dt)
    # positions += dt^2 a_p of the density solve (:250-255)
    S.positions = _add_positions(params, S.positions, (dt * dt) * dvdt_incomp, int(config.dim))
    system.adjacency = adjacency
    returnValues[-1] = tuple(returnValues[-1][:3]) + ((errors_incomp, pressures_incomp),)
    return system


def finalize_weakly_compressible(system, initialState, dt, returnValues, updateValues, config, schemeConfig):
    """systems/weaklyCompressible.py:73-200: the last stage's fields, the delta-plus shift
    (computed before the density update, added after it), and the exponential density
    update rho0 exp(dt drhodt / rho) from the last stage (:179-186)."""
    last = returnValues[-1][1]
    S = system.state
    for name in _LAST_STAGE_FIELDS:
        setattr(S, name, getattr(last, name))
    sp = schemeConfig.shiftProperties
    adjacency = returnValues[-1][0]
    dx = None
    if sp.active:
        if sp.correctdrhodt or sp.correctdvdt:
            raise NotImplementedError("the shift corrections of drho/dt and dv/dt are not on the GPU path (off by default)")
        dx, adjacency = solveShifting(S, config, schemeConfig, adjacency, dt)
    rho_mid = last.densities
    S.densities = initialState.state.densities * torch.exp(dt * updateValues[-1].drhodt / rho_mid)
    if dx is not None:
        S.positions = _add_positions(make_params(config), S.positions, dx, int(config.dim))
    system.adjacency = adjacency
    return system
