"""Case builders for the synthetic benchmark workloads.

``buildSod1D`` follows src/warpSPH/caseUtils/compressible/sod/sod.py:21-236: the
mirrored periodic layout on [-1, 1] (dense left state for |x| < 1/2, the right state
with samplingRatio-times coarser spacing and equal masses outside), supports from 16
gather Newton iterations, the ideal-gas state from the prescribed density, and the
logistic ramp of the internal energy across both interfaces when ``smoothIC``.

``buildPointCloud`` follows src/warpSPH/sample/regular.py:6-50 (cell-centred lattice
for periodic axes, 'xy' meshgrid order).  ``buildSedov`` follows
src/warpSPH/caseUtils/compressible/sedov/initial.py:24-218, including the 'hat'
initialisation that the reference leaves unimplemented (initial.py:144-153 raises):
the energy E0 is distributed over the particles with weights W(|x_i|, H_i) (the
kernel evaluated at the centre with each particle's own support), normalised to
sum to one, on top of the background pressure p0.
"""
from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np
import torch

from . import ops
from .configurations import CompressibleSPHConfig, SimulationConfig, make_params
from .core import DomainDescription, SupportScheme, buildDomainDescription, kernel_constants, volumeToSupportHelper
from .enumTypes import AdaptiveSupportScheme
from .schemes import computeTimestep, evaluateOptimalSupport


def buildPointCloud(nx, domain, targetNeighbors=16, device=None, dtype=torch.float32):
    dmin, dmax, per = domain.host()
    dim = domain.dim
    dxs = [(dmax[d] - dmin[d]) / (nx if per[d] else nx - 1) for d in range(dim)]
    dx = min(dxs)
    spaces = []
    for d in range(dim):
        l = dmax[d] - dmin[d]
        nd = int(math.ceil(l / dx - 1e-9))
        off = dx / 2 if per[d] else 0.0
        spaces.append(torch.linspace(dmin[d] + off, dmax[d] - off, nd, device=device, dtype=torch.float64))
    grid = torch.meshgrid(*spaces, indexing="xy")
    pos = torch.stack([g.flatten() for g in grid], dim=1).to(dtype)
    area = dx ** dim
    support = volumeToSupportHelper(area, targetNeighbors, dim)
    return pos.contiguous(), torch.full((pos.shape[0],), float(support), device=device, dtype=dtype), area, support


def kernel_weight(kernel, dim, r: torch.Tensor, H: torch.Tensor) -> torch.Tensor:
    """W(r, H) of the Wendland family and of B7 on torch tensors (set-up only)."""
    C, _ = kernel_constants(kernel, dim)
    q = (r / H).clamp(max=1.0)
    t = 1 - q
    k = kernel.value
    if k == 4:
        tp = lambda a: (a - q).clamp(min=0.0) ** 7
        return C / H ** dim * (tp(1.0) - 8 * tp(0.75) + 28 * tp(0.5) - 56 * tp(0.25))
    if k == 1:
        f = t ** 3 * (1 + 3 * q) if dim == 1 else t ** 4 * (1 + 4 * q)
    elif k == 2:
        f = t ** 5 * (1 + 5 * q + 8 * q * q) if dim == 1 else t ** 6 * (1 + 6 * q + 35 / 3 * q * q)
    else:
        f = t ** 7 * (1 + 7 * q + 19 * q * q + 21 * q ** 3) if dim == 1 else t ** 8 * (1 + 8 * q + 25 * q * q + 32 * q ** 3)
    return C / H ** dim * f


def buildSedov(SimulationSystem, SimulationState, config: SimulationConfig, nx: int = 200, dim: int = 2,
               domainExtent: float = 1.0, periodicDomain: bool = True, rho0: float = 1.0, E0: float = 1.0,
               p0: float = 1e-6, initialization: str = "hat", gamma: float = 5 / 3, kernel=None, targetNeighbors=32,
               device=None, dtype=torch.float32, supportIterations: int = 16, computeDt: bool = True):
    """Sedov-Taylor blast: lattice of nx^dim particles in [-L/2, L/2]^dim, density rho0,
    pressure p0, energy E0 deposited at the origin."""
    device = device or config.device
    kernel = kernel or config.kernel
    domain = buildDomainDescription(domainExtent, dim, periodic=periodicDomain, device=device, dtype=dtype)
    config.domain = domain
    config.dim = dim
    config.kernel = kernel
    config.targetNeighbors = targetNeighbors
    pos, H, area, support = buildPointCloud(nx, domain, targetNeighbors, device=device, dtype=dtype)
    n = pos.shape[0]
    masses = torch.full((n,), float(area * rho0), device=device, dtype=dtype)
    ones = torch.ones(n, device=device, dtype=dtype)
    state = SimulationState(positions=pos, velocities=torch.zeros_like(pos), supports=H, masses=masses, densities=ones.clone(),
                            kinds=torch.zeros(n, device=device, dtype=torch.int32),
                            materials=torch.zeros(n, device=device, dtype=torch.int32),
                            UIDs=torch.arange(n, device=device, dtype=torch.int32), UIDcounter=n,
                            divergence=torch.zeros(n, device=device, dtype=dtype), alpha0s=ones.clone(), alphas=ones.clone())
    params = make_params(config)
    adj = ops.buildVerletList(state.positions, state.supports, params, config.verletScale)
    state.densities = ops.density(params, state.positions, state.supports, state.masses, adj, SupportScheme.Gather)
    setup = CompressibleSPHConfig(adaptiveSupportIterations=supportIterations, adaptiveSupportThreshold=1e-3,
                                  adaptiveSupportScheme=AdaptiveSupportScheme.Monaghan, gamma=gamma)
    rho, Hn, adj, *_ = evaluateOptimalSupport(state, config, setup, SupportScheme.Gather, adj)
    state.densities = rho
    state.supports = Hn
    u_bg = p0 / ((gamma - 1) * rho)
    if initialization == "hat":
        r = torch.linalg.norm(state.positions.double(), dim=-1)
        W = kernel_weight(kernel, dim, r, state.supports.double())
        W = W / W.sum()
        u = (u_bg.double() + E0 * W / state.masses.double()).to(dtype)
    elif initialization == "singular":
        r = torch.linalg.norm(state.positions, dim=-1)
        u = u_bg.clone()
        k = int(torch.argmin(r))
        u[k] += E0 / state.masses[k]
    else:
        raise ValueError(f"Unknown initialization {initialization}")
    state.internalEnergies = u.contiguous()
    state.entropies, state.pressures, state.soundspeeds = ops.eos_ideal_gas(make_params(config, setup), state.internalEnergies,
                                                                            state.densities)
    state.totalEnergies = state.internalEnergies * state.masses
    system = SimulationSystem(state=state, adjacency=adj, domain=domain)
    config.dx = float(area)
    if computeDt:
        config.dt = computeTimestep(system, config, setup, dt=config.dt)
    return system


class sodInitialState(NamedTuple):
    p: float
    rho: float
    v: float


def buildSod1D(SimulationSystem, SimulationState, samplingRatio: int, leftState: sodInitialState, rightState: sodInitialState,
               gamma: float, config: SimulationConfig, smoothIC: bool = False,
               adaptiveSupportScheme: AdaptiveSupportScheme = AdaptiveSupportScheme.Monaghan, smoothingSpacings: float = 0.5):
    """caseUtils/compressible/sod/sod.py:21-236.  config.nx dense particles on |x| < 1/2 and
    config.nx // samplingRatio coarse ones on 1/2 < |x| < 1 in the periodic domain
    config.domain = [-1, 1]; each half is a tube with reflecting walls at its ends.
    ``smoothingSpacings`` is the logistic ramp's scale in dense spacings (the reference's
    0.5, sod.py:173-174)."""
    nx = int(config.nx)
    dev, dtype = config.device, config.dtype
    actualRatio = nx / (nx // samplingRatio)
    unit = buildDomainDescription(1, config.dim, periodic=True, device=dev, dtype=dtype)
    pos_l, H_l, area_l, _ = buildPointCloud(nx, unit, config.targetNeighbors, device=dev, dtype=dtype)
    pos_r, H_r, area_r, _ = buildPointCloud(nx // samplingRatio, unit, config.targetNeighbors, device=dev, dtype=dtype)
    pos_r = pos_r.clone()
    neg = pos_r[:, 0] < 0
    pos_r[neg, 0] -= 0.5
    pos_r[~neg & (pos_r[:, 0] > 0), 0] += 0.5
    pos = torch.cat([pos_l, pos_r], 0).contiguous()
    nl, nr = pos_l.shape[0], pos_r.shape[0]
    tags = torch.cat([torch.zeros(nl, dtype=torch.int32, device=dev), torch.ones(nr, dtype=torch.int32, device=dev)])
    left = tags == 0
    leftMass = float(area_l) * leftState.rho
    rightMass = float(area_l) * rightState.rho * actualRatio
    masses = torch.where(left, leftMass, rightMass).to(dtype)
    supports = torch.where(left, float(H_l.min()), float(H_r.min())).to(dtype)
    densities = torch.where(left, leftState.rho, rightState.rho).to(dtype)
    velocities = torch.where(left[:, None], float(leftState.v), float(rightState.v)).to(dtype).contiguous()
    UIDs = torch.cat([torch.arange(nl, dtype=torch.int32, device=dev), torch.arange(nr, dtype=torch.int32, device=dev)])
    state = SimulationState(positions=pos, velocities=velocities, supports=supports, masses=masses, densities=densities,
                            kinds=torch.zeros_like(tags), materials=tags, UIDs=UIDs, UIDcounter=int(UIDs.max()) + 1,
                            divergence=torch.zeros_like(densities), alpha0s=torch.ones_like(densities),
                            alphas=torch.ones_like(densities))
    prescribed = densities.clone()
    compParams = CompressibleSPHConfig(gamma=gamma, adaptiveSupportCorrections=True, adaptiveSupportIterations=16,
                                       adaptiveSupportThreshold=1e-3, adaptiveSupportScheme=adaptiveSupportScheme)
    rho_opt, h_opt, adjacency, *_ = evaluateOptimalSupport(state, config, compParams, SupportScheme.Gather)
    state.supports = h_opt
    eosRho = rho_opt if smoothIC else prescribed
    P_initial = torch.where(left, leftState.p, rightState.p).to(dtype)
    u = 1 / (gamma - 1) * (P_initial / eosRho)
    if smoothIC:
        dx = float(pos_l[1, 0] - pos_l[0, 0]) * smoothingSpacings

        def ramped(a, b, x):
            return (a - b) / (torch.exp(x / dx) + 1) + b

        left_u = 1 / (gamma - 1) * (leftState.p / leftState.rho)
        right_u = 1 / (gamma - 1) * (rightState.p / rightState.rho)
        x = state.positions[:, 0]
        u = torch.where(x > 0.0, ramped(left_u, right_u, x - 0.5), u)
        u = torch.where(x < 0.0, ramped(right_u, left_u, x + 0.5), u).to(dtype)
    state.densities = eosRho.contiguous()
    state.internalEnergies = u.contiguous()
    state.entropies, state.pressures, state.soundspeeds = ops.eos_ideal_gas(make_params(config, compParams), state.internalEnergies,
                                                                            state.densities)
    state.totalEnergies = (state.internalEnergies + 0.5 * (state.velocities ** 2).sum(-1)) * state.masses
    adjacency = ops.buildVerletList(state.positions, state.supports, make_params(config), 2 ** (1 / config.dim))
    system = SimulationSystem(state=state, adjacency=adjacency, domain=config.domain)
    compParams.gamma = gamma
    config.dx = float(masses.min())
    config.dt = computeTimestep(system, config, compParams, dt=None)
    return system


def tank_particles(dim: int, dx: float, column, tank, layers: int = 3, jitter: float = 0.0, seed: int = 0):
    """The particles of a dam break in an open-topped box tank (numpy, FP32).

    The tank's interior is [0, tank[a]] along every axis; axis 1 is vertical and the top is
    open.  The fluid column fills [0, column[a]] in the corner at the origin on the
    cell-centred lattice of spacing dx (optionally jittered by jitter * dx).  The walls are
    `layers` lattice layers outside the floor and the side walls, up to the tank's height.
    Each wall particle has one ghost point, its mirror image through the closest point of
    the interior box: x_g = 2 c(x_b) - x_b, which for the reference's SDF construction
    (rigidBody/ghostParticles.py:30-54, offset = (d - min(-d, 1.5 H)) n) is the same point
    whenever the wall depth is below 1.5 supports.  Returns (fluid [nf, d], walls [nw, d],
    ghosts [nw, d])."""
    rng = np.random.default_rng(seed)
    col = [int(round(c / dx)) for c in column]
    axes = [(np.arange(c) + 0.5) * dx for c in col]
    grids = np.meshgrid(*axes, indexing="ij")
    fluid = np.stack([g.ravel() for g in grids], 1)
    if jitter > 0:
        fluid = fluid + jitter * dx * (rng.random(fluid.shape) - 0.5)
    ncell = [int(round(t / dx)) for t in tank]
    waxes = []
    for a in range(dim):
        hi = ncell[a] if a == 1 else ncell[a] + layers
        waxes.append((np.arange(-layers, hi) + 0.5) * dx)
    wg = np.meshgrid(*waxes, indexing="ij")
    pts = np.stack([g.ravel() for g in wg], 1)
    lo = np.zeros(dim)
    hi = np.asarray(tank[:dim], dtype=np.float64)
    outside = np.any((pts < lo) | (pts > hi), axis=1)
    walls = pts[outside]
    closest = np.clip(walls, lo, hi)
    ghosts = 2 * closest - walls
    return fluid.astype(np.float32), walls.astype(np.float32), ghosts.astype(np.float32)


def buildDamBreak(SimulationSystem, SimulationState, config: SimulationConfig, dx: float, column=(0.5, 1.0, 0.5),
                  tank=(1.6, 1.2, 0.6), layers: int = 3, rho0: float = 1.0, jitter: float = 0.0, seed: int = 0, device=None,
                  dtype=torch.float32):
    """A dam break with mDBC walls in the layout of the reference's
    initializeSimulation / addBoundaryGhostParticles (initializers/weaklyCompressible.py:230,
    rigidBody/ghostParticles.py:6-79): fluid (kind 0), then walls (kind 1), then one ghost
    point per wall particle (kind 2); ghostIndices link a wall particle and its ghost,
    ghostOffsets hold x_wall - x_ghost for the wall particle and the negative for its ghost.
    Masses rho0 dx^d, supports from config.targetNeighbors, densities rho0, at rest.  Sets
    config.domain to a non-periodic box around the tank (open above the tank's top)."""
    dim = int(config.dim)
    device = device or config.device
    fluid, walls, ghosts = tank_particles(dim, dx, column[:dim], tank[:dim], layers, jitter, seed)
    nf, nw = len(fluid), len(walls)
    x = np.concatenate([fluid, walls, ghosts])
    n = len(x)
    kinds = np.concatenate([np.zeros(nf), np.ones(nw), np.full(nw, 2)]).astype(np.int32)
    gidx = np.full(n, -1, np.int64)
    gidx[nf:nf + nw] = np.arange(nf + nw, n)
    gidx[nf + nw:] = np.arange(nf, nf + nw)
    goff = np.zeros_like(x)
    goff[nf:nf + nw] = walls - ghosts
    goff[nf + nw:] = ghosts - walls
    pad = (layers + 2) * dx
    lo = [-pad] * dim
    hi = [t + pad for t in tank[:dim]]
    hi[1] = tank[1] + 2.0 * tank[1]          # room for the splash above the open top
    config.domain = DomainDescription(torch.tensor(lo, device=device, dtype=dtype), torch.tensor(hi, device=device, dtype=dtype),
                                      torch.zeros(dim, dtype=torch.bool, device=device), dim)
    H = float(volumeToSupportHelper(dx ** dim, config.targetNeighbors, dim))
    t = lambda a, dt_=dtype: torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dt_)
    state = SimulationState(positions=t(x), velocities=torch.zeros((n, dim), device=device, dtype=dtype),
                            supports=torch.full((n,), H, device=device, dtype=dtype),
                            masses=torch.full((n,), rho0 * dx ** dim, device=device, dtype=dtype),
                            densities=torch.full((n,), rho0, device=device, dtype=dtype), kinds=t(kinds, torch.int32),
                            materials=torch.zeros(n, dtype=torch.int32, device=device),
                            UIDs=torch.arange(n, dtype=torch.int64, device=device), UIDcounter=n,
                            ghostIndices=t(gidx, torch.int64), ghostOffsets=t(goff))
    return SimulationSystem(state=state, adjacency=None, domain=config.domain)
