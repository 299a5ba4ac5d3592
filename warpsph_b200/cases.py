"""Case builders for the synthetic benchmark workloads.

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

import torch

from . import ops
from .configurations import CompressibleSPHConfig, SimulationConfig, make_params
from .core import SupportScheme, buildDomainDescription, kernel_constants, volumeToSupportHelper
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
    """W(r, H) of the Wendland family on torch tensors (set-up only)."""
    C, _ = kernel_constants(kernel, dim)
    q = (r / H).clamp(max=1.0)
    t = 1 - q
    k = kernel.value
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
