"""DFSPH pressure solves with the reference's module-level names and return values.

  computeAlpha                   modules/incompressible/wp_alpha.py:294-313
  computeMomentumIncompressible  modules/momentum/incompressible.py:9-34
  computePressureAccelIISPH      modules/pressure/iisph.py:7-24
  computePressureShiftIISPH      modules/incompressible/drift.py:38-57
  solveDivergenceFree            modules/incompressible/divergenceFree.py:23-139
  solveIncompressible            modules/incompressible/incompressible.py:21-143

Each solve is ONE persistent cooperative kernel (sph_dfsph_div_solve /
sph_dfsph_density_solve); the reference launches two kernels and synchronises with
the host every iteration.  ``errors`` and ``pressures`` are returned as the
reference's Python lists, which costs one device-to-host read after the solve;
pass ``device_history=True`` to get them as device tensors instead (no sync).
``initialPressure`` replaces the reference's initial guess (a learned warm start);
None keeps the reference's rule (0.75 p_prev, or 0 for the density solve).
"""
from __future__ import annotations

from typing import Any, Optional

import torch

from . import ops
from .configurations import SimulationConfig, jacobi_config, make_params
from .core import AdjacencyList, SupportScheme


def computeAlpha(currentState: Any, config: SimulationConfig, schemeConfig: Any, adjacency: AdjacencyList,
                 apparentVolumes: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Returns -alpha (the reference's sign).  apparentVolumes must be m/rho, which is
    what every reference call site passes."""
    S = currentState
    return ops.dfsph_alpha(make_params(config), S.positions, S.supports, S.masses, S.densities, adjacency)


def computeMomentumIncompressible(currentState: Any, config: SimulationConfig, schemeConfig: Any, adjacency: AdjacencyList,
                                  advectionVelocities: torch.Tensor) -> torch.Tensor:
    S = currentState
    return ops.incompressible_divergence(make_params(config), schemeConfig.fluid.restDensity, S.positions, S.supports, S.masses,
                                         S.densities, advectionVelocities.contiguous(), adjacency)


def computePressureAccelIISPH(state: Any, pressureValues: torch.Tensor, config: SimulationConfig,
                              supportScheme: SupportScheme = SupportScheme.Scatter, adjacency: Optional[AdjacencyList] = None):
    if supportScheme != SupportScheme.Scatter:
        raise NotImplementedError("the pressure acceleration is implemented for the scatter support scheme")
    return ops.pressure_accel_iisph(make_params(config), state.positions, state.supports, state.masses, state.densities,
                                    pressureValues.contiguous(), adjacency)


def computePressureShiftIISPH(state: Any, config: SimulationConfig, pressureAccels: torch.Tensor,
                              supportScheme: SupportScheme = SupportScheme.Scatter, adjacency: Optional[AdjacencyList] = None):
    return ops.pressure_shift_iisph(make_params(config), state.positions, state.supports, state.masses, state.densities,
                                    pressureAccels.contiguous(), adjacency)


def _solve(mode, particles, config, schemeConfig, adjacency, dvdt, dt, initialPressure, device_history):
    if adjacency is None:
        raise ValueError("an AdjacencyList is required")
    S = particles
    solver = (schemeConfig.solverConfig.divergenceFreeSolver if mode == ops.DIVERGENCE_FREE
              else schemeConfig.solverConfig.pressureSolver)
    cfg = jacobi_config(solver, schemeConfig.fluid.restDensity, learned_init=initialPressure is not None)
    p_init = initialPressure if initialPressure is not None else S.pressures
    if p_init is None:
        p_init = torch.zeros_like(S.densities)
    pr, acc, hist, iters, status = ops.jacobi_solve(make_params(config), mode, cfg, S.positions, S.supports, S.masses, S.densities,
                                                    S.velocities, dvdt.contiguous(), p_init.contiguous(), dt, adjacency)
    if device_history:
        return acc, pr, hist, (iters, status)
    k = int(iters.item())
    h = hist[:k].cpu().tolist()
    if int(status.item()) & 0x8:
        raise RuntimeError("Jacobi solve: a grid barrier timed out")
    errors = [row[0] for row in h]
    pressures = [(row[1], row[2], row[3]) for row in h]
    return acc, pr, errors, pressures


def solveDivergenceFree(particles: Any, config: SimulationConfig, schemeConfig: Any, adjacency: AdjacencyList, dvdt: torch.Tensor,
                        dt: float, verbose: bool = False, initialPressure: Optional[torch.Tensor] = None,
                        device_history: bool = False):
    """Returns (a_p, pressureB, errors, pressures) as the reference does."""
    return _solve(ops.DIVERGENCE_FREE, particles, config, schemeConfig, adjacency, dvdt, dt, initialPressure, device_history)


def solveIncompressible(particles: Any, config: SimulationConfig, schemeConfig: Any, adjacency: AdjacencyList, dvdt: torch.Tensor,
                        dt: float, verbose: bool = False, initialPressure: Optional[torch.Tensor] = None,
                        device_history: bool = False):
    """Returns (a_p, pressureB, errors, pressures) as the reference does."""
    return _solve(ops.DENSITY, particles, config, schemeConfig, adjacency, dvdt, dt, initialPressure, device_history)
