"""State / system containers with the reference's field names.

CompSPHState / CompSPHSystem follow src/warpSPH/systems/compSPH.py:7-129 and
CompressibleSystemUpdate follows systems/compressibleMonaghan.py:31-37.  Fields the
reference tags ``integrated(...)`` (positions, velocities, internalEnergies) are
advanced by the integrator; the others are recomputed by the step function.
``finalize`` is the compatible-energy update of systems/compSPH.py:87-129, done on
the GPU by sph_finalize_compatible_energy.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Any, List, Optional

import torch

from .core import AdjacencyList, DomainDescription

INTEGRATED_FIELDS = ("positions", "velocities", "internalEnergies")


@dataclass
class CompSPHState:
    positions: torch.Tensor
    velocities: torch.Tensor
    supports: torch.Tensor
    masses: torch.Tensor
    densities: torch.Tensor
    kinds: Optional[torch.Tensor] = None
    materials: Optional[torch.Tensor] = None
    UIDs: Optional[torch.Tensor] = None
    UIDcounter: int = 0
    internalEnergies: Optional[torch.Tensor] = None
    totalEnergies: Optional[torch.Tensor] = None
    entropies: Optional[torch.Tensor] = None
    pressures: Optional[torch.Tensor] = None
    soundspeeds: Optional[torch.Tensor] = None
    divergence: Optional[torch.Tensor] = None
    alpha0s: Optional[torch.Tensor] = None
    alphas: Optional[torch.Tensor] = None
    ap_ij: Optional[torch.Tensor] = None
    av_ij: Optional[torch.Tensor] = None
    f_ij: Optional[torch.Tensor] = None

    def initializeNewState(self) -> "CompSPHState":
        """Shallow copy: step functions replace tensors rather than writing into them."""
        return dataclasses.replace(self)

    def clone(self) -> "CompSPHState":
        kw = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            kw[f.name] = v.clone() if isinstance(v, torch.Tensor) else v
        return CompSPHState(**kw)


CompressibleState = CompSPHState


@dataclass
class CompressibleSystemUpdate:
    dxdt: torch.Tensor
    dvdt: torch.Tensor
    dudt: torch.Tensor
    dEdt: Optional[torch.Tensor] = None
    drhodt: Optional[torch.Tensor] = None
    passive: Optional[torch.Tensor] = None


@dataclass
class CompSPHSystem:
    state: CompSPHState
    adjacency: Optional[AdjacencyList] = None
    domain: Optional[DomainDescription] = None
    t: float = 0.0

    def initializeNewState(self, *args, verbose=False, **kwargs) -> "CompSPHSystem":
        return CompSPHSystem(state=self.state.initializeNewState(), adjacency=self.adjacency, t=self.t, domain=self.domain)

    def finalize(self, initialState: "CompSPHSystem", dt, returnValues, updateValues, weights, config, compParams, *args, **kwargs):
        """systems/compSPH.py:87-129: compatible-energy u, then copy the last stage's
        non-integrated fields."""
        from . import ops
        from .configurations import make_params
        self.adjacency = returnValues[-1][0]
        last: CompSPHState = returnValues[-1][1]
        S0 = initialState.state
        if getattr(compParams, "compatibleEnergy", False):
            params = make_params(config, compParams)
            stages = [(upd.dvdt, adj, st.f_ij, st.ap_ij, st.av_ij) for (adj, st), upd in zip(returnValues, updateValues)]
            u, _ = ops.finalize_compatible_energy(params, weights, dt, S0.velocities, S0.internalEnergies, stages)
            self.state.internalEnergies = u
        for name in ("supports", "densities", "totalEnergies", "entropies", "pressures", "soundspeeds", "divergence",
                     "alpha0s", "alphas"):
            setattr(self.state, name, getattr(last, name))
        dt_t = dt if isinstance(dt, torch.Tensor) else float(dt)
        updateValues[-1].dudt = (self.state.internalEnergies - S0.internalEnergies) / dt_t
        return self


CompressibleSystem = CompSPHSystem


# ------------------------------------------------------------------ incompressible and weakly compressible
@dataclass
class IncompressibleState:
    """systems/incompressible.py:15-35: positions, velocities and densities are integrated
    (dxdt, dvdt, drhodt); the rest is recomputed by the step function."""
    positions: torch.Tensor
    velocities: torch.Tensor
    supports: torch.Tensor
    masses: torch.Tensor
    densities: Optional[torch.Tensor] = None
    kinds: Optional[torch.Tensor] = None
    materials: Optional[torch.Tensor] = None
    UIDs: Optional[torch.Tensor] = None
    UIDcounter: int = 0
    pressures: Optional[torch.Tensor] = None
    soundspeeds: Optional[torch.Tensor] = None
    surfaceIndicators: Optional[torch.Tensor] = None
    surfaceNormals: Optional[torch.Tensor] = None
    surfaceLambdas: Optional[torch.Tensor] = None
    ghostIndices: Optional[torch.Tensor] = None
    ghostOffsets: Optional[torch.Tensor] = None

    def initializeNewState(self):
        return dataclasses.replace(self)

    def clone(self):
        kw = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            kw[f.name] = v.clone() if isinstance(v, torch.Tensor) else v
        return type(self)(**kw)


@dataclass
class IncompressibleSystemUpdate:
    """systems/incompressible.py:37-42."""
    dxdt: torch.Tensor
    dvdt: torch.Tensor
    drhodt: torch.Tensor
    passive: Optional[torch.Tensor] = None


_DENSITY_FIELDS = (("positions", "dxdt", True), ("velocities", "dvdt", False), ("densities", "drhodt", False))
_LAST_STAGE_FIELDS = ("supports", "pressures", "soundspeeds", "surfaceIndicators", "surfaceNormals", "surfaceLambdas")


@dataclass
class IncompressibleSystem:
    """systems/incompressible.py:47-277.  ``finalize`` copies the last stage's fields,
    rebuilds the Verlet list, recomputes the gather density and moves the particles by
    dt^2 times the density solve's pressure acceleration (:213-256)."""
    state: IncompressibleState
    adjacency: Optional[AdjacencyList] = None
    domain: Optional[DomainDescription] = None
    t: float = 0.0
    INTEGRATED = _DENSITY_FIELDS

    def initializeNewState(self, *args, verbose=False, **kwargs):
        return type(self)(state=self.state.initializeNewState(), adjacency=self.adjacency, t=self.t, domain=self.domain)

    def finalize(self, initialState, dt, returnValues, updateValues, weights, config, schemeConfig, *args, **kwargs):
        from . import wcsph
        return wcsph.finalize_incompressible(self, initialState, dt, returnValues, updateValues, config, schemeConfig)


WeaklyCompressibleState = IncompressibleState   # systems/weaklyCompressible.py:14-35 declares the same fields
WeaklyCompressibleSystemUpdate = IncompressibleSystemUpdate


@dataclass
class WeaklyCompressibleSystem(IncompressibleSystem):
    """systems/weaklyCompressible.py:43-200.  ``finalize`` copies the last stage's fields,
    applies the delta-plus shift when shiftProperties.active (computed before the density
    update, added to the positions after it) and sets the density by the exponential
    update rho0 exp(dt drhodt_last / rho_last) of the last stage (:179-186)."""

    def finalize(self, initialState, dt, returnValues, updateValues, weights, config, schemeConfig, *args, **kwargs):
        from . import wcsph
        return wcsph.finalize_weakly_compressible(self, initialState, dt, returnValues, updateValues, config, schemeConfig)
