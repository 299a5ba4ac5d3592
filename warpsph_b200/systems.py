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
