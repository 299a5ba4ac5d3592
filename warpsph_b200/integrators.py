"""Explicit Runge-Kutta integrators with the call shape of the reference's absent
warpSPHIntegrators package: ``getIntegrator(type).function(state=system, f=step_fn,
dt=..., config=..., compParams=...)`` returning an object with ``.state`` and
``.stages`` (call site examples/compressible/01-sod-shock-tube-1d.py:196-210).

Tableaux (restated; the package's own choice is not visible):
  explicitEuler       c=[0],          b=[1]
  rungeKutta2 (Heun)  c=[0,1],        a21=1,                    b=[1/2,1/2]
  rungeKutta4         c=[0,1/2,1/2,1], a21=a32=1/2, a43=1,       b=[1/6,1/3,1/3,1/6]
Stage s starts from a copy of stage s-1's state (so non-integrated fields such as
the supports carry over), with the system's integrated fields (positions, velocities
and internal energies, or densities for the incompressible and weakly compressible
systems) set to y0 + dt * sum_k a_sk K_k; periodic positions are wrapped into the
domain.  Step functions may return more than (update, adjacency, state); the extra
values are kept in the stage's return values for ``finalize``.  After
the last stage the integrated fields are y0 + dt * sum_s b_s K_s and the system's
``finalize`` runs (compatible energy).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, List

import torch

from . import ops
from .core import IntegrationSchemeType


@dataclass
class StageRecord:
    update: Any
    aux: Any


@dataclass
class IntegrationResult:
    state: Any
    stages: List[StageRecord] = field(default_factory=list)


_TABLEAUX = {
    IntegrationSchemeType.explicitEuler: ([[]], [1.0], [0.0]),
    IntegrationSchemeType.rungeKutta2: ([[], [1.0]], [0.5, 0.5], [0.0, 1.0]),
    IntegrationSchemeType.rungeKutta4: ([[], [0.5], [0.0, 0.5], [0.0, 0.0, 1.0]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0.0, 0.5, 0.5, 1.0]),
}


# (state field, update field, wrap periodic positions) of the compressible systems;
# other systems declare their own table as INTEGRATED
_COMPRESSIBLE_FIELDS = (("positions", "dxdt", True), ("velocities", "dvdt", False), ("internalEnergies", "dudt", False))


class RungeKuttaIntegrator:
    def __init__(self, scheme: IntegrationSchemeType):
        if scheme not in _TABLEAUX:
            raise ValueError(f"integration scheme {scheme} is not available on this path")
        self.scheme = scheme
        self.a, self.b, self.c = _TABLEAUX[scheme]

    def _combine(self, params, y0, ks, ws, dt, wrap_dim):
        pairs = [(k, w) for k, w in zip(ks, ws) if w != 0.0]
        return ops.rk_combine(params, y0, [k for k, _ in pairs], [w for _, w in pairs], dt, wrap_dim)

    def function(self, state, f, dt, config, compParams, verbose=False, **kwargs) -> IntegrationResult:
        from .configurations import make_params
        params = make_params(config, compParams)
        sys0 = state
        S0 = sys0.state
        dim = int(config.dim)
        updates, returnValues = [], []
        prev = S0
        adjacency = sys0.adjacency
        fields = getattr(type(sys0), "INTEGRATED", _COMPRESSIBLE_FIELDS)

        def advance(Ss, weights):
            # every integrated field in one launch (sph_rk_combine_fields), same arithmetic as
            # one rk_combine per field
            keep = [q for q, w in enumerate(weights) if w != 0.0]
            todo = [(name, getattr(S0, name), [getattr(updates[q], deriv) for q in keep], dim if wrap else 0)
                    for name, deriv, wrap in fields if getattr(S0, name) is not None]
            if len(todo) > 4 or any(k is None for _, _, ks, _ in todo for k in ks):
                for name, y0, _, wrap_dim in todo:
                    deriv = next(d for nm, d, _ in fields if nm == name)
                    setattr(Ss, name, self._combine(params, y0, [getattr(u, deriv) for u in updates], weights, dt, wrap_dim))
                return
            outs = ops.rk_combine_fields(params, [(y0, ks, wrap_dim) for _, y0, ks, wrap_dim in todo], [weights[q] for q in keep], dt)
            for (name, _, _, _), y in zip(todo, outs):
                setattr(Ss, name, y)

        for s in range(len(self.b)):
            Ss = prev.initializeNewState()
            if s > 0:
                advance(Ss, self.a[s])
            t_s = sys0.t + self.c[s] * (float(dt) if not isinstance(dt, torch.Tensor) else 0.0)
            sys_s = type(sys0)(state=Ss, adjacency=adjacency, domain=sys0.domain, t=t_s)
            out = f(sys_s, dt, config, compParams, verbose=verbose)
            update, adjacency, Sout = out[0], out[1], out[2]
            updates.append(update)
            returnValues.append(tuple(out[1:]))
            prev = Sout
        Sf = prev.initializeNewState()
        advance(Sf, self.b)
        new_sys = type(sys0)(state=Sf, adjacency=adjacency, domain=sys0.domain, t=sys0.t)
        new_sys.finalize(sys0, dt, returnValues, updates, self.b, config, compParams)
        new_sys.t = sys0.t + (float(dt) if not isinstance(dt, torch.Tensor) else 0.0)
        if isinstance(dt, torch.Tensor):
            new_sys.t_device = getattr(sys0, "t_device", 0.0) + dt
        stages = [StageRecord(update=u, aux=rv) for u, rv in zip(updates, returnValues)]
        return IntegrationResult(state=new_sys, stages=stages)


def getIntegrator(scheme: IntegrationSchemeType) -> RungeKuttaIntegrator:
    return RungeKuttaIntegrator(scheme)
