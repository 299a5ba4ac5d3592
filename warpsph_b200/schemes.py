"""Step functions and scheme dispatch.

``buildScheme`` returns the reference's 7-tuple (src/warpSPH/schemes/builder.py:11-36).
``crkSPH_step`` follows src/warpSPH/schemes/crkSPH.py:19-366 call for call, with
every SPH operation executed by libwarpsph_b200 kernels:

  adaptive support (Monaghan Newton)  crkSPH.py:40  -> sph_adaptive_h_iter + sph_density_gather
  Verlet list                         crkSPH.py:54  -> sph_neighbors_build (unchanged prior reused)
  CRK volume / coefficients / rho     crkSPH.py:61  -> sph_crk_volume + sph_crk_factors_eos
  ideal-gas EOS                       crkSPH.py:95  -> the epilogue of sph_crk_factors_eos
  CRK velocity gradient               crkSPH.py:158 -> sph_grad_v (also the Cullen divergence)
  viscosity switch                    crkSPH.py:195 -> sph_switch_cullen (R and v_sig) / sph_switch_balsara
  momentum + energy RHS, dE/dt        crkSPH.py:241,263,330 -> sph_crk_accel_dudt (one fused pass)
  energy partition f_ij               crkSPH.py:343 -> sph_compsph_balance
"""
from __future__ import annotations

from typing import Optional, Union

import torch

from . import ops
from .configurations import (CompSPHConfig, CompressibleSPHConfig, CRKSPHConfig, SimulationConfig, compressibleConfigToDict,
                             compSPHConfigToDict, crkSPHConfigToDict, dictToCompressibleConfig, dictToCompSPHConfig,
                             dictToCRKSPHConfig, make_params)
from .core import AdjacencyList, SupportScheme, sphKernel_xi, volumeToSupportHelper
from .enumTypes import AdaptiveSupportScheme, CompressibleSPHScheme, IncompressibleSPHScheme, ViscositySwitch, WeaklyCompressibleSPHScheme
from .systems import CompressibleState, CompressibleSystem, CompressibleSystemUpdate, CompSPHState, CompSPHSystem


# ------------------------------------------------------------------ adaptive support
def evaluateOptimalSupport(particleState, config: SimulationConfig, compParams: CompressibleSPHConfig,
                           supportScheme: SupportScheme = SupportScheme.Scatter, adjacency: Optional[AdjacencyList] = None,
                           iterations: Optional[int] = None, threshold: Optional[float] = None, final_density: bool = True):
    """modules/adaptiveSupport/optimalSupport.py:12-43 and optimalSupportMonaghan.py:62-150.

    Returns (densities, supports, adjacency, None, None); the Owen scheme
    (optimalSupportOwen.py:35-127, ``owen.py``) returns its psi and support histories in
    the last two.  NoScheme returns the state unchanged.  With ``final_density=False``
    the closing gather density at the new supports is not evaluated and the densities
    of the last Newton iteration are returned (for callers that overwrite them)."""
    scheme = compParams.adaptiveSupportScheme
    if scheme == AdaptiveSupportScheme.NoScheme:
        return particleState.densities, particleState.supports, adjacency, None, None
    if scheme == AdaptiveSupportScheme.Owen:
        from .owen import evaluateOptimalSupportOwen
        return evaluateOptimalSupportOwen(particleState, config, compParams, kernel_=config.kernel, adjacency=adjacency,
                                          supportScheme=supportScheme)
    if supportScheme != SupportScheme.Gather:
        raise NotImplementedError("adaptive support is implemented for the gather support scheme")
    params = make_params(config, compParams)
    nIter = compParams.adaptiveSupportIterations if iterations is None else iterations
    hThreshold = compParams.adaptiveSupportThreshold if threshold is None else threshold
    S = particleState
    hb = ops.minmax(S.supports)
    if nIter == 1:
        # One Newton iteration on a list kept from the previous stage: its validity for the
        # moved positions and for the new supports is checked by two launches whose verdicts
        # are read together, after the iteration has run on the kept rows.  When the first
        # verdict says stale the iteration is discarded and the path below runs as usual.
        spec = ops.speculative_refresh(S.positions, S.supports, params, config.verletScale, adjacency)
        if spec is not None:
            adj1, f1 = spec
            rho, h_new, _ = ops.adaptive_h_iter(params, S.positions, S.supports, S.masses, adj1, hb)
            spec2 = ops.speculative_refresh(S.positions, h_new, params, config.verletScale, adj1)
            stale1, stale2 = ops.verdicts_stale([f1, spec2[1]])
            if not stale1:
                S.densities, S.supports = rho, h_new
                adjacency = (spec2[0] if not stale2
                             else ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adj1))
                if not final_density:
                    return S.densities, S.supports, adjacency, None, None
                densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
                return densities, S.supports, adjacency, None, None
    for it in range(nIter):
        adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adjacency)
        rho, h_new, ratio = ops.adaptive_h_iter(params, S.positions, S.supports, S.masses, adjacency, hb)
        S.densities = rho
        S.supports = h_new
        if it == nIter - 1:
            break
        hb = ops.minmax(h_new)      # the support bounds of the next iteration
        if float((ratio - 1).abs().max()) < hThreshold:
            break
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adjacency)
    if not final_density:
        return S.densities, S.supports, adjacency, None, None
    densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
    return densities, S.supports, adjacency, None, None


def computeCRKFactors(particleState, config: SimulationConfig, adjacency: AdjacencyList, params=None):
    """warpSPHCore computeCRKFactors (schemes/crkSPH.py:61): (apparentVolume, densities, crkState)."""
    params = make_params(config) if params is None else params
    S = particleState
    V = ops.crk_volume(params, S.positions, S.supports, adjacency)
    crk, rho = ops.crk_factors(params, S.positions, S.supports, S.masses, V, adjacency)
    return V, rho, crk


def idealGasEOS(A, u, P, rho, gamma):
    """modules/eos/idealGas.py:6-38 for the (u, rho) case used by the step functions.
    Returns (A, u, P, c)."""
    if A is not None or P is not None or u is None:
        raise NotImplementedError("only the (u, rho) form of the ideal-gas EOS is on the GPU path")
    from ._capi import SphParams
    p = SphParams()
    p.dim, p.kernel, p.verlet_scale, p.gamma = 1, 1, 1.0, float(gamma)
    p.domain_max[0] = 1.0
    A_, P_, c_ = ops.eos_ideal_gas(p, u, rho)
    return A_, u, P_, c_


def computeTimestep(system, config: SimulationConfig, compParams: CompressibleSPHConfig, dt=None, device_result: bool = False):
    """modules/timestep/compressible.py:12-66: CFL dt = min_i cfl*min(H)/(c_i xi), clamped
    to [minDt, maxDt] and to dtGrowthFactor*config.dt when dt is given.  With
    device_result=True the value stays on the GPU (no host sync)."""
    if not config.adaptiveDt:
        if dt is not None:
            return dt
        raise ValueError("dt must be provided if adaptiveDt is False")
    params = make_params(config, compParams)
    prev = config.dt if (dt is not None and config.dt is not None) else None
    S = system.state
    t = ops.cfl_dt(params, S.supports, S.internalEnergies, dt_prev=prev)
    return t if device_result else float(t.item())


# ------------------------------------------------------------------ CRKSPH step
def crkSPH_step(system: CompSPHSystem, dt, config: SimulationConfig, compParams: CRKSPHConfig, verbose: bool = False):
    """schemes/crkSPH.py:19-366 on the GPU.  Returns (update, adjacency, state)."""
    if compParams.boundaryConditions:
        raise NotImplementedError("boundary conditions are outside the GPU hot path")
    params = make_params(config, compParams)
    S = system.state
    # crkSPH.py:40-42 (the densities are replaced by the CRK densities at crkSPH.py:61 before
    # anything reads them, so the closing density pass is skipped)
    rho_opt, h_opt, system.adjacency, *_ = evaluateOptimalSupport(S, config, compParams, SupportScheme.Gather, system.adjacency,
                                                                  final_density=False)
    S.supports = h_opt
    S.densities = rho_opt
    # crkSPH.py:54-59
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, system.adjacency)
    system.adjacency = adjacency
    # crkSPH.py:61 (computeCRKFactors) with crkSPH.py:95-101 (the ideal-gas EOS of the CRK
    # density) in the epilogue of the same pass
    V = ops.crk_volume(params, S.positions, S.supports, adjacency)
    crk, S.densities, S.entropies, S.pressures, S.soundspeeds = ops.crk_factors_eos(params, S.positions, S.supports, S.masses, V,
                                                                                   adjacency, S.internalEnergies)
    if S.divergence is None:
        S.divergence = torch.zeros_like(S.densities)
    switch = compParams.viscositySwitchParams.scheme
    cullen = switch == ViscositySwitch.CullenDehnen2010
    # crkSPH.py:158-172 (+ the Cullen divergence in the same pass)
    DvDx, drhodt, div_cd, _ = ops.grad_v(params, S.positions, S.supports, S.masses, S.densities, V, crk, S.velocities,
                                         S.soundspeeds, adjacency, cullen)
    # crkSPH.py:195-200 (v_sig over the Verlet set is computed inside the switch pass)
    if cullen:
        S.alphas, _, _ = ops.switch_cullen(params, S.positions, S.supports, S.masses, S.densities, div_cd, S.divergence, None,
                                           S.alpha0s, dt, adjacency, v=S.velocities, c=S.soundspeeds)
    elif switch == ViscositySwitch.Balsara1995:
        S.alphas = ops.switch_balsara(params, DvDx, S.soundspeeds)
    elif switch == ViscositySwitch.CullenHopkins:
        # crkSPH.py:195-200 (the alpha0 update of crkSPH.py:308-314 is commented out there)
        S.alphas, _, _, _ = ops.switch_hopkins_terms(params, S.positions, S.supports, S.masses, S.densities, S.velocities, S.alpha0s,
                                                     adjacency)
    elif switch != ViscositySwitch.NoneSwitch:
        raise ValueError(f"Unsupported viscosity switch scheme: {switch}")
    # crkSPH.py:241-284
    # (dE/dt = m v.dv/dt + m du/dt of crkSPH.py:330 is written by the same pass)
    dvdt, dudt, S.ap_ij, S.av_ij, dEdt = ops.crk_accel_dudt(params, S.positions, S.supports, S.masses, S.densities, V, crk,
                                                            S.velocities, S.soundspeeds, S.pressures, DvDx, adjacency,
                                                            want_dEdt=True, reference_layout=False)
    # crkSPH.py:324-337
    S.divergence = -drhodt / S.densities
    update = CompressibleSystemUpdate(dxdt=S.velocities, dvdt=dvdt, dudt=dudt, drhodt=drhodt, dEdt=dEdt, passive=None)
    # crkSPH.py:341-363
    S.f_ij = ops.compsph_balance(params, S.masses, S.densities, S.pressures, S.internalEnergies, S.velocities, dvdt, dt, adjacency,
                                 S.ap_ij, S.av_ij)
    return update, adjacency, S


def buildScheme(schemeName: Union[str, CompressibleSPHScheme]):
    """schemes/builder.py:11-36: (System, State, SchemeConfig, Update, step_fn, export_fn, import_fn)."""
    if (isinstance(schemeName, str) and schemeName == "crkSPH") or schemeName == CompressibleSPHScheme.CRKSPH:
        return (CompSPHSystem, CompSPHState, CRKSPHConfig, CompressibleSystemUpdate, crkSPH_step, crkSPHConfigToDict,
                dictToCRKSPHConfig)
    if (isinstance(schemeName, str) and schemeName == "compSPH") or schemeName == CompressibleSPHScheme.CompSPH:
        from .compsph import compSPH_step
        return (CompSPHSystem, CompSPHState, CompSPHConfig, CompressibleSystemUpdate, compSPH_step, compSPHConfigToDict,
                dictToCompSPHConfig)
    if (isinstance(schemeName, str) and schemeName == "MonaghanCompressibleSPH") or schemeName == CompressibleSPHScheme.Monaghan:
        from .compsph import compressibleSPH_Monaghan
        return (CompressibleSystem, CompressibleState, CompressibleSPHConfig, CompressibleSystemUpdate, compressibleSPH_Monaghan,
                compressibleConfigToDict, dictToCompressibleConfig)
    if (isinstance(schemeName, str) and schemeName == "deltaSPH") or schemeName == WeaklyCompressibleSPHScheme.deltaSPH:
        from .configurations import WeaklyCompressibleSPHConfig, dictToWeaklyCompressibleConfig, weaklyCompressibleConfigToDict
        from .systems import WeaklyCompressibleState, WeaklyCompressibleSystem
        from .wcsph import deltaSPH_step
        # the reference's builder hands out CompressibleSystemUpdate here (builder.py:26-29),
        # although deltaSPH_step itself builds WeaklyCompressibleSystemUpdate
        return (WeaklyCompressibleSystem, WeaklyCompressibleState, WeaklyCompressibleSPHConfig, CompressibleSystemUpdate,
                deltaSPH_step, weaklyCompressibleConfigToDict, dictToWeaklyCompressibleConfig)
    if (isinstance(schemeName, str) and schemeName in ("divergenceFree", "dfsph")) or schemeName == IncompressibleSPHScheme.divergenceFree:
        from .configurations import IncompressibleSPHConfig, dictToIncompressibleSPHConfig, incompressibleConfigToDict
        from .systems import IncompressibleState, IncompressibleSystem, IncompressibleSystemUpdate
        from .wcsph import dfsph_step
        return (IncompressibleSystem, IncompressibleState, IncompressibleSPHConfig, IncompressibleSystemUpdate, dfsph_step,
                incompressibleConfigToDict, dictToIncompressibleSPHConfig)
    raise ValueError(f"Scheme {schemeName} not recognized.")
