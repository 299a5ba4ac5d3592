"""CompSPH and Monaghan compressible step functions on the GPU.

``compSPH_step`` follows src/warpSPH/schemes/compSPH.py:22-215 call for call and
``compressibleSPH_Monaghan`` follows src/warpSPH/schemes/monaghan.py:13-158; every SPH
operation runs in libwarpsph_b200:

  adaptive support (Monaghan Newton)    compSPH.py:36      -> sph_adaptive_h_iter + sph_density_gather
  Verlet list                           compSPH.py:42      -> sph_neighbors_build (the list just built for the
                                                              optimal supports is valid and is kept)
  gather density                        compSPH.py:57      -> sph_density_gather
  ideal-gas EOS                         compSPH.py:81      -> sph_eos_ideal_gas
  Omega, Cullen divergence, continuity  compSPH.py:89,105,162 -> sph_compsph_prep (one pass)
  Cullen-Dehnen switch                  compSPH.py:105,153 -> sph_switch_cullen (R and v_sig)
  momentum + energy RHS, dE/dt          compSPH.py:113,132,170 -> sph_compsph_accel_dudt (one pass)
  energy partition f_ij                 compSPH.py:193     -> sph_compsph_balance

The Monaghan step runs sph_compsph_prep (Omega and continuity) and sph_monaghan_rhs
(pressure force, PdV work, viscosity, conductivity and viscous heating in one pass).
"""
from __future__ import annotations

import torch

from . import ops
from .configurations import CompressibleSPHConfig, CompSPHConfig, SimulationConfig, make_params
from .core import SupportScheme
from .enumTypes import AdaptiveSupportScheme, ViscositySwitch
from .schemes import evaluateOptimalSupport
from .systems import CompressibleSystemUpdate, CompSPHSystem


def _no_boundaries(compParams) -> None:
    if getattr(compParams, "boundaryConditions", None):
        raise NotImplementedError("boundary conditions are outside the GPU hot path")


def compSPH_step(system: CompSPHSystem, dt, config: SimulationConfig, compParams: CompSPHConfig, verbose: bool = False):
    """schemes/compSPH.py:22-215 on the GPU.  Returns (update, adjacency, state).

    The reference computes the first-step divergence with a call that references the
    grad-h state before it exists (compSPH.py:67-76); here that first divergence is the
    consistent continuity without grad-h terms, which is what the call asks for."""
    _no_boundaries(compParams)
    params = make_params(config, compParams)
    S = system.state
    # compSPH.py:36-47
    rho_opt, h_opt, adj_opt, *_ = evaluateOptimalSupport(S, config, compParams, SupportScheme.Gather, system.adjacency)
    S.supports = h_opt
    S.densities = rho_opt
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adj_opt)
    system.adjacency = adjacency
    # compSPH.py:57-66: the gather density at the optimal supports.  When the adaptive
    # support ran and the list is the one it ended with, that is the density it returned
    # (the same pass over the same rows, so the same values) and is not recomputed.
    if adjacency is not adj_opt or compParams.adaptiveSupportScheme == AdaptiveSupportScheme.NoScheme:
        S.densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, SupportScheme.Gather)
    if S.divergence is None:
        _, _, dr0 = ops.compsph_prep(params, S.positions, S.supports, S.masses, S.densities, S.velocities, adjacency,
                                     grad_h=False, want_div=False)
        S.divergence = dr0
    # compSPH.py:81-87
    S.entropies, S.pressures, S.soundspeeds = ops.eos_ideal_gas(params, S.internalEnergies, S.densities)
    # compSPH.py:89-103, the Cullen divergence (CullenDehnen2010.py:246-257) and compSPH.py:162-168
    switch = compParams.viscositySwitchParams.scheme
    cullen = switch == ViscositySwitch.CullenDehnen2010
    omega, div, drhodt = ops.compsph_prep(params, S.positions, S.supports, S.masses, S.densities, S.velocities, adjacency,
                                          grad_h=bool(compParams.adaptiveSupportCorrections), want_div=cullen)
    # compSPH.py:105-110 (computeCullenTerms returns the updated alpha0 as the alphas;
    # computeHopkinsTerms returns max(Xi alpha0, alpha_min))
    hopkins = switch == ViscositySwitch.CullenHopkins
    if cullen:
        alphas, _, _ = ops.switch_cullen(params, S.positions, S.supports, S.masses, S.densities, div, S.divergence, None,
                                         S.alpha0s, dt, adjacency, v=S.velocities, c=S.soundspeeds)
        S.alphas = alphas
    elif hopkins:
        S.alphas, hop_div, _, _ = ops.switch_hopkins_terms(params, S.positions, S.supports, S.masses, S.densities, S.velocities,
                                                           S.alpha0s, adjacency)
    elif switch != ViscositySwitch.NoneSwitch:
        raise NotImplementedError(f"viscosity switch {switch} is not implemented on the GPU path")
    # compSPH.py:113-149 and :170
    dvdt, dudt, dEdt, S.ap_ij, S.av_ij = ops.compsph_accel_dudt(params, S.positions, S.supports, S.masses, S.densities, S.velocities,
                                                                S.soundspeeds, S.alphas, S.pressures, omega, adjacency,
                                                                reference_layout=False)
    # compSPH.py:153-159 (computeCullenUpdate hands back the same alpha0; computeHopkinsUpdate
    # relaxes alpha0 with the divergence of the previous step, CullenHopkins.py:48-149)
    if cullen:
        S.alpha0s = S.alphas
    elif hopkins:
        S.alpha0s, _ = ops.switch_hopkins_update(params, S.positions, S.supports, S.velocities, S.soundspeeds, hop_div, S.divergence,
                                                 S.alpha0s, dt, adjacency)
    # compSPH.py:169
    S.divergence = -drhodt / S.densities
    update = CompressibleSystemUpdate(dxdt=S.velocities.clone(), dvdt=dvdt, dudt=dudt, drhodt=drhodt, dEdt=dEdt,
                                      passive=torch.zeros(S.densities.shape, device=S.densities.device, dtype=torch.bool))
    # compSPH.py:191-213
    S.f_ij = ops.compsph_balance(params, S.masses, S.densities, S.pressures, S.internalEnergies, S.velocities, dvdt, dt, adjacency,
                                 S.ap_ij, S.av_ij)
    return update, adjacency, S


def compressibleSPH_Monaghan(system: CompSPHSystem, dt, config: SimulationConfig, compParams: CompressibleSPHConfig,
                             verbose: bool = False):
    """schemes/monaghan.py:13-158 on the GPU.  Returns (update, adjacency, state).

    The reference's own step fails before its first pair pass (enforceDirichlet and
    computeMomentumConsistent are called with signatures they do not have,
    monaghan.py:50 and :95); this is the step those calls describe, with the continuity
    of modules/momentum/consistent.py."""
    _no_boundaries(compParams)
    params = make_params(config, compParams)
    S = system.state
    # monaghan.py:23-35
    rho_opt, h_opt, system.adjacency, *_ = evaluateOptimalSupport(S, config, compParams, SupportScheme.Gather, system.adjacency)
    S.supports = h_opt
    S.densities = rho_opt
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, system.adjacency)
    system.adjacency = adjacency
    # monaghan.py:39-48 (config.supportMode density)
    S.densities = ops.density(params, S.positions, S.supports, S.masses, adjacency, config.supportMode)
    # monaghan.py:51-57
    S.entropies, S.pressures, S.soundspeeds = ops.eos_ideal_gas(params, S.internalEnergies, S.densities)
    # monaghan.py:59-73 and :95-101
    omega, _, drhodt = ops.compsph_prep(params, S.positions, S.supports, S.masses, S.densities, S.velocities, adjacency,
                                        grad_h=bool(compParams.adaptiveSupportCorrections), want_div=False)
    # monaghan.py:77-143
    dvdt, dudt, dEdt, _ = ops.monaghan_rhs(params, S.positions, S.supports, S.masses, S.densities, S.velocities, S.internalEnergies,
                                           S.soundspeeds, S.alphas, S.pressures, omega, adjacency)
    update = CompressibleSystemUpdate(dxdt=S.velocities, dvdt=dvdt, dudt=dudt, drhodt=drhodt, dEdt=dEdt)
    return update, adjacency, S
