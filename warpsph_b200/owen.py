"""Owen adaptive support: the n_h(psi_H) table and the support iteration.

``owen_table`` restates the table generator of
src/warpSPH/modules/adaptiveSupport/wp_psi.py:8-114 (computePsi, the psi_H branch the
lookup uses) and owenLUT.py:55-62 (computeOwen: n_h in [nMin, nMax] with nLUT entries):
for each n_h the kernel gradient magnitude |dk/dq| C_d is summed over the radial shells
eta = 1/n_h, 2/n_h, ... < 1 of a lattice with n_h particles per support, weighted by the
shell's particle count (2 in 1D, 2 pi eta/d_eta in 2D, 4 pi eta^2/d_eta^2 in 3D), and
psi_H = sum^(1/d).  The arithmetic is FP32 step for step, as the Warp kernel runs at the
reference's single precision, and the table is kept in FP64 as owenLUT.py keeps it.

``evaluateOptimalSupportOwen`` follows optimalSupportOwen.py:35-127 with the per-particle
work (psi0 pair sum, table lookup, support update) in one pass, sph_owen_iter.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from . import ops
from .core import KernelFunctions, SupportScheme, nH_to_n_h

F32 = np.float32
_TABLES: dict = {}


def _tpow(a, q, n):
    t = F32(F32(a) - q)
    if not t > 0:
        return F32(0)
    r = t
    for _ in range(n - 1):
        r = F32(r * t)
    return r


def _dkdq_C(kernel: int, dim: int, q):
    """|dk/dq| C_d of the dimensionless kernels (Wendland: dk/dq = -q p(q); B7: the
    derivative of the degree-7 B-spline's truncated powers)."""
    q = F32(q)
    t = F32(1) - q
    if kernel == 4:
        C = {1: F32(4096.0 / 315.0), 2: F32(589824.0 / (7435.0 * math.pi)), 3: F32(16384.0 / (105.0 * math.pi))}[dim]
        d = F32(-7) * (_tpow(1.0, q, 6) - F32(8) * _tpow(0.75, q, 6) + F32(28) * _tpow(0.5, q, 6) - F32(56) * _tpow(0.25, q, 6))
        return abs(F32(d * C))
    if kernel == 1:
        C = {1: F32(1.25), 2: F32(7.0 / math.pi), 3: F32(21.0 / (2.0 * math.pi))}[dim]
        p = F32(12) * t * t if dim == 1 else F32(20) * t * t * t
    elif kernel == 2:
        C = {1: F32(1.5), 2: F32(9.0 / math.pi), 3: F32(495.0 / (32.0 * math.pi))}[dim]
        t4 = (t * t) * (t * t)
        p = F32(14) * (F32(1) + F32(4) * q) * t4 if dim == 1 else (F32(56) / F32(3)) * (F32(1) + F32(5) * q) * t4 * t
    else:
        C = {1: F32(1.71875), 2: F32(78.0 / (7.0 * math.pi)), 3: F32(1365.0 / (64.0 * math.pi))}[dim]
        t6 = (t * t) * (t * t) * (t * t)
        p = (F32(6) * (F32(3) + F32(18) * q + F32(35) * q * q) * t6 if dim == 1
             else F32(22) * (F32(1) + F32(7) * q + F32(16) * q * q) * t6 * t)
    return abs(F32(q * p) * C)


def owen_table(kernel: KernelFunctions, dim: int, n_min: float = 2.0, n_max: float = 6.0, n_lut: int = 2 ** 12):
    """(n_h, psi_H) as FP64 numpy arrays of n_lut entries (the reference's table for the
    Owen scheme, optimalSupportOwen.py:49)."""
    key = (int(kernel.value), int(dim), float(n_min), float(n_max), int(n_lut))
    if key in _TABLES:
        return _TABLES[key]
    k = int(kernel.value)
    nh = np.zeros(n_lut, np.float64)
    psiH = np.zeros(n_lut, np.float64)
    dn = (F32(n_max) - F32(n_min)) / (F32(n_lut) - F32(1.0))
    for i in range(n_lut):
        n_h = F32(F32(n_min) + F32(i) * dn)
        deta = F32(1.0) / n_h
        etar = deta
        result = F32(0.0)
        while etar < F32(1.0):
            if dim == 1:
                corr = F32(2.0)
            elif dim == 2:
                corr = F32(F32(2.0) * F32(math.pi) * etar / deta)
            else:
                corr = F32(F32(4.0) * F32(math.pi) * (etar * etar) / (deta * deta))
            result = F32(result + _dkdq_C(k, dim, etar) * corr)
            etar = F32(etar + deta)
        nh[i] = n_h
        psiH[i] = F32(result ** (F32(1.0) / F32(dim)))
    _TABLES[key] = (nh, psiH)
    return nh, psiH


_DEVICE_TABLES: dict = {}


def _device_table(kernel, dim, device):
    key = (int(kernel.value), int(dim), str(device))
    if key not in _DEVICE_TABLES:
        nh, psiH = owen_table(kernel, dim)
        if not np.all(np.diff(psiH) > 0):
            raise RuntimeError("Owen table: psi_H must increase with n_h")
        _DEVICE_TABLES[key] = (torch.from_numpy(nh).to(device), torch.from_numpy(psiH).to(device))
    return _DEVICE_TABLES[key]


def evaluateOptimalSupportOwen(particles, config, compConfig, kernel_: Optional[KernelFunctions] = None, adjacency=None,
                               supportScheme: Optional[SupportScheme] = None, verbose: bool = False):
    """optimalSupportOwen.py:35-127.  Returns (densities, supports, adjacency, psis, hs)."""
    from .configurations import make_params
    kernel = kernel_ if kernel_ is not None else config.kernel
    S = particles
    dim = int(config.domain.dim)
    params = make_params(config, compConfig)
    lut_nh, lut_psiH = _device_table(kernel, dim, S.supports.device)
    target = float(nH_to_n_h(config.targetNeighbors, dim))
    n_iter = int(compConfig.adaptiveSupportIterations)
    threshold = float(compConfig.adaptiveSupportThreshold)
    hb = ops.minmax(S.supports)
    hs, psis = [S.supports], []
    for it in range(n_iter):
        adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adjacency)
        psiH, h, ratio = ops.owen_iter(params, S.positions, S.supports, adjacency, lut_nh, lut_psiH, target, hb)
        psis.append(psiH)
        hb = ops.minmax(h)
        S.supports = h
        hs.append(h)
        # the reference stops when max |h_new/h - 1| < threshold (a host read, as there);
        # after the last iteration the loop ends anyway
        if it < n_iter - 1 and float((ratio - 1).abs().max()) < threshold:
            break
    # the density at the new supports (optimalSupportOwen.py:116-125): the rows are made to
    # cover the new supports first (kept when the Verlet skin allows)
    adjacency = ops.buildVerletList(S.positions, S.supports, params, config.verletScale, adjacency)
    densities = ops.density(params, S.positions, S.supports, S.masses, adjacency,
                            supportScheme if supportScheme is not None else SupportScheme.Gather)
    return densities, hs[-1], adjacency, psis, hs
