"""Sedov initial state built entirely on the CPU oracle (test/baseline infrastructure).

Same recipe as warpsph_b200.cases.buildSedov (lattice of src/warpSPH/sample/regular.py:6-50,
Monaghan adaptive support, kernel-weighted energy deposit at the origin), so the CPU
baseline arm never runs the GPU engine.
"""
from __future__ import annotations

import numpy as np

from .steps import CRKSPHOracle

KSCALE_C = {(2, 2): 9 / np.pi, (1, 2): 7 / np.pi, (3, 2): 78 / (7 * np.pi)}


def _wendland(kernel, dim, r, H):
    q = np.minimum(r / H, 1.0)
    t = 1 - q
    if kernel == 1:
        f = t ** 3 * (1 + 3 * q) if dim == 1 else t ** 4 * (1 + 4 * q)
        C = {1: 1.25, 2: 7 / np.pi, 3: 21 / (2 * np.pi)}[dim]
    elif kernel == 2:
        f = t ** 5 * (1 + 5 * q + 8 * q * q) if dim == 1 else t ** 6 * (1 + 6 * q + 35 / 3 * q * q)
        C = {1: 1.5, 2: 9 / np.pi, 3: 495 / (32 * np.pi)}[dim]
    else:
        f = t ** 7 * (1 + 7 * q + 19 * q * q + 21 * q ** 3) if dim == 1 else t ** 8 * (1 + 8 * q + 25 * q * q + 32 * q ** 3)
        C = {1: 1.71875, 2: 78 / (7 * np.pi), 3: 1365 / (64 * np.pi)}[dim]
    return C / H ** dim * f


def sedov_state(params, nx: int, dim: int = 2, L: float = 1.0, rho0: float = 1.0, E0: float = 1.0, p0: float = 1e-6,
                gamma: float = 5 / 3, target_neighbors: float = 32.0, support_iterations: int = 16, precision: str = "f32"):
    dx = L / nx
    g = (np.arange(nx) + 0.5) * dx - L / 2
    mesh = np.meshgrid(*([g] * dim), indexing="xy")
    x = np.stack([a.ravel() for a in mesh], 1).astype(np.float32)
    n = x.shape[0]
    vol = dx ** dim
    if dim == 1:
        H0 = target_neighbors * vol / 2
    elif dim == 2:
        H0 = np.sqrt(target_neighbors * vol / np.pi)
    else:
        H0 = (target_neighbors * vol / np.pi * 3 / 4) ** (1 / 3)
    dt_ = np.float32 if precision == "f32" else np.float64
    st = dict(positions=x.astype(dt_), velocities=np.zeros_like(x, dtype=dt_), supports=np.full(n, H0, dt_),
              masses=np.full(n, vol * rho0, dt_), densities=np.ones(n, dt_), divergence=np.zeros(n, dt_),
              alpha0s=np.ones(n, dt_), alphas=np.ones(n, dt_))
    orc = CRKSPHOracle(params, precision, adaptive_iterations=support_iterations)
    st["densities"], st["supports"] = orc.optimal_support(st)
    u_bg = p0 / ((gamma - 1) * st["densities"].astype(np.float64))
    r = np.linalg.norm(st["positions"].astype(np.float64), axis=1)
    W = _wendland(int(params.kernel), dim, r, st["supports"].astype(np.float64))
    W = W / W.sum()
    st["internalEnergies"] = (u_bg + E0 * W / st["masses"].astype(np.float64)).astype(dt_)
    return st
