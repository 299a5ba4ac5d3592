"""Seeded synthetic particle sets shared by the tests."""
from __future__ import annotations

import numpy as np

from warpsph_b200 import configurations as cf
from warpsph_b200 import core
from warpsph_b200.enumTypes import ViscositySwitch

NEIGHBOURS = {1: 10.0, 2: 32.0, 3: 60.0}


def make_params(dim, kernel=core.KernelFunctions.Wendland4, periodic=True, L=1.0, switch=ViscositySwitch.CullenDehnen2010,
                energy_scheme=None, kahan=False):
    cfg = cf.SimulationConfig()
    cfg.domain = core.buildDomainDescription(L, dim, periodic)
    cfg.dim = dim
    cfg.kernel = kernel
    cfg.verletScale = 2.0 ** (1 / dim) if dim > 1 else 2.0 ** 0.5
    cfg.targetNeighbors = NEIGHBOURS[dim]
    sch = cf.CRKSPHConfig()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = switch
    sch.compensatedSums = kahan
    if energy_scheme is not None:
        sch.energyScheme = energy_scheme
    return cfg, sch, cf.make_params(cfg, sch)


def make_particles(dim, n_side, jitter=0.3, seed=0, L=1.0, periodic=True, h_spread=0.1, flow=1.0):
    rng = np.random.default_rng(seed)
    dx = L / n_side
    g = (np.arange(n_side) + 0.5) * dx - L / 2
    mesh = np.meshgrid(*([g] * dim), indexing="xy")
    x = np.stack([a.ravel() for a in mesh], 1)
    x = x + jitter * dx * (rng.random(x.shape) - 0.5)
    if periodic:
        x = (x + L / 2) % L - L / 2
    n = x.shape[0]
    H0 = float(core.volumeToSupportHelper(dx ** dim, NEIGHBOURS[dim], dim))
    H = H0 * (1 + h_spread * (rng.random(n) * 2 - 1))
    m = dx ** dim * (1 + 0.2 * (rng.random(n) - 0.5))
    k = 2 * np.pi / L
    v = np.zeros_like(x)
    for a in range(dim):
        v[:, a] = flow * np.sin(k * x[:, (a + 1) % dim] + a) + 0.1 * flow * (rng.random(n) - 0.5)
    u = 1.0 + 0.5 * rng.random(n)
    return dict(positions=x.astype(np.float32), supports=H.astype(np.float32), masses=m.astype(np.float32),
                velocities=v.astype(np.float32), internalEnergies=u.astype(np.float32))


def assert_close(got, ref, rtol, atol_rel=None, name=""):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    atol = (atol_rel if atol_rel is not None else rtol) * scale
    err = np.abs(got - ref)
    bad = err > atol + rtol * np.abs(ref)
    if bad.any():
        i = np.argmax(err - (atol + rtol * np.abs(ref)))
        raise AssertionError(f"{name}: {bad.sum()} / {bad.size} entries differ; worst flat index {i}: got {got.ravel()[i]!r} "
                             f"ref {ref.ravel()[i]!r} (rtol {rtol}, atol {atol:.3g})")
