"""Batched ensembles of independent periodic delta-SPH boxes.

Hundreds of weakly compressible boxes of uneven particle counts advance together:
  * one neighbour search over all of them (sph_ensemble_neighbors_build: per-box cell
    grids behind one cell table, segment offsets per box);
  * ONE cooperative persistent launch per time step for every box (sph_ensemble_step:
    Heun RK2 of the delta-SPH right-hand side of schemes/deltaSPH.py, per-box dt);
  * the launches of ``graph_steps`` steps captured once in a CUDA graph and replayed;
  * the tile shape of the step (lanes per particle x block size) chosen by a small
    autotuner (``Ensemble.autotune``) that times every candidate on a copy of the state;
  * the lists rebuilt between graph replays.  The rebuild writes into the same
    fixed-capacity buffers, so the captured graph stays valid.

The case (``build_boxes``) is a set of periodic unit boxes:
  * Sizes: particle counts log-uniform in [nmin, nmax] from one seed, each box a square
    lattice of round(sqrt(N_b))^2 particles.
  * Velocity: divergence-free, v = curl psi with
    psi = sum_k A(k) cos(2 pi k.x + phi_k) over integer wave vectors 2 <= |k| <= 16,
    |A(k)|^2 ~ |k|^-5/3 / |k| (the 2D shell of E(k) ~ k^-5/3), phases from the box's
    seed, scaled to U_max = 1.
  * Physics: stiff Tait EOS with c0 = 10 U_max, rho0 = 1, delta = 0.1, nu = 1e-3.
  * Time step: per box, the weakly compressible rule of
    modules/timestep/weaklyCompressible.py:13-88 (wcsph.weaklyCompressibleStepLimit): the
    smaller of the viscous limit 0.125 h^2 / nu / k and the acoustic limit CFL h / c0 / k
    (CFL 0.3), fixed at set-up; for these boxes the acoustic limit decides.

No counterpart in the reference, which runs one simulation per process.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _capi, ops
from ._capi import check, ptr
from .configurations import SimulationConfig, WeaklyCompressibleSPHConfig, make_params, wc_params
from .core import AdjacencyList, KernelFunctions, buildDomainDescription, n_h_to_nH, sphKernelScale, volumeToSupportHelper
from .wcsph import weaklyCompressibleStepLimit

TILE_CANDIDATES = [(4, 128), (4, 256), (8, 128), (8, 256), (16, 128), (16, 256)]


def box_sizes(nbox: int, seed: int = 0, nmin: int = 4096, nmax: int = 65536) -> List[int]:
    """Particle counts log-uniform in [nmin, nmax], rounded to square lattices."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nbox))
    return [int(round(math.sqrt(v))) ** 2 for v in n]


def shard_boxes(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of boxes to ranks (largest box to the least
    loaded rank); returns the box indices of every rank."""
    loads = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for b in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(b)
        loads[r] += sizes[b]
    return [sorted(o) for o in out]


def _stream_velocity(xy: torch.Tensor, seed: int, kmin: float = 2.0, kmax: float = 16.0) -> torch.Tensor:
    rng = np.random.default_rng(seed)
    ks = [(kx, ky) for kx in range(-16, 17) for ky in range(-16, 17) if kmin <= math.hypot(kx, ky) <= kmax]
    k = torch.tensor(ks, dtype=torch.float64, device=xy.device)
    kn = torch.linalg.norm(k, dim=1)
    amp = torch.sqrt(kn ** (-5.0 / 3.0) / kn)
    phi = torch.from_numpy(rng.uniform(0, 2 * math.pi, len(ks))).to(xy.device)
    arg = 2 * math.pi * (xy.double() @ k.T) + phi                 # [n, modes]
    s = -torch.sin(arg) * (2 * math.pi * amp)                      # d/dx_a cos(...) = -sin(...) 2 pi k_a
    dpsi_dx = s @ k[:, 0]
    dpsi_dy = s @ k[:, 1]
    v = torch.stack([dpsi_dy, -dpsi_dx], 1)
    return (v / torch.linalg.norm(v, dim=1).max()).float()


@dataclass
class BoxSet:
    sizes: List[int]
    seeds: List[int]


def build_boxes(nbox: int = 256, seed: int = 0, nmin: int = 4096, nmax: int = 65536, boxes: Optional[Sequence[int]] = None) -> BoxSet:
    sizes = box_sizes(nbox, seed, nmin, nmax)
    idx = list(range(nbox)) if boxes is None else list(boxes)
    return BoxSet([sizes[b] for b in idx], [seed * 100003 + b for b in idx])


class Ensemble:
    def __init__(self, boxes: BoxSet, device, kernel=KernelFunctions.Wendland2, target_neighbors: Optional[float] = None,
                 scheme: Optional[WeaklyCompressibleSPHConfig] = None, graph_steps: int = 6):
        dev = torch.device(device)
        self.device, self.graph_steps = dev, graph_steps
        self.scheme = scheme or WeaklyCompressibleSPHConfig()
        self.scheme.diffusionParams.inviscid = False          # nu = 1e-3 (viscous form)
        self.config = SimulationConfig(device=dev, domain=buildDomainDescription(1.0, 2, True, dev), dim=2, kernel=kernel,
                                       verletScale=2.0 ** 0.5,
                                       targetNeighbors=n_h_to_nH(4, 2) if target_neighbors is None else target_neighbors)
        self.params = make_params(self.config)
        self.wc = wc_params(self.scheme)
        kscale = float(sphKernelScale(kernel, 2))
        c0 = float(self.scheme.fluid.fixedSoundSpeed)
        xs, box_of, H, m, v, dts, grids = [], [], [], [], [], [], []
        for b, (nb, sd) in enumerate(zip(boxes.sizes, boxes.seeds)):
            nx = int(round(math.sqrt(nb)))
            dx = 1.0 / nx
            g = (torch.arange(nx, device=dev, dtype=torch.float64) + 0.5) * dx - 0.5
            gx, gy = torch.meshgrid(g, g, indexing="xy")
            xy = torch.stack([gx.reshape(-1), gy.reshape(-1)], 1)
            hb = float(volumeToSupportHelper(dx * dx, self.config.targetNeighbors, 2))
            xs.append(xy.float())
            v.append(_stream_velocity(xy, sd))
            box_of.append(torch.full((nx * nx,), b, dtype=torch.int32, device=dev))
            H.append(torch.full((nx * nx,), hb, device=dev))
            m.append(torch.full((nx * nx,), float(self.scheme.fluid.restDensity) * dx * dx, device=dev))
            nu = float(self.scheme.diffusionParams.viscidNu)
            dts.append(weaklyCompressibleStepLimit(hb, c0, nu, kscale, float(self.config.cflFactor), self.scheme))
            G = int(math.floor(1.0 / (self.config.verletScale * hb * (1 + 1e-5))))
            if G < 3:
                raise ValueError(f"box {b}: support {hb:.4g} too large for a 3-cell periodic grid")
            grids.append(G)
        self.sizes = list(boxes.sizes)
        self.n = int(sum(self.sizes))
        self.x = torch.cat(xs).contiguous()
        self.v = torch.cat(v).contiguous()
        self.H = torch.cat(H).contiguous()
        self.m = torch.cat(m).contiguous()
        self.box_of = torch.cat(box_of).contiguous()
        self.box_dt = torch.tensor(dts, device=dev, dtype=torch.float32)
        self.box_grid = torch.tensor(grids, device=dev, dtype=torch.int32)
        base = np.concatenate([[0], np.cumsum(np.array(grids, np.int64) ** 2)])
        self.total_cells = int(base[-1])
        self.box_base = torch.from_numpy(base[:-1].astype(np.int32)).to(dev)
        self.seg = torch.from_numpy(np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64))
        L = _capi.lib()
        self.nb_ws = torch.empty(int(L.sph_ensemble_neighbors_workspace_size(self.n, self.total_cells)), dtype=torch.uint8, device=dev)
        self.step_ws = torch.empty(int(L.sph_ensemble_step_workspace_size(self.n, 2)), dtype=torch.uint8, device=dev)
        self.offs = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.cnt = torch.empty(self.n, dtype=torch.int32, device=dev)
        per = self.config.verletScale ** 2 * self.config.targetNeighbors * 1.35 + 16   # Verlet rows ~ vs^2 N_H
        self.capacity = int(self.n * per)
        self.list = torch.empty(self.capacity, dtype=torch.int32, device=dev)
        self.flags = torch.zeros(4, dtype=torch.int64, device=dev)     # [nnz, status (low half), disp (low half), -]
        self.x_build = torch.empty_like(self.x)
        self.tile = (8, 128)
        self.graph = None
        self.steps_done = 0
        self.rebuilds = 0
        self.rebuild()
        adj = self.adjacency()
        self.rho = ops.density(self.params, self.x, self.H, self.m, adj)

    # -------------------------------------------------------------- neighbour lists
    def adjacency(self) -> AdjacencyList:
        return AdjacencyList(neighborOffsets=self.offs, numNeighbors=self.cnt, neighborList=self.list[: self.nnz], numRows=self.n,
                             numCols=self.n, nnz=self.nnz)

    def rebuild(self):
        L = _capi.lib()
        self.flags.zero_()
        check(L.sph_ensemble_neighbors_build(ops._p(self.params), self.n, len(self.sizes), ptr(self.box_of), ptr(self.box_grid),
                                             ptr(self.box_base), self.total_cells, ptr(self.x), ptr(self.H), ptr(self.nb_ws),
                                             self.nb_ws.numel(), ptr(self.offs), ptr(self.cnt), ptr(self.list), self.capacity,
                                             self.flags.data_ptr(), self.flags.data_ptr() + 8, ops.stream_ptr(self.device)),
              "sph_ensemble_neighbors_build")
        f = self.flags[:2].cpu()
        self.nnz = int(f[0])
        if int(f[1]) & _capi.STATUS_LIST_OVERFLOW:
            raise RuntimeError(f"ensemble list capacity {self.capacity} < {self.nnz} entries")
        self.x_build.copy_(self.x)
        self.flags[2].zero_()
        self._used_at_check = 0.0
        self.rebuilds += 1

    def skin_used(self) -> float:
        """Largest |x - x_build| / H since the last rebuild."""
        o = int(self.flags[2].item()) & 0xFFFFFFFF
        u = (o & 0x7FFFFFFF) if (o & 0x80000000) else (~o & 0xFFFFFFFF)
        return float(np.array([u], np.uint32).view(np.float32)[0]) if o else 0.0

    # -------------------------------------------------------------- stepping
    def _launch(self, tile=None, x=None, v=None, rho=None):
        lanes, block = tile or self.tile
        check(_capi.lib().sph_ensemble_step(ops._p(self.params), C.cast(C.pointer(self.wc), C.c_void_p), self.n, ptr(self.box_of),
                                            ptr(self.box_dt), ptr(self.H), ptr(self.m), ptr(self.x if x is None else x),
                                            ptr(self.v if v is None else v), ptr(self.rho if rho is None else rho), ptr(self.x_build),
                                            ptr(self.offs), ptr(self.cnt), ptr(self.list), ptr(self.step_ws), self.step_ws.numel(),
                                            lanes, block, self.flags.data_ptr() + 16, self.flags.data_ptr() + 8,
                                            ops.stream_ptr(self.device)), "sph_ensemble_step")

    def _capture(self):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(self.graph_steps):
                self._launch()
        self.graph = g

    def advance(self, nsteps: int, use_graph: bool = True):
        """At least nsteps time steps of every box.  The first step is a plain launch (it
        also resolves the launch configuration); after it the steps go in chunks of
        ``graph_steps`` (one replay of the captured graph, or the same launches issued
        one by one), each followed by the skin check that decides on a rebuild, so both
        modes take identical steps."""
        done = 0
        while done < nsteps:
            if self.steps_done == 0:
                self._launch()
                done += 1
                self.steps_done += 1
                continue
            if use_graph:
                if self.graph is None:
                    self._capture()
                self.graph.replay()
            else:
                for _ in range(self.graph_steps):
                    self._launch()
            done += self.graph_steps
            self.steps_done += self.graph_steps
            # the rows must hold until the next check: rebuild when the last chunk's growth
            # of the used skin, with a 1.5x margin, would exhaust it before then
            used = 2.0 * self.skin_used()
            skin = self.config.verletScale - 1.0
            if used >= skin:
                raise RuntimeError("ensemble: particles left the Verlet skin between two checks")
            if used + 1.5 * (used - self._used_at_check) >= skin:
                self.rebuild()
                used = 0.0
            self._used_at_check = used
        return done

    def status(self) -> int:
        return int(self.flags[1].item()) & 0xFFFFFFFF

    # -------------------------------------------------------------- autotuning
    def autotune(self, steps: int = 2) -> dict:
        """Times every (lanes, block) candidate for ``steps`` steps on a copy of the state
        and keeps the fastest; returns the ms per step of each candidate."""
        x0, v0, r0 = self.x.clone(), self.v.clone(), self.rho.clone()
        res = {}
        for tile in TILE_CANDIDATES:
            x, v, r = x0.clone(), v0.clone(), r0.clone()
            self._launch(tile, x, v, r)                 # warm-up (occupancy query, lazy load)
            torch.cuda.synchronize(self.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                self._launch(tile, x, v, r)
            e1.record()
            torch.cuda.synchronize(self.device)
            res[tile] = e0.elapsed_time(e1) / steps
        self.tile = min(res, key=res.get)
        self.rebuild()          # the candidates moved copies; restart the skin from the state
        self.graph = None
        return res
