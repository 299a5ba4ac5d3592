"""Learned warm start for the DFSPH pressure solves, and the dam-break case that trains
and judges it.

The plain solves start from the reference's guesses: 0.75 p_prev for the
divergence-free solve (modules/incompressible/divergenceFree.py:72) and 0 for the
density solve (modules/incompressible/incompressible.py:79).  ``WarmStartMLP``
predicts the initial pressure per particle from eight local features
(``sph_dfsph_features``) as P MLP(features), with P the features' pressure scale.  The
network is 8 -> 64 -> 64 -> 64 -> 1 with ReLU, trained by the library's own BF16
tensor-core kernels: ``sph_mlp_grad_tc`` (tcgen05) for the gradient and
``sph_mlp_adam`` for the update.  The solve then iterates from that guess
to the same tolerance, so it remains both the fallback and the judge of the network's
error (init_mode 1 of the solver).

``DamBreakMDBC`` is the dam break of the warm start in 3D (or 2D) with the reference's
mDBC wall particles and its DFSPH step order (the divergence-free solve in the step, the
density solve in the finalize).  ``DamBreak2D`` is the earlier small 2D stand-in, run
entirely by the library's kernels. Its parts:
  * Fluid column: the column sits in a tank lined with three layers of fixed boundary
    particles. These take part in every sum and are solved like fluid, but never move.
  * Step: the density solve, then the divergence-free solve on the predicted
    velocity, then symplectic Euler.
  * Training data: its trajectories over randomised column sizes give the
    (features, converged pressure) pairs.
  * Evaluation: it measures iterations and GPU time to tolerance, plain against learned.

There is no counterpart of either in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _capi, ops
from .configurations import RelaxedJacobiSolverConfig, jacobi_config, make_params
from .core import AdjacencyList, DomainDescription, KernelFunctions, volumeToSupportHelper

N_FEATURES = 8
HIDDEN = 64
PARAM_COUNT = 8961
# (name, shape, fan-in) in the parameter vector's order; names starting with "b" are biases
_SIZES = [("W1", (HIDDEN, N_FEATURES), N_FEATURES), ("b1", (HIDDEN,), 0), ("W2", (HIDDEN, HIDDEN), HIDDEN), ("b2", (HIDDEN,), 0),
          ("W3", (HIDDEN, HIDDEN), HIDDEN), ("b3", (HIDDEN,), 0), ("w4", (HIDDEN,), HIDDEN), ("b4", (1,), 0)]


class WarmStartMLP:
    """FP32 master parameters plus Adam moments on one device."""

    def __init__(self, device, seed: int = 0):
        assert int(_capi.lib().sph_mlp_param_count()) == PARAM_COUNT
        gen = torch.Generator().manual_seed(seed)
        parts = []
        for name, shape, fan_in in _SIZES:
            if name.startswith("b"):
                parts.append(torch.zeros(shape))
            else:
                lim = math.sqrt(6.0 / fan_in)                          # He-uniform
                parts.append((torch.rand(shape, generator=gen) * 2 - 1) * lim)
        self.theta = torch.cat([p.reshape(-1) for p in parts]).to(device=device, dtype=torch.float32).contiguous()
        self.m1 = torch.zeros_like(self.theta)
        self.m2 = torch.zeros_like(self.theta)
        self.step = 0

    # -------------------------------------------------------------- training
    def fit(self, feats: torch.Tensor, targets: torch.Tensor, epochs: int = 30, batch: int = 4096, lr: float = 2e-3,
            seed: int = 0, lr_decay: float = 0.97) -> List[float]:
        """Minibatch Adam on the mean squared error; returns the mean loss per epoch."""
        n = feats.shape[0]
        gen = torch.Generator(device=feats.device).manual_seed(seed)
        losses = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen, device=feats.device)
            tot = torch.zeros(1, device=feats.device, dtype=torch.float64)
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch]
                g, l = ops.mlp_grad(self.theta, feats[idx].contiguous(), targets[idx].contiguous())
                self.step += 1
                ops.mlp_adam(self.theta, g, self.m1, self.m2, self.step, lr * lr_decay ** ep)
                tot += l
            losses.append(float(tot.item()) / n)
        return losses

    def loss(self, feats, targets) -> float:
        _, l = ops.mlp_grad(self.theta, feats.contiguous(), targets.contiguous())
        return float(l.item()) / feats.shape[0]

    # -------------------------------------------------------------- inference
    def initial_pressure(self, params, mode: int, cfg, x, H, m, rho, v, dvdt, p_prev, dt, adj: AdjacencyList) -> torch.Tensor:
        """P MLP(features), with P the features' pressure scale."""
        feats, scale = ops.dfsph_features(params, mode, cfg, x, H, m, rho, v, dvdt, p_prev, dt, adj)
        return ops.mlp_forward(self.theta, feats, scale)

    def state_dict(self) -> dict:
        return {"theta": self.theta.detach().cpu(), "step": self.step}

    def load_state_dict(self, d: dict):
        self.theta.copy_(d["theta"].to(self.theta.device))
        self.step = int(d.get("step", 0))


# ------------------------------------------------------------------ dam break
@dataclass
class SolveStats:
    mode: int
    iterations: int
    ms: float          # GPU time of the solve, including the learned guess when used
    error: float       # final error in the reference's definition
    converged: bool


@dataclass
class DamBreak2D:
    """Fluid column width x height (m) in a tank_w x tank_h tank, spacing dx, gravity g;
    boundary: three layers of fixed particles under the floor and outside both walls.

    The reference's solves balance a source in density units (rho0 - rho*, or
    rho0 div v*) against dt^2 div a_p, which carries no density factor: they are
    consistent for the reference's default restDensity = 1 (configurations/
    moduleConfigurations/fluidProperties.py:12) and nothing else, so the case runs with
    rho0 = 1 (pressure in units of rho0 m^2/s^2).  The particle mass makes the kernel
    sum on the interior lattice equal rho0 exactly, so the column starts at rest density."""
    width: float = 0.5
    height: float = 1.0
    tank_w: float = 1.6
    tank_h: float = 1.2
    dx: float = 0.01
    rho0: float = 1.0
    g: float = -9.81
    dt: float = 1e-3
    target_neighbors: float = 20.0
    device: str = "cuda"
    kernel: KernelFunctions = KernelFunctions.Wendland2
    layers: int = 3
    seed: int = 0
    state: dict = field(default_factory=dict)

    def __post_init__(self):
        dev = torch.device(self.device)
        dx = self.dx
        rng = np.random.default_rng(self.seed)
        nfx, nfy = int(round(self.width / dx)), int(round(self.height / dx))
        fx, fy = np.meshgrid((np.arange(nfx) + 0.5) * dx, (np.arange(nfy) + 0.5) * dx, indexing="xy")
        fluid = np.stack([fx.ravel(), fy.ravel()], 1)
        fluid += 0.02 * dx * (rng.random(fluid.shape) - 0.5)     # break the lattice symmetry slightly
        bnd = []
        nbx = int(round(self.tank_w / dx))
        for k in range(self.layers):
            xs = (np.arange(-self.layers, nbx + self.layers) + 0.5) * dx
            bnd.append(np.stack([xs, np.full_like(xs, -(k + 0.5) * dx)], 1))
            ys = (np.arange(int(round(self.tank_h / dx))) + 0.5) * dx
            bnd.append(np.stack([np.full_like(ys, -(k + 0.5) * dx), ys], 1))
            bnd.append(np.stack([np.full_like(ys, self.tank_w + (k + 0.5) * dx), ys], 1))
        bnd = np.concatenate(bnd, 0)
        x = np.concatenate([fluid, bnd], 0).astype(np.float32)
        self.n_fluid, self.n = fluid.shape[0], x.shape[0]
        pad = (self.layers + 2) * dx
        self.domain = DomainDescription(torch.tensor([-pad, -pad], device=dev), torch.tensor([self.tank_w + pad, self.tank_h + pad], device=dev),
                                        torch.tensor([False, False], device=dev), 2)
        from .configurations import SimulationConfig
        self.config = SimulationConfig(device=dev, domain=self.domain, dim=2, kernel=self.kernel, verletScale=2.0 ** 0.5,
                                       targetNeighbors=self.target_neighbors)
        self.params = make_params(self.config)
        H = float(volumeToSupportHelper(dx * dx, self.target_neighbors, 2))
        S = self.state
        S["x"] = torch.from_numpy(x).to(dev)
        S["H"] = torch.full((self.n,), H, device=dev)
        S["m"] = torch.ones(self.n, device=dev)
        adj = ops.buildVerletList(S["x"], S["H"], self.params, self.config.verletScale)
        rho_unit = ops.density(self.params, S["x"], S["H"], S["m"], adj)
        interior = self._interior_index(fluid)
        S["m"] *= self.rho0 / float(rho_unit[interior].item())
        S["v"] = torch.zeros((self.n, 2), device=dev)
        S["p_rho"] = torch.zeros(self.n, device=dev)
        S["p_df"] = torch.zeros(self.n, device=dev)
        self.fluid = torch.zeros(self.n, dtype=torch.bool, device=dev)
        self.fluid[: self.n_fluid] = True
        self.gvec = torch.zeros((self.n, 2), device=dev)
        self.gvec[: self.n_fluid, 1] = self.g
        self.adj = None
        self.t = 0.0

    def _interior_index(self, fluid: np.ndarray) -> int:
        """A fluid particle at least three supports away from every free surface and wall."""
        c = np.array([0.5 * self.width, 0.5 * self.height])
        return int(np.argmin(np.linalg.norm(fluid - c, axis=1)))

    def _solve(self, mode, cfg, v, dvdt, p_init, rho):
        S = self.state
        return ops.jacobi_solve(self.params, mode, cfg, S["x"], S["H"], S["m"], rho, v, dvdt, p_init, self.dt, self.adj)

    def _arm(self, mode, solver: RelaxedJacobiSolverConfig, v, dvdt, p_prev, rho, net: Optional[WarmStartMLP]) -> SolveStats:
        """One solve of the current state from the plain guess (net None: the reference's
        rule) or the learned guess, timed on the GPU including the guess."""
        S = self.state
        cfg = jacobi_config(solver, self.rho0, learned_init=net is not None)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        p0 = p_prev
        if net is not None:
            p0 = net.initial_pressure(self.params, mode, cfg, S["x"], S["H"], S["m"], rho, v, dvdt, p_prev, self.dt, self.adj)
        pr, acc, hist, it, st = self._solve(mode, cfg, v, dvdt, p0, rho)
        ev1.record()
        torch.cuda.synchronize()
        k = int(it.item())
        err = float(hist[k - 1, 0].item()) if k > 0 else float("nan")
        return SolveStats(mode, k, ev0.elapsed_time(ev1), err, (int(st.item()) & _capi.STATUS_NOT_CONVERGED) == 0)

    def step(self, driver: tuple, collect: Optional[dict] = None, compare: Optional[dict] = None):
        """One DFSPH step: density solve, predicted velocity, divergence-free solve on it,
        symplectic Euler for the fluid.  ``driver`` = (density, divergence-free)
        RelaxedJacobiSolverConfig of the solves that advance the state; they start from
        the previous step's pressure.  ``collect`` (dict of lists) receives the features
        and the driver's pressures divided by the feature scale (training targets).
        ``compare`` = {"solvers": (density, div-free configs), "nets": (net_rho, net_df),
        "stats": list}: before each driver solve the same state is also solved from the
        plain and the learned guess, and their SolveStats are appended to stats."""
        S = self.state
        self.adj = ops.buildVerletList(S["x"], S["H"], self.params, self.config.verletScale, self.adj)
        rho = ops.density(self.params, S["x"], S["H"], S["m"], self.adj)
        zero = torch.zeros_like(S["v"])
        out = {}
        for mode, v, dvdt, key in ((ops.DENSITY, S["v"], self.gvec, "p_rho"), (ops.DIVERGENCE_FREE, None, zero, "p_df")):
            if mode == ops.DIVERGENCE_FREE:
                v = torch.where(self.fluid[:, None], S["v"] + self.dt * (self.gvec + out[ops.DENSITY]), zero).contiguous()
                vstar = v
            solver = driver[0] if mode == ops.DENSITY else driver[1]
            dcfg = jacobi_config(solver, self.rho0, learned_init=True)
            if compare is not None:
                ev = compare["solvers"][0] if mode == ops.DENSITY else compare["solvers"][1]
                net = compare["nets"][0] if mode == ops.DENSITY else compare["nets"][1]
                compare["stats"].append(("plain", self._arm(mode, ev, v, dvdt, S[key], rho, None)))
                compare["stats"].append(("learned", self._arm(mode, ev, v, dvdt, S[key], rho, net)))
            if collect is not None:
                f, sc = ops.dfsph_features(self.params, mode, dcfg, S["x"], S["H"], S["m"], rho, v, dvdt, S[key], self.dt, self.adj)
            pr, acc, hist, it, st = self._solve(mode, dcfg, v, dvdt, S[key], rho)
            out[mode] = acc
            if collect is not None:
                collect.setdefault(("feats", mode), []).append(f)
                collect.setdefault(("target", mode), []).append(pr / sc)
            S[key] = pr
        v = torch.where(self.fluid[:, None], vstar + self.dt * out[ops.DIVERGENCE_FREE], zero)
        S["x"] = (S["x"] + self.dt * v).contiguous()
        S["v"] = v.contiguous()
        self.t += self.dt


@dataclass
class DamBreakMDBC:
    """The dam break of the learned warm start with the reference's mDBC walls, in 2D or 3D:
    a column[:dim] fluid block in the corner of an open tank[:dim] tank (axis 1 vertical),
    three wall layers with one mirrored ghost point per wall particle (cases.tank_particles).

    Each step follows the reference's DFSPH (``step``): the gather density of fluid and
    walls with the walls' replaced by the mDBC pass (sph_mdbc_density, the Liu-Liu sums at
    the ghost points over a list of every particle); the no-penetration shift
    (sph_mdbc_nopen_shift) added to gravity over dt; the divergence-free solve; explicit
    Euler for the fluid; then the finalize's density solve at the new positions, whose
    acceleration shifts the fluid by dt^2 a_p.  The walls take part in both solves with
    their mDBC densities and zero velocities and never move.  rho0 = 1 for the reason
    DamBreak2D gives; masses are set so that an interior fluid particle of the lattice sums
    to rho0.  The kinematic viscosity of water (1e-6 m^2/s) is left out: its force, of
    order nu |v| / dx^2, is below 0.5 % of gravity at the spacings used here."""
    dim: int = 3
    column: tuple = (0.5, 1.0, 0.5)
    tank: tuple = (1.6, 1.2, 0.6)
    dx: float = 0.02
    rho0: float = 1.0
    sound_speed: float = 10.0
    g: float = -9.81
    dt: float = 1e-3
    target_neighbors: float = 40.0
    device: str = "cuda"
    kernel: KernelFunctions = KernelFunctions.Wendland2
    layers: int = 3
    seed: int = 0
    jitter: float = 0.02
    state: dict = field(default_factory=dict)

    def __post_init__(self):
        from .cases import tank_particles
        dev = torch.device(self.device)
        d, dx = self.dim, self.dx
        fluid, walls, ghosts = tank_particles(d, dx, self.column[:d], self.tank[:d], self.layers, self.jitter, self.seed)
        self.n_fluid, self.n_wall = len(fluid), len(walls)
        self.nfw = self.n_fluid + self.n_wall
        x = np.concatenate([fluid, walls, ghosts]).astype(np.float32)
        self.n = len(x)
        pad = (self.layers + 2) * dx
        hi = [t + pad for t in self.tank[:d]]
        hi[1] = 3.0 * self.tank[1]
        self.domain = DomainDescription(torch.full((d,), -pad, device=dev), torch.tensor(hi, device=dev, dtype=torch.float32),
                                        torch.zeros(d, dtype=torch.bool, device=dev), d)
        from .configurations import SimulationConfig
        self.config = SimulationConfig(device=dev, domain=self.domain, dim=d, kernel=self.kernel, verletScale=2.0 ** (1.0 / d),
                                       targetNeighbors=self.target_neighbors)
        self.params = make_params(self.config)
        S = self.state
        S["x"] = torch.from_numpy(x).to(dev)
        S["H"] = torch.full((self.n,), float(volumeToSupportHelper(dx ** d, self.target_neighbors, d)), device=dev)
        S["m"] = torch.ones(self.n, device=dev)
        kinds = np.concatenate([np.zeros(self.n_fluid), np.ones(self.n_wall), np.full(self.n_wall, 2)]).astype(np.int32)
        gidx = np.full(self.n, -1, np.int32)
        gidx[self.n_fluid:self.nfw] = np.arange(self.nfw, self.n)
        gidx[self.nfw:] = np.arange(self.n_fluid, self.nfw)
        goff = np.zeros_like(x)
        goff[self.n_fluid:self.nfw] = walls - ghosts
        goff[self.nfw:] = ghosts - walls
        S["kinds"] = torch.from_numpy(kinds).to(dev)
        S["gidx"] = torch.from_numpy(gidx).to(dev)
        S["goff"] = torch.from_numpy(goff).to(dev)
        adj = ops.buildVerletList(S["x"][: self.nfw], S["H"][: self.nfw], self.params, self.config.verletScale)
        rho_unit = ops.density(self.params, S["x"][: self.nfw], S["H"][: self.nfw], S["m"][: self.nfw], adj)
        c = np.asarray(self.column[:d]) * 0.5
        interior = int(np.argmin(np.linalg.norm(fluid - c, axis=1)))
        S["m"] *= self.rho0 / float(rho_unit[interior].item())
        S["v"] = torch.zeros((self.nfw, d), device=dev)
        S["p_rho"] = torch.zeros(self.nfw, device=dev)
        S["p_df"] = torch.zeros(self.nfw, device=dev)
        self.fluid = torch.zeros(self.nfw, dtype=torch.bool, device=dev)
        self.fluid[: self.n_fluid] = True
        self.gvec = torch.zeros((self.nfw, d), device=dev)
        self.gvec[: self.n_fluid, 1] = self.g
        self.gravity = [0.0] * d
        self.gravity[1] = self.g
        self.adj = None
        self.full = None
        self.t = 0.0

    def _solve(self, mode, cfg, v, dvdt, p_init, rho):
        S, k = self.state, self.nfw
        return ops.jacobi_solve(self.params, mode, cfg, S["x"][:k], S["H"][:k], S["m"][:k], rho, v, dvdt, p_init, self.dt, self.adj)

    def _arm(self, mode, solver: RelaxedJacobiSolverConfig, v, dvdt, p_prev, rho, net: Optional[WarmStartMLP],
             previous: bool = False) -> SolveStats:
        """One solve of the current state from the plain guess (the reference's rule), the
        learned guess (``net``) or, with ``previous``, the previous step's pressure as it is;
        timed on the GPU including the guess."""
        S, k = self.state, self.nfw
        cfg = jacobi_config(solver, self.rho0, learned_init=net is not None or previous)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        p0 = p_prev
        if net is not None:
            p0 = net.initial_pressure(self.params, mode, cfg, S["x"][:k], S["H"][:k], S["m"][:k], rho, v, dvdt, p_prev, self.dt, self.adj)
        pr, acc, hist, it, st = self._solve(mode, cfg, v, dvdt, p0, rho)
        ev1.record()
        torch.cuda.synchronize()
        n_it = int(it.item())
        err = float(hist[n_it - 1, 0].item()) if n_it > 0 else float("nan")
        return SolveStats(mode, n_it, ev0.elapsed_time(ev1), err, (int(st.item()) & _capi.STATUS_NOT_CONVERGED) == 0)

    def densities(self) -> torch.Tensor:
        """Gather density of fluid and walls with the walls' replaced by the mDBC pass."""
        S, k = self.state, self.nfw
        self.adj = ops.buildVerletList(S["x"][:k], S["H"][:k], self.params, self.config.verletScale, self.adj)
        self.full = ops.buildVerletList(S["x"], S["H"], self.params, self.config.verletScale, self.full)
        r = ops.density(self.params, S["x"][:k], S["H"][:k], S["m"][:k], self.adj)
        r_all = torch.cat([r, torch.full((self.n - k,), self.rho0, device=r.device)])
        r_all = ops.mdbc_density(self.params, S["x"], S["H"], S["m"], r_all, S["kinds"], S["gidx"], S["goff"], self.full, self.rho0,
                                 self.sound_speed, self.gravity)
        return r_all[:k].contiguous()

    def driver(self):
        """Solves that advance the case: the density solve to a tenth of the evaluation
        tolerance (3000 iterations at most), the divergence-free solve to half of its
        per-step tolerance in at most 200 iterations (run much longer, the reference's
        divergence-free Jacobi iteration, which has no free-surface condition and a
        zero-mean pressure gauge, grows again in a free-surface column)."""
        rho, df = solver_configs(self.rho0, 1e-5, 5e-4, 3000, dt=self.dt)
        df.maxIterations = 200
        return rho, df

    def _solve_mode(self, mode, key, v, dvdt, rho, solver, collect, compare):
        """Compare arms (``compare``), features (``collect``), then the driver solve from the
        previous pressure; stores the pressure under ``key`` and returns the acceleration."""
        S, k = self.state, self.nfw
        dcfg = jacobi_config(solver, self.rho0, learned_init=True)
        if compare is not None:
            ev = compare["solvers"][0] if mode == ops.DENSITY else compare["solvers"][1]
            net = compare["nets"][0] if mode == ops.DENSITY else compare["nets"][1]
            compare["stats"].append(("plain", self._arm(mode, ev, v, dvdt, S[key], rho, None)))
            compare["stats"].append(("learned", self._arm(mode, ev, v, dvdt, S[key], rho, net)))
            if compare.get("previous"):
                compare["stats"].append(("previous", self._arm(mode, ev, v, dvdt, S[key], rho, None, previous=True)))
        if collect is not None:
            f, sc = ops.dfsph_features(self.params, mode, dcfg, S["x"][:k], S["H"][:k], S["m"][:k], rho, v, dvdt, S[key], self.dt,
                                       self.adj)
        pr, acc, hist, it, st = self._solve(mode, dcfg, v, dvdt, S[key], rho)
        # a solve whose source vanishes (a column at rest) has no pressure scale and teaches nothing
        if collect is not None and float(sc.item()) > 1e-20:
            collect.setdefault(("feats", mode), []).append(f[: self.n_fluid])
            collect.setdefault(("target", mode), []).append((pr / sc)[: self.n_fluid])
        S[key] = pr
        return acc

    def step(self, driver: tuple, collect: Optional[dict] = None, compare: Optional[dict] = None):
        """One explicit-Euler step of the reference's DFSPH with mDBC walls: the step of
        schemes/dfsph.py:27-186 (wall densities, zero wall velocities, no-penetration
        shift over dt added to gravity, the divergence-free solve on v + dt dv/dt, the
        update with zero wall rows) and the finalize of systems/incompressible.py:212-249
        (the density at the new positions, the density solve with dv/dt = 0, and the
        position shift dt^2 a_p; velocities keep the step's values).  ``driver``,
        ``collect`` and ``compare`` as in DamBreak2D; samples are taken of fluid
        particles only."""
        S, k, nf = self.state, self.nfw, self.n_fluid
        rho = self.densities()
        zero = torch.zeros_like(S["v"])
        nopen = ops.mdbc_nopen_shift(self.params, S["x"][:k], S["H"][:k], S["m"][:k], S["v"], S["kinds"][:k], S["goff"][:k], self.adj)
        ext = (self.gvec + nopen / self.dt).contiguous()
        a_df = self._solve_mode(ops.DIVERGENCE_FREE, "p_df", S["v"], ext, rho, driver[1], collect, compare)
        v = torch.where(self.fluid[:, None], S["v"] + self.dt * (ext + a_df), zero).contiguous()
        S["v"] = v
        S["x"] = torch.cat([S["x"][:nf] + self.dt * v[:nf], S["x"][nf:]]).contiguous()
        rho = self.densities()
        a_rho = self._solve_mode(ops.DENSITY, "p_rho", v, zero, rho, driver[0], collect, compare)
        S["x"] = torch.cat([S["x"][:nf] + (self.dt * self.dt) * a_rho[:nf], S["x"][nf:]]).contiguous()
        self.t += self.dt


def solver_configs(rho0: float, density_tol_frac: float = 1e-4, div_tol_frac: float = 1e-3, max_iterations: int = 400,
                   dt: Optional[float] = None):
    """The reference's relaxed-Jacobi settings (solver.py:15-28) with the tolerances of
    a 0.01 % density error and a 0.1 % divergence error, both normalised by rho0.  The
    divergence-free solve's residual is a density rate (rho0 div v, in rho0 per second);
    with ``dt`` its tolerance is the 0.1 % per time step of Bender and Koschier's DFSPH
    (IEEE TVCG 2017), div_tol_frac rho0 / dt, else div_tol_frac rho0 per second."""
    return (RelaxedJacobiSolverConfig(minIterations=2, maxIterations=max_iterations, tolerance=density_tol_frac * rho0,
                                      relaxationFactor=0.3),
            RelaxedJacobiSolverConfig(minIterations=2, maxIterations=max_iterations,
                                      tolerance=div_tol_frac * rho0 / (dt if dt else 1.0),
                                      relaxationFactor=0.3))


def driver_configs(rho0: float):
    """Solves that advance the dam break, warm-started from the previous pressure: the
    density solve to a tenth of the evaluation tolerance (3000 iterations at most), so
    its pressures are converged targets; the divergence-free solve for 1000 iterations
    (in a free-surface column it stalls above 0.1 %, the reference having no free-surface
    treatment in that solve, so its targets are the pressure after 1000 iterations)."""
    rho, df = solver_configs(rho0, 1e-5, 1e-4, 3000)
    df.maxIterations = 1000
    return rho, df


def dam_break_2d(w, h, seed, dx, dt, device):
    return DamBreak2D(width=w, height=h, dx=dx, dt=dt, device=device, seed=seed)


def dam_break_mdbc_3d(w, h, seed, dx, dt, device):
    """The 3D mDBC dam break with a w x h x w column (the 1.6 x 1.2 x 0.6 m tank)."""
    return DamBreakMDBC(dim=3, column=(w, h, w), dx=dx, dt=dt, device=device, seed=seed)


def _driver(case):
    return case.driver() if hasattr(case, "driver") else driver_configs(case.rho0)


def generate_samples(geometries, steps: int, device="cuda", dx: float = 0.02, dt: float = 1e-3, make_case=dam_break_2d,
                     collect_every: int = 1, max_samples: Optional[int] = None, seed: int = 0, max_target: float = 1e3):
    """(features, targets) per solve mode from dam-break trajectories; ``geometries`` is a
    list of (width, height, seed); samples are collected every ``collect_every`` steps;
    rows with a non-finite feature or a target of magnitude max_target or more (solves
    whose pressure scale is a rounding residue) are dropped, and with ``max_samples`` a
    seeded random subset of that many rows is kept per mode."""
    collect: dict = {}
    for (w, h, gseed) in geometries:
        case = make_case(w, h, gseed, dx, dt, device)
        drv = _driver(case)
        for s_ in range(steps):
            case.step(drv, collect=collect if (s_ + 1) % collect_every == 0 else None)
    out = {}
    gen = torch.Generator(device="cpu").manual_seed(seed)
    for mode in (0, 1):
        f, t = torch.cat(collect[("feats", mode)]), torch.cat(collect[("target", mode)])
        ok = torch.isfinite(f).all(dim=1) & torch.isfinite(t) & (t.abs() < max_target)
        if not bool(ok.all()):
            f, t = f[ok], t[ok]
        if max_samples is not None and f.shape[0] > max_samples:
            keep = torch.randperm(f.shape[0], generator=gen)[:max_samples].to(f.device)
            f, t = f[keep], t[keep]
        out[mode] = (f.contiguous(), t.contiguous())
    return out


def compare_warm_starts(geometries, steps: int, nets, device="cuda", dx: float = 0.02, dt: float = 1e-3, skip: int = 2,
                        max_iterations: int = 2000, df_budget: Optional[int] = 32, make_case=dam_break_2d,
                        compare_every: int = 1, cases: Optional[list] = None, previous: bool = False):
    """Plain against learned initial pressure on the same states, every ``compare_every``
    steps after the first ``skip`` steps of each trajectory:
      density solve: summed iterations and GPU ms to the 0.01 % tolerance (cap
        ``max_iterations``), and how many solves missed it;
      divergence-free solve: with ``df_budget`` the error after the reference's budget of
        that many iterations (solver.py:22-28, maxIterations 32), summed, and the GPU ms;
        with ``df_budget`` None as the density solve, to the 0.1 % per-step tolerance.
    ``cases`` may hold prebuilt cases (one per geometry) instead of building them; with
    ``previous`` (cases that support it) a third arm starts from the previous step's
    pressure as it is.  Returns the sums and the per-solve statistics."""
    tot = {"density": {"plain": [0, 0.0, 0], "learned": [0, 0.0, 0], "previous": [0, 0.0, 0]},
           "divergence_free": {"plain": [0.0, 0.0, 0], "learned": [0.0, 0.0, 0], "previous": [0.0, 0.0, 0]}, "solves": []}
    for gi, (w, h, seed) in enumerate(geometries):
        case = cases[gi] if cases is not None else make_case(w, h, seed, dx, dt, device)
        drv = _driver(case)
        rho_ev, df_ev = solver_configs(case.rho0, max_iterations=max_iterations, dt=None if df_budget else case.dt)
        if df_budget:
            df_ev = RelaxedJacobiSolverConfig(minIterations=df_budget, maxIterations=df_budget, tolerance=0.0,
                                              relaxationFactor=df_ev.relaxationFactor)
        for k in range(steps):
            on = k >= skip and (k - skip) % compare_every == 0
            cmp = {"solvers": (rho_ev, df_ev), "nets": nets, "stats": [], "previous": previous} if on else None
            case.step(drv, compare=cmp)
            if cmp is not None:
                for arm, st in cmp["stats"]:
                    tot["solves"].append((gi, k, arm, st))
                    if st.mode == ops.DENSITY or not df_budget:
                        t = tot["density" if st.mode == ops.DENSITY else "divergence_free"][arm]
                        t[0] += st.iterations; t[1] += st.ms; t[2] += int(not st.converged)
                    else:
                        t = tot["divergence_free"][arm]
                        t[0] += st.error; t[1] += st.ms; t[2] += 1
    return tot
