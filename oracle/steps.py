"""CPU oracle of the full CRKSPH step (test infrastructure only).

Mirrors, on numpy arrays and the C oracle kernels, the reference's step order:
schemes/crkSPH.py:19-366 (one right-hand-side evaluation),
modules/adaptiveSupport/optimalSupportMonaghan.py:62-150 (adaptive support),
systems/compSPH.py:87-129 + modules/compSPH/multistep.py:52-94 (finalize with
compatible energy), and explicit Runge-Kutta staging (Heun RK2 / classic RK4; the
reference's integrator package is absent, so the tableaux are restated).

A state is a dict of numpy arrays with the reference's field names.
"""
from __future__ import annotations

import numpy as np

from . import oracle as _oracle

TABLEAUX = {
    "explicitEuler": ([[]], [1.0], [0.0]),
    "rungeKutta2": ([[], [1.0]], [0.5, 0.5], [0.0, 1.0]),
    "rungeKutta4": ([[], [0.5], [0.0, 0.5], [0.0, 0.0, 1.0]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0.0, 0.5, 0.5, 1.0]),
}

SWITCH_NONE, SWITCH_CULLEN, SWITCH_BALSARA, SWITCH_HOPKINS = 0, 1, 2, 3


def cell_capacity_for(n: int, dim: int) -> int:
    want = max(1024, n * (1 << dim))
    cap = 1
    while cap < want:
        cap <<= 1
    return min(cap, 1 << 24)


class CRKSPHOracle:
    def __init__(self, params, precision: str = "f32", adaptive_iterations: int = 1, adaptive_threshold: float = 1e-3,
                 switch: int = SWITCH_CULLEN, compatible_energy: bool = True, adaptive: bool = True, owen_table=None):
        self.o = _oracle.get(precision)
        self.p = params
        self.dt_ = self.o.dtype
        self.iters = adaptive_iterations
        self.thr = adaptive_threshold
        self.switch = switch
        self.compatible = compatible_energy
        self.adaptive = adaptive
        self.owen = owen_table          # (n_h, psi_H) table: the Owen scheme instead of Monaghan's
        self.dim = int(params.dim)

    # --------------------------------------------------------------- helpers
    def nb(self, x, H):
        return self.o.neighbors(self.p, x.astype(np.float32), H.astype(np.float32), cell_capacity_for(len(H), self.dim))

    def wrap(self, x):
        p = self.p
        x = x.copy()
        for a in range(self.dim):
            if p.periodic[a]:
                mn, mx = np.float32(p.domain_min[a]), np.float32(p.domain_max[a])
                L = np.float32(p.domain_max[a] - p.domain_min[a])
                col = x[:, a]
                hi = col >= mx
                lo = col < mn
                col[hi] = col[hi] - L.astype(self.dt_)
                col[lo] = col[lo] + L.astype(self.dt_)
        return x

    def combine(self, y0, ks, ws, dt, wrap=False):
        f = self.dt_
        s = np.zeros_like(y0, dtype=f)
        for k, w in zip(ks, ws):
            if w == 0.0:
                continue
            s = (s + (f(w) * k.astype(f)).astype(f)).astype(f)
        y = (y0.astype(f) + (f(dt) * s).astype(f)).astype(f)
        return self.wrap(y) if wrap else y

    # --------------------------------------------------------------- adaptive support
    def optimal_support(self, st):
        o, p = self.o, self.p
        x, H, m = st["positions"], st["supports"], st["masses"]
        hb = np.array([H.min(), H.max()], dtype=self.dt_)
        for it in range(self.iters):
            nb = self.nb(x, H)
            if self.owen is not None:       # modules/adaptiveSupport/optimalSupportOwen.py:70-114
                target = ((2.0 if self.dim == 1 else (np.pi if self.dim == 2 else 4 / 3 * np.pi)) / float(p.target_neighbors)) \
                    ** (-1.0 / self.dim)
                _, _, Hn, ratio = o.owen_iter(p, x, H, nb, self.owen[0], self.owen[1], target, hb)
                hb = np.array([Hn.min(), Hn.max()], dtype=self.dt_)
                H = Hn
                if it < self.iters - 1 and np.abs(ratio - 1).max() < self.thr:
                    break
                continue
            rho, Hn, ratio = o.adaptive_h_iter(p, x, H, m, nb, hb)
            hb = np.array([Hn.min(), Hn.max()], dtype=self.dt_)
            H = Hn
            if it < self.iters - 1 and np.abs(ratio - 1).max() < self.thr:
                break
        nb = self.nb(x, H)
        rho = o.density(p, 0, x, H, m, nb)
        return rho, H

    # --------------------------------------------------------------- one RHS evaluation
    def rhs(self, st, dt):
        o, p = self.o, self.p
        st = dict(st)
        if self.adaptive:
            st["densities"], st["supports"] = self.optimal_support(st)
        x, H, m, v, u = st["positions"], st["supports"], st["masses"], st["velocities"], st["internalEnergies"]
        nb = self.nb(x, H)
        V = o.crk_volume(p, x, H, nb)
        A, B, gA, gB, rho = o.crk_factors(p, x, H, m, V, nb)
        st["densities"] = rho
        st["entropies"], st["pressures"], st["soundspeeds"] = o.eos(p, u, rho)
        c, P = st["soundspeeds"], st["pressures"]
        cullen = self.switch == SWITCH_CULLEN
        G, drho, div, vs = o.grad_v(p, x, H, m, rho, V, A, B, gA, gB, v, c, nb, cullen=cullen)
        if cullen:
            st["alphas"], _ = o.switch_cullen(p, x, H, m, rho, div, st["divergence"], vs, st["alpha0s"], dt, nb)
        elif self.switch == SWITCH_BALSARA:
            st["alphas"] = o.switch_balsara(p, G, c)
        dvdt, dudt, ap, av = o.crk_accel_dudt(p, x, H, m, rho, V, A, B, gA, gB, v, c, P, G, nb)
        st["divergence"] = (-drho / rho).astype(self.dt_)
        st["ap_ij"], st["av_ij"] = ap, av
        st["f_ij"] = o.balance(p, m, rho, P, u, v, dvdt, dt, nb, ap, av)
        upd = dict(dxdt=v, dvdt=dvdt, dudt=dudt, drhodt=drho)
        extras = dict(V=V, A=A, B=B, gradA=gA, gradB=gB, DvDx=G, div_cd=div, vsig=vs)
        return upd, nb, st, extras

    # --------------------------------------------------------------- integrator step
    def step(self, st0, dt, scheme: str = "rungeKutta2"):
        a, b, _c = TABLEAUX[scheme]
        updates, rvs = [], []
        prev = dict(st0)
        for s in range(len(b)):
            Ss = dict(prev)
            if s > 0:
                Ss["positions"] = self.combine(st0["positions"], [u["dxdt"] for u in updates], a[s], dt, wrap=True)
                Ss["velocities"] = self.combine(st0["velocities"], [u["dvdt"] for u in updates], a[s], dt)
                Ss["internalEnergies"] = self.combine(st0["internalEnergies"], [u["dudt"] for u in updates], a[s], dt)
            upd, nb, Sout, _ = self.rhs(Ss, dt)
            updates.append(upd)
            rvs.append((nb, Sout))
            prev = Sout
        Sf = dict(prev)
        Sf["positions"] = self.combine(st0["positions"], [u["dxdt"] for u in updates], b, dt, wrap=True)
        Sf["velocities"] = self.combine(st0["velocities"], [u["dvdt"] for u in updates], b, dt)
        Sf["internalEnergies"] = self.combine(st0["internalEnergies"], [u["dudt"] for u in updates], b, dt)
        if self.compatible:
            stages = [dict(dvdt=u["dvdt"], nb=nb, f=S["f_ij"], ap=S["ap_ij"], av=S["av_ij"]) for u, (nb, S) in zip(updates, rvs)]
            Sf["internalEnergies"], _ = self.o.finalize(self.p, b, dt, st0["velocities"], st0["internalEnergies"], stages)
        return Sf, updates, rvs


class CompSPHOracle(CRKSPHOracle):
    """One right-hand-side evaluation of schemes/compSPH.py:22-215 on the C oracle
    (gather density, grad-h Omega, Cullen switch, CompSPH accel/dudt, energy partition);
    staging and compatible-energy finalize as in CRKSPHOracle."""

    def __init__(self, params, precision: str = "f32", grad_h: bool = True, **kw):
        super().__init__(params, precision, **kw)
        self.grad_h = grad_h

    def rhs(self, st, dt):
        o, p = self.o, self.p
        st = dict(st)
        if self.adaptive:
            st["densities"], st["supports"] = self.optimal_support(st)
        x, H, m, v, u = st["positions"], st["supports"], st["masses"], st["velocities"], st["internalEnergies"]
        nb = self.nb(x, H)
        rho = o.density(p, 0, x, H, m, nb)
        st["densities"] = rho
        if st.get("divergence") is None:
            st["divergence"] = o.compsph_prep(p, x, H, m, rho, v, nb, grad_h=False)[2]
        st["entropies"], st["pressures"], st["soundspeeds"] = o.eos(p, u, rho)
        c, P = st["soundspeeds"], st["pressures"]
        om, div, drho = o.compsph_prep(p, x, H, m, rho, v, nb, grad_h=self.grad_h)
        if self.switch == SWITCH_CULLEN:
            vs = o.vsig(p, x, H, v, c, nb)
            st["alphas"], _ = o.switch_cullen(p, x, H, m, rho, div, st["divergence"], vs, st["alpha0s"], dt, nb)
        elif self.switch == SWITCH_HOPKINS:       # modules/shockCapturing/CullenHopkins.py:7-45
            st["alphas"], hdiv, _, _ = o.switch_hopkins_terms(p, x, H, m, rho, v, st["alpha0s"], nb)
        dvdt, dudt, dEdt, ap, av = o.compsph_accel_dudt(p, x, H, m, rho, v, c, st.get("alphas"), P, om, nb)
        if self.switch == SWITCH_CULLEN:
            st["alpha0s"] = st["alphas"]
        elif self.switch == SWITCH_HOPKINS:       # CullenHopkins.py:48-149, before the divergence is replaced
            st["alpha0s"], _ = o.switch_hopkins_update(p, x, H, v, c, hdiv, st["divergence"], st["alpha0s"], dt, nb)
        st["divergence"] = (-drho / rho).astype(self.dt_)
        st["ap_ij"], st["av_ij"] = ap, av
        st["f_ij"] = o.balance(p, m, rho, P, u, v, dvdt, dt, nb, ap, av)
        upd = dict(dxdt=v, dvdt=dvdt, dudt=dudt, drhodt=drho, dEdt=dEdt)
        return upd, nb, st, dict(omega=om, div_cd=div)


class MonaghanOracle(CRKSPHOracle):
    """One right-hand-side evaluation of schemes/monaghan.py:13-158 on the C oracle;
    no compatible-energy finalize (the scheme integrates u directly)."""

    def __init__(self, params, precision: str = "f32", grad_h: bool = True, density_mode: int = 3, **kw):
        kw.setdefault("compatible_energy", False)
        kw.setdefault("switch", SWITCH_NONE)
        super().__init__(params, precision, **kw)
        self.grad_h = grad_h
        self.density_mode = density_mode

    def rhs(self, st, dt):
        o, p = self.o, self.p
        st = dict(st)
        if self.adaptive:
            st["densities"], st["supports"] = self.optimal_support(st)
        x, H, m, v, u = st["positions"], st["supports"], st["masses"], st["velocities"], st["internalEnergies"]
        nb = self.nb(x, H)
        rho = o.density(p, self.density_mode, x, H, m, nb)
        st["densities"] = rho
        st["entropies"], st["pressures"], st["soundspeeds"] = o.eos(p, u, rho)
        om, _, drho = o.compsph_prep(p, x, H, m, rho, v, nb, grad_h=self.grad_h)
        dvdt, dudt, dEdt, _ = o.monaghan_rhs(p, x, H, m, rho, v, u, st["soundspeeds"], st.get("alphas"), st["pressures"], om, nb)
        upd = dict(dxdt=v, dvdt=dvdt, dudt=dudt, drhodt=drho, dEdt=dEdt)
        return upd, nb, st, dict(omega=om)


class DFSPHOracle(CRKSPHOracle):
    """schemes/dfsph.py:13-218 for a fluid-only system, with the finalize of
    systems/incompressible.py:71-277: gather density (unless integrated), velocity
    diffusion and continuity, gravity, the divergence-free Jacobi solve; after the stages
    the gather density at the new positions and the density solve, whose acceleration
    moves the particles by dt^2 a_p.  Positions, velocities and densities are integrated."""

    def __init__(self, params, wc, df_cfg, rho_cfg, gravity=None, integrate_rho: bool = False, precision: str = "f32"):
        super().__init__(params, precision, adaptive=False, compatible_energy=False)
        self.wc, self.df_cfg, self.rho_cfg = wc, df_cfg, rho_cfg
        self.g = None if gravity is None else np.asarray(gravity, self.dt_)
        self.integrate_rho = integrate_rho

    def gravity(self, n):
        return np.zeros((n, self.dim), self.dt_) if self.g is None else np.tile(self.g, (n, 1)).astype(self.dt_)

    def rhs(self, st, dt):
        o, p = self.o, self.p
        st = dict(st)
        x, H, m, v = st["positions"], st["supports"], st["masses"], st["velocities"]
        nb = self.nb(x, H)
        if st.get("densities") is None or not self.integrate_rho:
            st["densities"] = o.density(p, 0, x, H, m, nb)
        rho = st["densities"]
        dvdt_diss, drhodt = o.visc_continuity(p, self.wc, x, H, m, rho, v, nb)
        dvdt = self.gravity(len(H))
        p0 = st.get("pressures")
        p0 = np.zeros(len(H), self.dt_) if p0 is None else p0
        src = (dvdt + dvdt_diss).astype(self.dt_)
        pr, acc, hist, it = o.jacobi_solve(p, 0, self.df_cfg, x, H, m, rho, v, src, p0, dt, nb)
        st["pressures"] = pr
        upd = dict(dxdt=v, dvdt=(src + acc).astype(self.dt_), drhodt=drhodt)
        return upd, nb, st, dict(errors=hist[:, 0].copy(), iterations=it)

    def step(self, st0, dt, scheme: str = "explicitEuler"):
        a, b, _c = TABLEAUX[scheme]
        updates, rvs = [], []
        prev = dict(st0)
        fields = (("positions", "dxdt", True), ("velocities", "dvdt", False), ("densities", "drhodt", False))
        for s in range(len(b)):
            Ss = dict(prev)
            if s > 0:
                for name, der, wr in fields:
                    if st0.get(name) is not None:
                        Ss[name] = self.combine(st0[name], [u[der] for u in updates], a[s], dt, wrap=wr)
            upd, nb, Sout, ex = self.rhs(Ss, dt)
            updates.append(upd)
            rvs.append((nb, Sout, ex))
            prev = Sout
        Sf = dict(prev)
        for name, der, wr in fields:
            if st0.get(name) is not None:
                Sf[name] = self.combine(st0[name], [u[der] for u in updates], b, dt, wrap=wr)
        self.finalize(Sf, st0, dt, updates, rvs)
        return Sf, updates, rvs

    def finalize(self, Sf, st0, dt, updates, rvs):
        o, p = self.o, self.p
        last = rvs[-1][1]
        Sf["pressures"] = last["pressures"]
        x, H, m, v = Sf["positions"], Sf["supports"], Sf["masses"], Sf["velocities"]
        nb = self.nb(x, H)
        rho = o.density(p, 0, x, H, m, nb)
        Sf["densities"] = rho
        zero = np.zeros_like(v)
        pr, acc, hist, it = o.jacobi_solve(p, 1, self.rho_cfg, x, H, m, rho, v, zero, Sf["pressures"], dt, nb)
        k = (self.dt_(self.dt_(dt) * self.dt_(dt)) * acc).astype(self.dt_)
        Sf["positions"] = self.combine(x, [k], [1.0], 1.0, wrap=True)
        Sf["density_solve_iterations"] = it


class DFSPHWallOracle(DFSPHOracle):
    """dfsph_step with wall particles and their ghost points (schemes/dfsph.py:27-126,
    170-186) and the incompressible finalize, in the library's arrangement: the first nfw
    particles (fluid and walls) take part in every pass, the ghosts only in the mDBC wall
    density (modules/mdbc/density2025.py), whose sums use a list over every particle; wall
    velocities are zero (mdbc/velocity.py, zeros walls); the no-penetration shift
    (mdbc/wp_nopenshift.py) enters dv/dt divided by dt; updates and the finalize's position
    shift are zero for walls and ghosts."""

    def __init__(self, params, wc, df_cfg, rho_cfg, walls: dict, gravity=None, precision: str = "f32"):
        super().__init__(params, wc, df_cfg, rho_cfg, gravity=gravity, precision=precision)
        self.w = walls      # kinds, ghost_indices, ghost_offsets, nfw, rho0, c_s

    def rhs(self, st, dt):
        o, p, w, f = self.o, self.p, self.w, self.dt_
        st = dict(st)
        nfw, kinds = w["nfw"], w["kinds"]
        x, H, m, v = st["positions"], st["supports"], st["masses"], st["velocities"]
        nb = self.nb(x[:nfw], H[:nfw])
        nb_all = self.nb(x, H)
        r = o.density(p, 0, x[:nfw], H[:nfw], m[:nfw], nb)
        rho_prev = st.get("densities")
        tail = rho_prev[nfw:] if rho_prev is not None else np.full(len(H) - nfw, w["rho0"], f)
        rho = np.concatenate([r, tail]).astype(f)
        g = [0.0] * self.dim if self.g is None else list(self.g)
        rho, _ = o.mdbc_density(p, x, H, m, rho, kinds, w["ghost_indices"], w["ghost_offsets"], nb_all, w["rho0"], w["c_s"], g)
        st["densities"] = rho
        v = np.where((kinds == 1)[:, None], f(0), v).astype(f)
        st["velocities"] = v
        xh, Hh, mh, rh, vh = x[:nfw], H[:nfw], m[:nfw], rho[:nfw], v[:nfw]
        dvdt_diss, drhodt = o.visc_continuity(p, self.wc, xh, Hh, mh, rh, vh, nb)
        dvdt = self.gravity(nfw)
        nopen = o.mdbc_nopen_shift(p, xh, Hh, mh, vh, kinds[:nfw], w["ghost_offsets"][:nfw], nb)
        dvdt = (dvdt + nopen / f(dt)).astype(f)
        p0 = st.get("pressures")
        p0 = np.zeros(nfw, f) if p0 is None else p0[:nfw]
        src = (dvdt + dvdt_diss).astype(f)
        pr, acc, hist, it = o.jacobi_solve(p, 0, self.df_cfg, xh, Hh, mh, rh, vh, src, p0, dt, nb)
        n = len(H)
        pad = lambda a: np.concatenate([a, np.zeros((n - nfw,) + a.shape[1:], f)]).astype(f)
        st["pressures"] = pad(pr)
        fluid = kinds[:nfw] == 0
        upd = dict(dxdt=pad(np.where(fluid[:, None], vh, f(0))), dvdt=pad(np.where(fluid[:, None], (src + acc).astype(f), f(0))),
                   drhodt=pad(np.where(fluid, drhodt, f(0))))
        return upd, nb, st, dict(errors=hist[:, 0].copy(), iterations=it)

    def finalize(self, Sf, st0, dt, updates, rvs):
        o, p, w, f = self.o, self.p, self.w, self.dt_
        nfw, kinds = w["nfw"], w["kinds"]
        last = rvs[-1][1]
        Sf["pressures"] = last["pressures"]
        x, H, m, v = Sf["positions"], Sf["supports"], Sf["masses"], Sf["velocities"]
        nb = self.nb(x[:nfw], H[:nfw])
        rho = o.density(p, 0, x[:nfw], H[:nfw], m[:nfw], nb)
        Sf["densities"] = np.concatenate([rho, Sf["densities"][nfw:]]).astype(f)
        zero = np.zeros_like(v[:nfw])
        pr, acc, hist, it = o.jacobi_solve(p, 1, self.rho_cfg, x[:nfw], H[:nfw], m[:nfw], rho, v[:nfw], zero, Sf["pressures"][:nfw],
                                           dt, nb)
        k = np.where((kinds[:nfw] == 0)[:, None], (f(f(dt) * f(dt)) * acc).astype(f), f(0)).astype(f)
        Sf["positions"] = np.concatenate([self.combine(x[:nfw], [k], [1.0], 1.0, wrap=True), x[nfw:]]).astype(f)
        Sf["density_solve_iterations"] = it


class DeltaSPHOracle(DFSPHOracle):
    """schemes/deltaSPH.py:11-208 for a fluid-only system with the finalize of
    systems/weaklyCompressible.py:73-200: the delta-SPH right-hand side plus gravity; after
    the stages the delta-plus shift (when active) at the integrated state, the exponential
    density update from the last stage, and the shift added to the positions.  With
    ``surface`` (dict limit=, iterations=) the colour-field free-surface detection of
    deltaSPH.py:86-91 runs before the right-hand side and its dilated indicators
    (> 0.5) enter the Antuono pressure term."""

    def __init__(self, params, wc, gravity=None, shift=None, precision: str = "f32", surface=None):
        CRKSPHOracle.__init__(self, params, precision, adaptive=False, compatible_energy=False)
        self.wc = wc
        self.surface = surface
        self.g = None if gravity is None else np.asarray(gravity, self.dt_)
        self.shift = shift      # None or dict(cfl=, c0=, iterations=)

    def rhs(self, st, dt):
        o, p = self.o, self.p
        st = dict(st)
        x, H, m, v = st["positions"], st["supports"], st["masses"], st["velocities"]
        nb = self.nb(x, H)
        if st.get("densities") is None:
            st["densities"] = o.density(p, 0, x, H, m, nb)
        mask = None
        if self.surface is not None:
            rho = st["densities"]
            c = o.surface_color_field(p, x, H, m, rho, nb)
            fs = o.surface_detect(p, x, H, m, rho, c, nb, self.surface["limit"])[0]
            for _ in range(int(self.surface.get("iterations", 1))):
                fs = o.surface_dilate(p, x, H, fs, nb)
            mask = (fs > 0.5).astype(np.int32)
            st["surfaceIndicators"] = mask
        dv, dr, _, P = o.deltasph_rhs(p, self.wc, x, H, m, st["densities"], v, nb, mask)
        st["pressures"] = P
        upd = dict(dxdt=v, dvdt=(dv + self.gravity(len(H))).astype(self.dt_), drhodt=dr)
        return upd, nb, st, {}

    def finalize(self, Sf, st0, dt, updates, rvs):
        o, p, f = self.o, self.p, self.dt_
        last = rvs[-1][1]
        Sf["pressures"] = last["pressures"]
        dx = None
        if self.shift is not None:
            x = Sf["positions"]
            dx = np.zeros_like(x)
            for _ in range(int(self.shift.get("iterations", 1))):
                nb = self.nb(x, Sf["supports"])
                upd = o.delta_shift(p, x, Sf["supports"], Sf["masses"], Sf["densities"], Sf["velocities"], nb, self.shift["cfl"],
                                    self.shift["c0"])
                dx = (dx + upd).astype(f)
                x = self.combine(x, [upd], [1.0], 1.0, wrap=True)
        t = ((f(dt) * updates[-1]["drhodt"]).astype(f) / last["densities"]).astype(f)
        Sf["densities"] = (st0["densities"] * np.exp(t).astype(f)).astype(f)
        if dx is not None:
            Sf["positions"] = self.combine(Sf["positions"], [dx], [1.0], 1.0, wrap=True)


def state_to_numpy(state, dtype=np.float32) -> dict:
    """Copies the tensors of a CompSPHState-like object into numpy arrays."""
    out = {}
    for name in ("positions", "velocities", "supports", "masses", "densities", "internalEnergies", "pressures", "soundspeeds",
                 "divergence", "alpha0s", "alphas", "entropies"):
        t = getattr(state, name, None)
        if t is not None:
            out[name] = t.detach().cpu().numpy().astype(dtype)
    return out
