"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the reference's algorithms in plain C (``sph_oracle.c``); this
module exposes it on numpy arrays.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import it: the product (``warpsph_b200``) never
does, and never falls back to it.

Two precisions are available: ``Oracle('f32')`` computes every float operation in
single precision (tight parity with the GPU), ``Oracle('f64')`` in double (the
"all-FP64 oracle" for error and drift measurements).  The neighbour search always
runs in single precision in both, so both produce the GPU's exact lists.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> None:
    """Compiles liboracle32.so / liboracle64.so with the committed Makefile."""
    args = ["make", "-C", str(HERE)]
    if force:
        args.append("-B")
    r = subprocess.run(args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def _nullable(arrtype):
    """ndpointer that also accepts None (passed as NULL)."""
    class _N(arrtype):  # type: ignore[misc, valid-type]
        @classmethod
        def from_param(cls, obj):
            if obj is None:
                return None
            return super().from_param(obj)
    return _N


class Oracle:
    def __init__(self, precision: str = "f64"):
        if precision not in ("f32", "f64"):
            raise ValueError("precision must be 'f32' or 'f64'")
        lib_path = BUILD / ("liboracle32.so" if precision == "f32" else "liboracle64.so")
        if not lib_path.exists():
            build()
        self.lib = C.CDLL(str(lib_path))
        self.precision = precision
        self.dtype = np.float32 if precision == "f32" else np.float64
        rp = _f32p if precision == "f32" else _f64p
        rpn = _nullable(rp)
        self._rp = rp
        L = self.lib
        L.oracle_real_size.restype = C.c_int
        assert L.oracle_real_size() == np.dtype(self.dtype).itemsize
        P = C.c_void_p
        i64 = C.c_int64
        L.oracle_neighbors_build.argtypes = [P, i64, _f32p, _f32p, i64, _i32p, _u32p, _i32p, _i32p, _i32p, _nullable(_i32p),
                                             _nullable(_i32p), i64, C.POINTER(C.c_int64)]
        L.oracle_density.argtypes = [P, i64, C.c_int, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_adaptive_h_iter.argtypes = [P, i64, rp, rp, rp, _i32p, _i32p, _i32p, rp, rp, rp, rpn]
        L.oracle_crk_volume.argtypes = [P, i64, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_crk_factors.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp, rp, rp, rp, rpn]
        L.oracle_eos_ideal_gas.argtypes = [P, i64, rp, rp, rpn, rpn, rpn]
        L.oracle_grad_v.argtypes = [P, i64, rp, rp, rpn, rp, rp, rp, rp, rp, rp, rp, rpn, _i32p, _i32p, _i32p,
                                    rp, rpn, rpn, rpn]
        real_c = C.c_float if precision == "f32" else C.c_double
        self._real_c = real_c
        L.oracle_switch_cullen.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, rp, rp, real_c, _i32p, _i32p, _i32p, rp, rpn]
        L.oracle_switch_balsara.argtypes = [P, i64, rp, rp, rp]
        L.oracle_crk_accel_dudt.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, rp, rp, rp, rp, rp, rp, rp,
                                            _i32p, _i32p, _i32p, rpn, rpn, rpn, rpn]
        L.oracle_compsph_balance.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, real_c, _i32p, _i32p, _i32p, rp, rp, rp]
        L.oracle_cfl_dt.argtypes = [P, i64, rp, rp, real_c, C.c_int]
        L.oracle_cfl_dt.restype = real_c
        L.oracle_finalize_compatible_energy.argtypes = [P, i64, C.c_int, P, real_c, rp, rp, P, P, P, P, P, P, P, rp, rpn]
        L.oracle_kernel_eval.argtypes = [C.c_int, C.c_int, i64, rp, real_c, rp, rp, rp]
        L.oracle_incompressible_divergence.argtypes = [P, i64, C.c_double, rp, rp, rp, rp, rp, rpn, real_c, _i32p, _i32p, _i32p, rp]
        L.oracle_dfsph_alpha.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_pressure_accel_iisph.argtypes = [P, i64, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_pressure_shift_iisph.argtypes = [P, i64, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_deltasph_rhs.argtypes = [P, P, i64, rp, rp, rp, rp, rp, _nullable(_i32p), _i32p, _i32p, _i32p, rp, rp, rp, rp]
        L.oracle_delta_shift.argtypes = [P, i64, rp, rp, rp, rp, rp, C.c_void_p, _i32p, _i32p, _i32p, real_c, real_c, real_c, C.c_int,
                                         real_c, rp]
        L.oracle_owen_iter.argtypes = [P, i64, rp, rp, _i32p, _i32p, _i32p, _f64p, _f64p, C.c_int, C.c_double, rp, rpn, rpn, rp, rpn]
        L.oracle_switch_hopkins_terms.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, rpn, rp, rp, rp, rpn]
        L.oracle_moment_matrix.argtypes = [P, i64, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_surface_color_field.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_surface_detect.argtypes = [P, i64, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, real_c, real_c, rp, rp, rp]
        L.oracle_surface_dilate.argtypes = [P, i64, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_surface_barecasco.argtypes = [P, i64, rp, rp, _i32p, _i32p, _i32p, real_c, rp, rp, rp]
        L.oracle_surface_maronne.argtypes = [P, i64, rp, rp, rp, _i32p, _i32p, _i32p, rp, rp]
        L.oracle_surface_color_gradient.argtypes = [P, i64, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, real_c, rp, rp]
        L.oracle_surface_moments.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_surface_renorm_normals.argtypes = [P, i64, C.c_int, rp, rp, rp, rp, rp, rpn, _i32p, _i32p, _i32p, rp, rpn]
        L.oracle_switch_hopkins_update.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, rp, real_c, _i32p, _i32p, _i32p, rp, rpn]
        L.oracle_vsig.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, rp]
        L.oracle_pi_pairs.argtypes = [P, i64, rp, rp, rp, rp, rpn, rpn, rp, _i32p, _i32p, _i32p, C.c_int, C.c_int, rp]
        L.oracle_compsph_prep.argtypes = [P, i64, rp, rp, rp, rp, rp, _i32p, _i32p, _i32p, rpn, rpn, rpn]
        L.oracle_compsph_accel_dudt.argtypes = [P, i64, rp, rp, rp, rp, rp, rpn, rpn, rp, rpn, _i32p, _i32p, _i32p,
                                                rpn, rpn, rpn, rpn, rpn]
        L.oracle_monaghan_rhs.argtypes = [P, i64, rp, rp, rp, rp, rp, rp, rpn, rpn, rp, rpn, _i32p, _i32p, _i32p,
                                          rpn, rpn, rpn, rpn]
        L.oracle_jacobi_solve.argtypes = [P, C.c_int, P, i64, rp, rp, rp, rp, rp, rpn, rp, real_c, _i32p, _i32p, _i32p, rp, rp,
                                          _f64p, C.POINTER(C.c_int)]
        L.oracle_liu_moments.argtypes = [P, i64, rp, rp, rp, rp, _i32p, _i32p, _i32p, _i32p, rp, rp, _i32p]
        L.oracle_mdbc_nopen_shift.argtypes = [P, i64, rp, rp, rp, rp, _i32p, rp, _i32p, _i32p, _i32p, rp]

    # ------------------------------------------------------------------ helpers
    def arr(self, a) -> np.ndarray:
        return np.ascontiguousarray(np.asarray(a), dtype=self.dtype)

    @staticmethod
    def _p(params) -> C.c_void_p:
        return C.c_void_p(C.addressof(params))

    # ------------------------------------------------------------------ neighbour search
    def neighbors(self, params, x, H, cell_capacity: int, list_capacity: int | None = None, partition: bool = True) -> dict:
        """Verlet list in the library's layout: with ``partition`` (the library's default)
        each row holds its interacting entries first (``inter_counts`` of them)."""
        x32 = np.ascontiguousarray(np.asarray(x), dtype=np.float32)
        H32 = np.ascontiguousarray(np.asarray(H), dtype=np.float32)
        n = H32.shape[0]
        si = np.zeros(n, np.int32); sk = np.zeros(n, np.uint32); grid = np.zeros(8, np.int32)
        offs = np.zeros(n, np.int32); cnt = np.zeros(n, np.int32)
        icnt = np.zeros(n, np.int32) if partition else None
        nnz = C.c_int64(0)
        # count first
        self.lib.oracle_neighbors_build(self._p(params), n, x32, H32, cell_capacity, si, sk, grid, offs, cnt, icnt, None, 0,
                                        C.byref(nnz))
        cap = nnz.value if list_capacity is None else list_capacity
        lst = np.zeros(max(cap, 1), np.int32)
        self.lib.oracle_neighbors_build(self._p(params), n, x32, H32, cell_capacity, si, sk, grid, offs, cnt, icnt, lst, cap,
                                        C.byref(nnz))
        out = dict(sort_index=si, sorted_keys=sk, grid=grid, offsets=offs, counts=cnt, list=lst[: nnz.value], nnz=nnz.value)
        if partition:
            out["inter_counts"] = icnt
        return out

    # ------------------------------------------------------------------ pair operations
    def density(self, params, mode, x, H, m, nb) -> np.ndarray:
        n = len(H)
        out = np.zeros(n, self.dtype)
        self.lib.oracle_density(self._p(params), n, mode, self.arr(x), self.arr(H), self.arr(m), nb["offsets"], nb["counts"], nb["list"], out)
        return out

    def adaptive_h_iter(self, params, x, H, m, nb, hb):
        n = len(H)
        rho = np.zeros(n, self.dtype); Hn = np.zeros(n, self.dtype); ratio = np.zeros(n, self.dtype)
        self.lib.oracle_adaptive_h_iter(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), nb["offsets"], nb["counts"], nb["list"],
                                        self.arr(hb), rho, Hn, ratio)
        return rho, Hn, ratio

    def crk_volume(self, params, x, H, nb):
        n = len(H)
        V = np.zeros(n, self.dtype)
        self.lib.oracle_crk_volume(self._p(params), n, self.arr(x), self.arr(H), nb["offsets"], nb["counts"], nb["list"], V)
        return V

    def crk_factors(self, params, x, H, m, V, nb):
        n, d = len(H), params.dim
        A = np.zeros(n, self.dtype); B = np.zeros((n, d), self.dtype); gA = np.zeros((n, d), self.dtype)
        gB = np.zeros((n, d, d), self.dtype); rho = np.zeros(n, self.dtype)
        self.lib.oracle_crk_factors(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(V), nb["offsets"], nb["counts"],
                                    nb["list"], A, B, gA, gB, rho)
        return A, B, gA, gB, rho

    def eos(self, params, u, rho):
        n = len(u)
        A = np.zeros(n, self.dtype); P = np.zeros(n, self.dtype); c = np.zeros(n, self.dtype)
        self.lib.oracle_eos_ideal_gas(self._p(params), n, self.arr(u), self.arr(rho), A, P, c)
        return A, P, c

    def grad_v(self, params, x, H, m, rho, V, A, B, gA, gB, v, c, nb, cullen: bool = True):
        n, d = len(H), params.dim
        G = np.zeros((n, d, d), self.dtype); drho = np.zeros(n, self.dtype)
        div = np.zeros(n, self.dtype) if cullen else None
        vs = np.zeros(n, self.dtype) if cullen else None
        self.lib.oracle_grad_v(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(V), self.arr(A),
                               self.arr(B), self.arr(gA), self.arr(gB), self.arr(v), self.arr(c), nb["offsets"], nb["counts"], nb["list"],
                               G, drho, div, vs)
        return G, drho, div, vs

    def switch_cullen(self, params, x, H, m, rho, div, div_prev, vsig, alpha0, dt, nb):
        n = len(H)
        al = np.zeros(n, self.dtype); R = np.zeros(n, self.dtype)
        self.lib.oracle_switch_cullen(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(div),
                                      self.arr(div_prev), self.arr(vsig), self.arr(alpha0), float(dt), nb["offsets"], nb["counts"],
                                      nb["list"], al, R)
        return al, R

    def switch_balsara(self, params, G, c):
        n = len(c)
        al = np.zeros(n, self.dtype)
        self.lib.oracle_switch_balsara(self._p(params), n, self.arr(G), self.arr(c), al)
        return al

    def crk_accel_dudt(self, params, x, H, m, rho, V, A, B, gA, gB, v, c, P, G, nb):
        n, d = len(H), params.dim
        nnz = int(nb["list"].shape[0])
        dvdt = np.zeros((n, d), self.dtype); dudt = np.zeros(n, self.dtype)
        ap = np.zeros((max(nnz, 1), d), self.dtype); av = np.zeros((max(nnz, 1), d), self.dtype)
        self.lib.oracle_crk_accel_dudt(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(V), self.arr(A),
                                       self.arr(B), self.arr(gA), self.arr(gB), self.arr(v), self.arr(c), self.arr(P), self.arr(G),
                                       nb["offsets"], nb["counts"], nb["list"], dvdt, dudt, ap, av)
        return dvdt, dudt, ap[:nnz], av[:nnz]

    def balance(self, params, m, rho, P, u, v, dvdt, dt, nb, ap, av):
        n = len(m)
        nnz = int(nb["list"].shape[0])
        f = np.zeros(max(nnz, 1), self.dtype)
        self.lib.oracle_compsph_balance(self._p(params), n, self.arr(m), self.arr(rho), self.arr(P), self.arr(u), self.arr(v), self.arr(dvdt),
                                        float(dt), nb["offsets"], nb["counts"], nb["list"], self.arr(ap).reshape(-1), self.arr(av).reshape(-1), f)
        return f[:nnz]

    def cfl_dt(self, params, H, u, dt_prev=None) -> float:
        return float(self.lib.oracle_cfl_dt(self._p(params), len(H), self.arr(H), self.arr(u), float(dt_prev or 0.0), 1 if dt_prev else 0))

    def finalize(self, params, weights, dt, v0, u0, stages):
        """stages: list of dicts with dvdt, nb, f, ap, av (numpy)."""
        n = len(u0)
        ns = len(stages)
        keep = []

        def ptrs(arrs):
            a = (C.c_void_p * ns)(*[x.ctypes.data for x in arrs])
            keep.append(a)
            keep.extend(arrs)
            return C.cast(a, C.c_void_p)

        dv = [self.arr(s["dvdt"]) for s in stages]
        offs = [np.ascontiguousarray(s["nb"]["offsets"]) for s in stages]
        cnt = [np.ascontiguousarray(s["nb"]["counts"]) for s in stages]
        lst = [np.ascontiguousarray(s["nb"]["list"]) for s in stages]
        f = [self.arr(s["f"]) for s in stages]
        ap = [self.arr(s["ap"]) for s in stages]
        av = [self.arr(s["av"]) for s in stages]
        w = (C.c_double * ns)(*weights)
        u = np.zeros(n, self.dtype); du = np.zeros(n, self.dtype)
        self.lib.oracle_finalize_compatible_energy(self._p(params), n, ns, C.cast(w, C.c_void_p), float(dt), self.arr(v0), self.arr(u0),
                                                   ptrs(dv), ptrs(offs), ptrs(cnt), ptrs(lst), ptrs(f), ptrs(ap), ptrs(av), u, du)
        return u, du

    # ------------------------------------------------------------------ incompressible (DFSPH)
    def incompressible_divergence(self, params, rho0, x, H, m, rho, v, dvdt, dt, nb):
        out = np.zeros(len(H), self.dtype)
        self.lib.oracle_incompressible_divergence(self._p(params), len(H), float(rho0), self.arr(x), self.arr(H), self.arr(m),
                                                  self.arr(rho), self.arr(v), None if dvdt is None else self.arr(dvdt), float(dt),
                                                  nb["offsets"], nb["counts"], nb["list"], out)
        return out

    def dfsph_alpha(self, params, x, H, m, rho, nb):
        out = np.zeros(len(H), self.dtype)
        self.lib.oracle_dfsph_alpha(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(m), self.arr(rho), nb["offsets"],
                                    nb["counts"], nb["list"], out)
        return out

    def pressure_accel_iisph(self, params, x, H, m, rho, pr, nb):
        out = np.zeros((len(H), params.dim), self.dtype)
        self.lib.oracle_pressure_accel_iisph(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(pr),
                                             nb["offsets"], nb["counts"], nb["list"], out)
        return out

    def pressure_shift_iisph(self, params, x, H, m, rho, acc, nb):
        out = np.zeros(len(H), self.dtype)
        self.lib.oracle_pressure_shift_iisph(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(m), self.arr(rho),
                                             self.arr(acc), nb["offsets"], nb["counts"], nb["list"], out)
        return out

    def jacobi_solve(self, params, mode, cfg, x, H, m, rho, v, dvdt, p_init, dt, nb):
        """mode 0: solveDivergenceFree, mode 1: solveIncompressible.  cfg is a
        warpsph_b200._capi.SphJacobiConfig.  Returns (p, accel, history[iters, 4], iters)."""
        n, d = len(H), params.dim
        p = np.zeros(n, self.dtype); acc = np.zeros((n, d), self.dtype)
        hist = np.zeros((max(cfg.max_iterations, 1), 4), np.float64)
        it = C.c_int(0)
        self.lib.oracle_jacobi_solve(self._p(params), int(mode), C.c_void_p(C.addressof(cfg)), n, self.arr(x), self.arr(H), self.arr(m),
                                     self.arr(rho), self.arr(v), None if dvdt is None else self.arr(dvdt), self.arr(p_init), float(dt),
                                     nb["offsets"], nb["counts"], nb["list"], p, acc, hist, C.byref(it))
        return p, acc, hist[: it.value], it.value

    # ------------------------------------------------------------------ weakly compressible delta-SPH
    def deltasph_rhs(self, params, wc, x, H, m, rho, v, nb, surface_mask=None):
        """(dvdt, drhodt, gradRhoL, P); wc is a warpsph_b200._capi.SphWcParams; surface_mask
        the int32 free-surface indicators or None."""
        n, d = len(H), params.dim
        gL = np.zeros((n, d), self.dtype); P = np.zeros(n, self.dtype)
        dv = np.zeros((n, d), self.dtype); dr = np.zeros(n, self.dtype)
        sm = None if surface_mask is None else np.ascontiguousarray(surface_mask, np.int32)
        self.lib.oracle_deltasph_rhs(self._p(params), C.c_void_p(C.addressof(wc)), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho),
                                     self.arr(v), sm, nb["offsets"], nb["counts"], nb["list"], gL, P, dv, dr)
        return dv, dr, gL, P

    def visc_continuity(self, params, wc, x, H, m, rho, v, nb):
        """(dvdt, drhodt) of the DFSPH step's velocity diffusion and continuity: the
        delta-SPH right-hand side with zero pressure (Tait, kappa 0) and no density
        diffusion."""
        import copy
        w = copy.copy(wc)
        w.eos, w.kappa, w.density_delta = 1, 0.0, 0.0
        dv, dr, _, _ = self.deltasph_rhs(params, w, x, H, m, rho, v, nb)
        return dv, dr

    def delta_shift(self, params, x, H, m, rho, v, nb, cfl, c0, kinds=None, R=0.25, nexp=4, rho0=1.0):
        """One delta-plus shift [n, dim] (modules/shifting/delta.py, sample/wp_deltaShift.py)."""
        n, d = len(H), params.dim
        out = np.zeros((n, d), self.dtype)
        kp = None if kinds is None else np.ascontiguousarray(kinds, np.int32)
        self.lib.oracle_delta_shift(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(v),
                                    None if kp is None else kp.ctypes.data, nb["offsets"], nb["counts"], nb["list"], cfl, c0, R,
                                    int(nexp), rho0, out)
        return out

    def owen_iter(self, params, x, H, nb, lut_nh, lut_psiH, target, hb):
        """(psi0, psiH, H_new, ratio) of one Owen support iteration."""
        n = len(H)
        psi0, psiH, Hn, ratio = (np.zeros(n, self.dtype) for _ in range(4))
        self.lib.oracle_owen_iter(self._p(params), n, self.arr(x), self.arr(H), nb["offsets"], nb["counts"], nb["list"],
                                  np.ascontiguousarray(lut_nh, np.float64), np.ascontiguousarray(lut_psiH, np.float64), len(lut_nh),
                                  float(target), self.arr(hb), psi0, psiH, Hn, ratio)
        return psi0, psiH, Hn, ratio

    def moment_matrix(self, params, x, H, m, nb):
        """M_i = -sum_j m_j x_ij (x) grad W(r_ij, H_i), shape (n, D, D)."""
        n, D = len(H), int(params.dim)
        M = np.zeros((n, D, D), self.dtype)
        self.lib.oracle_moment_matrix(self._p(params), n, self.arr(x), self.arr(H), self.arr(m),
                                      nb["offsets"], nb["counts"], nb["list"], M)
        return M

    @staticmethod
    def moment_pinv(M):
        """torch.linalg.pinv's default for a float32 input (CullenHopkins.py:27): singular
        values at or below D * eps_float32 * sigma_max are dropped.  LAPACK's SVD in float64."""
        D = M.shape[-1]
        return np.linalg.pinv(np.asarray(M, np.float64), rcond=D * float(np.finfo(np.float32).eps))

    def surface_color_field(self, params, x, H, m, rho, nb):
        n = len(H)
        c = np.zeros(n, self.dtype)
        self.lib.oracle_surface_color_field(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho),
                                            nb["offsets"], nb["counts"], nb["list"], c)
        return c

    def surface_detect(self, params, x, H, m, rho, c, nb, limit, normal_sign=-1.0):
        """(fs mask, normals [n, D], neighbour counts)"""
        n, D = len(H), int(params.dim)
        fs, nn, nrm = np.zeros(n, self.dtype), np.zeros(n, self.dtype), np.zeros((n, D), self.dtype)
        self.lib.oracle_surface_detect(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(c),
                                       nb["offsets"], nb["counts"], nb["list"], float(limit), float(normal_sign), fs, nrm, nn)
        return fs, nrm, nn

    def surface_dilate(self, params, x, H, fs, nb):
        out = np.zeros(len(H), self.dtype)
        self.lib.oracle_surface_dilate(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(fs),
                                       nb["offsets"], nb["counts"], nb["list"], out)
        return out

    def surface_barecasco(self, params, x, H, nb, threshold):
        """(mask, normalised cover vectors [n, D], cone counts)"""
        n, D = len(H), int(params.dim)
        fs, cnt, nrm = np.zeros(n, self.dtype), np.zeros(n, self.dtype), np.zeros((n, D), self.dtype)
        self.lib.oracle_surface_barecasco(self._p(params), n, self.arr(x), self.arr(H), nb["offsets"], nb["counts"], nb["list"],
                                          float(threshold), fs, nrm, cnt)
        return fs, nrm, cnt

    def surface_maronne(self, params, x, H, normals, nb):
        """(mask, counts)"""
        n = len(H)
        fs, cnt = np.zeros(n, self.dtype), np.zeros(n, self.dtype)
        self.lib.oracle_surface_maronne(self._p(params), n, self.arr(x), self.arr(H), self.arr(normals), nb["offsets"], nb["counts"],
                                        nb["list"], fs, cnt)
        return fs, cnt

    def surface_color_gradient(self, params, x, H, m, rho, c, nb, threshold):
        """(mask, normals)"""
        n, D = len(H), int(params.dim)
        fs, nrm = np.zeros(n, self.dtype), np.zeros((n, D), self.dtype)
        self.lib.oracle_surface_color_gradient(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(c),
                                               nb["offsets"], nb["counts"], nb["list"], float(threshold), fs, nrm)
        return fs, nrm

    def surface_renormalization(self, params, x, H, m, rho, nb):
        """(L = pinv(M) [n, D, D] by LAPACK in FP64 with torch's FP32 cutoff, the smallest
        |eigenvalue| of the symmetric M [n], M [n, D, D])"""
        n, D = len(H), int(params.dim)
        M = np.zeros((n, D, D), self.dtype)
        self.lib.oracle_surface_moments(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), nb["offsets"],
                                        nb["counts"], nb["list"], M)
        M64 = M.astype(np.float64)
        L = np.linalg.pinv(M64, rcond=D * np.finfo(np.float32).eps).astype(self.dtype)
        lam = np.abs(np.linalg.eigvalsh(0.5 * (M64 + M64.transpose(0, 2, 1)))).min(axis=1).astype(self.dtype)
        return L, lam, M

    def surface_renorm_normals(self, params, mode, x, H, m, rho, L, lam, nb):
        """(normals, renormalised gradient)"""
        n, D = len(H), int(params.dim)
        nrm, g = np.zeros((n, D), self.dtype), np.zeros((n, D), self.dtype)
        self.lib.oracle_surface_renorm_normals(self._p(params), n, int(mode), self.arr(x), self.arr(H), self.arr(m), self.arr(rho),
                                               self.arr(L), None if lam is None else self.arr(lam), nb["offsets"], nb["counts"],
                                               nb["list"], nrm, g)
        return nrm, g

    # ------------------------------------------------------------------ mDBC
    def liu_moments(self, params, x, H, m, rho, kinds, nb):
        """(b [n, D+1], A [n, D+1, D+1], neighbour counts [n]) at the ghost rows."""
        n, D = len(H), int(params.dim)
        b = np.zeros((n, D + 1), self.dtype)
        A = np.zeros((n, D + 1, D + 1), self.dtype)
        nbrs = np.zeros(n, np.int32)
        self.lib.oracle_liu_moments(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho),
                                    np.ascontiguousarray(kinds, np.int32), nb["offsets"], nb["counts"], nb["list"], b, A, nbrs)
        return b, A, nbrs

    def mdbc_density(self, params, x, H, m, rho, kinds, ghost_indices, ghost_offsets, nb, rho0, c_s, g):
        """modules/mdbc/density2025.py:20-85 with the Liu-Liu interpolation of liu/interp.py:
        the moments from the C restatement, the pseudo-inverse by LAPACK's SVD (numpy, the
        rtol torch.linalg.pinv uses for float32) and the density formula in numpy."""
        D = int(params.dim)
        b, A, nbrs = self.liu_moments(params, x, H, m, rho, kinds, nb)
        ghost = np.nonzero(np.asarray(kinds) == 2)[0]
        f = self.dtype
        out = np.array(rho, f, copy=True)
        # the pseudo-inverse and product at the oracle's precision (the reference's torch
        # pinv runs at the moments' float32)
        bg, Ag, ng = b[ghost], A[ghost], nbrs[ghost]
        res = np.zeros_like(bg)
        for k in range(len(ghost)):
            if ng[k] > 4:
                res[k] = (np.linalg.pinv(Ag[k], rcond=(D + 1) * np.finfo(np.float32).eps) @ bg[k]).astype(f)
        res = res.astype(f)
        rho0, cs2 = f(rho0), f(c_s * c_s)
        shep = np.where(Ag[:, 0, 0] > 0, (bg[:, 0] / np.where(Ag[:, 0, 0] > 0, Ag[:, 0, 0], 1)).astype(f), rho0).astype(f)
        rho_g = np.where(ng > 1, shep, rho0).astype(f)
        P_g = (cs2 * (rho_g - rho0)).astype(f)
        rel = (-np.asarray(ghost_offsets, f)[ghost]).astype(f)
        nrm = (rel / np.maximum(np.linalg.norm(rel, axis=1, keepdims=True), 1e-12)).astype(f)
        gv = np.asarray(g, f)[:D]
        dot = (nrm * gv).sum(1).astype(f)
        dot2 = (rel * nrm).sum(1).astype(f)
        rho_b = np.maximum((rho0 + (P_g + rho0 * (dot * dot2)) / cs2).astype(f), rho0)
        rho_proj = (res[:, 0] - (rel * res[:, 1:]).sum(1)).astype(f)
        out[np.asarray(ghost_indices)[ghost]] = np.where(ng > 9, rho_proj, rho_b)
        return out, nbrs

    def mdbc_nopen_shift(self, params, x, H, m, v, kinds, ghost_offsets, nb):
        n, D = len(H), int(params.dim)
        out = np.zeros((n, D), self.dtype)
        self.lib.oracle_mdbc_nopen_shift(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(v),
                                         np.ascontiguousarray(kinds, np.int32), self.arr(ghost_offsets), nb["offsets"], nb["counts"],
                                         nb["list"], out)
        return out

    def switch_hopkins_terms(self, params, x, H, m, rho, v, alpha0, nb):
        """(alphas, div, |S|^2, R); with params.correct_velocity_gradient the gradient is
        pinv(M) V (CullenHopkins.py:24-34)."""
        n = len(H)
        al, div, s2, R = (np.zeros(n, self.dtype) for _ in range(4))
        Minv = None
        if int(getattr(params, "correct_velocity_gradient", 0)):
            Minv = self.arr(self.moment_pinv(self.moment_matrix(params, x, H, m, nb)))
        self.lib.oracle_switch_hopkins_terms(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(v),
                                             self.arr(alpha0), nb["offsets"], nb["counts"], nb["list"], Minv, div, s2, al, R)
        return al, div, s2, R

    def switch_hopkins_update(self, params, x, H, v, c, div, div_prev, alpha0, dt, nb):
        """(alpha0_next, v_sig) over whole Verlet rows."""
        n = len(H)
        a0 = np.zeros(n, self.dtype); vs = np.zeros(n, self.dtype)
        self.lib.oracle_switch_hopkins_update(self._p(params), n, self.arr(x), self.arr(H), self.arr(v), self.arr(c), self.arr(div),
                                              self.arr(div_prev), self.arr(alpha0), float(dt), nb["offsets"], nb["counts"], nb["list"],
                                              a0, vs)
        return a0, vs

    def vsig(self, params, x, H, v, c, nb):
        out = np.zeros(len(H), self.dtype)
        self.lib.oracle_vsig(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(v), self.arr(c), nb["offsets"], nb["counts"],
                             nb["list"], out)
        return out

    def _opt(self, a):
        return None if a is None else self.arr(a)

    def pi_pairs(self, params, x, H, rho, v, c, alpha, P, nb, useJ: bool = False, thermal: bool = False):
        """Pi_ij * rho_j of computePi_actual for every Verlet entry."""
        out = np.zeros(len(nb["list"]), self.dtype)
        self.lib.oracle_pi_pairs(self._p(params), len(H), self.arr(x), self.arr(H), self.arr(rho), self.arr(v), self._opt(c),
                                 self._opt(alpha), self.arr(P), nb["offsets"], nb["counts"], nb["list"], int(useJ), int(thermal), out)
        return out

    def compsph_prep(self, params, x, H, m, rho, v, nb, grad_h: bool = True):
        """(omega or None, div, drhodt)"""
        n = len(H)
        om = np.zeros(n, self.dtype) if grad_h else None
        div = np.zeros(n, self.dtype); dr = np.zeros(n, self.dtype)
        self.lib.oracle_compsph_prep(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(v),
                                     nb["offsets"], nb["counts"], nb["list"], om, div, dr)
        return om, div, dr

    def compsph_accel_dudt(self, params, x, H, m, rho, v, c, alpha, P, omega, nb):
        """(dvdt, dudt, dEdt, ap_ij, av_ij)"""
        n, d = len(H), params.dim
        nnz = len(nb["list"])
        dv = np.zeros((n, d), self.dtype); du = np.zeros(n, self.dtype); dE = np.zeros(n, self.dtype)
        ap = np.zeros((nnz, d), self.dtype); av = np.zeros((nnz, d), self.dtype)
        self.lib.oracle_compsph_accel_dudt(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(v),
                                           self._opt(c), self._opt(alpha), self.arr(P), self._opt(omega), nb["offsets"], nb["counts"],
                                           nb["list"], dv, du, dE, ap, av)
        return dv, du, dE, ap, av

    def monaghan_rhs(self, params, x, H, m, rho, v, u, c, alpha, P, omega, nb):
        """(dvdt, dudt, dEdt, terms) with terms = dict(pressure, viscosity, pdv, conductivity, heating)."""
        n, d = len(H), params.dim
        dv = np.zeros((n, d), self.dtype); du = np.zeros(n, self.dtype); dE = np.zeros(n, self.dtype)
        o5 = np.zeros((n, 2 * d + 3), self.dtype)
        self.lib.oracle_monaghan_rhs(self._p(params), n, self.arr(x), self.arr(H), self.arr(m), self.arr(rho), self.arr(v), self.arr(u),
                                     self._opt(c), self._opt(alpha), self.arr(P), self._opt(omega), nb["offsets"], nb["counts"],
                                     nb["list"], dv, du, dE, o5)
        terms = dict(pressure=o5[:, :d], viscosity=o5[:, d:2 * d], pdv=o5[:, 2 * d], conductivity=o5[:, 2 * d + 1],
                     heating=o5[:, 2 * d + 2])
        return dv, du, dE, terms

    def kernel_eval(self, kernel, dim, r, H):
        r = self.arr(r)
        W = np.zeros_like(r); dWdr = np.zeros_like(r); dWdH = np.zeros_like(r)
        self.lib.oracle_kernel_eval(kernel, dim, len(r), r, float(H), W, dWdr, dWdH)
        return W, dWdr, dWdH


_cache: dict[str, Oracle] = {}


def get(precision: str = "f64") -> Oracle:
    if precision not in _cache:
        _cache[precision] = Oracle(precision)
    return _cache[precision]


if __name__ == "__main__":  # pragma: no cover
    build(force=bool(os.environ.get("FORCE")))
    print("oracle built:", sorted(p.name for p in BUILD.glob("*.so")))
