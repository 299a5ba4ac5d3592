"""Generates the golden vectors in tests/golden/ by executing the reference's own
Python source (wi-re/warpSPH, read from /root/reference at generation time only).

The hot-path arithmetic that lives in the reference repository is plain Python:
Warp @wp.func bodies (modules/crk/accel.py, modules/crk/dudt.py, modules/crk/limiter.py,
modules/compSPH/balance.py, modules/shockCapturing/wp_vsig.py, modules/dissipation/pi.py,
modules/dissipation/util.py) and torch code (modules/eos/idealGas.py,
modules/compSPH/multistep.py, modules/shockCapturing/CullenDehnen2010.py,
modules/timestep/compressible.py, modules/adaptiveSupport/optimalSupportMonaghan.py).
This script runs those function bodies unmodified, with
  * a numpy stand-in for the Warp builtins they call (wp.dot, wp.min/max with Warp's
    `a < b ? a : b` semantics, wp.exp, wp.pow, ...; decorators are identities), all
    arithmetic in numpy float32 scalars and arrays;
  * the pieces the reference imports from its absent sibling package warpSPHCore
    (minimum-image distance, Wendland kernel and gradient, the CRK-corrected gradient,
    particle accessors, generic interpolation) supplied by this project's restatement,
    operation for operation as in oracle/sph_oracle.c.
Inputs that come from warpSPHCore in the reference (CRK coefficients, volumes,
densities) are computed by the FP32 oracle and stored with the outputs, so a test
can feed identical inputs to the oracle or the GPU and compare with the reference's
own results.

Usage (in a container that has the reference checkout):
    python tests/golden/make_golden.py --reference <reference checkout> [--which ...]
"""
from __future__ import annotations

import argparse
import inspect
import re
import sys
import types
from dataclasses import dataclass, field
from enum import Enum
from pathlib import Path
from typing import Any, List, Optional, Tuple, Union

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

F = np.float32


# ---------------------------------------------------------------- Warp stand-in
def _ident(*a, **k):
    if len(a) == 1 and callable(a[0]) and not k:
        return a[0]
    return lambda f: f


wp = types.SimpleNamespace(
    func=_ident, kernel=_ident, struct=_ident, static=lambda x: x,
    dot=lambda a, b: F(np.dot(np.asarray(a, F), np.asarray(b, F))),
    min=lambda a, b: a if a < b else b, max=lambda a, b: a if a > b else b,
    abs=lambda x: abs(x), exp=lambda x: F(np.exp(F(x))), pow=lambda a, b: F(np.power(F(a), F(b))),
    sqrt=lambda x: F(np.sqrt(F(x))),
    clamp=lambda x, lo, hi: (lo if x < lo else (hi if x > hi else x)),
    outer=lambda a, b: np.outer(np.asarray(a, F), np.asarray(b, F)).astype(F),
    acos=lambda x: F(np.arccos(np.clip(F(x), F(-1), F(1)))),     # Warp clamps the argument
    normalize=lambda v: (np.asarray(v, F) / F(np.sqrt(F(np.dot(np.asarray(v, F), np.asarray(v, F)))))).astype(F)
    if F(np.dot(np.asarray(v, F), np.asarray(v, F))) > 0 else np.zeros_like(np.asarray(v, F)),
    int32=int, int64=int, bool=bool, float32=F, array=lambda *a, **k: None, tid=lambda: 0,
)
vector = matrix = lambda *a, **k: None


# ---------------------------------------------------------------- warpSPHCore restatement (ours)
class OperationDirection(Enum):
    TrueAllToToAll = 0
    AllToAll = 1
    FluidToGhost = 2
    BoundaryToFluid = 3


KSCALE = {(1, 1): 1.620185175, (1, 2): 1.897366596, (1, 3): 1.936491673,
          (2, 1): 1.936491673, (2, 2): 2.171240593, (2, 3): 2.207940217,
          (3, 1): 2.207940217, (3, 2): 2.415229458, (3, 3): 2.449489743}


def kernel_C(K, D):
    pi = 3.14159265358979323846
    if K == 1:
        return F(1.25) if D == 1 else (F(7.0 / pi) if D == 2 else F(21.0 / (2.0 * pi)))
    if K == 2:
        return F(1.5) if D == 1 else (F(9.0 / pi) if D == 2 else F(495.0 / (32.0 * pi)))
    return F(1.71875) if D == 1 else (F(78.0 / (7.0 * pi)) if D == 2 else F(1365.0 / (64.0 * pi)))


def kernel_kp(K, D, q):
    t = F(1) - q
    if K == 1:
        if D == 1:
            t2 = t * t
            return t2 * t * (F(1) + F(3) * q), F(12) * t2
        t3 = t * t * t
        return t3 * t * (F(1) + F(4) * q), F(20) * t3
    if K == 2:
        if D == 1:
            t4 = (t * t) * (t * t)
            return t4 * t * (F(1) + F(5) * q + F(8) * q * q), F(14) * (F(1) + F(4) * q) * t4
        t5 = (t * t) * (t * t) * t
        return t5 * t * (F(1) + F(6) * q + (F(35) / F(3)) * q * q), (F(56) / F(3)) * (F(1) + F(5) * q) * t5
    if D == 1:
        t6 = (t * t) * (t * t) * (t * t)
        return t6 * t * (F(1) + F(7) * q + F(19) * q * q + F(21) * q * q * q), F(6) * (F(3) + F(18) * q + F(35) * q * q) * t6
    t7 = (t * t) * (t * t) * (t * t) * t
    return t7 * t * (F(1) + F(8) * q + F(25) * q * q + F(32) * q * q * q), F(22) * (F(1) + F(7) * q + F(16) * q * q) * t7


def ipowD(h, D):
    return h if D == 1 else (h * h if D == 2 else h * h * h)


class Ctx:
    kernel = 2
    dim = 2
    L = F(1.0)
    halfL = F(0.5)
    periodic = True


def computeDistanceVec(xi, xj, domainState=None):
    d = (np.asarray(xi, F) - np.asarray(xj, F)).astype(F)
    if Ctx.periodic:
        d = np.where(d > Ctx.halfL, (d - Ctx.L).astype(F), np.where(d < -Ctx.halfL, (d + Ctx.L).astype(F), d)).astype(F)
    return d


def safe_sqrt(x):
    return F(np.sqrt(F(x if x > 0 else 0)))


def kWG(x, r, H):
    K, D = Ctx.kernel, Ctx.dim
    q = F(r) / F(H)
    if not (q < F(1)):
        return F(0), np.zeros(D, F)
    k, p = kernel_kp(K, D, q)
    cH = kernel_C(K, D) / ipowD(F(H), D)
    W = cH * k
    s = -cH * p / (F(H) * F(H))
    return F(W), (F(s) * np.asarray(x, F)).astype(F)


def kWdH(r, H):
    K, D = Ctx.kernel, Ctx.dim
    q = F(r) / F(H)
    if not (q < F(1)):
        return F(0), F(0)
    k, p = kernel_kp(K, D, q)
    cH = kernel_C(K, D) / ipowD(F(H), D)
    return F(cH * k), F(-cH / F(H) * (F(D) * k - q * q * p))


def computeKernelGradientCRK(xi, xj, hi, hj, kernelProperties, domainState, useCRK, A, B, gradA, gradB):
    # The CRK call sites pass equal supports; the CompSPH / Monaghan call sites pass
    # (H_i, H_j) and the operation's support scheme picks the gradient: gather uses H_i,
    # the kernel-mean scheme averages the two gradients.
    D = Ctx.dim
    x = computeDistanceVec(xi, xj, domainState)
    r = safe_sqrt(wp.dot(x, x))
    mode = getattr(kernelProperties, "supportMode", None)
    if mode == "gather":
        W, gW = kWG(x, r, hi)
    elif mode == "superSymmetric":
        W, gW = kWG(x, r, wp.max(hi, hj))
    elif mode == "kernelMeanSymmetric":
        Wi, gi = kWG(x, r, hi)
        Wj, gj = kWG(x, r, hj)
        W, gW = F(F(0.5) * (Wi + Wj)), (F(0.5) * (gi + gj)).astype(F)
    else:
        W, gW = kWG(x, r, hj)
    if not useCRK:
        return gW
    B = np.asarray(B, F)
    bx = F(1) + wp.dot(B, x)
    out = np.zeros(D, F)
    for g in range(D):
        gbx = F(gradB[0][g]) * x[0]
        for a in range(1, D):
            gbx = gbx + F(gradB[a][g]) * x[a]
        out[g] = F(A) * bx * gW[g] + F(A) * B[g] * W + F(gradA[g]) * bx * W + F(A) * gbx * W
    return out


def computeKernelCRK(xi, xj, hi, hj, kernelProperties, domainState, useCRK, A, B):
    # the kernel value under the operation's support scheme (no CRK call site here)
    x = computeDistanceVec(xi, xj, domainState)
    r = safe_sqrt(wp.dot(x, x))
    mode = getattr(kernelProperties, "supportMode", None)
    h = hi if mode == "gather" else (wp.max(hi, hj) if mode == "superSymmetric" else hj)
    return kWG(x, r, h)[0]


def sphKernelDkDh(xi, xj, hi, hj, kernelProperties, domainState):
    # gather support (the only call site, wp_omega.py:71, runs under SupportScheme.Gather)
    x = computeDistanceVec(xi, xj, domainState)
    return kWdH(safe_sqrt(wp.dot(x, x)), hi)[1]


def iPow(x, n):
    out = F(x)
    for _ in range(int(n) - 1):
        out = F(out * F(x))
    return out


def sphKernelScale(kernel, dim):
    return F(KSCALE[(int(kernel), int(dim))])


sphKernel_xi = sphKernelScale


def zero_like_warp(v):
    return np.zeros_like(np.asarray(v, F)) if np.ndim(v) else F(0)


def matmul(M, x):
    M = np.asarray(M, F)
    x = np.asarray(x, F)
    D = len(x)
    out = np.zeros(D, F)
    for a in range(D):
        s = M[a, 0] * x[0]
        for b in range(1, D):
            s = s + M[a, b] * x[b]
        out[a] = s
    return out


class SoA:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def getParticle(state, j):
    return state.positions[j], F(state.supports[j]), F(state.masses[j]), F(state.densities[j]), int(state.kinds[j])


def getVolume_j(cd, j):
    return True, F(cd.V[j])


def getCRK_j(cd, j):
    return True, F(cd.A[j]), cd.B[j], cd.gA[j], cd.gB[j]


def checkDirectionality_j(k, mode):
    return True


CORE = dict(scalar_t=F, vector=vector, matrix=matrix, Any=Any, OperationDirection=OperationDirection,
            computeDistanceVec=computeDistanceVec, safe_sqrt=safe_sqrt, computeKernelGradientCRK=computeKernelGradientCRK,
            sphKernelScale=sphKernelScale, sphKernel_xi=sphKernel_xi, zero_like_warp=zero_like_warp, matmul=matmul,
            getParticle=getParticle, getVolume_j=getVolume_j, getCRK_j=getCRK_j, checkDirectionality_j=checkDirectionality_j,
            sphKernelDkDh=sphKernelDkDh, iPow=iPow, computeKernelCRK=computeKernelCRK,
            domainData=None, kernelState=None, adjacencyData=None, gridData=None)


# ---------------------------------------------------------------- loading reference files
def load(ref: Path, rel: str, extra: dict | None = None) -> dict:
    src = (ref / "src" / "warpSPH" / rel).read_text()
    lines = src.split("\n")
    out, skip = [], False
    for ln in lines:
        if skip:
            out.append("")
            skip = "(" in ln and ")" not in ln or (skip and ")" not in ln)
            continue
        if re.match(r"^(from|import)\s", ln):
            out.append("")
            skip = "(" in ln and ")" not in ln
        else:
            out.append(ln)
    ns = dict(CORE)
    ns.update(wp=wp, torch=torch, np=np, Optional=Optional, Union=Union, Tuple=Tuple, List=List, dataclass=dataclass, field=field,
              Enum=Enum, record_function=torch.profiler.record_function, __name__="ref_" + rel.replace("/", "_"))
    if extra:
        ns.update(extra)
    sys.modules.setdefault(ns["__name__"], types.ModuleType(ns["__name__"]))   # dataclasses look their module up
    exec(compile("\n".join(out), str(ref / "src" / "warpSPH" / rel), "exec"), ns)
    return ns


def call(fn, **values):
    names = list(inspect.signature(fn).parameters)
    missing = [n for n in names if n not in values]
    if missing:
        raise KeyError(f"{fn.__name__}: no value for {missing}")
    return fn(*[values[n] for n in names])


# ---------------------------------------------------------------- inputs
def make_case(seed=0, n_side=14):
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params, make_particles
    import warpsph_b200 as ws
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    P = make_particles(2, n_side, seed=seed, jitter=0.4, flow=1.0)
    n = len(P["masses"])
    rng = np.random.default_rng(seed + 100)
    x, H, m, v = P["positions"], P["supports"], P["masses"], P["velocities"]
    # compressive + shearing flow so the limiters and the viscosity are exercised
    v = (v - 2.0 * x + 0.3 * rng.standard_normal(x.shape)).astype(F)
    u = (1.0 + 3.0 * rng.random(n)).astype(F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    V = o.crk_volume(p, x, H, nb)
    A, B, gA, gB, rho = o.crk_factors(p, x, H, m, V, nb)
    Aent, Pr, c = o.eos(p, u, rho)
    G, drho, div, vsig = o.grad_v(p, x, H, m, rho, V, A, B, gA, gB, v, c, nb, cullen=True)
    dvdt_guess = (0.5 * rng.standard_normal(x.shape)).astype(F)
    return dict(params=p, x=x, H=H, m=m, v=v, u=u, V=V, A=A, B=B, gA=gA, gB=gB, rho=rho, P=Pr, c=c, G=G, drho=drho, div=div,
                vsig=vsig, nb=nb, dvdt_guess=dvdt_guess, n=n)


def run_reference(ref: Path, case: dict) -> dict:
    import warpsph_b200 as ws
    p = case["params"]
    n = case["n"]
    nb = case["nb"]
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    nnz = len(lst)
    state = SoA(positions=case["x"], supports=case["H"], masses=case["m"], densities=case["rho"], kinds=np.zeros(n, np.int32))
    cd = SoA(V=case["V"], A=case["A"], B=case["B"], gA=case["gA"], gB=case["gB"])
    dp = ws.configurations.buildDefaultDiffusionParamsCRKSPH()
    visc = SoA(C_l=F(dp.C_l), C_q=F(dp.C_q), Cu_l=F(dp.Cu_l), Cu_q=F(dp.Cu_q), K=F(dp.K), viscosityTerm=dp.viscosityTerm,
               thermalConducitiyTerm=dp.thermalConducitiyTerm, scaleBeta=dp.scaleBeta, monaghanSwitch=dp.monaghanSwitch,
               correctXi=dp.correctXi)
    crkv = SoA(eta_fold=F(0.2), eta_crit=F(0.3333333), enableCRKLimiter=True, enableVanLeerLimiter=True,
               forceVanLeerOff=False, forceVanLeerOn=False)
    kp = SoA(operationMode=OperationDirection.TrueAllToToAll.value, kernelFunction=int(p.kernel))
    dom = SoA(dim=2)
    diff = load(ref, "configurations/moduleConfigurations/diffusionParameters.py")
    util = load(ref, "modules/dissipation/util.py", {"ViscosityTerms": diff["ViscosityTerms"]})
    pi = load(ref, "modules/dissipation/pi.py", {"ViscosityTerms": diff["ViscosityTerms"], "DiffusionParameters": None,
                                               "compute_mu_ij": util["compute_mu_ij"], "compute_bars": util["compute_bars"]})
    lim = load(ref, "modules/crk/limiter.py")
    common = dict(CRKViscosity=None, DiffusionParameters=None, computePi_actual=pi["computePi_actual"],
                  computeVanLeer=lim["computeVanLeer"], crkLimiter=lim["crkLimiter"])
    acc = load(ref, "modules/crk/accel.py", common)
    dud = load(ref, "modules/crk/dudt.py", common)
    out = {}
    ap = np.zeros((nnz, 2), F)
    av = np.zeros((nnz, 2), F)
    accel = np.zeros((n, 2), F)
    dudt = np.zeros(n, F)
    with np.errstate(all="ignore"):
        for i in range(n):
            vals = dict(i=i, dim=2, xi=case["x"][i], hi=F(case["H"][i]), mi=F(case["m"][i]), rhoi=F(case["rho"][i]),
                        referenceState=state, correctionData=cd, domainState=dom, kernelProperties=kp,
                        beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                        useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1), useVolume=True,
                        Vi=F(case["V"][i]), useCRK=True, Ai=F(case["A"][i]), Bi=case["B"][i], gradAi=case["gA"][i],
                        gradBi=case["gB"][i], vel_i=case["v"][i], referenceVelocities=case["v"], u_i=F(case["u"][i]),
                        referenceEnergies=case["u"], cs_i=F(case["c"][i]), referenceCs=case["c"], viscositySwitch=True,
                        alpha_i=F(1), referenceAlphas=np.ones(n, F), P_i=F(case["P"][i]), referencePressures=case["P"],
                        viscosityParams=visc, crkViscosityParams=crkv, gradV_i=case["G"][i],
                        referenceVelocityTensor=case["G"], pressureAccel_ij=ap, viscosityAccel_ij=av)
            accel[i] = call(acc["computeCrkSPHAccel_Func_i"], **vals)
            dudt[i] = call(dud["computeCrkSPHdudt_Func_i"], **vals)
    out.update(accel=accel, dudt=dudt, ap=ap, av=av)

    # energy partition f_ij for the six schemes (modules/compSPH/balance.py)
    bal = load(ref, "modules/compSPH/balance.py", {"EnergyScheme": ws.EnergyScheme})
    dt = F(1e-3)
    vh = (case["v"] + F(0.5) * dt * case["dvdt_guess"]).astype(F)
    fs = np.zeros((6, nnz), F)
    with np.errstate(all="ignore"):
        for es in ws.EnergyScheme:
            f_ij = np.zeros(nnz, F)
            for i in range(n):
                call(bal["computeCompSPHBalanceTerm_Func_i"], i=i, dim=2, xi=case["x"][i], hi=F(case["H"][i]), mi=F(case["m"][i]),
                     rhoi=F(case["rho"][i]), referenceState=state, domainState=dom, kernelProperties=kp,
                     beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                     useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1), referenceOmegas=None,
                     useVolume=True, Vi=F(case["V"][i]), referenceVolumes=case["V"], useCRK=True, Ai=F(case["A"][i]),
                     Bi=case["B"][i], gradAi=case["gA"][i], gradBi=case["gB"][i], vel_i=vh[i], referenceVelocities=vh,
                     u_i=F(case["u"][i]), referenceEnergies=case["u"], P_i=F(case["P"][i]), referencePressures=case["P"],
                     ap_ij=ap, av_ij=av, energyScheme_int=es.value, dt=dt, gamma=F(p.gamma), f_ij=f_ij)
            fs[es.value] = f_ij
    out.update(f_ij=fs, balance_dt=np.array([dt], F), dvdt_guess=case["dvdt_guess"])

    # signal velocity (modules/shockCapturing/wp_vsig.py)
    vs_ns = load(ref, "modules/shockCapturing/wp_vsig.py")
    vsig = np.zeros(n, F)
    with np.errstate(all="ignore"):
        for i in range(n):
            vsig[i] = call(vs_ns["computeVsig_Func_i"], i=i, dim=2, xi=case["x"][i], hi=F(case["H"][i]), mi=F(case["m"][i]),
                           rhoi=F(case["rho"][i]), referenceState=state, domainState=dom, kernelProperties=kp,
                           beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                           useGradientRenormalization=False, Li=None, useGradHTerms=False, Viscosity_i=F(1),
                           referenceViscositys=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                           Bi=None, gradAi=None, gradBi=None, vel_i=case["v"][i], referenceVelocities=case["v"],
                           individual_cs=True, cs_i=F(case["c"][i]), referenceCs=case["c"], outputValue=F(0))
    out["vsig"] = np.abs(vsig)

    # ideal-gas EOS (modules/eos/idealGas.py)
    eos = load(ref, "modules/eos/idealGas.py")
    Aent, _, Pt, ct = eos["idealGasEOS"](A=None, u=torch.from_numpy(case["u"]), P=None, rho=torch.from_numpy(case["rho"]),
                                           gamma=float(p.gamma))
    out.update(eos_A=Aent.numpy(), eos_P=Pt.numpy(), eos_c=ct.numpy())

    # Cullen-Dehnen switch algebra (modules/shockCapturing/CullenDehnen2010.py:218-331) with the
    # generic SPH operations (warpSPHCore warpOperation) restated here in numpy
    H, m, rho, x = case["H"], case["m"], case["rho"], case["x"]

    def warpOperation(state, props, domain=None, adjacency=None, queryValues=None, **kw):
        op = props.operation
        if op == "Divergence":
            return torch.from_numpy(case["div"])
        if op == "Interpolate":
            qv = queryValues.numpy() if isinstance(queryValues, torch.Tensor) else queryValues
            outv = np.zeros(n, F)
            for i in range(n):
                s = F(0)
                for k in range(offs[i], offs[i] + cnt[i]):
                    j = lst[k]
                    d = computeDistanceVec(x[i], x[j])
                    W, _ = kWG(d, safe_sqrt(wp.dot(d, d)), H[i])
                    s = s + m[j] / rho[j] * qv[j] * W
                outv[i] = s
            return torch.from_numpy(outv)
        raise NotImplementedError(op)

    class OperationProperties:
        def __init__(self, kernel=None, operation=None, supportMode=None, gradientMode=None):
            self.operation = operation

    WarpOperation = types.SimpleNamespace(Divergence="Divergence", Interpolate="Interpolate", Gradient="Gradient")
    cd_ns = load(ref, "modules/shockCapturing/CullenDehnen2010.py", dict(
        warpOperation=warpOperation, OperationProperties=OperationProperties, WarpOperation=WarpOperation,
        GradientScheme=types.SimpleNamespace(Difference=1), SupportScheme=types.SimpleNamespace(Gather=0, SuperSymmetric=3),
        ViscositySwitchState=lambda **kw: SoA(**kw), CompressibleState=None, SimulationConfig=None, CompressibleSPHConfig=None,
        AdjacencyList=None, CompactHashMap=None, computeM=None,
        computeVsigWarp=lambda *a, **k: torch.from_numpy(out["vsig"])))
    div_prev = (case["div"] * 0.7 + 0.05).astype(F)
    alpha0 = np.full(n, 0.6, F)
    ps = SoA(positions=torch.from_numpy(x), supports=torch.from_numpy(H), densities=torch.from_numpy(rho),
             divergence=torch.from_numpy(div_prev), alpha0s=torch.from_numpy(alpha0), velocities=torch.from_numpy(case["v"]),
             soundspeeds=torch.from_numpy(case["c"]))
    swc = SoA(alpha_min=0.02, alpha_max=2.0, beta_xi=2.0, limitXi=True, correctVelocityGradient=False)
    sim = SoA(kernel=types.SimpleNamespace(value=int(p.kernel)), supportMode=3, domain=None)
    a0s, sst = cd_ns["computeCullenTerms"](1e-3, ps, sim, SoA(viscositySwitchParams=swc), None, None)
    out.update(cullen_alpha=a0s.numpy().astype(F), cullen_R=sst.R.numpy().astype(F), cullen_div_prev=div_prev,
               cullen_alpha0=alpha0)

    # compatible energy (modules/compSPH/multistep.py:52-94), two stages
    ms = load(ref, "modules/compSPH/multistep.py", {"EnergyScheme": ws.EnergyScheme, "CompressibleSystemUpdate": None,
                                                     "CompSPHConfig": None, "SimulationConfig": None})
    i_idx = torch.from_numpy(np.repeat(np.arange(n), cnt).astype(np.int64))
    j_idx = torch.from_numpy(lst)
    rng = np.random.default_rng(7)
    stages, updates = [], []
    f_stage = [fs[5], fs[0]]
    for s in range(2):
        dv = (case["dvdt_guess"] * (1 + 0.3 * s)).astype(F)
        stages.append((SoA(i=i_idx, j=j_idx), SoA(f_ij=torch.from_numpy(f_stage[s]), ap_ij=torch.from_numpy(ap * F(1 + 0.1 * s)),
                                                   av_ij=torch.from_numpy(av * F(1 - 0.1 * s)))))
        updates.append(SoA(dvdt=torch.from_numpy(dv)))
    init = SoA(velocities=torch.from_numpy(case["v"]), internalEnergies=torch.from_numpy(case["u"]), positions=torch.from_numpy(x))
    for es in (ws.EnergyScheme.CRK, ws.EnergyScheme.PdV):
        du = ms["compSPH_deltaU_multistep"](float(dt), init, stages, updates, np.array([0.5, 0.5]), None, SoA(energyScheme=es))
        out[f"multistep_du_{es.name}"] = du.numpy().astype(F)
    out["multistep_dvdt"] = np.stack([u.dvdt.numpy() for u in updates])

    # CFL time step (modules/timestep/compressible.py:12-61)
    ts = load(ref, "modules/timestep/compressible.py", {"idealGasEOS": eos["idealGasEOS"], "volumeToSupportHelper": lambda *a: 0.0,
                                                        "CompressibleState": None, "CompressibleSystem": None,
                                                        "CompressibleSPHConfig": None, "SimulationConfig": None})
    sysobj = SoA(state=SoA(internalEnergies=torch.from_numpy(case["u"]), densities=torch.from_numpy(rho), supports=torch.from_numpy(H)))
    conf = SoA(adaptiveDt=True, cflFactor=0.3, dx=1.0, targetNeighbors=32, dim=2, kernel=types.SimpleNamespace(value=int(p.kernel)),
               minDt=1e-6, maxDt=1e-2, dt=1e-4, dtGrowthFactor=1.1)
    out["cfl_dt_grow"] = np.array([ts["computeTimestep"](sysobj, conf, SoA(gamma=float(p.gamma)), dt=1e-4)], np.float64)
    out["cfl_dt_first"] = np.array([ts["computeTimestep"](sysobj, conf, SoA(gamma=float(p.gamma)), dt=None)], np.float64)
    return out


# ---------------------------------------------------------------- DFSPH pressure solves
def make_dfsph_case(seed=3, n_side=16):
    """Periodic unit box, rest density 1, uniform support, a divergent velocity field,
    gravity plus noise as the non-pressure acceleration and a positive previous pressure."""
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params, make_particles
    import warpsph_b200 as ws
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    P = make_particles(2, n_side, seed=seed, jitter=0.3, flow=1.0, h_spread=0.0)
    n = len(P["masses"])
    rng = np.random.default_rng(seed + 200)
    x, H, m = P["positions"], P["supports"], P["masses"]
    v = (P["velocities"] + 0.5 * x + 0.1 * rng.standard_normal(x.shape)).astype(F)
    dvdt = (np.array([0.0, -1.0]) + 0.2 * rng.standard_normal(x.shape)).astype(F)
    p_prev = (0.1 + 0.05 * rng.random(n)).astype(F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    rho = o.density(p, 0, x, H, m, nb)
    return dict(params=p, x=x, H=H, m=m, v=v, dvdt=dvdt, p_prev=p_prev, rho=rho, nb=nb, n=n, dt=F(2e-3))


def run_reference_dfsph(ref: Path, case: dict) -> dict:
    """Runs solveDivergenceFree (modules/incompressible/divergenceFree.py) and
    solveIncompressible (modules/incompressible/incompressible.py) unmodified, with
    computeAlpha from modules/incompressible/wp_alpha.py (its Warp function body run
    per particle), computeMomentumIncompressible (modules/momentum/incompressible.py),
    computePressureAccelIISPH (modules/pressure/iisph.py) and computePressureShiftIISPH
    (modules/incompressible/drift.py).  The generic operations those call
    (warpSPHCore warpOperation: symmetric gradient, difference divergence, scatter
    support) are this project's restatement, in float32 with the oracle's order."""
    n = case["n"]
    nb = case["nb"]
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    x, H, m, rho = case["x"], case["H"], case["m"], case["rho"]
    i_idx = np.repeat(np.arange(n), cnt)
    # per-pair scatter gradients (H_j) in the oracle's operation order; H is uniform so
    # the gather gradient of computeAlpha is the same field
    gS = np.zeros((len(lst), 2), F)
    for k in range(len(lst)):
        i, j = i_idx[k], lst[k]
        d = computeDistanceVec(x[i], x[j])
        _, g = kWG(d, safe_sqrt(wp.dot(d, d)), H[j])
        gS[k] = g

    def seg_sum(vals):
        """Row sums accumulated in list order (float32, like the oracle's loop)."""
        out = np.zeros((n,) + vals.shape[1:], F)
        for k in range(len(lst)):
            out[i_idx[k]] = (out[i_idx[k]] + vals[k]).astype(F)
        return out

    def warpOperation(state, props, queryValues=None, domain=None, adjacency=None, consistentDivergence=True, **kw):
        q = queryValues.numpy().astype(F)
        rj = rho[lst]
        if props.operation == "Gradient" and props.gradientMode == "Symmetric":
            qi = (q / (rho * rho)).astype(F)
            c = (m[lst] * (qi[i_idx] + (q[lst] / (rj * rj)).astype(F))).astype(F)
            s = seg_sum((c[:, None] * gS).astype(F))
            return torch.from_numpy((rho[:, None] * s).astype(F))
        if props.operation == "Divergence" and props.gradientMode == "Difference" and not consistentDivergence:
            dq = (q[lst] - q[i_idx]).astype(F)
            t = (dq[:, 0] * gS[:, 0]).astype(F)
            for a in range(1, dq.shape[1]):
                t = (t + dq[:, a] * gS[:, a]).astype(F)
            return torch.from_numpy(seg_sum(((m[lst] / rj).astype(F) * t).astype(F)))
        raise NotImplementedError((props.operation, props.gradientMode, consistentDivergence))

    class OperationProperties:
        def __init__(self, kernel=None, operation=None, gradientMode=None, supportMode=None, **kw):
            self.operation, self.gradientMode = operation, gradientMode

    names = dict(warpOperation=warpOperation, OperationProperties=OperationProperties,
                 WarpOperation=types.SimpleNamespace(Gradient="Gradient", Divergence="Divergence", Density="Density"),
                 GradientScheme=types.SimpleNamespace(Symmetric="Symmetric", Difference="Difference"),
                 SupportScheme=types.SimpleNamespace(Scatter=1, Gather=0), CompressibleState=None, SimulationConfig=None,
                 AdjacencyList=None, CompactHashMap=None, ParticleState=None, DomainDescription=None, CRKState=None,
                 GradHState=None, RenormalizationState=None)
    mom = load(ref, "modules/momentum/incompressible.py", names)
    iis = load(ref, "modules/pressure/iisph.py", names)
    dri = load(ref, "modules/incompressible/drift.py", names)
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))

    def computeAlphaWarp(queryParticles=None, operationProperties=None, domain=None, adjacency=None, queryApparentAreas=None, **kw):
        A = queryApparentAreas.numpy().astype(F)
        out = np.zeros(n, F)
        for i in range(n):
            out[i] = alpha_ns["computeAlpha_Func_i_first"](
                i, 2, x[i], F(H[i]), F(m[i]), F(rho[i]), state, None, SoA(operationMode=0, kernelFunction=2),
                int(offs[i]), int(cnt[i]), lst, 0, None, False, None, False, F(0), None, False, F(0), None,
                False, F(1), np.zeros(2, F), np.zeros(2, F), np.zeros((2, 2), F), F(A[i]), A)
        return torch.from_numpy(out)

    alpha_names = dict(names, computeAlphaWarp=computeAlphaWarp, warpWrapper2=None, launch_kernel=None,
                       castTorchToWarpAsBuiltins=None, getL_i=None, getGradH_i=None, getVolume_i=None, getCRK_i=None,
                       checkDirectionality_i=None, checkOffset=None, particleDataSoA=None)
    alpha_ns = load(ref, "modules/incompressible/wp_alpha.py", alpha_names)
    alpha_ns["computeAlphaWarp"] = computeAlphaWarp   # the Warp launch wrapper; its per-particle body runs as is
    solver_names = dict(names, computeAlpha=alpha_ns["computeAlpha"], computeMomentumIncompressible=mom["computeMomentumIncompressible"],
                        computePressureAccelIISPH=iis["computePressureAccelIISPH"],
                        computePressureShiftIISPH=dri["computePressureShiftIISPH"])
    dfs = load(ref, "modules/incompressible/divergenceFree.py", solver_names)
    inc = load(ref, "modules/incompressible/incompressible.py", solver_names)
    particles = SoA(positions=torch.from_numpy(x), supports=torch.from_numpy(H), masses=torch.from_numpy(m),
                    densities=torch.from_numpy(rho), velocities=torch.from_numpy(case["v"]), pressures=torch.from_numpy(case["p_prev"]))
    conf = SoA(kernel=SoA(value=2), domain=None, dt=float(case["dt"]))
    out = {}
    mom_div = mom["computeMomentumIncompressible"](particles, conf, SoA(fluid=SoA(restDensity=1.0)), None, torch.from_numpy(case["v"]))
    out["alpha"] = alpha_ns["computeAlpha"](particles, conf, None, None, torch.from_numpy((m / rho).astype(F))).numpy()
    out["divergence"] = mom_div.numpy()
    pr = torch.from_numpy(case["p_prev"])
    acc = iis["computePressureAccelIISPH"](particles, pr, conf, 1, None)
    out["accel_iisph"] = acc.numpy()
    out["shift_iisph"] = dri["computePressureShiftIISPH"](particles, conf, acc, 1, None).numpy()
    runs = {"df_fixed": ("divergenceFreeSolver", dfs["solveDivergenceFree"], 2, 6, 0.0, 0.3),
            "df_default": ("divergenceFreeSolver", dfs["solveDivergenceFree"], 2, 32, 2.5e-3, 0.3),
            "rho_fixed": ("pressureSolver", inc["solveIncompressible"], 2, 6, 0.0, 0.3),
            "rho_default": ("pressureSolver", inc["solveIncompressible"], 2, 64, 5e-4, 0.3)}
    for name, (key, fn, mn, mx, tol, om) in runs.items():
        solver = SoA(minIterations=mn, maxIterations=mx, tolerance=tol, relaxationFactor=om)
        sc = SoA(fluid=SoA(restDensity=1.0), solverConfig=SoA(**{key: solver}))
        with np.errstate(all="ignore"):
            a_p, pB, errors, pressures = fn(particles, conf, sc, None, torch.from_numpy(case["dvdt"]), float(case["dt"]))
        out[f"{name}_accel"] = a_p.numpy().astype(F)
        out[f"{name}_p"] = pB.numpy().astype(F)
        out[f"{name}_errors"] = np.array(errors, np.float64)
        out[f"{name}_pressures"] = np.array(pressures, np.float64).reshape(-1, 3)
        out[f"{name}_config"] = np.array([mn, mx, tol, om], np.float64)
    return out


# ---------------------------------------------------------------- CompSPH and Monaghan-scheme pair bodies
PI_VARIANTS = np.array([[1, 0, 1], [0, 1, 0]], np.int32)   # (monaghanSwitch, scaleBeta, correctXi)
PI_COEFFS = np.array([1.0, 2.0, 0.7, 1.3, 1.0], np.float64)  # C_l, C_q, Cu_l, Cu_q, c_s


def make_compsph_case(seed=5, n_side=14):
    """Periodic unit box, varied supports, compressive + shearing flow, gather density,
    ideal-gas pressure and sound speed, a spread of switch values."""
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params, make_particles
    import warpsph_b200 as ws
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    P = make_particles(2, n_side, seed=seed, jitter=0.4, flow=1.0, h_spread=0.15)
    n = len(P["masses"])
    rng = np.random.default_rng(seed + 300)
    x, H, m = P["positions"], P["supports"], P["masses"]
    v = (P["velocities"] - 1.5 * x + 0.3 * rng.standard_normal(x.shape)).astype(F)
    u = (1.0 + 3.0 * rng.random(n)).astype(F)
    alpha = (0.2 + 1.3 * rng.random(n)).astype(F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    rho = o.density(p, 0, x, H, m, nb)
    _, Pr, c = o.eos(p, u, rho)
    sel = np.sort(rng.choice(len(nb["list"]), 512, replace=False)).astype(np.int64)
    return dict(params=p, x=x, H=H, m=m, v=v, u=u, alpha=alpha, rho=rho, P=Pr, c=c, nb=nb, n=n, pi_sel=sel)


def run_reference_compsph(ref: Path, case: dict) -> dict:
    """Executes, per particle and unmodified: computeOmega_Func_i (wp_omega.py), the
    CompSPH pair bodies computeCompSPHAccel_Func_i / computeCompSPHdudt_Func_i
    (modules/compSPH/accel.py, dudt.py) for every ViscosityTerms form, computePi_actual
    (modules/dissipation/pi.py) on a sample of pairs for every form and two flag
    settings, and the Monaghan-scheme dissipation bodies (wp_diffusion.py,
    wp_conductivity.py, wp_dissipation.py) under the kernel-mean support."""
    p = case["params"]
    n, nb = case["n"], case["nb"]
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    nnz = len(lst)
    row = np.repeat(np.arange(n), cnt)
    x, H, m, v, u, rho, Pr, c, alpha = (case[k] for k in ("x", "H", "m", "v", "u", "rho", "P", "c", "alpha"))
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))
    dom = SoA(dim=2)
    diff = load(ref, "configurations/moduleConfigurations/diffusionParameters.py")
    util = load(ref, "modules/dissipation/util.py", {"ViscosityTerms": diff["ViscosityTerms"]})
    pi = load(ref, "modules/dissipation/pi.py", {"ViscosityTerms": diff["ViscosityTerms"], "DiffusionParameters": None,
                                               "compute_mu_ij": util["compute_mu_ij"], "compute_bars": util["compute_bars"]})
    common = dict(DiffusionParameters=None, computePi_actual=pi["computePi_actual"])
    om_ns = load(ref, "modules/adaptiveSupport/wp_omega.py")
    acc = load(ref, "modules/compSPH/accel.py", common)
    dud = load(ref, "modules/compSPH/dudt.py", common)
    vis = load(ref, "modules/dissipation/wp_diffusion.py", common)
    con = load(ref, "modules/dissipation/wp_conductivity.py", common)
    dis = load(ref, "modules/dissipation/wp_dissipation.py", common)
    C_l, C_q, Cu_l, Cu_q, c_s = (F(a) for a in PI_COEFFS)

    def visc_params(term, cterm, sw=True, sb=False, cx=True):
        return SoA(c_s=c_s, C_l=C_l, C_q=C_q, Cu_l=Cu_l, Cu_q=Cu_q, K=F(1), thermalConductivity=F(0.5), viscosityTerm=int(term),
                   thermalConducitiyTerm=int(cterm), scaleBeta=bool(sb), monaghanSwitch=bool(sw), correctXi=bool(cx))

    def base(i, kp, vp):
        return dict(i=i, dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]), referenceState=state, domainState=dom,
                    kernelProperties=kp, beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, ki=0,
                    referenceKinds=state.kinds, useGradientRenormalization=False, Li=None, useGradHTerms=True,
                    omega_i=F(omega[i]) if omega is not None else F(1), referenceOmegas=omega, Viscosity_i=F(1),
                    referenceViscositys=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                    Bi=np.zeros(2, F), gradAi=np.zeros(2, F), gradBi=np.zeros((2, 2), F), vel_i=v[i], referenceVelocities=v,
                    u_i=F(u[i]), referenceEnergies=u, individual_cs=True, cs_i=F(c[i]), referenceCs=c, viscositySwitch=True,
                    alpha_i=F(alpha[i]), referenceAlphas=alpha, explicitPressure=True, P_i=F(Pr[i]), referencePressures=Pr,
                    viscosityParams=vp, outputValue=F(0))

    out = {}
    omega = None
    kp_g = SoA(operationMode=0, kernelFunction=int(p.kernel), supportMode="gather")
    om = np.zeros(n, F)
    with np.errstate(all="ignore"):
        for i in range(n):
            vals = base(i, kp_g, None)
            vals["useGradHTerms"] = False
            s = call(om_ns["computeOmega_Func_i"], **vals)
            om[i] = F(1) - s
    out["omega"] = om
    omega = om

    # computePi_actual on the sampled pairs: [variant, term, (i, j, thermal), pair]
    sel = case["pi_sel"]
    pis = np.zeros((len(PI_VARIANTS), 12, 3, len(sel)), F)
    with np.errstate(all="ignore"):
        for vi_, (sw, sb, cx) in enumerate(PI_VARIANTS):
            for t in range(12):
                vp = visc_params(t, t, sw, sb, cx)
                for q, k in enumerate(sel):
                    i, j = row[k], lst[k]
                    args = (x[i], x[j], F(H[i]), F(H[j]), F(m[i]), F(m[j]), F(rho[i]), F(rho[j]), True, F(Pr[i]), F(Pr[j]),
                            v[i], v[j], dom, int(p.kernel), F(c[i]), F(c[j]), F(alpha[i]), F(alpha[j]), vp)
                    pis[vi_, t, 0, q] = pi["computePi_actual"](*args, False, False)
                    pis[vi_, t, 1, q] = pi["computePi_actual"](*args, True, False)
                    pis[vi_, t, 2, q] = pi["computePi_actual"](*args, False, True)
    out["pi"] = pis

    # CompSPH accel (kernel-mean via explicit (H_i,H_i) / (H_j,H_j) calls) and dudt (gather)
    kp_a = SoA(operationMode=0, kernelFunction=int(p.kernel), supportMode=None)
    acc_t = np.zeros((12, n, 2), F)
    dud_t = np.zeros((12, n), F)
    ap = np.zeros((nnz, 2), F)
    av = np.zeros((nnz, 2), F)
    with np.errstate(all="ignore"):
        for t in range(12):
            vp = visc_params(t, t)
            ap_t = np.zeros((nnz, 2), F)
            av_t = np.zeros((nnz, 2), F)
            for i in range(n):
                vals = base(i, kp_a, vp)
                vals.update(pressureAccel_ij=ap_t, viscosityAccel_ij=av_t)
                acc_t[t, i] = call(acc["computeCompSPHAccel_Func_i"], **vals)
                vals["kernelProperties"] = kp_g
                dud_t[t, i] = call(dud["computeCompSPHdudt_Func_i"], **vals)
            if t == 3:      # Monaghan1992, the CompSPH default
                ap[:], av[:] = ap_t, av_t
    out.update(compsph_accel=acc_t, compsph_dudt=dud_t, compsph_ap=ap, compsph_av=av)

    # Monaghan-scheme dissipation bodies, kernel-mean support, two parameter sets
    kp_k = SoA(operationMode=0, kernelFunction=int(p.kernel), supportMode="kernelMeanSymmetric")
    sets = np.array([[7, 9], [3, 7]], np.int32)   # (viscosityTerm, thermalConducitiyTerm)
    visc_o = np.zeros((len(sets), n, 2), F)
    cond_o = np.zeros((len(sets), n), F)
    heat_o = np.zeros((len(sets), n), F)
    with np.errstate(all="ignore"):
        for si, (t, ct) in enumerate(sets):
            vp = visc_params(t, ct)
            for i in range(n):
                vals = base(i, kp_k, vp)
                vals["useGradHTerms"] = False
                vals["outputValue"] = np.zeros(2, F)
                visc_o[si, i] = call(vis["computeViscosity_Func_i"], **vals)
                vals["outputValue"] = F(0)
                cond_o[si, i] = call(con["computeConductivity_Func_i"], **vals)
                heat_o[si, i] = call(dis["computeThermalDissipation_Func_i"], **vals)
    out.update(monaghan_sets=sets, monaghan_viscosity=visc_o, monaghan_conductivity=cond_o, monaghan_heating=heat_o)
    return out


# ---------------------------------------------------------------- Cullen-Hopkins switch
def run_reference_hopkins(ref: Path, g: dict) -> dict:
    """computeHopkinsTerms and computeHopkinsUpdate (modules/shockCapturing/CullenHopkins.py)
    run unmodified on the CompSPH fixture's particles, with computeR / computeXi /
    computeShearTensor from CullenDehnen2010.py and common.py, v_sig from the wp_vsig.py
    pair body, and warpSPHCore's generic gather operations restated in numpy (difference
    gradient sum_j V_j (q_j - q_i) (x) grad W(H_i); interpolation sum_j V_j q_j W(H_i)).
    A second run sets correctVelocityGradient: computeM (common.py) then negates the
    reference's own moment-matrix pair body (wp_computeM.py computeM_Func_i, gather support)
    and torch.linalg.pinv inverts it, as CullenHopkins.py does; its results carry "cvg"."""
    Ctx.kernel, Ctx.dim = 2, 2
    x, H, m, rho, v, c = (g[k] for k in ("x", "H", "m", "rho", "v", "c"))
    offs, cnt, lst = g["offsets"], g["counts"], g["list"].astype(np.int64)
    n = len(H)
    rng = np.random.default_rng(17)
    alpha0 = (0.1 + 1.5 * rng.random(n)).astype(F)
    dt = F(2e-3)
    dvdt = (0.5 * rng.standard_normal((n, 2))).astype(F)
    pairs = []
    for i in range(n):
        for k in range(offs[i], offs[i] + cnt[i]):
            j = lst[k]
            d = computeDistanceVec(x[i], x[j])
            W, gW = kWG(d, safe_sqrt(wp.dot(d, d)), H[i])
            pairs.append((i, j, W, gW))

    def warpOperation(state, props, domain=None, adjacency=None, queryValues=None, **kw):
        q = queryValues.numpy().astype(F) if isinstance(queryValues, torch.Tensor) else np.asarray(queryValues, F)
        if props.operation == "Gradient":
            outv = np.zeros((n, 2, 2), F)
            for i, j, W, gW in pairs:
                if W == 0:
                    continue
                Vj = F(m[j] / rho[j])
                for a in range(2):
                    dq = F(Vj * (q[j, a] - q[i, a]))
                    for b in range(2):
                        outv[i, a, b] = F(outv[i, a, b] + dq * gW[b])
            return torch.from_numpy(outv)
        if props.operation == "Interpolate":
            outv = np.zeros(n, F)
            for i, j, W, gW in pairs:
                if W == 0:
                    continue
                outv[i] = F(outv[i] + m[j] / rho[j] * q[j] * W)
            return torch.from_numpy(outv)
        if props.operation == "Divergence":
            return torch.zeros(n)          # used only by computeSecondOrderV, whose result is discarded
        raise NotImplementedError(props.operation)

    class OperationProperties:
        def __init__(self, kernel=None, operation=None, supportMode=None, gradientMode=None):
            self.operation = operation

    vs_ns = load(ref, "modules/shockCapturing/wp_vsig.py")
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))
    vsig = np.zeros(n, F)
    kp = SoA(operationMode=0, kernelFunction=2)
    with np.errstate(all="ignore"):
        for i in range(n):
            vsig[i] = call(vs_ns["computeVsig_Func_i"], i=i, dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]),
                           referenceState=state, domainState=SoA(dim=2), kernelProperties=kp, beginIndex=int(offs[i]),
                           numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                           useGradientRenormalization=False, Li=None, useGradHTerms=False, Viscosity_i=F(1),
                           referenceViscositys=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                           Bi=None, gradAi=None, gradBi=None, vel_i=v[i], referenceVelocities=v, individual_cs=True,
                           cs_i=F(c[i]), referenceCs=c, outputValue=F(0))
    m_ns = load(ref, "modules/shockCapturing/wp_computeM.py")
    kpm = SoA(operationMode=OperationDirection.TrueAllToToAll.value, supportMode="gather")

    def computeMWarp(*a, **kw):
        outm = np.zeros((n, 2, 2), F)
        for i in range(n):
            outm[i] = call(m_ns["computeM_Func_i"], i=i, dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]),
                           referenceState=state, domainState=None, kernelProperties=kpm, beginIndex=int(offs[i]),
                           numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                           useGradientRenormalization=False, Li=None, useGradHTerms=False, Viscosity_i=F(1),
                           referenceViscositys=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                           Bi=None, gradAi=None, gradBi=None, outputValue=np.zeros((2, 2), F))
        return torch.from_numpy(outm)

    names = dict(warpOperation=warpOperation, OperationProperties=OperationProperties,
                 WarpOperation=types.SimpleNamespace(Divergence="Divergence", Interpolate="Interpolate", Gradient="Gradient"),
                 GradientScheme=types.SimpleNamespace(Difference=1), SupportScheme=types.SimpleNamespace(Gather=0, SuperSymmetric=3),
                 ViscositySwitchState=lambda **kw: SoA(**kw), CompressibleState=None, SimulationConfig=None,
                 CompressibleSPHConfig=None, AdjacencyList=None, CompactHashMap=None, computeMWarp=computeMWarp,
                 computeVsigWarp=lambda *a, **k: torch.from_numpy(vsig), Union=Union, Tuple=Tuple, Dict=dict, Optional=Optional)
    common = load(ref, "modules/shockCapturing/common.py", names)
    names.update({k: common[k] for k in ("computeM", "computeShearTensor")})
    cd_ns = load(ref, "modules/shockCapturing/CullenDehnen2010.py", names)
    names.update({k: cd_ns[k] for k in ("computeR", "computeXi", "computeSecondOrderV", "compute_vsig")})
    hop = load(ref, "modules/shockCapturing/CullenHopkins.py", names)
    div_prev = (0.3 * rng.standard_normal(n)).astype(F)
    ps = SoA(positions=torch.from_numpy(x), supports=torch.from_numpy(H), densities=torch.from_numpy(rho),
             divergence=torch.from_numpy(div_prev), alpha0s=torch.from_numpy(alpha0), velocities=torch.from_numpy(v),
             soundspeeds=torch.from_numpy(c))
    out = dict(hopkins_alpha0=alpha0, hopkins_div_prev=div_prev, hopkins_dt=np.array([dt], F), hopkins_vsig=np.abs(vsig))
    for tag, correct in (("hopkins", False), ("hopkins_cvg", True)):
        swc = SoA(alpha_min=0.02, alpha_max=2.0, beta_xi=2.0, limitXi=False, correctVelocityGradient=correct, beta_c=0.7,
                  beta_d=0.05)
        sim = SoA(kernel=types.SimpleNamespace(value=2), supportMode=3, domain=None)
        sch = SoA(viscositySwitchParams=swc)
        alphas, st = hop["computeHopkinsTerms"](float(dt), ps, sim, sch, None, None)
        a0n, st2 = hop["computeHopkinsUpdate"](st, float(dt), torch.from_numpy(dvdt), ps, sim, sch, None, None)
        out.update({f"{tag}_alphas": alphas.numpy().astype(F), f"{tag}_div": st.div.numpy().astype(F),
                    f"{tag}_R": st.R.numpy().astype(F), f"{tag}_Xi": st.Xi.numpy().astype(F),
                    f"{tag}_alpha0_next": a0n.numpy().astype(F)})
    out["hopkins_cvg_M"] = common["computeM"](ps, sim, sch, None, None).numpy().astype(F)
    return out


# ---------------------------------------------------------------- free-surface detection
def make_surface_case(seed=21, nx=22, ny=12):
    """A jittered 2D block of fluid in the lower half of a closed unit box: a free surface on
    top and three walls without boundary particles, so the block's edges are surface."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / 32
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * dx - 0.5, (np.arange(ny) + 0.5) * dx - 0.5, indexing="xy")
    x = np.stack([gx.ravel(), gy.ravel()], 1) + 0.2 * dx * (rng.random((nx * ny, 2)) - 0.5)
    x = x.astype(F)
    n = len(x)
    H = (dx * np.sqrt(32 / np.pi) * (1 + 0.05 * (2 * rng.random(n) - 1))).astype(F)
    m = np.full(n, dx * dx, F)
    Ctx.kernel, Ctx.dim = 2, 2
    rows = []
    for i in range(n):
        d = x[i] - x
        r = np.sqrt((d.astype(np.float64) ** 2).sum(1))
        rows.append(np.nonzero(r < 1.5 * np.maximum(H[i], H))[0].astype(np.int32))
    counts = np.array([len(r) for r in rows], np.int32)
    offsets = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32)
    lst = np.concatenate(rows).astype(np.int32)
    rho = np.zeros(n, F)
    for i in range(n):
        for j in rows[i]:
            d = computeDistanceVec(x[i], x[j])
            rho[i] = F(rho[i] + m[j] * kWG(d, safe_sqrt(wp.dot(d, d)), H[i])[0])
    return dict(x=x, H=H, m=m, rho=rho, offsets=offsets, counts=counts, list=lst)


def run_reference_surface(ref: Path, case: dict) -> dict:
    """detectFreeSurface (surfaceDetection/wrapper.py) with the SurfaceDetectionConfig
    dataclass defaults (colour-field scheme, colour-field-gradient normals, one dilation),
    run unmodified with computeColorField (colorFieldCompute.py), detectFreeSurfaceColorField
    (colorFieldDetection.py) and dilateSurface (dilation.py).  The pair bodies of
    countNeighborsWarp (util/wp_numNeighbors.py), warpSum (util/wp_sum.py) and
    dilateSurfaceMaskWarp (wp_dilate.py) are the reference's own, run per particle under
    super-symmetric support; warpSPHCore's gather interpolation and difference gradient are
    restated in numpy as for the switches."""
    Ctx.kernel, Ctx.dim = 2, 2
    x, H, m, rho = (case[k] for k in ("x", "H", "m", "rho"))
    offs, cnt, lst = case["offsets"], case["counts"], case["list"].astype(np.int64)
    n = len(H)
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))

    def warpOperation(st, props, domain=None, adjacency=None, queryValues=None, **kw):
        q = queryValues.numpy().astype(F) if isinstance(queryValues, torch.Tensor) else np.asarray(queryValues, F)
        outv = np.zeros((n, 2) if props.operation == "Gradient" else n, F)
        for i in range(n):
            for k in range(offs[i], offs[i] + cnt[i]):
                j = lst[k]
                d = computeDistanceVec(x[i], x[j])
                W, gW = kWG(d, safe_sqrt(wp.dot(d, d)), H[i])
                if W == 0:
                    continue
                Vj = F(m[j] / rho[j])
                if props.operation == "Interpolate":
                    outv[i] = F(outv[i] + Vj * q[j] * W)
                else:
                    outv[i] = (outv[i] + F(Vj * (q[j] - q[i])) * gW).astype(F)
        return torch.from_numpy(outv)

    class OperationProperties:
        def __init__(self, kernel=None, operation=None, supportMode=None, gradientMode=None, operationMode=None):
            self.operation = operation

    kp = SoA(operationMode=OperationDirection.TrueAllToToAll.value, supportMode="superSymmetric")
    common_args = dict(dim=2, referenceState=state, domainState=None, kernelProperties=kp, offsetArray=lst, ki=0,
                       referenceKinds=state.kinds, useGradientRenormalization=False, Li=None, useGradHTerms=False,
                       omega_i=F(1), referenceOmegas=None, Viscosity_i=F(1), referenceViscositys=None, useVolume=False, Vi=F(0),
                       referenceVolumes=None, useCRK=False, Ai=F(1), Bi=None, gradAi=None, gradBi=None, outputValue=F(0))

    def per_particle(fn, **extra):
        out = np.zeros(n, F)
        for i in range(n):
            out[i] = call(fn, i=i, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]), beginIndex=int(offs[i]),
                          numIndices=int(cnt[i]), **common_args, **extra)
        return torch.from_numpy(out)

    nn_ns = load(ref, "modules/util/wp_numNeighbors.py")
    sum_ns = load(ref, "modules/util/wp_sum.py")
    dil_ns = load(ref, "modules/surfaceDetection/wp_dilate.py")
    fnames = [k for k in nn_ns if k.endswith("_Func_i")]
    count_fn = nn_ns[fnames[0]]
    sum_fn = sum_ns["warpSum_Func_i"]
    dil_fn = dil_ns["dilateSurfaceMask_Func_i"]
    countNeighborsWarp = lambda *a, **k: per_particle(count_fn)
    warpSum = lambda *a, queryValues=None, **k: per_particle(sum_fn, queryValues=np.asarray(queryValues, F))
    dilateSurfaceMaskWarp = lambda *a, freeSurfaceMask=None, **k: per_particle(dil_fn, freeSurfaceMask=np.asarray(freeSurfaceMask, F))
    names = dict(warpOperation=warpOperation, OperationProperties=OperationProperties,
                 WarpOperation=types.SimpleNamespace(Interpolate="Interpolate", Gradient="Gradient"),
                 GradientScheme=types.SimpleNamespace(Difference=1, Naive=0),
                 SupportScheme=types.SimpleNamespace(Gather=0, SuperSymmetric=3), SimulationConfig=None,
                 SurfaceDetectionConfig=None, AdjacencyList=None, CompactHashMap=None, RenormalizationState=None,
                 countNeighborsWarp=countNeighborsWarp, warpSum=warpSum, dilateSurfaceMaskWarp=dilateSurfaceMaskWarp)
    cfg_ns = load(ref, "configurations/moduleConfigurations/surfaceDetection.py")
    names.update(SurfaceDetectionScheme=cfg_ns["SurfaceDetectionScheme"], NormalSource=cfg_ns["NormalSource"])
    cf_ns = load(ref, "modules/surfaceDetection/colorFieldCompute.py", names)
    names["computeColorField"] = cf_ns["computeColorField"]
    det_ns = load(ref, "modules/surfaceDetection/colorFieldDetection.py", names)
    names["detectFreeSurfaceColorField"] = det_ns["detectFreeSurfaceColorField"]
    dl_ns = load(ref, "modules/surfaceDetection/dilation.py", names)
    names["dilateSurface"] = dl_ns["dilateSurface"]
    wr_ns = load(ref, "modules/surfaceDetection/wrapper.py", names)
    sd = cfg_ns["SurfaceDetectionConfig"]()
    ps = SoA(positions=torch.from_numpy(x))
    sim = SoA(kernel=types.SimpleNamespace(value=2), domain=None, targetNeighbors=32.0)
    fsm, fs, normals, _, _ = wr_ns["detectFreeSurface"](ps, sim, None, sd, None, returnNormals=True)
    c, gc = cf_ns["computeColorField"](ps, sim, None, None)
    nnb = per_particle(count_fn)
    return dict(surface_color=c.numpy().astype(F), surface_color_grad=gc.numpy().astype(F), surface_num_neighbors=nnb.numpy(),
                surface_fsm=fsm.numpy().astype(F), surface_fs=fs.numpy().astype(F), surface_normals=normals.numpy().astype(F),
                surface_target_neighbors=np.array([32.0], F), surface_threshold=np.array([sd.colorFieldThreshold], F),
                surface_expansion=np.array([sd.expansionIterations], np.int32))


def run_reference_surface_schemes(ref: Path, case: dict, base: dict) -> dict:
    """The other detection schemes on the surface case, with the reference's own bodies:
    Barecasco (wp_barecasco.py computeBarecascoSurfaceDetection_Func_i_first / _second and
    the kernel's normalisation, barecascoDetection.py's mask) at the buildDefault threshold
    pi/3 and the dataclass default 1.5; Maronne (wp_maronne.py
    computeMaronneSurfaceDetection_Func_i and computeMaronneSurfaceDetection's mask) with two
    normal fields, the colour-field normals and the Barecasco cover directions; and the
    colour-field-gradient scheme (colorFieldGradientDetection.py), run unmodified on the
    restated colour field.  All under super-symmetric support."""
    import math
    Ctx.kernel, Ctx.dim = 2, 2
    x, H, m, rho = (case[k] for k in ("x", "H", "m", "rho"))
    offs, cnt, lst = case["offsets"], case["counts"], case["list"].astype(np.int64)
    n = len(H)
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))
    kp = SoA(operationMode=OperationDirection.TrueAllToToAll.value, supportMode="superSymmetric", kernelFunction=2)
    common = dict(dim=2, referenceState=state, domainState=None, kernelProperties=kp, offsetArray=lst, ki=0,
                  referenceKinds=state.kinds, useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1),
                  referenceOmegas=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1), Bi=None, gradAi=None,
                  gradBi=None)
    out = {}
    bc = load(ref, "modules/surfaceDetection/wp_barecasco.py")
    first, second = bc["computeBarecascoSurfaceDetection_Func_i_first"], bc["computeBarecascoSurfaceDetection_Func_i_second"]
    for tag, theta in (("pi3", F(math.pi / 3)), ("1p5", F(1.5))):
        nrm = np.zeros((n, 2), F)
        count = np.zeros(n, F)
        for i in range(n):
            pi_ = dict(i=i, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]), beginIndex=int(offs[i]), numIndices=int(cnt[i]))
            cv = call(first, **pi_, **common)
            ch = wp.normalize(cv)
            nrm[i] = ch
            count[i] = call(second, **pi_, **common, coverVector=ch, threshold=theta)
        out[f"barecasco_{tag}_normals"] = nrm
        out[f"barecasco_{tag}_count"] = count
        out[f"barecasco_{tag}_fsm"] = (count < 0.5).astype(F)
        out[f"barecasco_{tag}_threshold"] = np.array([theta], F)
    mr = load(ref, "modules/surfaceDetection/wp_maronne.py")
    mfn = mr["computeMaronneSurfaceDetection_Func_i"]
    for tag, normals in (("colour", base["surface_normals"]), ("cover", out["barecasco_pi3_normals"])):
        count = np.zeros(n, F)
        for i in range(n):
            count[i] = call(mfn, i=i, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]), beginIndex=int(offs[i]),
                            numIndices=int(cnt[i]), **common, normals=np.asarray(normals, F))
        out[f"maronne_{tag}_normals"] = np.asarray(normals, F)
        out[f"maronne_{tag}_count"] = count
        out[f"maronne_{tag}_fsm"] = (count < 0.5).astype(F)
    # colour-field-gradient scheme, unmodified, on the colour field of run_reference_surface
    names = dict(SimulationConfig=None, SurfaceDetectionConfig=None, AdjacencyList=None, CompactHashMap=None,
                 computeColorField=lambda *a, **k: (torch.from_numpy(base["surface_color"]), torch.from_numpy(base["surface_color_grad"])))
    cg = load(ref, "modules/surfaceDetection/colorFieldGradientDetection.py", names)
    cfg_ns = load(ref, "configurations/moduleConfigurations/surfaceDetection.py")
    sd = cfg_ns["SurfaceDetectionConfig"]()
    ps = SoA(positions=torch.from_numpy(x), supports=torch.from_numpy(H))
    sim = SoA(kernel=types.SimpleNamespace(value=2), dim=2)
    fs, nrm = cg["detectFreeSurfaceColorFieldGradient"](ps, sim, None, sd, None, returnNormals=True)
    out["cfgrad_fsm"] = fs.numpy().astype(F)
    out["cfgrad_normals"] = nrm.numpy().astype(F)
    out["cfgrad_threshold"] = np.array([sd.colorFieldGradThreshold], F)
    return out


# ---------------------------------------------------------------- Owen adaptive support
def _eval_C_d(dim, kernel):
    return kernel_C(int(kernel), int(dim))


def _eval_k(q, dim, kernel):
    q = F(q)
    if not (q < F(1)):
        return F(0)
    return F(kernel_kp(int(kernel), int(dim), q)[0])


def _eval_dkdq(q, dim, kernel):
    q = F(q)
    if not (q < F(1)):
        return F(0)
    return F(-(q * kernel_kp(int(kernel), int(dim), q)[1]))


def run_reference_owen(ref: Path) -> dict:
    """The reference's table generator (wp_psi.py computePsi, its per-entry body run with
    wp.tid() set to the entry), the psi0 pair body (wp_psi0.py computePsi0_Func_i, gather
    support), the table lookup (owenLUT.py interpolateLUT) and the support update
    (optimalSupportOwen.py computeNewSupport), with this project's Wendland restatement
    for the absent warpSPHCore kernel functions."""
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params, make_particles
    import warpsph_b200 as ws
    from warpsph_b200.owen import owen_table
    psi_ns = load(ref, "modules/adaptiveSupport/wp_psi.py", dict(eval_k=_eval_k, eval_dkdq=_eval_dkdq, eval_C_d=_eval_C_d,
                                                                  math=__import__("math")))
    out = {}
    rng = np.random.default_rng(11)
    for (kern, dim, nsel) in ((1, 1, 64), (2, 2, 48), (2, 3, 4)):
        nlut = 2 ** 12
        sel = np.sort(rng.choice(nlut, nsel, replace=False))
        n_out, psi, psiH, NH = (np.zeros(nlut, F) for _ in range(4))
        for i in sel:
            wp.tid = (lambda k: (lambda: int(k)))(i)
            with np.errstate(all="ignore"):
                psi_ns["computePsi"](kern, dim, F(2.0), F(6.0), nlut, n_out, psi, psiH, NH)
        out[f"owen_lut_sel_k{kern}_d{dim}"] = sel
        out[f"owen_lut_nh_k{kern}_d{dim}"] = n_out[sel].astype(np.float64)
        out[f"owen_lut_psiH_k{kern}_d{dim}"] = psiH[sel].astype(np.float64)
    wp.tid = lambda: 0
    # per-particle iteration, 2D Wendland C4
    Ctx.kernel, Ctx.dim = 2, 2
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    P = make_particles(2, 16, seed=21, jitter=0.4, h_spread=0.15)
    x, H, m = P["positions"], P["supports"], P["masses"]
    n = len(H)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    rho = o.density(p, 0, x, H, m, nb)
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))

    def sphKernel(xi, xj, hi, hj, kp, dom):
        d = computeDistanceVec(xi, xj)
        return kWG(d, safe_sqrt(wp.dot(d, d)), hi)[0]

    def sphKernelGradient(xi, xj, hi, hj, kp, dom):
        d = computeDistanceVec(xi, xj)
        return kWG(d, safe_sqrt(wp.dot(d, d)), hi)[1]

    psi0_ns = load(ref, "modules/adaptiveSupport/wp_psi0.py", dict(sphKernel=sphKernel, sphKernelGradient=sphKernelGradient,
                                                                    dim_t=None))
    psi0 = np.zeros(n, F)
    psi0H = np.zeros(n, F)
    kp = SoA(operationMode=0, kernelFunction=2, supportMode="gather")
    with np.errstate(all="ignore"):
        for i in range(n):
            a, b = call(psi0_ns["computePsi0_Func_i"], i=i, dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]),
                        referenceState=state, domainState=SoA(dim=2), kernelProperties=kp, beginIndex=int(offs[i]),
                        numIndices=int(cnt[i]), offsetArray=lst, ki=0, referenceKinds=state.kinds,
                        useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1), referenceOmegas=None,
                        useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1), Bi=np.zeros(2, F),
                        gradAi=np.zeros(2, F), gradBi=np.zeros((2, 2), F))
            psi0[i], psi0H[i] = a, b
    lut_ns = load(ref, "modules/adaptiveSupport/owenLUT.py", dict(generatePSILut_warp=None))
    nh_tab, psiH_tab = owen_table(ws.KernelFunctions.Wendland4, 2)
    LUT = [torch.from_numpy(nh_tab), [torch.from_numpy(psiH_tab)], [torch.from_numpy(psiH_tab)], [torch.from_numpy(nh_tab)]]
    n_h = lut_ns["interpolateLUT"](LUT, 2, which="n_h", psiH=torch.from_numpy(psi0H).to(torch.float64)).to(torch.float32)
    own_ns = load(ref, "modules/adaptiveSupport/optimalSupportOwen.py", dict(computePsi0Warp=None, computeOwen=None,
                                                                             interpolateLUT=None, CompressibleState=None,
                                                                             SimulationConfig=None, CompressibleSPHConfig=None,
                                                                             KernelFunctions=None, AdjacencyList=None,
                                                                             CompactHashMap=None, SupportScheme=None))
    target = own_ns["nH_to_n_h"](float(p.target_neighbors), 2)
    Ht = torch.from_numpy(H)
    h = own_ns["computeNewSupport"](target, n_h, Ht)
    h = h.clamp(min=Ht.min() * 0.25, max=Ht.max() * 4.0)
    out.update(owen_x=x, owen_H=H, owen_m=m, owen_offsets=offs, owen_counts=cnt, owen_list=nb["list"], owen_psi0=psi0,
               owen_psi0H=psi0H, owen_nh=n_h.numpy(), owen_Hnew=h.numpy(), owen_target=np.array([target]))
    return out


# ---------------------------------------------------------------- delta-SPH pair bodies
WC_COEFFS = np.array([0.05, 10.0, 1e-3], np.float64)   # inviscid alpha, c_s, viscid nu


def make_deltasph_case(seed=9, n_side=16):
    """Periodic unit box, varied supports (the super-symmetric support max(H_i, H_j)),
    a compressive + shearing flow, densities from the gather sum perturbed by a few
    per cent, and the renormalised density gradient and stiff-Tait pressure of the
    oracle's first delta-SPH pass (warpSPHCore quantities in the reference)."""
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params, make_particles
    import warpsph_b200 as ws
    from warpsph_b200.configurations import WeaklyCompressibleSPHConfig, wc_params
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    P = make_particles(2, n_side, seed=seed, jitter=0.3, flow=1.0, h_spread=0.15)
    n = len(P["masses"])
    rng = np.random.default_rng(seed + 400)
    x, H, m = P["positions"], P["supports"], P["masses"]
    v = (P["velocities"] - 1.2 * x + 0.3 * rng.standard_normal(x.shape)).astype(F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    rho0 = o.density(p, 0, x, H, m, nb)
    rho = (rho0 * (1.0 + 0.03 * rng.standard_normal(n))).astype(F)
    wc = wc_params(WeaklyCompressibleSPHConfig())
    _, _, gL, Pr = o.deltasph_rhs(p, wc, x, H, m, rho, v, nb)
    return dict(params=p, x=x, H=H, m=m, v=v, rho=rho, gL=gL.astype(F), P=Pr.astype(F), nb=nb, n=n)


def run_reference_deltasph(ref: Path, case: dict) -> dict:
    """Executes, per particle and unmodified, the delta-SPH pair bodies under the
    super-symmetric support: computeVelocityDiffusionDeltaSPH_Func_i
    (modules/deltaSPH/wp_viscosityDelta.py; inviscid and viscid), 
    computeDensityDiffusionDeltaSPH_Func_i (modules/deltaSPH/wp_densityDelta.py; the
    deltaSPH, densityOnly and deltaOnly schemes) and computePressureSurfaceAware_Func_i
    (modules/pressure/wp_surfaceAware.py; every pressure term without a surface mask, and
    the Antuono term with every third particle marked as free surface)."""
    p = case["params"]
    n, nb = case["n"], case["nb"]
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    x, H, m, v, rho, gL, Pr = (case[k] for k in ("x", "H", "m", "v", "rho", "gL", "P"))
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=np.zeros(n, np.int32))
    dom = SoA(dim=2)
    enums = load(ref, "enumTypes.py")
    extra = dict(DensityDiffusionScheme=enums["DensityDiffusionScheme"], PressureForceScheme=enums["PressureForceScheme"])
    vis = load(ref, "modules/deltaSPH/wp_viscosityDelta.py", extra)
    den = load(ref, "modules/deltaSPH/wp_densityDelta.py", extra)
    prs = load(ref, "modules/pressure/wp_surfaceAware.py", extra)
    kp = SoA(operationMode=0, kernelFunction=int(p.kernel), supportMode="superSymmetric")
    alpha, c_s, nu = (F(a) for a in WC_COEFFS)

    def base(i):
        return dict(i=i, dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]), referenceState=state, domainState=dom,
                    kernelProperties=kp, beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, ki=0,
                    referenceKinds=state.kinds, useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1),
                    referenceOmegas=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                    Bi=np.zeros(2, F), gradAi=np.zeros(2, F), gradBi=np.zeros((2, 2), F), vel_i=v[i], referenceVelocities=v,
                    alpha=alpha, c_s=c_s, nu=nu, n=2, gradRho_i=np.zeros(2, F), referenceGradRho=np.zeros((n, 2), F),
                    gradRhoL_i=gL[i], referenceGradRhoL=gL, P_i=F(Pr[i]), referencePressures=Pr, mask_i=0,
                    referenceSurfaceMask=np.zeros(n, np.int32), PressureSurfaceAware_i=F(0), referencePressureSurfaceAwares=None,
                    outputValue=np.zeros(2, F))

    out = {"visc_inviscid": np.zeros((n, 2), F), "visc_viscid": np.zeros((n, 2), F),
           "dd": np.zeros((3, n), F), "pf": np.zeros((6, n, 2), F)}
    schemes = [enums["DensityDiffusionScheme"].deltaSPH.value, enums["DensityDiffusionScheme"].densityOnly.value,
               enums["DensityDiffusionScheme"].deltaOnly.value]
    with np.errstate(all="ignore"):
        for i in range(n):
            b = base(i)
            out["visc_inviscid"][i] = call(vis["computeVelocityDiffusionDeltaSPH_Func_i"], inviscid=True, **b)
            out["visc_viscid"][i] = call(vis["computeVelocityDiffusionDeltaSPH_Func_i"], inviscid=False, **b)
            for s_, sch in enumerate(schemes):
                bb = dict(b, outputValue=F(0))
                out["dd"][s_, i] = call(den["computeDensityDiffusionDeltaSPH_Func_i"], densityScheme=sch, **bb)
            for t in range(6):
                out["pf"][t, i] = call(prs["computePressureSurfaceAware_Func_i"], pressureTerm=t, **b)
    # the Antuono switch with free-surface particles (mask_i == 1 forces P_j + P_i)
    smask = (np.arange(n) % 3 == 0).astype(np.int32)
    antuono = enums["PressureForceScheme"].Antuono.value
    out["pf_antuono_mask"] = np.zeros((n, 2), F)
    with np.errstate(all="ignore"):
        for i in range(n):
            b = dict(base(i), mask_i=int(smask[i]), referenceSurfaceMask=smask)
            out["pf_antuono_mask"][i] = call(prs["computePressureSurfaceAware_Func_i"], pressureTerm=antuono, **b)
    out["surface_mask"] = smask
    out["dd_schemes"] = np.array(schemes, np.int32)
    out["wc_coeffs"] = WC_COEFFS

    # delta-plus shift: computeDeltaShift (modules/shifting/delta.py) unmodified, with the
    # Warp launch wrapper replaced by the per-particle body computeDeltaShift_Func_i
    # (sample/wp_deltaShift.py) under the gather support
    def eval_k(q, dim, kf):
        return kernel_kp(int(kf), int(dim), F(q))[0] if F(q) < F(1) else F(0)

    def computeKernelCRK(xi_, xj_, hi_, hj_, kernelProperties, domainState, useCRK, A, B):
        d = computeDistanceVec(xi_, xj_, domainState)
        return kWG(d, safe_sqrt(wp.dot(d, d)), hi_)[0]

    sh_names = dict(computeKernelCRK=computeKernelCRK, computePairwiseSupport=lambda hi_, hj_, mode: hi_, eval_k=eval_k,
                    eval_C_d=lambda dim, kf: kernel_C(int(kf), int(dim)), eval_dkdq=None)
    ds = load(ref, "sample/wp_deltaShift.py", sh_names)
    kp_g = SoA(operationMode=0, kernelFunction=int(p.kernel), supportMode="gather")

    def computeDeltaShiftWarp(state_, operationProperties=None, referenceParticles=None, domain=None, adjacency=None, CFL=0.0,
                              computeMach=True, c_max=0.0, rho0=1.0, dx=0.0, R=0.25, n=4):
        xs = state_.positions.numpy().astype(F)
        outv = np.zeros((len(xs), 2), F)
        st = SoA(positions=xs, supports=H, masses=m, densities=rho, kinds=np.zeros(len(xs), np.int32))
        with np.errstate(all="ignore"):
            for i in range(len(xs)):
                b = base(i)
                b.update(xi=xs[i], referenceState=st, kernelProperties=kp_g, correctionData=None, outputValue=np.zeros(2, F))
                b.pop("n")   # the viscosity bodies' dimension argument; here n is the exponent
                outv[i] = call(ds["computeDeltaShift_Func_i"], R=R, n=n, CFL=CFL, computeMach=computeMach, c_max=c_max, rho0=rho0,
                               dx=dx, **b)
        return torch.from_numpy(outv)

    dl = load(ref, "modules/shifting/delta.py", dict(computeDeltaShiftWarp=computeDeltaShiftWarp, OperationProperties=lambda **k: None,
                                                     WarpOperation=SoA(Density=0), SupportScheme=SoA(Gather=0),
                                                     sphKernelScale=sphKernelScale))
    cfl, c0 = F(0.3), F(10.0)
    st = SoA(positions=torch.from_numpy(x.copy()), velocities=torch.from_numpy(v), supports=torch.from_numpy(H),
             densities=torch.from_numpy(rho), masses=torch.from_numpy(m))
    conf = SoA(dt=1e-3, dx=0.0625, kernel=SoA(value=int(p.kernel)), dim=2)
    sconf = SoA(shiftProperties=SoA(iterations=1, CFL=float(cfl), computeMach=True), fluid=SoA(fixedSoundSpeed=float(c0)))
    delta, _ = dl["computeDeltaShift"](st, conf, sconf, None, None, iters=1)
    out["shift"] = delta.numpy().astype(F)
    out["shift_coeffs"] = np.array([cfl, c0], np.float64)
    return out


# ---------------------------------------------------------------- mDBC (wall particles)
def make_mdbc_case(seed=11):
    """A 2D fluid block resting on a wall of three particle layers, with one ghost point per
    wall particle mirrored across the wall surface y = 0 (the layout addBoundaryGhostParticles
    builds, rigidBody/ghostParticles.py:6-79: fluid, wall, ghosts; a wall particle's ghost
    offset is x_b - x_g, its ghost's the negative).  The lowest fluid row is pressed against
    the wall and moves into it, so the no-penetration shift acts; densities are perturbed
    by a few per cent; gravity points down."""
    from oracle import oracle
    from oracle.steps import cell_capacity_for
    from tests.cases import make_params
    import warpsph_b200 as ws
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    rng = np.random.default_rng(seed)
    dx = F(1 / 32)
    fx, fy = np.meshgrid((np.arange(16) + 0.5) * dx - F(0.25), (np.arange(8) + 0.5) * dx, indexing="xy")
    fluid = np.stack([fx.ravel(), fy.ravel()], 1) + F(0.15) * dx * (rng.random((128, 2)) - F(0.5))
    fluid[:16, 1] = F(0.2) * dx
    bx, by = np.meshgrid((np.arange(20) + 0.5) * dx - F(0.3125), -(np.arange(3) + 0.5) * dx, indexing="xy")
    wall = np.stack([bx.ravel(), by.ravel()], 1)
    ghost = wall * np.array([1, -1], F)
    x = np.concatenate([fluid, wall, ghost]).astype(F)
    nf, nw = len(fluid), len(wall)
    n = len(x)
    kinds = np.concatenate([np.zeros(nf), np.ones(nw), np.full(nw, 2)]).astype(np.int32)
    gidx = np.full(n, -1, np.int32)
    gidx[nf:nf + nw] = np.arange(nf + nw, n)
    gidx[nf + nw:] = np.arange(nf, nf + nw)
    goff = np.zeros((n, 2), F)
    goff[nf:nf + nw] = (wall - ghost).astype(F)
    goff[nf + nw:] = -goff[nf:nf + nw]
    H = np.full(n, ws.volumeToSupportHelper(float(dx) ** 2, cfg.targetNeighbors, 2), F)
    m = np.full(n, float(dx) ** 2, F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    rho = (o.density(p, 0, x, H, m, nb) * (1 + 0.02 * rng.standard_normal(n))).astype(F)
    v = (0.3 * rng.standard_normal((n, 2))).astype(F)
    v[:16, 1] = -np.abs(v[:16, 1]) - F(0.1)
    v[kinds != 0] = 0
    return dict(params=p, x=x, H=H, m=m, rho=rho, v=v, kinds=kinds, ghost_indices=gidx, ghost_offsets=goff, nb=nb, n=n,
                rho0=np.array([1.0]), c_s=np.array([10.0]), gravity=np.array([0.0, -9.81]))


def run_reference_mdbc(ref: Path, case: dict) -> dict:
    """Executes the reference's mDBC code unmodified: the Liu-Liu moment body
    computeLiuMatrices_Func_i (modules/liu/wp_mat.py) for every ghost point, interpolateLiuLiu
    (modules/liu/interp.py; torch.linalg.pinv) over those moments, computeMdbcDensity
    (modules/mdbc/density2025.py) on top, and the no-penetration body
    computeMdbcNoPenShift_Func_i (modules/mdbc/wp_nopenshift.py) for every fluid particle with
    its kernel's per-axis average (:413-415, restated: a @wp.kernel body)."""
    p = case["params"]
    n, nb = case["n"], case["nb"]
    offs, cnt, lst = nb["offsets"], nb["counts"], nb["list"].astype(np.int64)
    x, H, m, rho, v, kinds = (case[k] for k in ("x", "H", "m", "rho", "v", "kinds"))
    goff, gidx = case["ghost_offsets"], case["ghost_indices"]
    state = SoA(positions=x, supports=H, masses=m, densities=rho, kinds=kinds)
    dom = SoA(dim=2)
    ghosts = np.nonzero(kinds == 2)[0]
    mat = load(ref, "modules/liu/wp_mat.py", dict(checkDirectionality_j=lambda k, mode: k == 0))
    kp = SoA(operationMode=OperationDirection.FluidToGhost.value, kernelFunction=int(p.kernel), supportMode="scatter")
    cd = SoA(V=(m / rho).astype(F))
    shep, bs, As, nbrs = [], [], [], []
    with np.errstate(all="ignore"):
        for i in ghosts:
            r = call(mat["computeLiuMatrices_Func_i"], i=int(i), dim=2, xi=x[i], referenceState=state, correctionData=cd, domainState=dom,
                     kernelProperties=kp, beginIndex=int(offs[i]), numIndices=int(cnt[i]), offsetArray=lst, referenceKinds=kinds,
                     useGradientRenormalization=False, Li=None, useGradHTerms=False, omega_i=F(1), useVolume=False, Vi=F(0),
                     useCRK=False, Ai=F(1), Bi=np.zeros(2, F), gradAi=np.zeros(2, F), gradBi=np.zeros((2, 2), F),
                     referenceQuantities=rho, vector_out=np.zeros(3, F), matrix_out=np.zeros((3, 3), F), shep_out=F(0))
            shep.append(F(r[0])); bs.append(np.asarray(r[1], F)); As.append(np.asarray(r[2], F)); nbrs.append(int(r[3]))
    moments = (torch.tensor(np.array(shep, F)), torch.tensor(np.array(bs, F)), torch.tensor(np.array(As, F)),
               torch.tensor(np.array(nbrs, np.int32)))

    def computeLiuMatricesWarp(queryPositions, referenceParticles, referenceQuantities, operationProperties, domain, adjacency=None):
        return moments

    interp = load(ref, "modules/liu/interp.py", dict(computeLiuMatricesWarp=computeLiuMatricesWarp, OperationProperties=lambda **k: SoA(**k),
                                                    SupportScheme=SoA(Scatter="scatter"), AdjacencyList=type("AdjacencyList", (), {}),
                                                    SimulationConfig=object))
    dens = load(ref, "modules/mdbc/density2025.py", dict(interpolateLiuLiu=interp["interpolateLiuLiu"],
                                                          AdjacencyList=type("AdjacencyList", (), {}), CompactHashMap=object,
                                                          SimulationConfig=object))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    st = SoA(positions=T(x), supports=T(H), masses=T(m), densities=T(rho), velocities=T(v), kinds=T(kinds), ghostIndices=T(gidx),
             ghostOffsets=T(goff))
    rho0, c_s = float(case["rho0"][0]), float(case["c_s"][0])
    sc = SoA(fluid=SoA(restDensity=rho0, fixedSoundSpeed=c_s), gravityConfig=SoA(direction=[0.0, -1.0], magnitude=9.81, active=True))
    out = {"mdbc_density": dens["computeMdbcDensity"](st, SoA(kernel=None, domain=None), sc, None).numpy().astype(F),
           "liu_b": np.array(bs, F), "liu_A": np.array(As, F), "liu_nbrs": np.array(nbrs, np.int32)}
    nps = load(ref, "modules/mdbc/wp_nopenshift.py", dict(checkDirectionality_j=lambda k, mode: k == 1))
    kpg = SoA(operationMode=OperationDirection.BoundaryToFluid.value, kernelFunction=int(p.kernel), supportMode="gather")
    shift = np.zeros((n, 2), F)
    with np.errstate(all="ignore"):
        for i in np.nonzero(kinds == 0)[0]:
            o_, c_ = call(nps["computeMdbcNoPenShift_Func_i"], i=int(i), dim=2, xi=x[i], hi=F(H[i]), mi=F(m[i]), rhoi=F(rho[i]),
                          referenceState=state, domainState=dom, kernelProperties=kpg, beginIndex=int(offs[i]), numIndices=int(cnt[i]),
                          offsetArray=lst, ki=0, referenceKinds=kinds, useGradientRenormalization=False, Li=None, useGradHTerms=False,
                          omega_i=F(1), referenceOmegas=None, useVolume=False, Vi=F(0), referenceVolumes=None, useCRK=False, Ai=F(1),
                          Bi=np.zeros(2, F), gradAi=np.zeros(2, F), gradBi=np.zeros((2, 2), F), vel_i=v[i], referenceVelocities=v,
                          ghostOffset_i=goff[i], referenceGhostOffsets=goff, outCtr=np.zeros(2, np.int32))
            shift[i] = [F(o_[d]) / (F(c_[d]) + F(1e-12)) for d in range(2)]
    out["nopen_shift"] = shift
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout (wi-re/warpSPH)")
    ap.add_argument("--which", choices=["all", "crk", "dfsph", "compsph", "owen", "hopkins", "deltasph", "surface", "mdbc"], default="all")
    a = ap.parse_args()
    ref = Path(a.reference)
    if a.which in ("all", "crk"):
        case = make_case()
        out = run_reference(ref, case)
        nb = case["nb"]
        np.savez_compressed(Path(__file__).parent / "crk_pair_golden.npz",
                            x=case["x"], H=case["H"], m=case["m"], v=case["v"], u=case["u"], V=case["V"], A=case["A"], B=case["B"],
                            gA=case["gA"], gB=case["gB"], rho=case["rho"], P=case["P"], c=case["c"], G=case["G"], div=case["div"],
                            offsets=nb["offsets"], counts=nb["counts"], list=nb["list"], **out)
        print("wrote", Path(__file__).parent / "crk_pair_golden.npz", "particles", case["n"], "pairs", len(nb["list"]))
    if a.which in ("all", "dfsph"):
        case = make_dfsph_case()
        out = run_reference_dfsph(ref, case)
        nb = case["nb"]
        np.savez_compressed(Path(__file__).parent / "dfsph_golden.npz",
                            x=case["x"], H=case["H"], m=case["m"], v=case["v"], dvdt=case["dvdt"], p_prev=case["p_prev"],
                            rho=case["rho"], dt=np.array([case["dt"]], F), offsets=nb["offsets"], counts=nb["counts"], list=nb["list"],
                            **out)
        print("wrote", Path(__file__).parent / "dfsph_golden.npz", "particles", case["n"], "pairs", len(nb["list"]),
              {k: len(out[k]) for k in out if k.endswith("_errors")})
    if a.which in ("all", "compsph"):
        case = make_compsph_case()
        out = run_reference_compsph(ref, case)
        nb = case["nb"]
        np.savez_compressed(Path(__file__).parent / "compsph_golden.npz",
                            x=case["x"], H=case["H"], m=case["m"], v=case["v"], u=case["u"], alpha=case["alpha"], rho=case["rho"],
                            P=case["P"], c=case["c"], offsets=nb["offsets"], counts=nb["counts"], list=nb["list"],
                            pi_sel=case["pi_sel"], pi_variants=PI_VARIANTS, pi_coeffs=PI_COEFFS, **out)
        print("wrote", Path(__file__).parent / "compsph_golden.npz", "particles", case["n"], "pairs", len(nb["list"]))
    if a.which in ("all", "hopkins"):
        g = dict(np.load(Path(__file__).parent / "compsph_golden.npz"))
        out = run_reference_hopkins(ref, g)
        np.savez_compressed(Path(__file__).parent / "hopkins_golden.npz", **out)
        print("wrote", Path(__file__).parent / "hopkins_golden.npz")
    if a.which in ("all", "surface"):
        case = make_surface_case()
        out = run_reference_surface(ref, case)
        np.savez_compressed(Path(__file__).parent / "surface_golden.npz", **case, **out)
        print("wrote", Path(__file__).parent / "surface_golden.npz", "particles", len(case["H"]), "surface", int(out["surface_fsm"].sum()))
        out2 = run_reference_surface_schemes(ref, case, out)
        np.savez_compressed(Path(__file__).parent / "surface_schemes_golden.npz", **out2)
        print("wrote", Path(__file__).parent / "surface_schemes_golden.npz",
              {k: int(v.sum()) for k, v in out2.items() if k.endswith("_fsm")})
    if a.which in ("all", "deltasph"):
        case = make_deltasph_case()
        out = run_reference_deltasph(ref, case)
        nb = case["nb"]
        np.savez_compressed(Path(__file__).parent / "deltasph_golden.npz",
                            x=case["x"], H=case["H"], m=case["m"], v=case["v"], rho=case["rho"], gL=case["gL"], P=case["P"],
                            offsets=nb["offsets"], counts=nb["counts"], list=nb["list"], **out)
        print("wrote", Path(__file__).parent / "deltasph_golden.npz", "particles", case["n"], "pairs", len(nb["list"]))
    if a.which in ("all", "mdbc"):
        case = make_mdbc_case()
        out = run_reference_mdbc(ref, case)
        nb = case["nb"]
        keep = ("x", "H", "m", "rho", "v", "kinds", "ghost_indices", "ghost_offsets", "rho0", "c_s", "gravity")
        np.savez_compressed(Path(__file__).parent / "mdbc_golden.npz", **{k: case[k] for k in keep}, offsets=nb["offsets"],
                            counts=nb["counts"], list=nb["list"], **out)
        print("wrote", Path(__file__).parent / "mdbc_golden.npz", "particles", case["n"], "pairs", len(nb["list"]),
              "ghost neighbours", out["liu_nbrs"].min(), out["liu_nbrs"].max(),
              "shifted", int((np.abs(out["nopen_shift"]).sum(1) > 0).sum()))
    if a.which in ("all", "owen"):
        out = run_reference_owen(ref)
        np.savez_compressed(Path(__file__).parent / "owen_golden.npz", **out)
        print("wrote", Path(__file__).parent / "owen_golden.npz")


if __name__ == "__main__":
    main()
