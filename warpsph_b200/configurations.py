"""Configuration dataclasses with the reference's names, fields and defaults.

Mirrors src/warpSPH/configurations/: SimulationConfig / buildConfig
(simulationConfig.py:15-121), DiffusionParameters and ViscosityTerms
(moduleConfigurations/diffusionParameters.py:8-37, a Warp struct in the reference,
a plain dataclass here), ViscositySwitchConfig (moduleConfigurations/viscositySwitchParameters.py:11-26),
CompressibleSPHConfig (compressibleConfig.py:16-30), CompSPHConfig (compSPHConfig.py:32-40),
CRKViscosity / CRKSPHConfig (crkSPH.py:16-80), with the *ToDict / dictTo* round trips.
``make_params`` packs a configuration into the C ABI's SphParams block.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from enum import Enum
from typing import Any, Dict, List, Optional

import torch

from . import _capi
from .core import (DomainDescription, GradientScheme, IntegrationSchemeType, KernelFunctions, LaplacianScheme,
                   SamplingScheme, SupportScheme, buildDomainDescription, n_h_to_nH)
from .enumTypes import AdaptiveSupportScheme, EnergyScheme, ViscositySwitch


# ------------------------------------------------------------------ simulation config
@dataclass
class SimulationConfig:
    device: torch.device = field(default_factory=lambda: torch.device("cuda:0") if torch.cuda.is_available() else torch.device("cpu"))
    dtype: torch.dtype = torch.float32
    domain: DomainDescription = field(default_factory=lambda: buildDomainDescription(l=2, dim=2, periodic=True))
    dim: int = 2
    verletScale: float = 2.0 ** 0.5
    kernel: KernelFunctions = KernelFunctions.Wendland2
    integrationScheme: IntegrationSchemeType = IntegrationSchemeType.rungeKutta4
    cflFactor: float = 0.3
    dt: Optional[float] = None
    minDt: Optional[float] = 1e-6
    maxDt: Optional[float] = 1e-2
    dtGrowthFactor: Optional[float] = 1.1
    adaptiveDt: bool = True
    dx: Optional[float] = None
    nx: Optional[int] = None
    targetNeighbors: float = field(default_factory=lambda: n_h_to_nH(4, 2))
    supportMode: SupportScheme = SupportScheme.SuperSymmetric
    gradientMode: GradientScheme = GradientScheme.Difference
    laplacianMode: LaplacianScheme = LaplacianScheme.Brookshaw
    samplingScheme: SamplingScheme = SamplingScheme.regular


def buildConfig(device=None, dtype=None, domain=None, dim=None, verletScale=None, kernel=None, integrationScheme=None,
                cflFactor=None, dt=None, minDt=None, maxDt=None, dtGrowthFactor=None, adaptiveDt=None,
                targetNeighbors=None, supportMode=None, gradientMode=None, laplacianMode=None, samplingScheme=None):
    """simulationConfig.py:47-121: fills defaults and returns (config, integrator)."""
    from .integrators import getIntegrator
    if device is None:
        device = torch.device("cuda:0") if torch.cuda.is_available() else torch.device("cpu")
    dtype = torch.float32 if dtype is None else dtype
    dim = 2 if dim is None else dim
    domain = buildDomainDescription(l=2, dim=dim, periodic=True) if domain is None else domain
    verletScale = 2.0 ** (1 / dim) if verletScale is None else verletScale
    kernel = KernelFunctions.Wendland2 if kernel is None else kernel
    integrationScheme = IntegrationSchemeType.rungeKutta2 if integrationScheme is None else integrationScheme
    cflFactor = 0.3 if cflFactor is None else cflFactor
    adaptiveDt = True if adaptiveDt is None else adaptiveDt
    targetNeighbors = n_h_to_nH(4, dim) if targetNeighbors is None else targetNeighbors
    supportMode = SupportScheme.SuperSymmetric if supportMode is None else supportMode
    gradientMode = GradientScheme.Difference if gradientMode is None else gradientMode
    laplacianMode = LaplacianScheme.Brookshaw if laplacianMode is None else laplacianMode
    samplingScheme = SamplingScheme.regular if samplingScheme is None else samplingScheme
    minDt = 1e-6 if minDt is None else minDt
    maxDt = 1e-2 if maxDt is None else maxDt
    dtGrowthFactor = 1.1 if dtGrowthFactor is None else dtGrowthFactor
    cfg = SimulationConfig(device=device, dtype=dtype, domain=domain, dim=dim, verletScale=verletScale, kernel=kernel,
                           integrationScheme=integrationScheme, cflFactor=cflFactor, dt=dt, minDt=minDt, maxDt=maxDt,
                           dtGrowthFactor=dtGrowthFactor, adaptiveDt=adaptiveDt, targetNeighbors=targetNeighbors,
                           supportMode=supportMode, gradientMode=gradientMode, laplacianMode=laplacianMode,
                           samplingScheme=samplingScheme)
    return cfg, getIntegrator(integrationScheme)


def configurationToDict(config: SimulationConfig) -> Dict[str, Any]:
    dmin, dmax, per = config.domain.host()
    return {
        "device": str(config.device), "dtype": str(config.dtype),
        "domain": {"min": dmin, "max": dmax, "periodic": per, "dim": config.domain.dim},
        "dim": config.dim, "verletScale": config.verletScale, "kernel": config.kernel.name,
        "integrationScheme": config.integrationScheme.name, "cflFactor": config.cflFactor,
        "dt": float(config.dt) if config.dt is not None else None, "minDt": config.minDt, "maxDt": config.maxDt,
        "dtGrowthFactor": config.dtGrowthFactor, "adaptiveDt": config.adaptiveDt,
        "targetNeighbors": config.targetNeighbors, "supportMode": config.supportMode.name,
        "gradientMode": config.gradientMode.name, "laplacianMode": config.laplacianMode.name,
        "samplingScheme": config.samplingScheme.name,
    }


def dictToConfig(d: Dict[str, Any]) -> SimulationConfig:
    device = torch.device(d["device"])
    dtype = getattr(torch, d["dtype"].split(".")[-1])
    dd = d["domain"]
    domain = DomainDescription(torch.tensor(dd["min"], device=device, dtype=dtype), torch.tensor(dd["max"], device=device, dtype=dtype),
                               torch.tensor(dd["periodic"], device=device, dtype=torch.bool), dd["dim"])
    return SimulationConfig(device=device, dtype=dtype, domain=domain, dim=int(d["dim"]), verletScale=float(d["verletScale"]),
                            kernel=KernelFunctions[d["kernel"]], integrationScheme=IntegrationSchemeType[d["integrationScheme"]],
                            cflFactor=float(d["cflFactor"]), dt=None if d["dt"] is None else float(d["dt"]),
                            minDt=float(d["minDt"]), maxDt=float(d["maxDt"]), dtGrowthFactor=float(d["dtGrowthFactor"]),
                            adaptiveDt=bool(d["adaptiveDt"]), targetNeighbors=float(d["targetNeighbors"]),
                            supportMode=SupportScheme[d["supportMode"]], gradientMode=GradientScheme[d["gradientMode"]],
                            laplacianMode=LaplacianScheme[d["laplacianMode"]], samplingScheme=SamplingScheme[d["samplingScheme"]])


# ------------------------------------------------------------------ module parameters
class ViscosityTerms(Enum):
    Default = 0
    MonaghanGingold1983 = 1
    Cleary1998 = 2
    Monaghan1992 = 3
    Monaghan1997a = 4
    Monaghan1997b = 5
    Dukowicz = 6
    Price2012_98 = 7
    Price2012 = 8
    Price2008 = 9
    Wadsley2008 = 10
    DeltaSPH = 11


@dataclass
class DiffusionParameters:
    c_s: float = 1.0
    C_l: float = 1.0
    C_q: float = 2.0
    Cu_l: float = 1.0
    Cu_q: float = 2.0
    K: float = 1.0
    thermalConductivity: float = 0.5
    viscosityTerm: int = ViscosityTerms.Price2012_98.value
    thermalConducitiyTerm: int = ViscosityTerms.Price2012_98.value
    scaleBeta: bool = False
    monaghanSwitch: bool = True
    correctXi: bool = True


def buildDefaultDiffusionParamsCompressibleSPH() -> DiffusionParameters:
    return DiffusionParameters(c_s=1, C_l=1, C_q=0, Cu_l=1, Cu_q=0, K=1.0, thermalConductivity=0.5,
                               viscosityTerm=ViscosityTerms.Price2012_98.value, thermalConducitiyTerm=ViscosityTerms.Price2008.value,
                               scaleBeta=False, monaghanSwitch=True, correctXi=True)


def buildDefaultDiffusionParamsCRKSPH() -> DiffusionParameters:
    return DiffusionParameters(c_s=1, C_l=1, C_q=1, Cu_l=1, Cu_q=1, K=1.0, thermalConductivity=0.5,
                               viscosityTerm=ViscosityTerms.Monaghan1992.value, thermalConducitiyTerm=ViscosityTerms.Price2012_98.value,
                               scaleBeta=False, monaghanSwitch=True, correctXi=True)


def buildDefaultDiffusionParamsCompSPH() -> DiffusionParameters:
    return DiffusionParameters(c_s=1, C_l=1, C_q=2, Cu_l=1, Cu_q=2, K=1.0, thermalConductivity=0.5,
                               viscosityTerm=ViscosityTerms.Monaghan1992.value, thermalConducitiyTerm=ViscosityTerms.Price2012_98.value,
                               scaleBeta=False, monaghanSwitch=True, correctXi=True)


def _term_value(t) -> int:
    return t.value if isinstance(t, ViscosityTerms) else int(t)


def diffusionParamsToDict(p: DiffusionParameters) -> Dict[str, Any]:
    return {"c_s": p.c_s, "C_l": p.C_l, "C_q": p.C_q, "Cu_l": p.Cu_l, "Cu_q": p.Cu_q, "K": p.K,
            "thermalConductivity": p.thermalConductivity, "viscosityTerm": ViscosityTerms(_term_value(p.viscosityTerm)).name,
            "thermalConducitiyTerm": ViscosityTerms(_term_value(p.thermalConducitiyTerm)).name, "scaleBeta": p.scaleBeta,
            "monaghanSwitch": p.monaghanSwitch, "correctXi": p.correctXi}


def dictToDiffusionParams(d: Dict[str, Any]) -> DiffusionParameters:
    vt = d["viscosityTerm"]
    tt = d["thermalConducitiyTerm"]
    return DiffusionParameters(c_s=d["c_s"], C_l=d["C_l"], C_q=d["C_q"], Cu_l=d["Cu_l"], Cu_q=d["Cu_q"], K=d["K"],
                               thermalConductivity=d["thermalConductivity"],
                               viscosityTerm=ViscosityTerms[vt].value if isinstance(vt, str) else vt,
                               thermalConducitiyTerm=ViscosityTerms[tt].value if isinstance(tt, str) else tt,
                               scaleBeta=d["scaleBeta"], monaghanSwitch=d["monaghanSwitch"], correctXi=d["correctXi"])


@dataclass
class ViscositySwitchConfig:
    scheme: ViscositySwitch = ViscositySwitch.NoneSwitch
    correctVelocityGradient: bool = False
    divergenceScheme: Optional[str] = "naive"
    alpha_min: float = 0.02
    alpha_max: float = 2.0
    beta_c: float = 0.7
    beta_d: float = 0.05
    beta_xi: float = 2.0
    limitXi: bool = True   # the reference declares the field twice; the later default (True) is the effective one


def viscositySwitchConfigToDict(c: ViscositySwitchConfig) -> Dict[str, Any]:
    return {"scheme": c.scheme.name, "limitXi": c.limitXi, "correctVelocityGradient": c.correctVelocityGradient,
            "divergenceScheme": c.divergenceScheme, "alpha_min": c.alpha_min, "alpha_max": c.alpha_max,
            "beta_c": c.beta_c, "beta_d": c.beta_d, "beta_xi": c.beta_xi}


def dictToViscositySwitchConfig(d: Dict[str, Any]) -> ViscositySwitchConfig:
    s = d["scheme"]
    return ViscositySwitchConfig(scheme=ViscositySwitch[s] if isinstance(s, str) else s, limitXi=d["limitXi"],
                                 correctVelocityGradient=d["correctVelocityGradient"], divergenceScheme=d["divergenceScheme"],
                                 alpha_min=d["alpha_min"], alpha_max=d["alpha_max"], beta_c=d["beta_c"], beta_d=d["beta_d"],
                                 beta_xi=d["beta_xi"])


@dataclass
class CRKViscosity:
    eta_fold: float = 0.2
    eta_crit: float = 0.3333333
    enableCRKLimiter: bool = True
    enableVanLeerLimiter: bool = True
    forceVanLeerOff: bool = False
    forceVanLeerOn: bool = False


def buildDefaultCRKViscosityParams() -> CRKViscosity:
    return CRKViscosity()


# ------------------------------------------------------------------ scheme configs
@dataclass
class CompressibleSPHConfig:
    gamma: float = 1.4
    backgroundPressure: float = 0.0
    rho0: float = 1.0
    adaptiveSupportScheme: AdaptiveSupportScheme = AdaptiveSupportScheme.Monaghan
    adaptiveSupportIterations: int = 1
    adaptiveSupportThreshold: float = 1e-3
    adaptiveSupportCorrections: bool = True
    diffusionParams: DiffusionParameters = field(default_factory=buildDefaultDiffusionParamsCompressibleSPH)
    viscositySwitchParams: ViscositySwitchConfig = field(default_factory=ViscositySwitchConfig)
    schemeName: str = "Compressible SPH"
    boundaryConditions: List[Any] = field(default_factory=list)
    # B200 build option: Neumaier-compensated accumulation of dv/dt and du/dt
    compensatedSums: bool = False


def compressibleConfigToDict(c: CompressibleSPHConfig) -> Dict[str, Any]:
    if c.boundaryConditions:
        raise NotImplementedError("boundary conditions are outside the GPU hot path")
    return {"gamma": c.gamma, "backgroundPressure": c.backgroundPressure, "rho0": c.rho0,
            "adaptiveSupportScheme": c.adaptiveSupportScheme.name, "adaptiveSupportIterations": c.adaptiveSupportIterations,
            "adaptiveSupportThreshold": c.adaptiveSupportThreshold, "adaptiveSupportCorrections": c.adaptiveSupportCorrections,
            "diffusionParams": diffusionParamsToDict(c.diffusionParams),
            "viscositySwitchParams": viscositySwitchConfigToDict(c.viscositySwitchParams), "schemeName": c.schemeName,
            "boundaryConditions": [], "compensatedSums": c.compensatedSums}


def dictToCompressibleConfig(d: Dict[str, Any]) -> CompressibleSPHConfig:
    a = d["adaptiveSupportScheme"]
    return CompressibleSPHConfig(gamma=d["gamma"], backgroundPressure=d["backgroundPressure"], rho0=d["rho0"],
                                 adaptiveSupportScheme=AdaptiveSupportScheme[a] if isinstance(a, str) else a,
                                 adaptiveSupportIterations=d["adaptiveSupportIterations"],
                                 adaptiveSupportThreshold=d["adaptiveSupportThreshold"],
                                 adaptiveSupportCorrections=d["adaptiveSupportCorrections"],
                                 diffusionParams=dictToDiffusionParams(d["diffusionParams"]),
                                 viscositySwitchParams=dictToViscositySwitchConfig(d["viscositySwitchParams"]),
                                 schemeName=d["schemeName"], boundaryConditions=[],
                                 compensatedSums=bool(d.get("compensatedSums", False)))


@dataclass
class CompSPHConfig(CompressibleSPHConfig):
    energyScheme: EnergyScheme = EnergyScheme.CRK
    diffusionParams: DiffusionParameters = field(default_factory=buildDefaultDiffusionParamsCompSPH)
    schemeName: str = "CompSPH"
    compatibleEnergy: bool = True


def compSPHConfigToDict(c: CompSPHConfig) -> Dict[str, Any]:
    d = compressibleConfigToDict(c)
    d.update({"energyScheme": c.energyScheme.name, "compatibleEnergy": c.compatibleEnergy})
    return d


def dictToCompSPHConfig(d: Dict[str, Any]) -> CompSPHConfig:
    base = dictToCompressibleConfig(d)
    c = CompSPHConfig(**base.__dict__)
    e = d["energyScheme"]
    c.energyScheme = EnergyScheme[e] if isinstance(e, str) else e
    c.compatibleEnergy = d["compatibleEnergy"]
    return c


@dataclass
class CRKSPHConfig(CompressibleSPHConfig):
    energyScheme: EnergyScheme = EnergyScheme.CRK
    diffusionParams: DiffusionParameters = field(default_factory=buildDefaultDiffusionParamsCRKSPH)
    crkViscosityParams: CRKViscosity = field(default_factory=buildDefaultCRKViscosityParams)
    schemeName: str = "CRKSPH"
    compatibleEnergy: bool = True


def crkSPHConfigToDict(c: CRKSPHConfig) -> Dict[str, Any]:
    d = compressibleConfigToDict(c)
    v = c.crkViscosityParams
    d.update({"energyScheme": c.energyScheme.name, "compatibleEnergy": c.compatibleEnergy,
              "crkViscosityParams": {"eta_fold": v.eta_fold, "eta_crit": v.eta_crit, "enableCRKLimiter": v.enableCRKLimiter,
                                     "enableVanLeerLimiter": v.enableVanLeerLimiter, "forceVanLeerOff": v.forceVanLeerOff,
                                     "forceVanLeerOn": v.forceVanLeerOn}})
    return d


def dictToCRKSPHConfig(d: Dict[str, Any]) -> CRKSPHConfig:
    base = dictToCompressibleConfig(d)
    c = CRKSPHConfig(**base.__dict__)
    e = d["energyScheme"]
    c.energyScheme = EnergyScheme[e] if isinstance(e, str) else e
    c.compatibleEnergy = d["compatibleEnergy"]
    v = d["crkViscosityParams"]
    c.crkViscosityParams = CRKViscosity(eta_fold=v["eta_fold"], eta_crit=v["eta_crit"], enableCRKLimiter=v["enableCRKLimiter"],
                                        enableVanLeerLimiter=v["enableVanLeerLimiter"], forceVanLeerOff=v["forceVanLeerOff"],
                                        forceVanLeerOn=v["forceVanLeerOn"])
    return c


# ------------------------------------------------------------------ incompressible (DFSPH)
@dataclass
class RelaxedJacobiSolverConfig:
    """configurations/moduleConfigurations/solver.py:7-12 (same defaults)."""
    minIterations: int = 1
    maxIterations: int = 10
    tolerance: float = 1e-3
    relaxationFactor: float = 0.5


def buildDefaultPSConfig() -> RelaxedJacobiSolverConfig:
    """solver.py:15-21: the density (pressure) solver."""
    return RelaxedJacobiSolverConfig(minIterations=2, maxIterations=64, tolerance=5e-4, relaxationFactor=0.3)


def buildDefaultDFConfig() -> RelaxedJacobiSolverConfig:
    """solver.py:22-28: the divergence-free solver."""
    return RelaxedJacobiSolverConfig(minIterations=2, maxIterations=32, tolerance=2.5e-3, relaxationFactor=0.3)


@dataclass
class IncompressibleSolverConfig:
    """solver.py:31-35."""
    pressureSolver: RelaxedJacobiSolverConfig = field(default_factory=buildDefaultPSConfig)
    divergenceFreeSolver: RelaxedJacobiSolverConfig = field(default_factory=buildDefaultDFConfig)
    integrateRho: bool = False


def buildDefaultIncompressibleSolverConfig() -> IncompressibleSolverConfig:
    return IncompressibleSolverConfig(pressureSolver=buildDefaultPSConfig(), divergenceFreeSolver=buildDefaultDFConfig(),
                                      integrateRho=False)


@dataclass
class fluidProperties:
    """moduleConfigurations/fluidProperties.py:9-30 (the fields the solves read).  eosType
    None defers to the scheme configuration's own eosType."""
    restDensity: float = 1.0
    polytropicExponent: Optional[float] = 7.0
    kappa: Optional[float] = 1.3
    fixedSoundSpeed: Optional[float] = 10.0
    eosType: Optional[Any] = None


# ------------------------------------------------------------------ gravity, surface detection, shifting
class GravityType(Enum):
    """moduleConfigurations/gravity.py:7-10."""
    Directional = 0
    PointSource = 1
    PotentialField = 2


@dataclass
class gravityConfiguration:
    """moduleConfigurations/gravity.py:18-27 (same defaults: inactive, 9.81 along -y)."""
    active: bool = False
    type: GravityType = GravityType.Directional
    magnitude: float = 9.81
    direction: List[float] = field(default_factory=lambda: [0.0, -1.0])
    origin: List[float] = field(default_factory=lambda: [0.0, 0.0])


def buildDefaultGravityConfiguration() -> gravityConfiguration:
    return gravityConfiguration()


class SurfaceDetectionScheme(Enum):
    ColorField = 0
    ColorFieldGrad = 1
    Barecasco = 2
    Maronne = 3


class NormalSource(Enum):
    Native = 0
    ColorFieldGrad = 1
    LambdaGrad = 2
    Maronne = 3


@dataclass
class SurfaceDetectionConfig:
    """moduleConfigurations/surfaceDetection.py:22-35 (the dataclass defaults: active,
    colour-field scheme, colour-field-gradient normals).  The schemes take the inactive
    buildDefaultSurfaceDetectionConfig (:38-48)."""
    active: bool = True
    colorFieldThreshold: float = 0.75
    colorFieldGradThreshold: float = 10.0
    barecascoThreshold: float = 1.5
    expansionIterations: int = 1
    scheme: SurfaceDetectionScheme = SurfaceDetectionScheme.ColorField
    normalSource: NormalSource = NormalSource.ColorFieldGrad


def buildDefaultSurfaceDetectionConfig() -> SurfaceDetectionConfig:
    return SurfaceDetectionConfig(active=False, colorFieldThreshold=0.75, colorFieldGradThreshold=10.0,
                                  barecascoThreshold=math.pi / 3, expansionIterations=1,
                                  scheme=SurfaceDetectionScheme.Barecasco, normalSource=NormalSource.LambdaGrad)


@dataclass
class ShiftProperties:
    """moduleConfigurations/shifting.py:18-37 with the defaults of
    buildDefaultShiftProperties (:40-53): one delta-plus iteration, CFL 0.3, active."""
    iterations: int = 1
    CFL: float = 0.3
    computeMach: bool = True
    maxC: float = 0.3
    active: bool = True
    scheme: str = "deltaSPH"
    projectionScheme: str = "mat"
    summationDensity: bool = False
    surfaceScaling: float = 0.1
    threshold: float = 0.5
    projectQuantities: bool = False
    correctdrhodt: bool = False
    correctdvdt: bool = False
    reuseNormals: bool = True


def buildDefaultShiftProperties() -> ShiftProperties:
    return ShiftProperties()


def buildDefaultFluidProperties() -> fluidProperties:
    return fluidProperties(restDensity=1.0, polytropicExponent=7.0, kappa=1.3, fixedSoundSpeed=10.0)


@dataclass
class WeaklyCompressibleDiffusionParams:
    """configurations/moduleConfigurations/weaklyCompressibleDiffusionParams.py:10-26."""
    inviscid: bool = True
    inviscidAlpha: float = 0.01
    viscidNu: float = 1e-3
    densityDelta: float = 0.1
    densityDiffusionTerm: Any = "deltaSPH"


@dataclass
class IncompressibleSPHConfig:
    """configurations/incompressible.py:32-68: the fields dfsph_step and its finalize read.
    Boundary conditions, regions and rigid bodies are accepted as the reference declares
    them and rejected by the step when non-empty."""
    fluid: fluidProperties = field(default_factory=buildDefaultFluidProperties)
    adaptiveSupportScheme: Any = None
    adaptiveSupportIterations: int = 1
    adaptiveSupportThreshold: float = 1e-3
    adaptiveSupportCorrections: bool = True
    diffusionParams: WeaklyCompressibleDiffusionParams = field(default_factory=WeaklyCompressibleDiffusionParams)
    schemeName: str = "Compressible SPH"
    boundaryConditions: List[Any] = field(default_factory=list)
    dt_viscosityConstraint: bool = True
    dt_accelerationConstraint: bool = True
    dt_acousticConstraint: bool = True
    pressureForceTerm: Any = "Antuono"
    shiftProperties: ShiftProperties = field(default_factory=buildDefaultShiftProperties)
    regions: List[Any] = field(default_factory=list)
    rigidBodies: List[Any] = field(default_factory=list)
    surfaceDetectionConfig: SurfaceDetectionConfig = field(default_factory=buildDefaultSurfaceDetectionConfig)
    gravityConfig: gravityConfiguration = field(default_factory=buildDefaultGravityConfiguration)
    solverConfig: IncompressibleSolverConfig = field(default_factory=buildDefaultIncompressibleSolverConfig)


def jacobi_config(solver: RelaxedJacobiSolverConfig, restDensity: float, learned_init: bool = False) -> _capi.SphJacobiConfig:
    """Packs a RelaxedJacobiSolverConfig into the C ABI's SphJacobiConfig."""
    c = _capi.SphJacobiConfig()
    c.rest_density = float(restDensity)
    c.tolerance = float(solver.tolerance)
    c.relaxation = float(solver.relaxationFactor)
    c.min_iterations = int(solver.minIterations)
    c.max_iterations = int(solver.maxIterations)
    c.init_mode = 1 if learned_init else 0
    return c


# ------------------------------------------------------------------ weakly compressible (delta-SPH)
@dataclass
class WeaklyCompressibleSPHConfig:
    """configurations/weaklyCompressible.py:35-65: the fields deltaSPH_step and its
    finalize read.  eosType here is used when fluid.eosType is None."""
    fluid: fluidProperties = field(default_factory=lambda: fluidProperties(restDensity=1.0, polytropicExponent=7.0, kappa=1.3,
                                                                           fixedSoundSpeed=10.0))
    eosType: Any = "stiffTait"
    adaptiveSupportScheme: Any = None
    adaptiveSupportIterations: int = 1
    adaptiveSupportThreshold: float = 1e-3
    adaptiveSupportCorrections: bool = True
    diffusionParams: WeaklyCompressibleDiffusionParams = field(default_factory=WeaklyCompressibleDiffusionParams)
    schemeName: str = "Compressible SPH"
    boundaryConditions: List[Any] = field(default_factory=list)
    dt_viscosityConstraint: bool = True
    dt_accelerationConstraint: bool = True
    dt_acousticConstraint: bool = True
    pressureForceTerm: Any = "Antuono"
    shiftProperties: ShiftProperties = field(default_factory=buildDefaultShiftProperties)
    regions: List[Any] = field(default_factory=list)
    rigidBodies: List[Any] = field(default_factory=list)
    surfaceDetectionConfig: SurfaceDetectionConfig = field(default_factory=buildDefaultSurfaceDetectionConfig)
    gravityConfig: gravityConfiguration = field(default_factory=buildDefaultGravityConfiguration)


_EOS = {"stiffTait": 0, "Tait": 1, "isoThermal": 2, "polytropic": 3, "murnaghan": 4}
_DDIFF = {"deltaSPH": 0, "densityOnly": 2, "deltaOnly": 3}
_PTERM = {"conservative": 0, "nonConservative": 1, "Antuono": 2, "i": 3, "j": 4, "symmetric": 5}


def _name(v) -> str:
    """An enum member's name or the string itself (the reference passes enums)."""
    return v.name if isinstance(v, Enum) else str(v)


def wc_params(cfg) -> _capi.SphWcParams:
    """Packs a WeaklyCompressibleSPHConfig (or IncompressibleSPHConfig) into the C ABI's
    SphWcParams."""
    w = _capi.SphWcParams()
    f, d = cfg.fluid, cfg.diffusionParams
    w.rest_density, w.sound_speed = float(f.restDensity), float(f.fixedSoundSpeed if f.fixedSoundSpeed is not None else 1.0)
    w.polytropic_exponent, w.kappa = float(f.polytropicExponent), float(f.kappa)
    w.density_delta, w.viscosity_nu, w.inviscid_alpha = float(d.densityDelta), float(d.viscidNu), float(d.inviscidAlpha)
    w.inviscid = int(bool(d.inviscid))
    w.density_scheme = _DDIFF[_name(d.densityDiffusionTerm)]
    w.pressure_term = _PTERM[_name(cfg.pressureForceTerm)]
    eos = f.eosType if getattr(f, "eosType", None) is not None else getattr(cfg, "eosType", "isoThermal")
    w.eos = _EOS[_name(eos)]
    return w


# ------------------------------------------------------------------ C ABI parameter block
def make_params(config: SimulationConfig, scheme: Optional[CompressibleSPHConfig] = None) -> _capi.SphParams:
    """Packs the configuration into the C ABI's SphParams (host-side, no device sync
    beyond a cached read of the domain tensors)."""
    p = _capi.SphParams()
    dmin, dmax, per = config.domain.host()
    dim = int(config.dim)
    for a in range(3):
        p.domain_min[a] = dmin[a] if a < dim else 0.0
        p.domain_max[a] = dmax[a] if a < dim else 1.0
        p.periodic[a] = int(per[a]) if a < dim else 0
    p.dim = dim
    p.kernel = int(config.kernel.value)
    p.verlet_scale = float(config.verletScale)
    p.target_neighbors = float(config.targetNeighbors)
    p.cfl = float(config.cflFactor)
    p.min_dt = float(config.minDt if config.minDt is not None else 0.0)
    p.max_dt = float(config.maxDt if config.maxDt is not None else 1e30)
    p.dt_growth = float(config.dtGrowthFactor if config.dtGrowthFactor is not None else 1e30)
    # the weakly compressible and incompressible configurations carry their parameters in
    # SphWcParams / SphJacobiConfig (wc_params, jacobi_config)
    if isinstance(scheme, CompressibleSPHConfig):
        dp = scheme.diffusionParams
        p.C_l, p.C_q, p.Cu_l, p.Cu_q, p.K = float(dp.C_l), float(dp.C_q), float(dp.Cu_l), float(dp.Cu_q), float(dp.K)
        p.viscosity_term = _term_value(dp.viscosityTerm)
        p.conductivity_term = _term_value(dp.thermalConducitiyTerm)
        p.c_s = float(dp.c_s)
        p.monaghan_switch = int(bool(dp.monaghanSwitch))
        p.correct_xi = int(bool(dp.correctXi))
        p.scale_beta = int(bool(dp.scaleBeta))
        p.gamma = float(scheme.gamma)
        sw = scheme.viscositySwitchParams
        p.alpha_min, p.alpha_max, p.beta_xi = float(sw.alpha_min), float(sw.alpha_max), float(sw.beta_xi)
        p.beta_c, p.beta_d = float(sw.beta_c), float(sw.beta_d)
        p.limit_xi = int(bool(sw.limitXi))
        p.correct_velocity_gradient = int(bool(sw.correctVelocityGradient))
        p.kahan = int(bool(getattr(scheme, "compensatedSums", False)))
        es = getattr(scheme, "energyScheme", EnergyScheme.CRK)
        p.energy_scheme = int(es.value)
        cv = getattr(scheme, "crkViscosityParams", None)
        if cv is not None:
            p.eta_crit, p.eta_fold = float(cv.eta_crit), float(cv.eta_fold)
            p.enable_crk_limiter = int(bool(cv.enableCRKLimiter))
            p.enable_vanleer_limiter = int(bool(cv.enableVanLeerLimiter))
            p.force_vanleer_off = int(bool(cv.forceVanLeerOff))
            p.force_vanleer_on = int(bool(cv.forceVanLeerOn))
    return p


# ------------------------------------------------------------------ dict round trips of the WC / DFSPH configs
def _to_dict(obj) -> Any:
    import dataclasses
    if dataclasses.is_dataclass(obj):
        return {f.name: _to_dict(getattr(obj, f.name)) for f in dataclasses.fields(obj)}
    if isinstance(obj, Enum):
        return obj.name
    if isinstance(obj, torch.Tensor):
        return obj.detach().cpu().tolist()
    if isinstance(obj, (list, tuple)):
        return [_to_dict(v) for v in obj]
    return obj


def _from_dict(cls, d: Dict[str, Any]):
    import dataclasses
    import typing
    hints = typing.get_type_hints(cls)
    kw = {}
    defaults = cls()
    for f in dataclasses.fields(cls):
        if f.name not in d:
            continue
        v, cur = d[f.name], getattr(defaults, f.name)
        if dataclasses.is_dataclass(cur) and isinstance(v, dict):
            v = _from_dict(type(cur), v)
        elif isinstance(cur, Enum) and isinstance(v, str):
            v = type(cur)[v]
        kw[f.name] = v
    return cls(**kw)


def weaklyCompressibleConfigToDict(config: WeaklyCompressibleSPHConfig) -> Dict[str, Any]:
    """configurations/weaklyCompressible.py (weaklyCompressibleConfigToDict): enums by name."""
    return _to_dict(config)


def dictToWeaklyCompressibleConfig(d: Dict[str, Any]) -> WeaklyCompressibleSPHConfig:
    return _from_dict(WeaklyCompressibleSPHConfig, d)


def incompressibleConfigToDict(config: IncompressibleSPHConfig) -> Dict[str, Any]:
    """configurations/incompressible.py:71-130 (incompressibleConfigToDict): enums by name."""
    return _to_dict(config)


def dictToIncompressibleSPHConfig(d: Dict[str, Any]) -> IncompressibleSPHConfig:
    return _from_dict(IncompressibleSPHConfig, d)

