"""warpsph_b200: the warpSPH per-step particle hot path on NVIDIA B200 (sm_100a).

A drop-in for the reference's buildScheme(...) / SimulationState / SimulationConfig /
step-function API (wi-re/warpSPH).  All SPH work runs in hand-written CUDA kernels
in libwarpsph_b200.so, called through a ctypes C ABI on torch CUDA tensors; there is
no CPU fallback.
"""
from .core import (AdjacencyList, CRKState, DomainDescription, GradientScheme, IntegrationSchemeType, KernelFunctions,
                   LaplacianScheme, OperationProperties, SamplingScheme, SupportScheme, WarpOperation, buildDomainDescription,
                   n_h_to_nH, nH_to_n_h, sphKernel_xi, sphKernelScale, volumeToSupportHelper)
from .enumTypes import (AdaptiveSupportScheme, CompressibleSPHScheme, DensityDiffusionScheme, EnergyScheme, EquationOfState,
                        IncompressibleSPHScheme, PressureForceScheme, ViscositySwitch, WeaklyCompressibleSPHScheme)
from .configurations import (CompressibleSPHConfig, CompSPHConfig, CRKSPHConfig, CRKViscosity, DiffusionParameters,
                             SimulationConfig, ViscositySwitchConfig, ViscosityTerms, buildConfig, compSPHConfigToDict,
                             configurationToDict, crkSPHConfigToDict, dictToCompSPHConfig, dictToConfig, dictToCRKSPHConfig,
                             make_params)
from .systems import CompressibleState, CompressibleSystem, CompressibleSystemUpdate, CompSPHState, CompSPHSystem
from .integrators import IntegrationResult, getIntegrator
from .schemes import buildScheme, computeCRKFactors, computeTimestep, crkSPH_step, evaluateOptimalSupport, idealGasEOS
from .cases import buildPointCloud, buildSedov, buildSod1D, sodInitialState
from .io import exportSimulationSystem, importConfigs, importSimulationSystem, prepExport

__version__ = "0.1.0"
