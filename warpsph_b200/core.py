"""Core types that the reference imports from its absent sibling package warpSPHCore.

Names and meanings follow their call sites in the reference (wi-re/warpSPH):
KernelFunctions (configurations/simulationConfig.py:25), SupportScheme
(simulationConfig.py:39), GradientScheme / LaplacianScheme (simulationConfig.py:42-43),
IntegrationSchemeType (simulationConfig.py:27), WarpOperation (modules/density/density.py:16-28),
DomainDescription / buildDomainDescription (utils/domain.py:7-22), the support helpers
(utils/support.py:6-44) and AdjacencyList (field names from io.py:8-20).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from enum import Enum
from typing import Optional

import numpy as np
import torch


class KernelFunctions(Enum):
    Wendland2 = 1
    Wendland4 = 2
    Wendland6 = 3
    B7 = 4          # degree-7 B-spline, the compressible notebooks' kernel


class SupportScheme(Enum):
    Gather = 0
    Scatter = 1
    Symmetric = 2
    SuperSymmetric = 3
    KernelMeanSymmetric = 4


class GradientScheme(Enum):
    Naive = 0
    Difference = 1
    Symmetric = 2
    Summation = 3


class LaplacianScheme(Enum):
    Brookshaw = 0


class IntegrationSchemeType(Enum):
    explicitEuler = 0
    semiImplicitEuler = 1
    rungeKutta2 = 2
    rungeKutta4 = 3


class WarpOperation(Enum):
    Density = 0
    Interpolate = 1
    Gradient = 2
    Divergence = 3
    Curl = 4
    Laplacian = 5


class SamplingScheme(Enum):
    regular = 0


def kernel_constants(kernel: KernelFunctions, dim: int) -> tuple[float, float]:
    """(normalisation C_d, kernel scale H/h).

    Wendland kernels: Wendland (1995) normalisations and Dehnen & Aly (2012) Table 1 scales;
    the 2D values reproduce the reference notebooks' printed lattice densities and c0
    (examples/incompressible/01-taylor-green-vortex.ipynb, periodic-random-flow.ipynb).
    B7 (degree-7 B-spline): C_d integrates it to one; the scale is the factor the
    reference's CFL step divides by, read from the printed initial time steps of
    examples/compressible/05-Woodward_Colella.ipynb (1D) and 09-Gresho_Chan_Vortex.ipynb
    (2D), and continued to 3D by the quintic spline's moment ratio sqrt(15/14)."""
    pi = np.pi
    norms = {1: {1: 1.25, 2: 7 / pi, 3: 21 / (2 * pi)},
             2: {1: 1.5, 2: 9 / pi, 3: 495 / (32 * pi)},
             3: {1: 1.71875, 2: 78 / (7 * pi), 3: 1365 / (64 * pi)},
             4: {1: 4096 / 315, 2: 589824 / (7435 * pi), 3: 16384 / (105 * pi)}}
    scales = {1: {1: 1.620185175, 2: 1.897366596, 3: 1.936491673},
              2: {1: 1.936491673, 2: 2.171240593, 3: 2.207940217},
              3: {1: 2.207940217, 2: 2.415229458, 3: 2.449489743},
              4: {1: 3.865656972, 2: 3.932734728, 3: 4.001335111}}
    k = kernel.value
    return norms[k][dim], scales[k][dim]


def sphKernelScale(kernel: KernelFunctions, dim: int) -> float:
    return kernel_constants(kernel, dim)[1]


def sphKernel_xi(kernel: KernelFunctions, dim: int) -> float:
    """The kernel 'xi' of the CFL condition, the viscosity correction and the switches.
    Taken equal to the kernel scale H/h (support radius over smoothing length)."""
    return kernel_constants(kernel, dim)[1]


# ------------------------------------------------------------------ support helpers (utils/support.py)
def n_h_to_nH(n_h, dim):
    spacing = 1 / n_h
    v = spacing ** dim
    vH = 2.0 if dim == 1 else (np.pi if dim == 2 else (4 / 3) * np.pi)
    return vH / v


def nH_to_n_h(nH, dim):
    vH = 2.0 if dim == 1 else (np.pi if dim == 2 else (4 / 3) * np.pi)
    v = vH / nH
    return (1 / v) ** (1 / dim)


def volumeToSupportHelper(volume, targetNeighbors, dim):
    if dim == 1:
        return targetNeighbors * volume / 2
    if dim == 2:
        return torch.sqrt(targetNeighbors * volume / np.pi) if isinstance(volume, torch.Tensor) else np.sqrt(targetNeighbors * volume / np.pi)
    if isinstance(volume, torch.Tensor):
        return torch.pow(targetNeighbors * volume / np.pi * 3 / 4, 1 / 3)
    return np.power(targetNeighbors * volume / np.pi * 3 / 4, 1 / 3)


# ------------------------------------------------------------------ domain (utils/domain.py:7-22)
@dataclass
class DomainDescription:
    min: torch.Tensor
    max: torch.Tensor
    periodic: torch.Tensor
    dim: int
    _host: Optional[tuple] = field(default=None, repr=False, compare=False)

    def host(self) -> tuple:
        """(min list, max list, periodic list) as Python values, cached per tensor version."""
        key = (id(self.min), self.min._version, id(self.max), self.max._version, id(self.periodic), self.periodic._version)
        if self._host is None or self._host[0] != key:
            self._host = (key, [float(v) for v in self.min.tolist()], [float(v) for v in self.max.tolist()],
                          [bool(v) for v in self.periodic.tolist()])
        return self._host[1], self._host[2], self._host[3]


def buildDomainDescription(l, dim, periodic=False, device="cpu", dtype=torch.float32):
    minDomain = [-l / 2] * dim
    maxDomain = [l / 2] * dim
    per = torch.tensor([periodic] * dim, dtype=torch.bool, device=device) if isinstance(periodic, bool) else periodic
    return DomainDescription(torch.tensor(minDomain, device=device, dtype=dtype),
                             torch.tensor(maxDomain, device=device, dtype=dtype), per, dim)


# ------------------------------------------------------------------ adjacency (io.py:8-20 field names)
@dataclass
class AdjacencyList:
    """CSR Verlet list built on the GPU.

    neighborOffsets / numNeighbors are int32 [N]; neighborList is int32 [nnz] (the
    reference stores int64; ``i``/``j`` give the expanded int64 row/column arrays the
    reference's torch code indexes with).  Each row lists its interacting neighbours
    first (``interCounts``); pairwise arrays are indexed by position in neighborList."""
    neighborOffsets: torch.Tensor
    numNeighbors: torch.Tensor
    neighborList: torch.Tensor
    numRows: int
    numCols: int
    nnz: int
    sortIndex: Optional[torch.Tensor] = None
    sortedKeys: Optional[torch.Tensor] = None
    grid: Optional[torch.Tensor] = None
    queryPositions: Optional[torch.Tensor] = None
    querySupports: Optional[torch.Tensor] = None
    verletScale: float = 1.0
    # interacting prefix: row i holds its entries with r < max(H_i, H_j) first, so the
    # pair passes walk neighborList[off_i : off_i + interCounts[i]]
    interCounts: Optional[torch.Tensor] = None
    interNnz: int = 0
    _x_version: Optional[tuple] = field(default=None, repr=False)
    _h_version: Optional[tuple] = field(default=None, repr=False)
    _ij: Optional[tuple] = field(default=None, repr=False)
    # positions / supports the Verlet rows were built from (for the validity check)
    _x0: Optional[torch.Tensor] = field(default=None, repr=False)
    _h0: Optional[torch.Tensor] = field(default=None, repr=False)
    _dim: int = field(default=0, repr=False)
    # SphParams of a kept prior list whose interacting subset is filtered on first use
    _pending: Optional[object] = field(default=None, repr=False)
    _inter_nnz_dev: Optional[torch.Tensor] = field(default=None, repr=False)
    # rows kept in fixed buffers and updated on the GPU (ops.DeviceLists): nnz is the capacity
    _device_rows: bool = field(default=False, repr=False)

    @property
    def edgeOffsets(self) -> torch.Tensor:
        return self.neighborOffsets

    def _expand(self):
        if self._ij is None:
            from . import ops
            self._ij = ops.expand_adjacency(self)
        return self._ij

    @property
    def i(self) -> torch.Tensor:
        return self._expand()[0]

    @property
    def j(self) -> torch.Tensor:
        return self._expand()[1]

    @property
    def referencePositions(self) -> Optional[torch.Tensor]:
        return self.queryPositions

    @property
    def referenceSupports(self) -> Optional[torch.Tensor]:
        return self.querySupports


@dataclass
class CRKState:
    """CRK correction coefficients: A [N], B [N,d], gradA [N,d], gradB [N,d,d] with
    gradB[i][a][g] = dB^a/dx^g."""
    A: torch.Tensor
    B: torch.Tensor
    gradA: torch.Tensor
    gradB: torch.Tensor


@dataclass
class OperationProperties:
    kernel: KernelFunctions = KernelFunctions.Wendland2
    operation: WarpOperation = WarpOperation.Density
    supportMode: SupportScheme = SupportScheme.Gather
    gradientMode: GradientScheme = GradientScheme.Difference
