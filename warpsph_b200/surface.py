"""Free-surface detection (modules/surfaceDetection/wrapper.py:84-149) on the GPU passes.

Built: the colour-field scheme (SurfaceDetectionScheme.ColorField), normals from the
colour-field gradient (NormalSource.ColorFieldGrad) or the scheme's own (Native), and the
dilation iterations.  The Barecasco, Maronne and colour-field-gradient schemes and the
renormalisation-matrix normal sources (LambdaGrad, Maronne) raise NotImplementedError."""
from __future__ import annotations

from typing import Any

import torch

from . import ops
from .configurations import NormalSource, SurfaceDetectionScheme, make_params


def detectFreeSurface(currentState: Any, config: Any, schemeConfig: Any, surfaceConfig: Any, adjacency,
                      renormalizationState=None, returnNormals: bool = True):
    """Returns (fsm, fs, normals, renormalizationState, lambdas) with returnNormals, else
    (fsm, fs, renormalizationState, lambdas), in the reference's order: fsm is the 0/1 mask
    of the scheme and fs its dilation (a sum over super-symmetric neighbours, as in
    wp_dilate.py)."""
    x = currentState.positions
    if not surfaceConfig.active:
        fsm = torch.zeros(x.shape[0], device=x.device, dtype=x.dtype)
        return (fsm, fsm, torch.zeros_like(x), None, None) if returnNormals else (fsm, fsm, None, None)
    if surfaceConfig.scheme != SurfaceDetectionScheme.ColorField:
        raise NotImplementedError(f"surface detection scheme {surfaceConfig.scheme} is not on the GPU path")
    if surfaceConfig.normalSource not in (NormalSource.ColorFieldGrad, NormalSource.Native):
        raise NotImplementedError(f"normal source {surfaceConfig.normalSource} is not on the GPU path")
    params = make_params(config)
    S = currentState
    c = ops.surface_color_field(params, S.positions, S.supports, S.masses, S.densities, adjacency)
    sign = -1.0 if surfaceConfig.normalSource == NormalSource.ColorFieldGrad else 1.0
    fsm, normals, _ = ops.surface_detect_color_field(params, S.positions, S.supports, S.masses, S.densities, c, adjacency,
                                                     float(config.targetNeighbors) * float(surfaceConfig.colorFieldThreshold), sign)
    fs = fsm
    for _ in range(int(surfaceConfig.expansionIterations)):
        fs = ops.surface_dilate(params, S.positions, S.supports, fs, adjacency)
    return (fsm, fs, normals, renormalizationState, None) if returnNormals else (fsm, fs, renormalizationState, None)
