"""Free-surface detection (modules/surfaceDetection/wrapper.py:84-149) on the GPU passes.

Schemes: ColorField (colorFieldDetection.py), ColorFieldGrad
(colorFieldGradientDetection.py), Barecasco (barecascoDetection.py, wp_barecasco.py) and
Maronne (maronneDetection.py, wp_maronne.py); normal sources: the colour-field gradient,
the renormalised lambda gradient (lambdaGrad.py), Maronne's normals (maronneNormals.py) and
the scheme's own (Native); then the dilation iterations.

The renormalisation matrices and their eigenvalues come from warpSPHCore's
computeRenormalizationMatrices in the reference (absent here); sph_surface_renormalization
restates them (L = pinv(M), M = sum_j V_j (x_j - x_i) (x) grad_i W under super-symmetric
support; lambda = the smallest |eigenvalue| of M).  The returned renormalisation state is
that L tensor [n, d, d]."""
from __future__ import annotations

from typing import Any

import torch

from . import ops
from .configurations import NormalSource, SurfaceDetectionScheme, make_params


def _normals(S, params, config, surfaceConfig, adjacency, renormalizationState):
    """computeNormals (wrapper.py:18-64): (normals or None, renormalisation state, lambdas)."""
    src = surfaceConfig.normalSource
    L, lambdas = renormalizationState, None
    if src in (NormalSource.LambdaGrad, NormalSource.Maronne):
        L, lambdas = ops.surface_renormalization(params, S.positions, S.supports, S.masses, S.densities, adjacency)
    if src == NormalSource.ColorFieldGrad:
        c = ops.surface_color_field(params, S.positions, S.supports, S.masses, S.densities, adjacency)
        _, normals, _ = ops.surface_detect_color_field(params, S.positions, S.supports, S.masses, S.densities, c, adjacency,
                                                       0.0, -1.0)
        return normals, L, lambdas
    if src == NormalSource.LambdaGrad:
        return ops.surface_renormalized_normals(params, 0, S.positions, S.supports, S.masses, S.densities, L, lambdas, adjacency), \
            L, lambdas
    if src == NormalSource.Maronne:
        return ops.surface_renormalized_normals(params, 1, S.positions, S.supports, S.masses, S.densities, L, None, adjacency), \
            L, lambdas
    if src == NormalSource.Native:
        return None, L, lambdas
    raise ValueError(f"Unknown normal source: {src}")


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
    scheme = surfaceConfig.scheme
    if scheme not in (SurfaceDetectionScheme.ColorField, SurfaceDetectionScheme.ColorFieldGrad, SurfaceDetectionScheme.Barecasco,
                      SurfaceDetectionScheme.Maronne):
        raise ValueError(f"Unknown surface detection scheme: {scheme}")
    if surfaceConfig.normalSource not in (NormalSource.ColorFieldGrad, NormalSource.LambdaGrad, NormalSource.Maronne,
                                          NormalSource.Native):
        raise ValueError(f"Unknown normal source: {surfaceConfig.normalSource}")
    params = make_params(config)
    S = currentState
    colour_scheme = scheme in (SurfaceDetectionScheme.ColorField, SurfaceDetectionScheme.ColorFieldGrad)
    # with a colour-field scheme the colour-field-gradient normals are the scheme's own
    # gradient pass, taken from it below instead of a second pass
    from_scheme = colour_scheme and surfaceConfig.normalSource == NormalSource.ColorFieldGrad
    if from_scheme:
        normals, L, lambdas = None, renormalizationState, None
    else:
        normals, L, lambdas = _normals(S, params, config, surfaceConfig, adjacency, renormalizationState)
    if colour_scheme:
        c = ops.surface_color_field(params, S.positions, S.supports, S.masses, S.densities, adjacency)
        if scheme == SurfaceDetectionScheme.ColorField:
            fsm, normals2, _ = ops.surface_detect_color_field(params, S.positions, S.supports, S.masses, S.densities, c, adjacency,
                                                              float(config.targetNeighbors) * float(surfaceConfig.colorFieldThreshold),
                                                              1.0)
        else:
            fsm, normals2 = ops.surface_detect_color_gradient(params, S.positions, S.supports, S.masses, S.densities, c, adjacency,
                                                              float(surfaceConfig.colorFieldGradThreshold))
    elif scheme == SurfaceDetectionScheme.Barecasco:
        fsm, normals2, _ = ops.surface_barecasco(params, S.positions, S.supports, adjacency, float(surfaceConfig.barecascoThreshold))
    else:
        if normals is None:
            if L is None:
                L, _ = ops.surface_renormalization(params, S.positions, S.supports, S.masses, S.densities, adjacency)
            normals = ops.surface_renormalized_normals(params, 1, S.positions, S.supports, S.masses, S.densities, L, None, adjacency)
        fsm, _ = ops.surface_maronne(params, S.positions, S.supports, normals, adjacency)
        normals2 = normals
    if from_scheme:     # -normalize(grad c): the ColorField pass returns +normalize(grad c)
        normals = -normals2 if scheme == SurfaceDetectionScheme.ColorField else normals2
    if surfaceConfig.normalSource == NormalSource.Native:
        normals = normals2
    fs = fsm
    for _ in range(int(surfaceConfig.expansionIterations)):
        fs = ops.surface_dilate(params, S.positions, S.supports, fs, adjacency)
    return (fsm, fs, normals, L, lambdas) if returnNormals else (fsm, fs, L, lambdas)
