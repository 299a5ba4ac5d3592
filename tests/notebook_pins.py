"""Numbers the reference's notebooks print, used to pin the kernel constants, the
density summation, the adaptive support and the time-step rules to the reference's own
(absent) warpSPHCore.

Each entry names the notebook, the printed line and the set-up that produced it (the
notebook cells' parameters).  The values are copied from the notebooks' stored outputs;
nothing here runs the reference.

- examples/incompressible/01-taylor-green-vortex.ipynb (Wendland4, 2D, nx = 128 on
  [0, 2 pi]^2, n_h = 4): "Initial density stats: mean: 1.00042, min: 1.00041, max:
  1.00042", after the mass correction "mean: 1, min: 0.999993, max: 1", "Computed c0:
  27.129610061645508", "Initial kinetic energy from simulation: 9.8655".
- examples/incompressible/periodic-random-flow.ipynb (Wendland2, same lattice): "mean:
  1.00121, min: 1.0012, max: 1.00121", after correction "min: 0.999994", "Computed c0:
  31.045583724975586", "Initial kinetic energy from simulation: 9.85772".
- examples/incompressible/1d-test.ipynb (Wendland4, 1D, nx = 192 on [-1, 1], a fluid block
  |x| < 0.5): "Computed c0: 4.593486785888672", "Computed dt: 0.0014052445767447352",
  "Initial density stats: mean: 0.992127, min: 0.687559, max: 1.00012".
- examples/compressible/05-Woodward_Colella.ipynb (B7, 1D, nx = 2000 on [-1, 1], gamma
  1.4, p = 1000 for |x| < 0.1): "Running with dt: 8.29648161015939e-06".
- examples/compressible/09-Gresho_Chan_Vortex.ipynb (B7, 2D, nx = 200 on [-0.5, 0.5]^2,
  gamma 5/3, p = 3 + 4 ln 2 outside r = 0.4): "Running with dt: 0.0004918661434203386".
- examples/compressible/12-Kelvin-Helmholtz.ipynb (B7, 2D, nx = 256 on [0, 1]^2, p = 2.5,
  rho = 1 or 2, dt scaled by 2/3): "Running with dt: 0.0003892789827659726".
- examples/compressible/01-Sod_Shock_Tube_1D.ipynb (B7, 1D, nx = 800, samplingRatio 4,
  Owen adaptive support, gamma 5/3, left (p, rho) = (1, 1), right (0.1795, 0.25)):
  "Initial internal energy: 0.7121 to  2.138", "Running with dt: 0.00030056745163165033".
"""
from __future__ import annotations

import math

import numpy as np

TGV = {
    "Wendland4": dict(rho=("1.00042", "1.00041", "1.00042"), rho_corrected_min="0.999993", c0=27.129610061645508, ke="9.8655"),
    "Wendland2": dict(rho=("1.00121", "1.0012", "1.00121"), rho_corrected_min="0.999994", c0=31.045583724975586, ke="9.85772"),
}
TGV_NX, TGV_L, TGV_TARGET_DT = 128, 2 * math.pi, 1e-3

BLOCK_1D = dict(nx=192, L=2.0, c0=4.593486785888672, dt=0.0014052445767447352, target_dt=5e-4,
                rho=(0.992127, 0.687559, 1.00012))

WOODWARD_COLELLA = dict(nx=2000, L=2.0, gamma=1.4, p_max=1000.0, dt=8.29648161015939e-06)
GRESHO = dict(nx=200, L=1.0, gamma=5 / 3, p_max=3 + 4 * math.log(2), dt=0.0004918661434203386)
KELVIN_HELMHOLTZ = dict(nx=256, L=1.0, gamma=5 / 3, p=2.5, rho_min=1.0, dt=0.0003892789827659726)

SOD = dict(nx=800, ratio=4, gamma=5 / 3, left=(1.0, 1.0), right=(0.1795, 0.25), u_range=("0.7121", "2.138"),
           dt=0.00030056745163165033)


def fmt6(x) -> str:
    """The notebooks' {:.6g} formatting of a statistic."""
    return f"{float(x):.6g}"


def lattice_1d(nx: int, L: float):
    """Cell-centred 1D lattice on [-L/2, L/2] in FP32 (sample/regular.py with jitter 0)."""
    dx = np.float32(L / nx)
    return (np.float32(-L / 2) + dx / np.float32(2) + np.arange(nx, dtype=np.float32) * dx).astype(np.float32), dx


def tgv_velocities(x: np.ndarray) -> np.ndarray:
    """The notebook's Taylor-Green field, k = 2 (wave number 1, phase pi/2)."""
    v = np.zeros_like(x)
    v[:, 0] = np.cos(x[:, 0] + np.pi / 2) * np.sin(x[:, 1] + np.pi / 2)
    v[:, 1] = -np.sin(x[:, 0] + np.pi / 2) * np.cos(x[:, 1] + np.pi / 2)
    return v
