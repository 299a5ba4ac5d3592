"""The CPU oracle and the host-side constants against numbers the reference's notebooks
print (tests/notebook_pins.py lists them): the Wendland lattice densities and kinetic
energies through the oracle's neighbour search and gather density, and the kernel scales
behind the printed sound speeds and time steps (the same FP32 arithmetic the reference's
torch code does on its FP32 tensors).  test_gpu_notebook_pins.py runs the same checks
through the GPU path."""
import numpy as np
import pytest
import torch

from oracle import oracle
from oracle.steps import cell_capacity_for
from tests import notebook_pins as NB
from tests.cases import make_params
from warpsph_b200 import core
from warpsph_b200.core import KernelFunctions, n_h_to_nH, sphKernelScale, volumeToSupportHelper

F = np.float32


def lattice_2d(nx, L):
    dx = F(L / nx)
    g = (dx / F(2) + np.arange(nx, dtype=F) * dx).astype(F)
    X, Y = np.meshgrid(g, g, indexing="xy")
    return np.stack([X.ravel(), Y.ravel()], 1).astype(F), dx


@pytest.mark.parametrize("kernel", ["Wendland4", "Wendland2"])
def test_oracle_taylor_green_lattice(kernel):
    want = NB.TGV[kernel]
    kf = getattr(KernelFunctions, kernel)
    # the notebook's domain is [0, 2 pi]^2; the periodic lattice is shifted onto the
    # centred domain of make_params (the sums are translation invariant)
    _, _, p = make_params(2, kernel=kf, periodic=True, L=NB.TGV_L)
    x0, dx = lattice_2d(NB.TGV_NX, NB.TGV_L)
    x = (x0 - F(NB.TGV_L / 2)).astype(F)
    n = len(x)
    H = np.full(n, volumeToSupportHelper(float(dx) ** 2, n_h_to_nH(4, 2), 2), F)
    m = np.full(n, float(dx) ** 2, F)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 2))
    rho = o.density(p, 0, x, H, m, nb)
    assert (NB.fmt6(rho.mean()), NB.fmt6(rho.min()), NB.fmt6(rho.max())) == want["rho"]
    m = (m / rho.astype(np.float64).mean()).astype(F)
    v = NB.tgv_velocities(x0)
    assert NB.fmt6((0.5 * m * (v * v).sum(-1)).sum()) == want["ke"]


def test_kernel_scales_behind_printed_sound_speeds_and_steps():
    """c0 = 0.3 H_2D(dx) / k / targetDt (timestep/weaklyCompressible.py:94) and the
    CFL step 0.3 H / (c k) (timestep/compressible.py:49-55) in FP32 arithmetic."""
    for kernel, want in NB.TGV.items():
        dx = F(NB.TGV_L / NB.TGV_NX)
        H = torch.sqrt(torch.tensor(n_h_to_nH(4, 2)) * torch.tensor(dx) ** 2 / np.pi).to(torch.float32)
        c0 = float(0.3 * H / sphKernelScale(getattr(KernelFunctions, kernel), 2) / NB.TGV_TARGET_DT)
        assert abs(c0 / want["c0"] - 1) < 1e-6
    b = NB.BLOCK_1D
    dx = F(b["L"] / b["nx"])
    c0 = float(0.3 * np.sqrt(n_h_to_nH(4, 1) * float(dx) ** 2 / np.pi) / sphKernelScale(KernelFunctions.Wendland4, 2) / b["target_dt"])
    assert abs(c0 / b["c0"] - 1) < 1e-6
    dt = float(F(0.3) * F(4 * dx) / F(c0) / F(sphKernelScale(KernelFunctions.Wendland4, 1)))
    assert abs(dt / b["dt"] - 1) < 1e-6

    def cfl(nx, L, dim, gamma, p, rho=1.0):
        dx = torch.tensor(L / nx, dtype=torch.float32)
        H = (n_h_to_nH(4, 1) * dx / 2) if dim == 1 else torch.sqrt(n_h_to_nH(4, 2) * dx * dx / np.pi)
        u = torch.tensor([p], dtype=torch.float32) / torch.tensor([rho], dtype=torch.float32) / (gamma - 1)
        c = torch.sqrt(u.abs() * gamma * (gamma - 1))
        return float((0.3 * H / (c * sphKernelScale(KernelFunctions.B7, dim))).min())
    wc, gr, kh = NB.WOODWARD_COLELLA, NB.GRESHO, NB.KELVIN_HELMHOLTZ
    assert abs(cfl(wc["nx"], wc["L"], 1, wc["gamma"], wc["p_max"]) / wc["dt"] - 1) < 1e-6
    assert abs(cfl(gr["nx"], gr["L"], 2, gr["gamma"], gr["p_max"]) / gr["dt"] - 1) < 1e-6
    assert abs(cfl(kh["nx"], kh["L"], 2, kh["gamma"], kh["p"], kh["rho_min"]) * 2 / 3 / kh["dt"] - 1) < 1e-6
