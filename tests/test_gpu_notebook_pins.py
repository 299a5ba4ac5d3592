"""The GPU path against numbers the reference's notebooks print (tests/notebook_pins.py
lists them with their notebooks).  These pin the parts of the path whose reference code
lives in the absent warpSPHCore package:

- the Wendland4 and Wendland2 normalisations and profiles, the gather density summation
  and the neighbour search, through the printed lattice densities (six significant
  digits, as printed) and the kinetic energy after the mass correction;
- the kernel scales of Wendland4 (1D and 2D) and Wendland2 (2D), through the printed
  sound speeds c0 and the weakly compressible time step;
- the B7 kernel's CFL factor, through the initial time steps of three compressible
  notebooks (Woodward-Colella 1D, Gresho-Chan and Kelvin-Helmholtz 2D; the 1D and 2D
  factors were read from the first two, Kelvin-Helmholtz checks the 2D one independently);
- the B7 profile, the Owen adaptive support, the gather density and the CFL reduction,
  through the Sod notebook's printed internal-energy range and initial time step.

Tolerances: the printed digits for the statistics, except the minimum density after the
mass correction on the exact lattice, which is the FP32 rounding spread of identical
sums (4e-6 absolute), and the kinetic energy, an FP32 sum whose sixth digit depends on
the summation order (2e-6 relative); 1e-6 relative for time steps that the
reference computes from FP32 inputs alone; 2e-5 for the Sod step, whose smallest support
comes out of 16 FP32 support iterations (the reference's and this path's differ in their
last bits); 5e-6 for the 1D block densities, whose edge values the notebook's particle
sampler places a few ulps differently (the edge minimum differs by 3.7e-6)."""

import pytest
import torch

import warpsph_b200 as ws
from tests import notebook_pins as NB
from warpsph_b200 import ops, wcsph
from warpsph_b200.configurations import IncompressibleSPHConfig
from warpsph_b200.core import DomainDescription, KernelFunctions, SupportScheme, n_h_to_nH
from warpsph_b200.enumTypes import AdaptiveSupportScheme
from warpsph_b200.systems import CompressibleState, CompressibleSystem

pytestmark = pytest.mark.gpu


def domain(lo, hi, dim, cuda):
    return DomainDescription(torch.full((dim,), float(lo), device=cuda), torch.full((dim,), float(hi), device=cuda),
                             torch.ones(dim, dtype=torch.bool, device=cuda), dim)


def lattice(cuda, nx, lo, hi, dim, kernel):
    dom = domain(lo, hi, dim, cuda)
    cfg, _ = ws.buildConfig(device=cuda, domain=dom, dim=dim, kernel=kernel, targetNeighbors=n_h_to_nH(4, dim),
                            supportMode=SupportScheme.KernelMeanSymmetric, adaptiveDt=True, cflFactor=0.3)
    cfg.minDt = 1e-8
    x, H, area, _ = ws.buildPointCloud(nx, dom, cfg.targetNeighbors, device=cuda)
    m = torch.full((x.shape[0],), float(area), device=cuda)
    return cfg, x, H, m


def gather_density(cfg, x, H, m):
    p = ws.make_params(cfg)
    adj = ops.buildVerletList(x, H, p, cfg.verletScale)
    return ops.density(p, x, H, m, adj, SupportScheme.Gather)


@pytest.mark.parametrize("kernel", ["Wendland4", "Wendland2"])
def test_taylor_green_lattice_density_energy_and_c0(cuda, kernel):
    want = NB.TGV[kernel]
    cfg, x, H, m = lattice(cuda, NB.TGV_NX, 0.0, NB.TGV_L, 2, getattr(KernelFunctions, kernel))
    rho = gather_density(cfg, x, H, m)
    assert (NB.fmt6(rho.mean()), NB.fmt6(rho.min()), NB.fmt6(rho.max())) == want["rho"]
    m = m / rho.mean()
    rho = gather_density(cfg, x, H, m)
    assert (NB.fmt6(rho.mean()), NB.fmt6(rho.max())) == ("1", "1")
    # on the exact lattice every density is the same sum; the corrected minimum is the FP32
    # rounding spread of that sum over the particles (the reference sums in its own order)
    assert abs(float(rho.min()) - float(want["rho_corrected_min"])) < 4e-6
    v = torch.from_numpy(NB.tgv_velocities(x.cpu().numpy())).to(cuda)
    ke = (0.5 * m * (v * v).sum(-1)).sum()
    # the printed energy (a torch FP32 sum over 16,384 particles) to 2e-6 relative: the
    # summation order moves its sixth digit
    assert abs(float(ke) / float(want["ke"]) - 1) < 2e-6, float(ke)
    cfg.dx = NB.TGV_L / NB.TGV_NX      # masses.min() ** (1 / dim) before the correction
    sch = IncompressibleSPHConfig()
    state = CompressibleState(positions=x, supports=H, masses=m, densities=rho, velocities=v)
    c0, dt = wcsph.setupWeaklyCompressibleTimestep(cfg, sch, CompressibleSystem(state=state), NB.TGV_TARGET_DT, verbose=False)
    assert abs(c0 / want["c0"] - 1) < 1e-6 and dt == NB.TGV_TARGET_DT


def test_wendland4_block_1d_density_c0_and_dt(cuda):
    b = NB.BLOCK_1D
    cfg, x, H, m = lattice(cuda, b["nx"], -b["L"] / 2, b["L"] / 2, 1, KernelFunctions.Wendland4)
    keep = x[:, 0].abs() < 0.5
    x, H, m = x[keep].contiguous(), H[keep].contiguous(), m[keep].contiguous()
    rho = gather_density(cfg, x, H, m)
    for got, w in zip((rho.mean(), rho.min(), rho.max()), b["rho"]):
        assert abs(float(got) / w - 1) < 5e-6, (float(got), w)
    cfg.dx = b["L"] / b["nx"]
    sch = IncompressibleSPHConfig()
    state = CompressibleState(positions=x, supports=H, masses=m, densities=rho, velocities=torch.zeros_like(x))
    system = CompressibleSystem(state=state)
    c0, _ = wcsph.setupWeaklyCompressibleTimestep(cfg, sch, system, b["target_dt"], verbose=False)
    assert abs(c0 / b["c0"] - 1) < 1e-6
    # the notebook's version of the set-up returns computeTimestep(dt=None): the acoustic
    # limit 0.3 H_1D / c0 / k_1D, with the Wendland4 1D kernel scale
    dt = float(wcsph.computeTimestep(system, cfg, sch, dt=None))
    assert abs(dt / b["dt"] - 1) < 1e-6


def compressible_dt(cuda, case, lo, hi, dim, u_of, dt_prev=None):
    """computeTimestep (timestep/compressible.py) on the notebook's lattice: supports from
    the sampler (n_h = 4), internal energies from the case's pressure and density."""
    cfg, x, H, m = lattice(cuda, case["nx"], lo, hi, dim, KernelFunctions.B7)
    sch = ws.CRKSPHConfig()
    sch.gamma = case["gamma"]
    u = u_of(x).to(torch.float32).contiguous()
    state = CompressibleState(positions=x, velocities=torch.zeros_like(x), supports=H, masses=m, densities=torch.ones_like(m),
                              internalEnergies=u)
    cfg.dt = dt_prev
    return ws.computeTimestep(CompressibleSystem(state=state), cfg, sch, dt=dt_prev)


def test_b7_cfl_factor_woodward_colella_1d(cuda):
    c = NB.WOODWARD_COLELLA
    g = c["gamma"]

    def u_of(x):
        p = torch.where(x[:, 0].abs() < 0.1, c["p_max"], torch.where(x[:, 0].abs() < 0.9, 0.1, 100.0)).to(torch.float32)
        return p / torch.ones_like(p) / (g - 1)
    dt = compressible_dt(cuda, c, -1.0, 1.0, 1, u_of)
    assert abs(dt / c["dt"] - 1) < 1e-6, dt


def test_b7_cfl_factor_gresho_and_kelvin_helmholtz_2d(cuda):
    c = NB.GRESHO
    g = c["gamma"]

    def u_gresho(x):
        r = torch.linalg.norm(x, dim=-1)
        p = torch.where(r < 0.2, 12.5 * r * r + 5, torch.where(r < 0.4, 12.5 * r * r - 20 * r + 4 * torch.log(5 * r) + 9,
                                                                c["p_max"]))
        return 1 / (g - 1) * (p.to(torch.float32) / 1.0)
    dt = compressible_dt(cuda, c, -0.5, 0.5, 2, u_gresho)
    assert abs(dt / c["dt"] - 1) < 1e-6, dt
    k = NB.KELVIN_HELMHOLTZ
    g = k["gamma"]

    def u_kh(x):
        y = x[:, 1]
        rho = torch.where((y >= 0.25) & (y < 0.75), 2.0, 1.0).to(torch.float32)
        return (k["p"] / rho / (g - 1)).to(torch.float32)
    # setupBasicCompressibleInitialState leaves config.dt = maxDt (zero pressure); sampleKHH
    # then scales the CFL step by 2/3 (kelvinHelmholtz/sample.py:71)
    dt = compressible_dt(cuda, k, 0.0, 1.0, 2, u_kh, dt_prev=1e-2) * 2 / 3
    assert abs(dt / k["dt"] - 1) < 1e-6, dt


def test_b7_sod_owen_support_density_and_dt(cuda):
    s = NB.SOD
    dom = ws.buildDomainDescription(2, 1, True, cuda)
    cfg, integ = ws.buildConfig(device=cuda, domain=dom, dim=1, kernel=KernelFunctions.B7, targetNeighbors=n_h_to_nH(4, 1),
                                supportMode=SupportScheme.Gather, dt=1e-3, adaptiveDt=True, cflFactor=0.3)
    cfg.nx = s["nx"]
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    left, right = ws.sodInitialState(*s["left"], 0.0), ws.sodInitialState(*s["right"], 0.0)
    system = ws.buildSod1D(System, State, s["ratio"], left, right, s["gamma"], cfg, True,
                           adaptiveSupportScheme=AdaptiveSupportScheme.Owen)
    S = system.state
    # the notebook prints u = P / ((gamma - 1) rho) at the Owen densities, before the ramp
    P = torch.where(S.materials == 0, s["left"][0], s["right"][0]).to(torch.float32)
    u = 1 / (s["gamma"] - 1) * (P / S.densities)
    assert (f"{float(u.min()):6.4g}".strip(), f"{float(u.max()):6.4g}".strip()) == s["u_range"]
    assert abs(cfg.dt / s["dt"] - 1) < 2e-5, cfg.dt
    # the smallest support is the dense lattice's: four spacings
    assert abs(float(S.supports.min()) / (4.0 / s["nx"]) - 1) < 2e-5
