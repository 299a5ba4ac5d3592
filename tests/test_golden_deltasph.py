"""The CPU oracle's delta-SPH right-hand side against golden vectors produced by the
reference's own pair bodies (tests/golden/make_golden.py --which deltasph runs
modules/deltaSPH/wp_viscosityDelta.py, modules/deltaSPH/wp_densityDelta.py and
modules/pressure/wp_surfaceAware.py unmodified, under the super-symmetric support).

The oracle combines the terms (dv/dt = -pressure / rho_i + viscosity, the division being
the one the reference's kernel wrapper applies at wp_surfaceAware.py:207-218; drho/dt =
-rho continuity + delta (H / xi) c0 diffusion); each term is isolated by a parameter
choice: a Tait EOS
with kappa = 0 gives P = 0 (no pressure term), inviscid alpha = 0 gives no viscosity,
and two densityDelta values separate the diffusion from the continuity.  Tolerances are
a few FP32 ulps of each field's scale (1e-5 relative; 1e-4 where a difference of two
oracle outputs is taken)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core
from warpsph_b200.configurations import WeaklyCompressibleSPHConfig, wc_params

GOLD = Path(__file__).resolve().parent / "golden" / "deltasph_golden.npz"
PTERMS = ["conservative", "nonConservative", "Antuono", "i", "j", "symmetric"]
DSCHEMES = {0: "deltaSPH", 2: "densityOnly", 3: "deltaOnly"}


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def run(g, surface_mask=None, **kw):
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    cfg = WeaklyCompressibleSPHConfig()
    for k, v in kw.items():
        if k in ("inviscid", "inviscidAlpha", "viscidNu", "densityDelta", "densityDiffusionTerm"):
            setattr(cfg.diffusionParams, k, v)
        elif k in ("kappa", "fixedSoundSpeed"):
            setattr(cfg.fluid, k, v)
        else:
            setattr(cfg, k, v)
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    return oracle.get("f32").deltasph_rhs(p, wc_params(cfg), g["x"], g["H"], g["m"], g["rho"], g["v"], nb, surface_mask)


def test_golden_inputs_reproduced(gold):
    """The renormalised density gradient and pressure stored with the golden case are the
    oracle's first pass on the same inputs (the reference takes them from warpSPHCore)."""
    _, _, gL, P = run(gold)
    assert np.array_equal(gL, gold["gL"]) and np.array_equal(P, gold["P"])


@pytest.mark.parametrize("inviscid", [True, False])
def test_golden_velocity_diffusion(gold, inviscid):
    alpha, c_s, nu = gold["wc_coeffs"]
    dv, _, _, _ = run(gold, eosType="Tait", kappa=0.0, inviscid=inviscid, inviscidAlpha=float(alpha), fixedSoundSpeed=float(c_s),
                      viscidNu=float(nu))
    want = gold["visc_inviscid"] if inviscid else gold["visc_viscid"]
    assert_close(dv, want, 1e-5, 1e-5, f"velocity diffusion (inviscid={inviscid})")


@pytest.mark.parametrize("t", range(6))
def test_golden_pressure_force(gold, t):
    dv, _, _, P = run(gold, inviscid=True, inviscidAlpha=0.0, pressureForceTerm=PTERMS[t])
    assert np.array_equal(P, gold["P"])
    want = -gold["pf"][t] / gold["rho"][:, None]      # the wrapper's -sum / rho_i
    assert_close(dv, want, 1e-5, 1e-5, f"pressure force {PTERMS[t]}")


def test_golden_pressure_force_surface_mask(gold):
    """The Antuono term with free-surface particles: mask_i == 1 selects P_j + P_i even
    where both pressures are negative (wp_surfaceAware.py:89-92)."""
    mask = gold["surface_mask"]
    assert np.any((mask == 1) & (gold["P"] < 0))
    dv, _, _, _ = run(gold, surface_mask=mask, inviscid=True, inviscidAlpha=0.0, pressureForceTerm="Antuono")
    assert_close(dv, -gold["pf_antuono_mask"] / gold["rho"][:, None], 1e-5, 1e-5, "Antuono pressure force with surface mask")
    # without the mask the masked particles with negative pressure differ
    dv0, _, _, _ = run(gold, inviscid=True, inviscidAlpha=0.0, pressureForceTerm="Antuono")
    assert not np.allclose(dv0, dv)


@pytest.mark.parametrize("s", range(3))
def test_golden_density_diffusion(gold, s):
    scheme = DSCHEMES[int(gold["dd_schemes"][s])]
    c0 = 10.0
    _, d0, _, _ = run(gold, densityDelta=0.0, densityDiffusionTerm=scheme, fixedSoundSpeed=c0)
    _, d1, _, _ = run(gold, densityDelta=1.0, densityDiffusionTerm=scheme, fixedSoundSpeed=c0)
    xi = float(core.sphKernelScale(core.KernelFunctions.Wendland4, 2))
    dd = (d1.astype(np.float64) - d0) / (gold["H"].astype(np.float64) / xi * c0)
    assert_close(dd, gold["dd"][s], 1e-4, 1e-4, f"density diffusion {scheme}")


def test_golden_delta_shift(gold):
    """computeDeltaShift (modules/shifting/delta.py) with the reference's pair body: the
    oracle agrees to 5e-5 of the field's scale (the (W/W0)^4 factor and the torch norm
    behind Ma amplify FP32 rounding a little)."""
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    nb = dict(offsets=gold["offsets"], counts=gold["counts"], list=gold["list"])
    cfl, c0 = gold["shift_coeffs"]
    s = oracle.get("f32").delta_shift(p, gold["x"], gold["H"], gold["m"], gold["rho"], gold["v"], nb, float(cfl), float(c0))
    assert_close(s, gold["shift"], 5e-5, 5e-5, "delta-plus shift")
    # boundary particles (kind != 0) do not move
    kinds = np.zeros(len(gold["H"]), np.int32)
    kinds[::7] = 1
    s2 = oracle.get("f32").delta_shift(p, gold["x"], gold["H"], gold["m"], gold["rho"], gold["v"], nb, float(cfl), float(c0), kinds=kinds)
    assert np.all(s2[::7] == 0) and np.array_equal(s2[kinds == 0], s[kinds == 0])
