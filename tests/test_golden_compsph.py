"""The CPU oracle against golden vectors produced by the reference's own Python source
for the CompSPH and Monaghan schemes (tests/golden/make_golden.py --which compsph runs
modules/adaptiveSupport/wp_omega.py, modules/dissipation/pi.py + util.py,
modules/compSPH/accel.py, modules/compSPH/dudt.py, modules/dissipation/wp_diffusion.py,
wp_conductivity.py and wp_dissipation.py unmodified).

Both sides compute in FP32 with the same operation order; the tolerances are a few
ulps of each field's scale."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core

GOLD = Path(__file__).resolve().parent / "golden" / "compsph_golden.npz"
TERMS = range(12)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def params_for(g, term=3, cterm=None, flags=(1, 0, 1)):
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    p.C_l, p.C_q, p.Cu_l, p.Cu_q, p.c_s = (float(a) for a in g["pi_coeffs"])
    p.viscosity_term = int(term)
    p.conductivity_term = int(term if cterm is None else cterm)
    p.monaghan_switch, p.scale_beta, p.correct_xi = (int(a) for a in flags)
    return p


def nbl(g):
    return dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])


def test_golden_omega(gold):
    g = gold
    om, _, _ = oracle.get("f32").compsph_prep(params_for(g), g["x"], g["H"], g["m"], g["rho"], g["v"], nbl(g))
    assert_close(om, g["omega"], 1e-6, 1e-7, "Omega vs reference wp_omega.py")
    assert g["omega"].min() < 0.95 and g["omega"].max() > 1.02


@pytest.mark.parametrize("variant", [0, 1])
def test_golden_pi_all_forms(gold, variant):
    """computePi_actual for all twelve ViscosityTerms forms, i / j / conductivity roles."""
    g = gold
    o = oracle.get("f32")
    sel = g["pi_sel"]
    for t in TERMS:
        p = params_for(g, t, t, g["pi_variants"][variant])
        for w, (useJ, thermal) in enumerate([(False, False), (True, False), (False, True)]):
            got = o.pi_pairs(p, g["x"], g["H"], g["rho"], g["v"], g["c"], g["alpha"], g["P"], nbl(g), useJ, thermal)[sel]
            assert_close(got, g["pi"][variant, t, w], 1e-6, 1e-7, f"Pi term {t} role {w} variant {variant} vs reference pi.py")
    # the forms differ from one another and the switch zeroes receding pairs only when on
    assert len({float(np.abs(g["pi"][variant, t, 0]).sum()) for t in TERMS}) >= 8
    zero_frac = (g["pi"][variant, 3, 0] == 0).mean()
    assert (zero_frac > 0.2) if g["pi_variants"][variant][0] else (zero_frac < 0.05)


@pytest.mark.parametrize("term", list(TERMS))
def test_golden_compsph_accel_dudt(gold, term):
    g = gold
    p = params_for(g, term)
    dvdt, dudt, dEdt, ap, av = oracle.get("f32").compsph_accel_dudt(p, g["x"], g["H"], g["m"], g["rho"], g["v"], g["c"], g["alpha"],
                                                                    g["P"], g["omega"], nbl(g))
    assert_close(dvdt, g["compsph_accel"][term], 1e-5, 1e-6, f"dv/dt vs reference compSPH/accel.py (term {term})")
    assert_close(dudt, g["compsph_dudt"][term], 1e-5, 1e-6, f"du/dt vs reference compSPH/dudt.py (term {term})")
    if term == 3:
        assert_close(ap, g["compsph_ap"], 1e-5, 1e-6, "ap_ij vs reference compSPH/accel.py")
        assert_close(av, g["compsph_av"], 1e-5, 1e-6, "av_ij vs reference compSPH/accel.py")
    ref_dE = g["m"] * np.sum(g["v"] * dvdt, 1) + g["m"] * dudt
    assert_close(dEdt, ref_dE, 1e-5, 1e-6, "dE/dt")


@pytest.mark.parametrize("which", [0, 1])
def test_golden_monaghan_dissipation(gold, which):
    g = gold
    t, ct = g["monaghan_sets"][which]
    p = params_for(g, t, ct)
    dv, du, dE, T = oracle.get("f32").monaghan_rhs(p, g["x"], g["H"], g["m"], g["rho"], g["v"], g["u"], g["c"], g["alpha"], g["P"],
                                                   g["omega"], nbl(g))
    assert_close(T["viscosity"], g["monaghan_viscosity"][which], 1e-5, 1e-6, "viscosity vs reference wp_diffusion.py")
    assert_close(T["conductivity"], g["monaghan_conductivity"][which], 1e-5, 1e-6, "conductivity vs reference wp_conductivity.py")
    assert_close(T["heating"], g["monaghan_heating"][which], 1e-5, 1e-6, "heating vs reference wp_dissipation.py")
    assert_close(dv, T["pressure"] + T["viscosity"], 1e-6, 1e-7, "dv/dt = pressure + viscosity")
    assert_close(du, T["pdv"] + T["conductivity"] + T["heating"], 1e-6, 1e-7, "du/dt = PdV + conductivity + heating")


def test_fp64_oracle_close_to_fp32_reference(gold):
    """The all-FP64 oracle agrees with the FP32 reference to FP32 rounding of the sums."""
    g = gold
    p = params_for(g)
    dvdt, dudt, *_ = oracle.get("f64").compsph_accel_dudt(p, g["x"], g["H"], g["m"], g["rho"], g["v"], g["c"], g["alpha"], g["P"],
                                                          g["omega"], nbl(g))
    assert_close(dvdt, g["compsph_accel"][3], 1e-4, 1e-5, "FP64 dv/dt")
    assert_close(dudt, g["compsph_dudt"][3], 1e-4, 1e-5, "FP64 du/dt")
