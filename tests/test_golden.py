"""The CPU oracle against golden vectors produced by the reference's own Python source
(tests/golden/make_golden.py runs modules/crk/accel.py, modules/crk/dudt.py,
modules/crk/limiter.py, modules/compSPH/balance.py, modules/shockCapturing/wp_vsig.py,
modules/shockCapturing/CullenDehnen2010.py, modules/eos/idealGas.py,
modules/compSPH/multistep.py and modules/timestep/compressible.py unmodified).

Both sides compute in FP32 with the same operation order, so the tolerances only
absorb libm differences (expf, powf) between numpy and glibc."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core
from warpsph_b200.enumTypes import EnergyScheme

GOLD = Path(__file__).resolve().parent / "golden" / "crk_pair_golden.npz"


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


@pytest.fixture(scope="module")
def setup(gold):
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    nb = dict(offsets=gold["offsets"], counts=gold["counts"], list=gold["list"])
    return p, nb


def test_golden_accel_dudt(gold, setup):
    p, nb = setup
    o = oracle.get("f32")
    g = gold
    dvdt, dudt, ap, av = o.crk_accel_dudt(p, g["x"], g["H"], g["m"], g["rho"], g["V"], g["A"], g["B"], g["gA"], g["gB"], g["v"],
                                          g["c"], g["P"], g["G"], nb)
    assert_close(ap, g["ap"], 1e-5, 1e-6, "ap_ij vs reference accel.py")
    assert_close(av, g["av"], 1e-5, 1e-6, "av_ij vs reference accel.py")
    assert_close(dvdt, g["accel"], 1e-5, 1e-6, "dv/dt vs reference accel.py")
    assert_close(dudt, g["dudt"], 1e-5, 1e-6, "du/dt vs reference dudt.py")
    assert np.abs(g["ap"]).max() > 0 and np.abs(g["av"]).max() > 0


@pytest.mark.parametrize("scheme", list(EnergyScheme))
def test_golden_energy_partition(gold, setup, scheme):
    p, nb = setup
    p.energy_scheme = scheme.value
    g = gold
    f = oracle.get("f32").balance(p, g["m"], g["rho"], g["P"], g["u"], g["v"], g["dvdt_guess"], float(g["balance_dt"][0]), nb,
                                  g["ap"], g["av"])
    ref = g["f_ij"][scheme.value]
    assert_close(f, ref, 1e-5, 1e-6, f"f_ij {scheme.name} vs reference balance.py")


def test_golden_vsig_eos_switch_timestep(gold, setup):
    p, nb = setup
    o = oracle.get("f32")
    g = gold
    _, _, div, vs = o.grad_v(p, g["x"], g["H"], g["m"], g["rho"], g["V"], g["A"], g["B"], g["gA"], g["gB"], g["v"], g["c"], nb, True)
    assert_close(vs, g["vsig"], 1e-6, 1e-7, "v_sig vs reference wp_vsig.py")
    A, P, c = o.eos(p, g["u"], g["rho"])
    assert_close(P, g["eos_P"], 1e-6, 1e-7, "P vs reference idealGas.py")
    assert_close(c, g["eos_c"], 1e-6, 1e-7, "c vs reference idealGas.py")
    assert_close(A, g["eos_A"], 1e-5, 1e-6, "A vs reference idealGas.py")
    al, R = o.switch_cullen(p, g["x"], g["H"], g["m"], g["rho"], g["div"], g["cullen_div_prev"], g["vsig"], g["cullen_alpha0"],
                            1e-3, nb)
    assert_close(R, g["cullen_R"], 1e-5, 1e-6, "R vs reference CullenDehnen2010.py")
    assert_close(al, g["cullen_alpha"], 1e-5, 1e-6, "alpha vs reference CullenDehnen2010.py")
    assert abs(o.cfl_dt(p, g["H"], g["u"], 1e-4) - g["cfl_dt_grow"][0]) <= 1e-6 * g["cfl_dt_grow"][0]
    assert abs(o.cfl_dt(p, g["H"], g["u"], None) - g["cfl_dt_first"][0]) <= 1e-6 * g["cfl_dt_first"][0]


@pytest.mark.parametrize("scheme", [EnergyScheme.CRK, EnergyScheme.PdV])
def test_golden_compatible_energy(gold, setup, scheme):
    p, nb = setup
    p.energy_scheme = scheme.value
    g = gold
    stages = [dict(dvdt=g["multistep_dvdt"][s], nb=nb, f=g["f_ij"][5 if s == 0 else 0], ap=g["ap"] * np.float32(1 + 0.1 * s),
                   av=g["av"] * np.float32(1 - 0.1 * s)) for s in range(2)]
    u, du = oracle.get("f32").finalize(p, [0.5, 0.5], float(g["balance_dt"][0]), g["v"], g["u"], stages)
    assert_close(du, g[f"multistep_du_{scheme.name}"], 1e-5, 1e-6, f"du vs reference multistep.py ({scheme.name})")
