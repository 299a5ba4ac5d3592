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


# ---------------------------------------------------------------- DFSPH (tests/golden/dfsph_golden.npz)
DF_GOLD = Path(__file__).resolve().parent / "golden" / "dfsph_golden.npz"


@pytest.fixture(scope="module")
def dgold():
    return dict(np.load(DF_GOLD))


def jacobi_cfg(g, name):
    from warpsph_b200._capi import SphJacobiConfig
    mn, mx, tol, om = g[name + "_config"]
    c = SphJacobiConfig()
    c.rest_density, c.tolerance, c.relaxation = 1.0, float(tol), float(om)
    c.min_iterations, c.max_iterations = int(mn), int(mx)
    return c


def test_golden_dfsph_operators(dgold):
    """computeAlpha (wp_alpha.py), computeMomentumIncompressible, computePressureAccelIISPH and
    computePressureShiftIISPH: identical float32 operation order, so exact."""
    g = dgold
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    o = oracle.get("f32")
    assert_close(o.dfsph_alpha(p, g["x"], g["H"], g["m"], g["rho"], nb), g["alpha"], 1e-6, 1e-7, "computeAlpha")
    assert_close(o.incompressible_divergence(p, 1.0, g["x"], g["H"], g["m"], g["rho"], g["v"], None, 0.0, nb), g["divergence"],
                 1e-6, 1e-7, "computeMomentumIncompressible")
    assert_close(o.pressure_accel_iisph(p, g["x"], g["H"], g["m"], g["rho"], g["p_prev"], nb), g["accel_iisph"], 1e-6, 1e-7,
                 "computePressureAccelIISPH")
    assert_close(o.pressure_shift_iisph(p, g["x"], g["H"], g["m"], g["rho"], g["accel_iisph"], nb), g["shift_iisph"], 1e-6, 1e-7,
                 "computePressureShiftIISPH")


@pytest.mark.parametrize("name,mode", [("df_fixed", 0), ("df_default", 0), ("rho_fixed", 1), ("rho_default", 1)])
def test_golden_dfsph_solves(dgold, name, mode):
    """solveDivergenceFree / solveIncompressible run from the reference source: the
    iteration count, the per-iteration errors and pressure statistics, the final
    pressure and acceleration.  The divergence-free gauge subtracts a mean that torch
    sums in float32 and the oracle in double: 1e-6 relative."""
    g = dgold
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    pr, acc, hist, it = oracle.get("f32").jacobi_solve(p, mode, jacobi_cfg(g, name), g["x"], g["H"], g["m"], g["rho"], g["v"],
                                                       g["dvdt"], g["p_prev"], float(g["dt"][0]), nb)
    assert it == len(g[name + "_errors"])
    assert_close(hist[:, 0], g[name + "_errors"], 1e-6, 1e-7, f"{name} errors")
    assert_close(hist[:, 1:], g[name + "_pressures"], 1e-6, 1e-6, f"{name} pressures")
    assert_close(pr, g[name + "_p"], 1e-6, 1e-6, f"{name} pressure")
    assert_close(acc, g[name + "_accel"], 1e-6, 1e-6, f"{name} acceleration")
