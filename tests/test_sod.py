"""The Sod shock tube on the CPU: the exact Riemann solver against the reference's own
solution (tests/golden/sod_exact.npz, from caseUtils/compressible/sod/sodSolution.py),
and the full CRKSPH run of the case (RK4, CFL 0.3, Balsara, to t = 0.2) on the CPU
oracle, whose L1 errors against the exact solution are bounded."""
from pathlib import Path

import numpy as np

import warpsph_b200 as ws
from oracle import riemann
from tests import sod_case as S

GOLD = Path(__file__).resolve().parent / "golden" / "sod_exact.npz"


def test_riemann_matches_reference_solution():
    g = np.load(GOLD)
    L, R = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)
    ps, us = riemann.star_state(L, R, 1.4)
    assert abs(ps - g["p_star"][0]) < 1e-9 and abs(us - g["u_star"][0]) < 1e-9
    w = riemann.wave_positions(float(g["t"][0]), L, R)
    for k in ("head", "tail", "contact", "shock"):
        assert abs(w[k] - g[k][0]) < 1e-9, k
    rho, u, p = riemann.sample(g["x"], float(g["t"][0]), L, R)
    np.testing.assert_allclose(rho, g["rho"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(u, g["u"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(p, g["p"], rtol=0, atol=1e-9)


def test_sod_initial_state():
    cfg, sch, _ = S.config("cpu")
    st = S.oracle_initial_state(ws.make_params(cfg, sch))
    m, x = st["masses"], st["positions"][:, 0]
    assert len(m) == S.NX + S.NX // S.RATIO == 1998
    assert np.ptp(m) <= 1e-6 * m.max()                       # 8:1 spacing with equal masses
    half = (x > 0) & (x < 1)
    assert half.sum() == 999
    # the ramped internal energy matches the states away from the interfaces
    u = st["internalEnergies"]
    assert abs(u[np.abs(x) < 0.3].mean() - 2.5) < 1e-4 and abs(u[np.abs(x) > 0.7].mean() - 2.0) < 1e-4


def test_sod_oracle_run_accuracy():
    cfg, sch, _ = S.config("cpu")
    p = ws.make_params(cfg, sch)
    st, t, steps = S.run_oracle(p, S.oracle_initial_state(p), 0.2)
    assert abs(t - 0.2) < 1e-9 and 300 < steps < 1000
    P = (S.GAMMA - 1) * st["densities"].astype(np.float64) * st["internalEnergies"]
    e = S.right_half_errors(st["positions"], st["densities"], st["velocities"], P, t)
    print("Sod CPU oracle L1 errors at t=0.2:", e)
    assert e["rho"] < 5e-3 and e["v"] < 1e-2 and e["p"] < 5e-3, e
