"""The Cullen-Hopkins switch on the CPU oracle against golden vectors from the reference's
own computeHopkinsTerms / computeHopkinsUpdate (modules/shockCapturing/CullenHopkins.py,
with computeR / computeXi / computeShearTensor and the wp_vsig.py pair body), generated by
tests/golden/make_golden.py --which hopkins on the CompSPH fixture's particles."""
from pathlib import Path

import numpy as np

import warpsph_b200 as ws
from oracle import oracle
from tests.cases import assert_close, make_params

HERE = Path(__file__).resolve().parent / "golden"


def hopkins_params():
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    p.alpha_min, p.alpha_max, p.beta_xi, p.limit_xi, p.beta_c, p.beta_d = 0.02, 2.0, 2.0, 0, 0.7, 0.05
    return p


def test_hopkins_switch_matches_reference():
    g, h = dict(np.load(HERE / "compsph_golden.npz")), dict(np.load(HERE / "hopkins_golden.npz"))
    p = hopkins_params()
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    o = oracle.get("f32")
    al, div, s2, R = o.switch_hopkins_terms(p, g["x"], g["H"], g["m"], g["rho"], g["v"], h["hopkins_alpha0"], nb)
    assert_close(div, h["hopkins_div"], 1e-6, 1e-7, "divergence vs reference common.py")
    assert_close(R, h["hopkins_R"], 1e-6, 1e-7, "R vs reference CullenDehnen2010.py")
    assert_close(al, h["hopkins_alphas"], 1e-6, 1e-7, "alphas vs reference CullenHopkins.py")
    a0, vs = o.switch_hopkins_update(p, g["x"], g["H"], g["v"], g["c"], div, h["hopkins_div_prev"], h["hopkins_alpha0"],
                                     h["hopkins_dt"][0], nb)
    assert_close(vs, h["hopkins_vsig"], 1e-6, 1e-7, "v_sig vs reference wp_vsig.py")
    assert_close(a0, h["hopkins_alpha0_next"], 1e-6, 1e-7, "alpha0 update vs reference CullenHopkins.py")
    # both branches of the update occur
    assert (h["hopkins_alpha0_next"] != h["hopkins_alpha0"]).mean() > 0.3
    assert h["hopkins_alphas"].min() == np.float32(0.02) and h["hopkins_alphas"].max() > 0.5


def test_moment_matrix_matches_reference():
    """M_i = -sum_j m_j x_ij (x) grad W(r_ij, H_i) against the reference's computeM
    (common.py negating the wp_computeM.py pair body)."""
    g, h = dict(np.load(HERE / "compsph_golden.npz")), dict(np.load(HERE / "hopkins_golden.npz"))
    p = hopkins_params()
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    for precision in ("f32", "f64"):
        M = oracle.get(precision).moment_matrix(p, g["x"], g["H"], g["m"], nb)
        assert_close(M, h["hopkins_cvg_M"], 1e-5, 1e-6, f"moment matrix ({precision}) vs reference wp_computeM.py")


def test_hopkins_corrected_gradient_matches_reference():
    """correctVelocityGradient: the gradient is pinv(M) V before its trace and shear
    (CullenHopkins.py:24-34, common.py:76-78)."""
    g, h = dict(np.load(HERE / "compsph_golden.npz")), dict(np.load(HERE / "hopkins_golden.npz"))
    p = hopkins_params()
    p.correct_velocity_gradient = 1
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    for precision, tol in (("f32", 1e-5), ("f64", 1e-5)):
        o = oracle.get(precision)
        al, div, s2, R = o.switch_hopkins_terms(p, g["x"], g["H"], g["m"], g["rho"], g["v"], h["hopkins_alpha0"], nb)
        assert_close(div, h["hopkins_cvg_div"], tol, tol, f"corrected divergence ({precision})")
        assert_close(R, h["hopkins_cvg_R"], tol, tol, f"R from the corrected divergence ({precision})")
        assert_close(al, h["hopkins_cvg_alphas"], 1e-4, 1e-5, f"alphas, corrected gradient ({precision})")
        a0, _ = o.switch_hopkins_update(p, g["x"], g["H"], g["v"], g["c"], div, h["hopkins_div_prev"], h["hopkins_alpha0"],
                                        h["hopkins_dt"][0], nb)
        assert_close(a0, h["hopkins_cvg_alpha0_next"], 1e-4, 1e-5, f"alpha0 update, corrected gradient ({precision})")
    # the correction changes the result by more than the tolerance
    assert np.abs(h["hopkins_cvg_div"] - h["hopkins_div"]).max() > 0.05 * np.abs(h["hopkins_div"]).max()


def test_moment_pinv_drops_singular_directions():
    """torch.linalg.pinv's default cutoff for float32: singular values at or below
    D * eps_float32 * sigma_max are dropped."""
    M = np.array([[[2.0, 0.0], [0.0, 1e-9]], [[1.0, 1.0], [1.0, 1.0]], [[0.0, 0.0], [0.0, 0.0]], [[0.0, 2.0], [-4.0, 0.0]]])
    P = oracle.get("f64").moment_pinv(M)
    want = np.array([[[0.5, 0.0], [0.0, 0.0]], [[0.25, 0.25], [0.25, 0.25]], [[0.0, 0.0], [0.0, 0.0]], [[0.0, -0.25], [0.5, 0.0]]])
    assert np.allclose(P, want, rtol=1e-12, atol=1e-12)
