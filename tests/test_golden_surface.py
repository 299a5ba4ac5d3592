"""Free-surface detection (colour-field scheme) on the CPU oracle against golden vectors
from the reference's own detectFreeSurface (modules/surfaceDetection/wrapper.py with
colorFieldCompute.py, colorFieldDetection.py, dilation.py and the wp_numNeighbors.py,
wp_sum.py and wp_dilate.py pair bodies), generated by
tests/golden/make_golden.py --which surface on a 2D block of fluid with free edges."""
from pathlib import Path

import numpy as np

import warpsph_b200 as ws
from oracle import oracle
from tests.cases import assert_close, make_params

HERE = Path(__file__).resolve().parent / "golden"


def surface_params():
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4, periodic=False)
    return p


def test_color_field_detection_matches_reference():
    g = dict(np.load(HERE / "surface_golden.npz"))
    p = surface_params()
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    limit = float(g["surface_target_neighbors"][0]) * float(g["surface_threshold"][0])
    for precision in ("f32", "f64"):
        o = oracle.get(precision)
        c = o.surface_color_field(p, g["x"], g["H"], g["m"], g["rho"], nb)
        assert_close(c, g["surface_color"], 1e-5, 1e-6, f"colour field ({precision})")
        fsm, normals, nn = o.surface_detect(p, g["x"], g["H"], g["m"], g["rho"], g["surface_color"], nb, limit, -1.0)
        assert np.array_equal(nn, g["surface_num_neighbors"]), "super-symmetric neighbour counts"
        assert np.array_equal(fsm, g["surface_fsm"]), f"surface mask ({precision})"
        assert_close(normals, g["surface_normals"], 1e-4, 1e-5, f"normals ({precision})")
        fs = o.surface_dilate(p, g["x"], g["H"], g["surface_fsm"], nb)
        assert np.array_equal(fs, g["surface_fs"]), "dilation"
    assert 0 < g["surface_fsm"].sum() < len(g["H"]) and g["surface_fs"].max() > 1


def test_barecasco_maronne_and_colour_gradient_match_reference():
    """The Barecasco, Maronne and colour-field-gradient schemes against the reference's own
    bodies (surface_schemes_golden.npz, make_golden.py --which surface): masks and counts
    exactly, directions to 1e-5 (FP32; FP64 to 2e-3, see below)."""
    g = dict(np.load(HERE / "surface_golden.npz"))
    s = dict(np.load(HERE / "surface_schemes_golden.npz"))
    p = surface_params()
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    for precision in ("f32", "f64"):
        o = oracle.get(precision)
        for tag in ("pi3", "1p5"):
            fs, nrm, cnt = o.surface_barecasco(p, g["x"], g["H"], nb, float(s[f"barecasco_{tag}_threshold"][0]))
            assert np.array_equal(cnt, s[f"barecasco_{tag}_count"]), f"Barecasco counts {tag} ({precision})"
            assert np.array_equal(fs, s[f"barecasco_{tag}_fsm"]), f"Barecasco mask {tag} ({precision})"
            # the direction of an interior particle's near-zero cover vector is rounding noise:
            # FP32 follows the reference's FP32 sums, FP64 only to 2e-3
            tol = (1e-5, 1e-6) if precision == "f32" else (0.0, 2e-3)
            assert_close(nrm, s[f"barecasco_{tag}_normals"], *tol, f"Barecasco cover directions {tag} ({precision})")
        for tag in ("colour", "cover"):
            fs, cnt = o.surface_maronne(p, g["x"], g["H"], s[f"maronne_{tag}_normals"], nb)
            assert np.array_equal(cnt, s[f"maronne_{tag}_count"]), f"Maronne counts {tag} ({precision})"
            assert np.array_equal(fs, s[f"maronne_{tag}_fsm"]), f"Maronne mask {tag} ({precision})"
        fs, nrm = o.surface_color_gradient(p, g["x"], g["H"], g["m"], g["rho"], g["surface_color"], nb, float(s["cfgrad_threshold"][0]))
        assert np.array_equal(fs, s["cfgrad_fsm"]), f"colour-gradient mask ({precision})"
        assert_close(nrm, s["cfgrad_normals"], 1e-4, 1e-5, f"colour-gradient normals ({precision})")
    for k in ("barecasco_pi3_fsm", "maronne_colour_fsm", "cfgrad_fsm"):
        assert 0 < s[k].sum() < len(g["H"]), k


def test_renormalization_oracle_is_consistent():
    """The restated renormalisation (warpSPHCore's computeRenormalizationMatrices is absent):
    M is the identity for an interior particle of a uniform lattice, L M = I where M is
    regular, and the smallest |eigenvalue| drops at the block's free edges."""
    g = dict(np.load(HERE / "surface_golden.npz"))
    p = surface_params()
    nb = dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])
    o = oracle.get("f64")
    L, lam, M = o.surface_renormalization(p, g["x"], g["H"], g["m"], g["rho"], nb)
    eye = np.eye(2)
    assert np.abs(np.einsum("nab,nbc->nac", L.astype(np.float64), M.astype(np.float64)) - eye).max() < 1e-6
    fsm = g["surface_fsm"] > 0
    assert lam[~fsm].mean() > 0.9 and lam[fsm].mean() < lam[~fsm].mean() - 0.1
    nrm, grad = o.surface_renorm_normals(p, 1, g["x"], g["H"], g["m"], g["rho"], L, None, nb)
    assert np.all(np.abs(np.linalg.norm(nrm, axis=1) - 1) < 1e-6)
