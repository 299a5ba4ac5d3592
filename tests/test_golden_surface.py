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
