"""The CPU oracle's mDBC passes against golden vectors made by executing the reference's
own code (tests/golden/make_golden.py --which mdbc): the Liu-Liu moments at the ghost
points (modules/liu/wp_mat.py), the wall density of computeMdbcDensity
(modules/mdbc/density2025.py, with interpolateLiuLiu of modules/liu/interp.py and
torch.linalg.pinv) and the no-penetration shift (modules/mdbc/wp_nopenshift.py), on a
fluid block resting on a three-layer wall with mirrored ghost points.  Tolerances: 1e-5
of each field's scale (FP32 sums in the same order).  The wall densities of ghosts whose
moment matrix is ill-conditioned (condition number above 1e3, ghosts near the fluid's
edge) are compared to 2e-4 of the scale: there torch's FP32 pseudo-inverse in the
reference is itself off by about that much from the FP64 one (checked against
numpy's FP64 SVD), and the oracle's LAPACK SVD sits with the FP64 answer."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core

GOLD = Path(__file__).resolve().parent / "golden" / "mdbc_golden.npz"


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def nbl(g):
    return dict(offsets=g["offsets"], counts=g["counts"], list=g["list"])


def wall_conditioning(g):
    """Masks of the wall particles whose ghost's Liu-Liu matrix is well / ill conditioned."""
    ghosts = np.nonzero(g["kinds"] == 2)[0]
    cond = np.array([np.linalg.cond(a.astype(np.float64)) for a in g["liu_A"]])
    well = np.zeros(len(g["kinds"]), bool)
    ill = np.zeros(len(g["kinds"]), bool)
    wall_of = g["ghost_indices"][ghosts]
    well[wall_of[cond <= 1e3]] = True
    ill[wall_of[cond > 1e3]] = True
    return well, ill


def test_golden_liu_moments(gold):
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    b, A, nbrs = oracle.get("f32").liu_moments(p, gold["x"], gold["H"], gold["m"], gold["rho"], gold["kinds"], nbl(gold))
    ghosts = gold["kinds"] == 2
    assert np.array_equal(nbrs[ghosts], gold["liu_nbrs"])
    assert_close(b[ghosts], gold["liu_b"], 1e-5, 1e-5, "Liu b")
    assert_close(A[ghosts], gold["liu_A"], 1e-5, 1e-5, "Liu A")


def test_golden_mdbc_density(gold):
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    rho, _ = oracle.get("f32").mdbc_density(p, gold["x"], gold["H"], gold["m"], gold["rho"], gold["kinds"], gold["ghost_indices"],
                                            gold["ghost_offsets"], nbl(gold), float(gold["rho0"][0]), float(gold["c_s"][0]),
                                            gold["gravity"])
    want = gold["mdbc_density"]
    wall = gold["kinds"] == 1
    assert np.array_equal(rho[~wall], want[~wall])                  # copied
    assert not np.allclose(want[wall], gold["rho"][wall])            # the walls got new densities
    well, ill = wall_conditioning(gold)
    assert well.sum() > 40 and ill.sum() > 0
    assert_close(rho[well], want[well], 1e-5, 1e-5, "mDBC wall density (well-conditioned moments)")
    scale = np.abs(want[wall]).max()
    assert np.abs(rho[ill] - want[ill]).max() < 2e-4 * scale, "mDBC wall density (ill-conditioned moments)"


def test_golden_mdbc_nopen_shift(gold):
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    s = oracle.get("f32").mdbc_nopen_shift(p, gold["x"], gold["H"], gold["m"], gold["v"], gold["kinds"], gold["ghost_offsets"], nbl(gold))
    assert (np.abs(gold["nopen_shift"]).sum(1) > 0).sum() > 0
    assert_close(s, gold["nopen_shift"], 1e-6, 1e-6, "no-penetration shift")
