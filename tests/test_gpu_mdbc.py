"""mDBC on the GPU (sph_mdbc_density, sph_mdbc_nopen_shift through the C ABI) against the
reference's own code (golden vectors from modules/liu/wp_mat.py, liu/interp.py,
mdbc/density2025.py and mdbc/wp_nopenshift.py) and against the CPU oracle in 3D.

Tolerances as in test_golden_mdbc.py: 1e-5 of the scale where the Liu-Liu moment matrix
is well conditioned, 2e-4 where its condition number exceeds 1e3 (the reference's FP32
torch pseudo-inverse there differs from the FP64 one by about that much; the GPU's
Jacobi pseudo-inverse is FP64).  The no-penetration shift: 1e-5."""
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle
from oracle.steps import cell_capacity_for
from tests.cases import assert_close, make_params
from tests.test_golden_mdbc import wall_conditioning
from warpsph_b200 import core, ops
from warpsph_b200.core import AdjacencyList

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "mdbc_golden.npz"


def test_mdbc_matches_reference(cuda):
    g = dict(np.load(GOLD))
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in g.items()}
    _, _, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    n = len(g["H"])
    fixture = AdjacencyList(neighborOffsets=t["offsets"], numNeighbors=t["counts"], neighborList=t["list"], numRows=n, numCols=n,
                            nnz=int(g["list"].shape[0]))
    built = ops.buildVerletList(t["x"], t["H"], p, float(p.verlet_scale))
    well, ill = wall_conditioning(g)
    want = g["mdbc_density"]
    scale = np.abs(want[g["kinds"] == 1]).max()
    for adj in (fixture, built):
        rho, nbrs = ops.mdbc_density(p, t["x"], t["H"], t["m"], t["rho"], t["kinds"], t["ghost_indices"], t["ghost_offsets"], adj,
                                     float(g["rho0"][0]), float(g["c_s"][0]), [float(a) for a in g["gravity"]], want_neighbors=True)
        r = rho.cpu().numpy()
        assert np.array_equal(nbrs.cpu().numpy()[g["kinds"] == 2], g["liu_nbrs"])
        assert np.array_equal(r[g["kinds"] != 1], want[g["kinds"] != 1])
        assert_close(r[well], want[well], 1e-5, 1e-5, "mDBC wall density (GPU)")
        assert np.abs(r[ill] - want[ill]).max() < 2e-4 * scale
        s = ops.mdbc_nopen_shift(p, t["x"], t["H"], t["m"], t["v"], t["kinds"], t["ghost_offsets"], adj)
        assert_close(s.cpu().numpy(), g["nopen_shift"], 1e-5, 1e-5, "no-penetration shift (GPU)")


def wall_case_3d(seed=5, nf=10, nw=14):
    """A 3D fluid block over a three-layer floor with ghosts mirrored across z = 0; the lowest
    fluid layer is pressed against the floor and moves into it."""
    rng = np.random.default_rng(seed)
    dx = np.float32(1 / 40)
    g = (np.arange(nf) + 0.5) * dx - nf * dx / 2
    X, Y, Z = np.meshgrid(g, g, (np.arange(nf) + 0.5) * dx, indexing="ij")
    fluid = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + 0.1 * dx * (rng.random((nf ** 3, 3)) - 0.5)
    low = Z.ravel() < dx
    fluid[low, 2] = 0.2 * dx
    gw = (np.arange(nw) + 0.5) * dx - nw * dx / 2
    WX, WY, WZ = np.meshgrid(gw, gw, -(np.arange(3) + 0.5) * dx, indexing="ij")
    wall = np.stack([WX.ravel(), WY.ravel(), WZ.ravel()], 1)
    ghost = wall * np.array([1, 1, -1])
    x = np.concatenate([fluid, wall, ghost]).astype(np.float32)
    a, b = len(fluid), len(wall)
    n = len(x)
    kinds = np.concatenate([np.zeros(a), np.ones(b), np.full(b, 2)]).astype(np.int32)
    gi = np.full(n, -1, np.int32)
    gi[a:a + b], gi[a + b:] = np.arange(a + b, n), np.arange(a, a + b)
    go = np.zeros((n, 3), np.float32)
    go[a:a + b] = wall - ghost
    go[a + b:] = -(wall - ghost)
    v = (0.3 * rng.standard_normal((n, 3))).astype(np.float32)
    v[:a][low, 2] = -0.5
    v[kinds != 0] = 0
    return x, kinds, gi, go, v, dx, rng


def test_mdbc_3d_matches_oracle(cuda):
    x, kinds, gi, go, v, dx, rng = wall_case_3d()
    cfg, _, p = make_params(3, kernel=core.KernelFunctions.Wendland4)
    n = len(x)
    H = np.full(n, core.volumeToSupportHelper(float(dx) ** 3, cfg.targetNeighbors, 3), np.float32)
    m = np.full(n, float(dx) ** 3, np.float32)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, cell_capacity_for(n, 3))
    rho = (o.density(p, 0, x, H, m, nb) * (1 + 0.02 * rng.standard_normal(n))).astype(np.float32)
    t = {k: torch.from_numpy(a).to(cuda) for k, a in dict(x=x, H=H, m=m, rho=rho, kinds=kinds, gi=gi, go=go, v=v).items()}
    adj = ops.buildVerletList(t["x"], t["H"], p, float(p.verlet_scale))
    grav = [0.0, 0.0, -9.81]
    got, nbrs = ops.mdbc_density(p, t["x"], t["H"], t["m"], t["rho"], t["kinds"], t["gi"], t["go"], adj, 1.0, 10.0, grav,
                                 want_neighbors=True)
    want, wn = o.mdbc_density(p, x, H, m, rho, kinds, gi, go, nb, 1.0, 10.0, grav)
    assert np.array_equal(nbrs.cpu().numpy()[kinds == 2], wn[kinds == 2])
    _, A, _ = o.liu_moments(p, x, H, m, rho, kinds, nb)
    ghosts = np.nonzero(kinds == 2)[0]
    cond = np.array([np.linalg.cond(A[k].astype(np.float64)) if wn[k] > 4 else 0.0 for k in ghosts])
    well = gi[ghosts[cond <= 1e3]]
    assert len(well) > 100
    assert_close(got.cpu().numpy()[well], want[well], 1e-4, 1e-4, "3D mDBC wall density")
    s = ops.mdbc_nopen_shift(p, t["x"], t["H"], t["m"], t["v"], t["kinds"], t["go"], adj)
    ws_ = o.mdbc_nopen_shift(p, x, H, m, v, kinds, go, nb)
    assert (np.abs(ws_).sum(1) > 0).sum() > 10
    assert_close(s.cpu().numpy(), ws_, 1e-5, 1e-5, "3D no-penetration shift")
