"""Free-surface detection on the GPU (colour-field scheme, sph_surface_* through the C ABI)
against the reference's detectFreeSurface (golden vectors) and the oracle."""
import types
from pathlib import Path

import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle import oracle
from tests.cases import assert_close, make_params, make_particles
from warpsph_b200 import core, ops, surface
from warpsph_b200.configurations import NormalSource, SurfaceDetectionConfig
from warpsph_b200.core import AdjacencyList

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "surface_golden.npz"


def test_detect_free_surface_matches_reference(cuda):
    g = dict(np.load(GOLD))
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in g.items()}
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4, periodic=False)
    cfg.targetNeighbors = float(g["surface_target_neighbors"][0])
    n = len(g["H"])
    fixture = AdjacencyList(neighborOffsets=t["offsets"], numNeighbors=t["counts"], neighborList=t["list"], numRows=n, numCols=n,
                            nnz=int(g["list"].shape[0]))
    built = ops.buildVerletList(t["x"], t["H"], p, float(p.verlet_scale))
    state = types.SimpleNamespace(positions=t["x"], supports=t["H"], masses=t["m"], densities=t["rho"])
    for adj in (fixture, built):
        c = ops.surface_color_field(p, t["x"], t["H"], t["m"], t["rho"], adj)
        assert_close(c.cpu().numpy(), g["surface_color"], 1e-5, 1e-6, "colour field (GPU)")
        fsm, normals, nn = ops.surface_detect_color_field(p, t["x"], t["H"], t["m"], t["rho"], t["surface_color"], adj,
                                                          cfg.targetNeighbors * 0.75, -1.0)
        assert np.array_equal(nn.cpu().numpy(), g["surface_num_neighbors"]), "neighbour counts (GPU)"
        assert np.array_equal(fsm.cpu().numpy(), g["surface_fsm"]), "surface mask (GPU)"
        assert_close(normals.cpu().numpy(), g["surface_normals"], 1e-4, 1e-5, "normals (GPU)")
        fs = ops.surface_dilate(p, t["x"], t["H"], t["surface_fsm"], adj)
        assert np.array_equal(fs.cpu().numpy(), g["surface_fs"]), "dilation (GPU)"
        for _ in (0,):
            r = surface.detectFreeSurface(state, cfg, None, SurfaceDetectionConfig(), adj)
            assert np.array_equal(r[0].cpu().numpy(), g["surface_fsm"]) and np.array_equal(r[1].cpu().numpy(), g["surface_fs"])
            assert_close(r[2].cpu().numpy(), g["surface_normals"], 1e-4, 1e-5, "detectFreeSurface normals")
            r = surface.detectFreeSurface(state, cfg, None, SurfaceDetectionConfig(normalSource=NormalSource.Native), adj)
            assert_close(r[2].cpu().numpy(), -g["surface_normals"], 1e-4, 1e-5, "native normals (+ grad c)")


@pytest.mark.parametrize("dim,n_side", [(1, 300), (2, 40), (3, 14)])
def test_surface_passes_vs_oracle(cuda, dim, n_side):
    """A non-periodic block in each dimension: GPU passes against the FP64 oracle."""
    cfg, sch, p = make_params(dim, periodic=False)
    P = make_particles(dim, n_side, periodic=False, seed=4)
    G = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in P.items()}
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    nb = dict(offsets=adj.neighborOffsets.cpu().numpy(), counts=adj.numNeighbors.cpu().numpy(),
              list=adj.neighborList.cpu().numpy())
    rho = ops.density(p, G["positions"], G["supports"], G["masses"], adj, core.SupportScheme.Gather)
    o = oracle.get("f64")
    c = ops.surface_color_field(p, G["positions"], G["supports"], G["masses"], rho, adj)
    rc = o.surface_color_field(p, P["positions"], P["supports"], P["masses"], rho.cpu().numpy(), nb)
    assert_close(c.cpu().numpy(), rc, 2e-6, 2e-6, f"colour field {dim}D")
    limit = float(cfg.targetNeighbors) * 0.75
    fsm, normals, nn = ops.surface_detect_color_field(p, G["positions"], G["supports"], G["masses"], rho, c, adj, limit)
    rf, rn, rnn = o.surface_detect(p, P["positions"], P["supports"], P["masses"], rho.cpu().numpy(), c.cpu().numpy(), nb, limit)
    assert np.array_equal(nn.cpu().numpy(), rnn), f"neighbour counts {dim}D"
    assert np.array_equal(fsm.cpu().numpy(), rf), f"mask {dim}D"
    assert_close(normals.cpu().numpy(), rn, 1e-4, 1e-5, f"normals {dim}D")
    assert 0 < rf.sum() < len(rf)
    fs = ops.surface_dilate(p, G["positions"], G["supports"], fsm, adj)
    assert np.array_equal(fs.cpu().numpy(), o.surface_dilate(p, P["positions"], P["supports"], rf, nb)), f"dilation {dim}D"
