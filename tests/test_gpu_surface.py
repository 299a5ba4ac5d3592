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


def test_barecasco_maronne_colour_gradient_match_reference(cuda):
    """sph_surface_barecasco, sph_surface_maronne and sph_surface_detect_color_gradient against
    the reference's own bodies (surface_schemes_golden.npz): masks and counts exactly,
    directions to 2e-3 (near-zero cover vectors); and detectFreeSurface with each scheme."""
    g = dict(np.load(GOLD))
    s = dict(np.load(GOLD.parent / "surface_schemes_golden.npz"))
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in g.items()}
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4, periodic=False)
    cfg.targetNeighbors = float(g["surface_target_neighbors"][0])
    n = len(g["H"])
    fixture = AdjacencyList(neighborOffsets=t["offsets"], numNeighbors=t["counts"], neighborList=t["list"], numRows=n, numCols=n,
                            nnz=int(g["list"].shape[0]))
    built = ops.buildVerletList(t["x"], t["H"], p, float(p.verlet_scale))
    state = types.SimpleNamespace(positions=t["x"], supports=t["H"], masses=t["m"], densities=t["rho"])
    from warpsph_b200.configurations import SurfaceDetectionScheme
    for adj in (fixture, built):
        for tag in ("pi3", "1p5"):
            fs, nrm, cnt = ops.surface_barecasco(p, t["x"], t["H"], adj, float(s[f"barecasco_{tag}_threshold"][0]))
            assert np.array_equal(cnt.cpu().numpy(), s[f"barecasco_{tag}_count"]), f"Barecasco counts {tag}"
            assert np.array_equal(fs.cpu().numpy(), s[f"barecasco_{tag}_fsm"]), f"Barecasco mask {tag}"
            # an interior particle's near-zero cover vector points wherever the rounding of
            # its sum says: directions to 2e-3 (the counts and the mask above are exact)
            assert_close(nrm.cpu().numpy(), s[f"barecasco_{tag}_normals"], 0.0, 2e-3, f"Barecasco directions {tag}")
        for tag in ("colour", "cover"):
            nr = torch.from_numpy(s[f"maronne_{tag}_normals"]).to(cuda)
            fs, cnt = ops.surface_maronne(p, t["x"], t["H"], nr, adj)
            assert np.array_equal(cnt.cpu().numpy(), s[f"maronne_{tag}_count"]), f"Maronne counts {tag}"
            assert np.array_equal(fs.cpu().numpy(), s[f"maronne_{tag}_fsm"]), f"Maronne mask {tag}"
        fs, nrm = ops.surface_detect_color_gradient(p, t["x"], t["H"], t["m"], t["rho"], t["surface_color"], adj,
                                                    float(s["cfgrad_threshold"][0]))
        assert np.array_equal(fs.cpu().numpy(), s["cfgrad_fsm"]), "colour-gradient mask"
        assert_close(nrm.cpu().numpy(), s["cfgrad_normals"], 1e-4, 1e-5, "colour-gradient normals")
        # the scheme dispatch: Barecasco with its own directions, the colour-field-gradient scheme
        sd = SurfaceDetectionConfig(scheme=SurfaceDetectionScheme.Barecasco, normalSource=NormalSource.Native,
                                    barecascoThreshold=float(s["barecasco_pi3_threshold"][0]))
        r = surface.detectFreeSurface(state, cfg, None, sd, adj)
        assert np.array_equal(r[0].cpu().numpy(), s["barecasco_pi3_fsm"])
        assert_close(r[2].cpu().numpy(), s["barecasco_pi3_normals"], 0.0, 2e-3, "detectFreeSurface Barecasco normals")
        sd = SurfaceDetectionConfig(scheme=SurfaceDetectionScheme.ColorFieldGrad)
        r = surface.detectFreeSurface(state, cfg, None, sd, adj)
        assert np.array_equal(r[0].cpu().numpy(), s["cfgrad_fsm"])
        assert_close(r[2].cpu().numpy(), s["cfgrad_normals"], 1e-4, 1e-5, "detectFreeSurface colour-gradient normals")


@pytest.mark.parametrize("dim,n_side", [(2, 40), (3, 14)])
def test_renormalization_and_normal_sources_vs_oracle(cuda, dim, n_side):
    """The restated renormalisation on a non-periodic block: L against LAPACK's pinv and the
    smallest |eigenvalue| against eigvalsh (FP64 oracle sums), the lambda-gradient and Maronne
    normals, and the Maronne scheme through detectFreeSurface with each normal source."""
    cfg, sch, p = make_params(dim, periodic=False)
    P = make_particles(dim, n_side, periodic=False, seed=4)
    G = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in P.items()}
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    nb = dict(offsets=adj.neighborOffsets.cpu().numpy(), counts=adj.numNeighbors.cpu().numpy(),
              list=adj.neighborList.cpu().numpy())
    rho = ops.density(p, G["positions"], G["supports"], G["masses"], adj, core.SupportScheme.Gather)
    rn = rho.cpu().numpy()
    o = oracle.get("f64")
    L, lam = ops.surface_renormalization(p, G["positions"], G["supports"], G["masses"], rho, adj)
    rL, rlam, rM = o.surface_renormalization(p, P["positions"], P["supports"], P["masses"], rn, nb)
    assert_close(L.cpu().numpy(), rL, 1e-4, 1e-5, f"L {dim}D")
    assert_close(lam.cpu().numpy(), rlam, 1e-4, 1e-5, f"lambda {dim}D")
    for mode in (0, 1):
        nrm, gr = ops.surface_renormalized_normals(p, mode, G["positions"], G["supports"], G["masses"], rho, L, lam, adj,
                                                   want_grad=True)
        rnrm, rgr = o.surface_renorm_normals(p, mode, P["positions"], P["supports"], P["masses"], rn, L.cpu().numpy(),
                                             lam.cpu().numpy(), nb)
        assert_close(gr.cpu().numpy(), rgr, 1e-4, 1e-5, f"renormalised gradient mode {mode} {dim}D")
        # directions of weak gradients (interior particles) carry the rounding of their sums
        strong = np.linalg.norm(rgr, axis=1) > 1e-2 * np.abs(rgr).max()
        assert_close(nrm.cpu().numpy()[strong], rnrm[strong], 1e-3, 1e-4, f"normals mode {mode} {dim}D")
        fs, cnt = ops.surface_maronne(p, G["positions"], G["supports"], nrm, adj)
        rfs, rcnt = o.surface_maronne(p, P["positions"], P["supports"], nrm.cpu().numpy(), nb)
        assert np.array_equal(cnt.cpu().numpy(), rcnt) and np.array_equal(fs.cpu().numpy(), rfs), f"Maronne mode {mode} {dim}D"
        assert 0 < rfs.sum() < len(rfs)
    from warpsph_b200.configurations import SurfaceDetectionScheme
    state = types.SimpleNamespace(positions=G["positions"], supports=G["supports"], masses=G["masses"], densities=rho)
    for src, mode in ((NormalSource.LambdaGrad, 0), (NormalSource.Maronne, 1)):
        sd = SurfaceDetectionConfig(scheme=SurfaceDetectionScheme.Maronne, normalSource=src)
        fsm, fs, nrm, Lr, lamr = surface.detectFreeSurface(state, cfg, None, sd, adj)
        want, _ = ops.surface_renormalized_normals(p, mode, G["positions"], G["supports"], G["masses"], rho, L, lam, adj,
                                                   want_grad=True)
        assert torch.equal(nrm, want) and torch.equal(Lr, L) and torch.equal(lamr, lam)
        wfs, _ = ops.surface_maronne(p, G["positions"], G["supports"], want, adj)
        assert torch.equal(fsm, wfs)
