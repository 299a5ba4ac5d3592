"""The delta-SPH right-hand side and the batched ensemble on the GPU against the CPU
oracle.

The single right-hand side is compared with the FP32 oracle at 1e-4 of each field's
scale.  FMA contraction and summation order are the only differences, but the EOS
pressure multiplies density differences by c0^2 rho0 / gamma.

Ensemble checks:
  * lists: compared per box, row by row as sets, against the oracle's search on each
    box alone;
  * steps: compared after two Heun steps against the oracle stepping each box with its
    own lists, at 1e-3 of scale;
  * graph: replaying a captured CUDA graph is bit-identical to the same launches issued
    one by one."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200 import core, ops
from warpsph_b200.configurations import WeaklyCompressibleSPHConfig, wc_params
from warpsph_b200.ensemble import TILE_CANDIDATES, BoxSet, Ensemble

pytestmark = pytest.mark.gpu


def small_ensemble(cuda, sizes=(576, 784, 1024), graph_steps=4):
    return Ensemble(BoxSet(list(sizes), [11, 12, 13][: len(sizes)]), cuda, target_neighbors=core.n_h_to_nH(4, 2),
                    graph_steps=graph_steps)


def box_slice(E, b):
    return slice(int(E.seg[b]), int(E.seg[b + 1]))


def test_deltasph_rhs_matches_oracle(cuda):
    E = small_ensemble(cuda, sizes=(576,))
    p = E.params
    wc = E.wc
    x, H, m, v = (t.cpu().numpy() for t in (E.x, E.H, E.m, E.v))
    rng = np.random.default_rng(0)
    rho = (1.0 + 0.01 * rng.standard_normal(len(H))).astype(np.float32)
    o = oracle.get("f32")
    nb = o.neighbors(p, x, H, 1 << 14)
    adj = core.AdjacencyList(neighborOffsets=torch.from_numpy(nb["offsets"]).to(cuda), numNeighbors=torch.from_numpy(nb["counts"]).to(cuda),
                             neighborList=torch.from_numpy(nb["list"]).to(cuda), numRows=len(H), numCols=len(H), nnz=int(nb["nnz"]))
    dv, dr, gL, P = ops.deltasph_rhs(p, wc, E.x, E.H, E.m, torch.from_numpy(rho).to(cuda), E.v, adj)
    rdv, rdr, rgL, rP = o.deltasph_rhs(p, wc, x, H, m, rho, v, nb)
    assert_close(P.cpu().numpy(), rP, 1e-5, 1e-5, "stiff Tait pressure")
    assert_close(gL.cpu().numpy(), rgL, 1e-4, 1e-4, "renormalised density gradient")
    assert_close(dr.cpu().numpy(), rdr, 1e-4, 1e-4, "drho/dt")
    assert_close(dv.cpu().numpy(), rdv, 1e-4, 1e-4, "dv/dt")
    assert np.abs(rdv).max() > 0 and np.abs(rdr).max() > 0


def test_ensemble_lists_per_box(cuda):
    E = small_ensemble(cuda)
    offs, cnt, lst = (t.cpu().numpy() for t in (E.offs, E.cnt, E.list[: E.nnz]))
    o = oracle.get("f32")
    for b in range(len(E.sizes)):
        sl = box_slice(E, b)
        x, H = E.x[sl].cpu().numpy(), E.H[sl].cpu().numpy()
        nb = o.neighbors(E.params, x, H, 1 << 14)
        for i in range(len(H)):
            gi = sl.start + i
            row = lst[offs[gi]: offs[gi] + cnt[gi]]
            assert row.min() >= sl.start and row.max() < sl.stop, "a row crosses boxes"
            ref = nb["list"][nb["offsets"][i]: nb["offsets"][i] + nb["counts"][i]] + sl.start
            assert set(row.tolist()) == set(ref.tolist()), (b, i)


def test_ensemble_step_matches_oracle(cuda):
    E = small_ensemble(cuda)
    o = oracle.get("f32")
    states = []
    for b in range(len(E.sizes)):
        sl = box_slice(E, b)
        states.append({k: t[sl].cpu().numpy().copy() for k, t in dict(x=E.x, v=E.v, rho=E.rho, H=E.H, m=E.m).items()})
    dts = E.box_dt.cpu().numpy()
    E._launch()                            # exactly two steps (advance() works in whole chunks)
    E._launch()

    def wrap(x):
        return ((x + 0.5) % 1.0 - 0.5).astype(np.float32)

    for b, s in enumerate(states):
        dt = np.float32(dts[b])
        x0, v0, r0 = s["x"], s["v"], s["rho"]
        for _ in range(2):
            nb = o.neighbors(E.params, x0, s["H"], 1 << 14)
            k1v, k1r, _, _ = o.deltasph_rhs(E.params, E.wc, x0, s["H"], s["m"], r0, v0, nb)
            x1, v1, r1 = wrap(x0 + dt * v0), (v0 + dt * k1v).astype(np.float32), (r0 + dt * k1r).astype(np.float32)
            nb1 = o.neighbors(E.params, x1, s["H"], 1 << 14)
            k2v, k2r, _, _ = o.deltasph_rhs(E.params, E.wc, x1, s["H"], s["m"], r1, v1, nb1)
            h = np.float32(0.5) * dt
            x0 = wrap(x0 + h * (v0 + v1))
            v0 = (v0 + h * (k1v + k2v)).astype(np.float32)
            r0 = (r0 + h * (k1r + k2r)).astype(np.float32)
        sl = box_slice(E, b)
        d = E.x[sl].cpu().numpy() - x0
        assert np.abs(d - np.round(d)).max() < 1e-6, b
        assert_close(E.v[sl].cpu().numpy(), v0, 1e-3, 1e-3, f"v box {b}")
        assert_close(E.rho[sl].cpu().numpy(), r0, 1e-5, 1e-5, f"rho box {b}")
    assert E.status() == 0


def test_graph_replay_bit_identical_to_eager(cuda):
    A = small_ensemble(cuda, graph_steps=4)
    B = small_ensemble(cuda, graph_steps=4)
    A.advance(13, use_graph=True)          # capture (1 step) + 3 replays of 4 steps
    B.advance(13, use_graph=False)
    assert A.steps_done == B.steps_done == 13
    assert torch.equal(A.x, B.x) and torch.equal(A.v, B.v) and torch.equal(A.rho, B.rho)
    assert A.rebuilds == B.rebuilds
    assert A.status() == 0 and B.status() == 0


def test_autotune_chooses_a_measured_candidate(cuda):
    E = small_ensemble(cuda)
    x0 = E.x.clone()
    res = E.autotune(steps=1)
    assert set(res) == set(TILE_CANDIDATES) and E.tile in res and all(t > 0 for t in res.values())
    assert torch.equal(E.x, x0)             # the state is untouched
    # every candidate gives the same step
    outs = []
    for tile in TILE_CANDIDATES:
        x, v, r = E.x.clone(), E.v.clone(), E.rho.clone()
        E._launch(tile, x, v, r)
        outs.append((x, v, r))
    for x, v, r in outs[1:]:
        assert_close(v.cpu().numpy(), outs[0][1].cpu().numpy(), 1e-5, 1e-5, "v across tile shapes")
