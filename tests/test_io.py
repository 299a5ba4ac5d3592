"""Export and import with the reference's layout (src/warpSPH/io.py): a round trip of a
CRKSPH system with its adjacency, two stages and every kind of extra data, on CPU
tensors (the adjacency's expanded i/j arrays are given, so no kernel runs).  The GPU
resume test (a resumed run equal to an uninterrupted one bit for bit) is in
test_gpu_io.py."""
import json

import numpy as np
import torch

import warpsph_b200 as ws
from warpsph_b200 import io
from warpsph_b200.core import AdjacencyList
from warpsph_b200.integrators import StageRecord
from warpsph_b200.systems import CompressibleSystemUpdate, CompSPHState, CompSPHSystem


def make_state(n, rng):
    f = lambda *s: torch.from_numpy(rng.standard_normal(s).astype(np.float32))
    return CompSPHState(positions=f(n, 2), velocities=f(n, 2), supports=f(n).abs(), masses=f(n).abs(), densities=f(n).abs(),
                        kinds=torch.zeros(n, dtype=torch.int32), UIDs=torch.arange(n, dtype=torch.int32), UIDcounter=n,
                        internalEnergies=f(n).abs(), pressures=f(n), alphas=None, ap_ij=f(3 * n, 2))


def make_adjacency(n, rng):
    cnt = torch.from_numpy(rng.integers(1, 5, n).astype(np.int32))
    offs = torch.cumsum(cnt, 0).to(torch.int32) - cnt
    nnz = int(cnt.sum())
    lst = torch.from_numpy(rng.integers(0, n, nnz).astype(np.int32))
    adj = AdjacencyList(neighborOffsets=offs, numNeighbors=cnt, neighborList=lst, numRows=n, numCols=n, nnz=nnz,
                        queryPositions=torch.zeros(n, 2), querySupports=torch.ones(n), verletScale=1.4142,
                        interCounts=torch.minimum(cnt, torch.full_like(cnt, 2)))
    adj._ij = (torch.repeat_interleave(torch.arange(n), cnt.long()), lst.long())
    adj._x0, adj._h0, adj._dim = torch.zeros(n, 2), torch.ones(n), 2
    return adj


def test_export_import_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    n = 40
    S, adj = make_state(n, rng), make_adjacency(n, rng)
    system = CompSPHSystem(state=S, adjacency=adj, t=0.125)
    stages = []
    for k in range(2):
        upd = CompressibleSystemUpdate(dxdt=torch.randn(n, 2), dvdt=torch.randn(n, 2), dudt=torch.randn(n))
        stages.append(StageRecord(update=upd, aux=(adj, make_state(n, rng), (torch.zeros(3), torch.zeros(3)))))
    extra = {"kineticEnergy": torch.tensor(1.5), "frame_num": 7, "name": "sod", "d": {"a": torch.arange(3), "b": 2.5},
             "l": [torch.ones(2), {"x": torch.zeros(1), "y": 3}, 4.0]}
    path = io.exportSimulationSystem(str(tmp_path), "state_0003", ws.CompressibleSPHScheme.CRKSPH, system, stages=stages,
                                     extraData=extra)
    assert path.endswith("/trajectory/state_0003.npz")
    z = np.load(path)
    assert {"state/positions", "adjacency/i", "adjacency/j", "adjacency/numNeighbors", "adjacency/edgeOffsets",
            "stages/stage_1/dvdt", "stages/stage_0/aux/1_state/densities", "stages/stage_0/aux/0_adjacency/j"} <= set(z.files)
    attrs = json.loads(str(z["__attrs__"]))
    assert attrs[""]["scheme"] == "CRKSPH" and attrs[""]["time"] == 0.125 and attrs["state/"]["alphas"] == "None"
    sys2, st2, scheme, ex2 = io.importSimulationSystem(path, torch.device("cpu"))
    assert scheme == ws.CompressibleSPHScheme.CRKSPH and sys2.t == 0.125
    for name in ("positions", "velocities", "supports", "masses", "densities", "kinds", "UIDs", "internalEnergies", "pressures",
                 "ap_ij"):
        a, b = getattr(S, name), getattr(sys2.state, name)
        assert a.dtype == b.dtype and torch.equal(a, b), name
    assert sys2.state.alphas is None and sys2.state.UIDcounter == n
    a2 = sys2.adjacency
    assert torch.equal(a2.neighborList, adj.neighborList) and torch.equal(a2.numNeighbors, adj.numNeighbors)
    assert torch.equal(a2.neighborOffsets, adj.neighborOffsets) and torch.equal(a2.interCounts, adj.interCounts)
    assert torch.equal(a2._x0, adj._x0) and a2.verletScale == adj.verletScale and a2.numRows == n
    assert len(st2) == 2 and torch.equal(st2[1].update.dvdt, stages[1].update.dvdt)
    assert isinstance(st2[0].aux[0], AdjacencyList) and torch.equal(st2[0].aux[1].densities, stages[0].aux[1].densities)
    assert float(ex2["kineticEnergy"]) == 1.5 and ex2["frame_num"] == 7 and ex2["name"] == "sod"
    assert torch.equal(ex2["d"]["a"], torch.arange(3)) and ex2["d"]["b"] == 2.5
    assert torch.equal(ex2["l"][0], torch.ones(2)) and ex2["l"][1]["y"] == 3 and ex2["l"][2] == 4.0


def test_prep_export_and_import_configs(tmp_path):
    cfg, _ = ws.buildConfig(device=torch.device("cpu"), dim=1)
    sch = ws.CRKSPHConfig()
    sch.gamma = 1.4
    path = io.prepExport("case", cfg, sch, ws.CompressibleSPHScheme.CRKSPH, ws.crkSPHConfigToDict, exportRoot=str(tmp_path))
    cfg2, sch2 = io.importConfigs(f"{path}/config.json", ws.dictToCRKSPHConfig)
    assert cfg2.dim == 1 and sch2.gamma == 1.4 and cfg2.kernel == cfg.kernel
