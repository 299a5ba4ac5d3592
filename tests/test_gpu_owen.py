"""The Owen adaptive support on the GPU: sph_owen_iter against the reference's own psi0
pair body, table lookup and update (golden vectors) and against the oracle; the full
evaluateOptimalSupport with the Owen scheme; a CRKSPH step with Owen supports against the
oracle's step."""
from pathlib import Path

import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from oracle import oracle
from oracle.steps import CRKSPHOracle, SWITCH_CULLEN, cell_capacity_for, state_to_numpy
from tests.cases import assert_close, make_params, make_particles
from warpsph_b200 import ops
from warpsph_b200.core import AdjacencyList
from warpsph_b200.enumTypes import AdaptiveSupportScheme
from warpsph_b200.owen import owen_table

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "owen_golden.npz"


def test_owen_iter_matches_reference_and_oracle(cuda):
    g = dict(np.load(GOLD))
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    nh, psiH = owen_table(ws.KernelFunctions.Wendland4, 2)
    t = {k: torch.from_numpy(np.ascontiguousarray(g[k])).to(cuda) for k in ("owen_x", "owen_H", "owen_offsets", "owen_counts", "owen_list")}
    n = len(g["owen_H"])
    adj = AdjacencyList(neighborOffsets=t["owen_offsets"], numNeighbors=t["owen_counts"], neighborList=t["owen_list"], numRows=n,
                        numCols=n, nnz=int(g["owen_list"].shape[0]))
    hb = ops.minmax(t["owen_H"])
    psiH_t, Hn, ratio, psi0 = ops.owen_iter(p, t["owen_x"], t["owen_H"], adj, torch.from_numpy(nh).to(cuda),
                                            torch.from_numpy(psiH).to(cuda), float(g["owen_target"][0]), hb, want_psi0=True)
    assert_close(psi0.cpu().numpy(), g["owen_psi0"], 1e-5, 1e-6, "psi0 vs reference (GPU)")
    assert_close(psiH_t.cpu().numpy(), g["owen_psi0H"], 1e-5, 1e-6, "psi0_H vs reference (GPU)")
    assert_close(Hn.cpu().numpy(), g["owen_Hnew"], 1e-5, 1e-6, "new support vs reference (GPU)")
    # larger case, the library's own list, against the oracle
    P = make_particles(2, 48, seed=31, jitter=0.4, h_spread=0.2)
    x, H = P["positions"], P["supports"]
    nb = oracle.get("f32").neighbors(p, x, H, cell_capacity_for(len(H), 2))
    xg, Hg = torch.from_numpy(x).to(cuda), torch.from_numpy(H).to(cuda)
    adj = ops.buildVerletList(xg, Hg, p, p.verlet_scale)
    target = ws.core.nH_to_n_h(p.target_neighbors, 2)
    psiH_t, Hn, ratio = ops.owen_iter(p, xg, Hg, adj, torch.from_numpy(nh).to(cuda), torch.from_numpy(psiH).to(cuda), target,
                                      ops.minmax(Hg))
    _, rpsiH, rHn, rratio = oracle.get("f32").owen_iter(p, x, H, nb, nh, psiH, target, np.array([H.min(), H.max()], np.float32))
    assert_close(psiH_t.cpu().numpy(), rpsiH, 1e-5, 1e-6, "psi0_H vs oracle")
    assert_close(Hn.cpu().numpy(), rHn, 1e-5, 1e-6, "new support vs oracle")


def sedov_owen(nx, dev, iterations=1):
    cfg, integ = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                targetNeighbors=32, integrationScheme=ws.IntegrationSchemeType.rungeKutta2, device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    sch.adaptiveSupportScheme = AdaptiveSupportScheme.Owen
    sch.adaptiveSupportIterations = iterations
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=2, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=32, device=dev)
    return cfg, sch, integ, step, system


def test_owen_converges_to_target_neighbour_count(cuda):
    """16 Owen iterations on a jittered lattice: the supports stop moving and the kernel
    sum stays at the lattice density (the n_h(psi_H) table is that of a regular lattice)."""
    cfg, sch, integ, step, system = sedov_owen(40, cuda, iterations=16)
    S = system.state
    S.positions = (S.positions + 0.1 * (cfg.dx ** 0.5) * (torch.rand_like(S.positions) - 0.5)).contiguous()
    rho, H, adj, psis, hs = ws.schemes.evaluateOptimalSupport(S, cfg, sch, ws.SupportScheme.Gather, None)
    assert len(hs) >= 3
    last = (hs[-1] / hs[-2] - 1).abs().max().item()
    first = (hs[1] / hs[0] - 1).abs().max().item()
    assert last < 2e-3 and last < first
    assert abs(float(rho.mean()) - 1.0) < 5e-3


def test_crksph_step_with_owen_supports_matches_oracle(cuda):
    cfg, sch, integ, step, system = sedov_owen(32, cuda, iterations=2)
    dt = 2e-4
    st = state_to_numpy(system.state)
    nh, psiH = owen_table(ws.KernelFunctions.Wendland4, 2)
    orc = CRKSPHOracle(ws.make_params(cfg, sch), "f32", switch=SWITCH_CULLEN, adaptive_iterations=2, owen_table=(nh, psiH))
    for k in range(2):
        system = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch).state
        st, _, _ = orc.step(st, dt, "rungeKutta2")
        S = system.state
        assert_close(S.supports.cpu().numpy(), st["supports"], 1e-5, 1e-5, f"H step {k}")
        assert_close(S.densities.cpu().numpy(), st["densities"], 1e-5, 1e-5, f"rho step {k}")
        assert_close(S.velocities.cpu().numpy(), st["velocities"], 5e-4, 5e-4, f"v step {k}")
        assert_close(S.internalEnergies.cpu().numpy(), st["internalEnergies"], 5e-4, 5e-4, f"u step {k}")
