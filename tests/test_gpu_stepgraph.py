"""Device-decided neighbour lists (sph_neighbors_update / sph_neighbors_rewrite) and
whole steps recorded as CUDA graphs (warpsph_b200.stepgraph).

* the interacting rows of a device-decided list equal those of a fresh build, for a
  kept list (particles still inside the Verlet skin) and for a rebuilt one;
* Sedov CRKSPH steps with device-decided lists follow the ordinary eager steps;
* replayed graph steps equal eager steps with device-decided lists;
* a rebuild that overflows the list is reported by check() and stays in bounds."""
import numpy as np
import pytest
import torch

import warpsph_b200 as ws
from warpsph_b200 import ops
from warpsph_b200.stepgraph import StepGraph
from tests.cases import assert_close

pytestmark = pytest.mark.gpu


def sedov(nx, dev, scheme="crkSPH"):
    cfg, integrator = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                     targetNeighbors=32, integrationScheme=ws.IntegrationSchemeType.rungeKutta2, cflFactor=0.3,
                                     device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme(scheme)
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=2, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=32, device=dev)
    return cfg, sch, integrator, step, system


def wrap(x):
    """Positions wrapped into the periodic unit box [-0.5, 0.5)^2."""
    return torch.remainder(x + 0.5, 1.0) - 0.5


def interacting_pairs(adj, n):
    """Sorted i * n + j codes of the interacting prefixes of `adj`'s rows."""
    offs = adj.neighborOffsets.cpu().numpy().astype(np.int64)
    icnt = adj.interCounts.cpu().numpy().astype(np.int64)
    lst = adj.neighborList.cpu().numpy().astype(np.int64)
    rows = np.repeat(np.arange(n), icnt)
    pos = np.concatenate([np.arange(o, o + c) for o, c in zip(offs, icnt)]) if n else np.zeros(0, np.int64)
    return np.sort(rows * n + lst[pos])


def fresh_pairs(x, H, params, vs, n):
    with ops._suspend_device_lists():
        adj = ops.buildVerletList(x, H, params, vs, None)
    return interacting_pairs(adj, n)


def device_pairs(nb, x, H, params):
    adj = nb.update(x, H, params)
    ops._lists(params, adj, True)     # the rewrite, on first use of the interacting rows
    return interacting_pairs(adj, nb.n), adj


@pytest.fixture(autouse=True)
def _fresh_lists():
    ops.release_device_lists()
    yield
    ops.release_device_lists()


def test_device_lists_kept_and_rebuilt(cuda):
    cfg, sch, _, _, system = sedov(64, cuda)
    params = ws.make_params(cfg, sch)
    S = system.state
    n = S.positions.shape[0]
    x, H = S.positions.clone(), S.supports.clone()
    nb = ops.device_lists_for(x, H, params, cfg.verletScale)
    got, _ = device_pairs(nb, x, H, params)
    assert np.array_equal(got, fresh_pairs(x, H, params, cfg.verletScale, n))
    x0_first = nb.x0.clone()
    # a small move keeps the rows (the build-time positions stay), the interacting rows follow
    g = torch.Generator(device=cuda).manual_seed(3)
    skin = float((cfg.verletScale - 1.0) * H.min())
    x2 = wrap(x + 0.05 * skin * (torch.rand(x.shape, generator=g, device=cuda) - 0.5))
    got, _ = device_pairs(nb, x2, H, params)
    assert torch.equal(nb.x0, x0_first), "a move well inside the skin must keep the rows"
    assert np.array_equal(got, fresh_pairs(x2, H, params, cfg.verletScale, n))
    # a move across the skin rebuilds them
    x3 = wrap(x + 4.0 * skin * (torch.rand(x.shape, generator=g, device=cuda) - 0.5))
    got, _ = device_pairs(nb, x3, H, params)
    assert torch.equal(nb.x0, x3), "a move across the skin must rebuild the rows"
    assert np.array_equal(got, fresh_pairs(x3, H, params, cfg.verletScale, n))
    nb.check()


def test_device_list_steps_follow_eager(cuda):
    dt = 2e-4
    cfg, sch, integ, step, sys_a = sedov(48, cuda)
    *_, sys_b = sedov(48, cuda)
    for _ in range(6):
        sys_a = integ.function(state=sys_a, f=step, dt=dt, config=cfg, compParams=sch).state
    with ops.device_decided_lists():
        for _ in range(6):
            sys_b = integ.function(state=sys_b, f=step, dt=dt, config=cfg, compParams=sch).state
    A, B = sys_a.state, sys_b.state
    assert sys_b.adjacency._device_rows
    for name, tol in (("positions", 1e-6), ("velocities", 2e-4), ("internalEnergies", 2e-4), ("densities", 1e-5), ("supports", 1e-5)):
        assert_close(getattr(B, name).cpu().numpy(), getattr(A, name).cpu().numpy(), tol, tol, name)
    for nb in ops._device_lists.values():
        nb.check()


@pytest.mark.parametrize("scheme", ["crkSPH", "compSPH"])
def test_graph_replay_equals_eager_steps(cuda, scheme):
    warm, steps = 3, 5
    cfg, sch, integ, step, sys_a = sedov(48, cuda, scheme)
    *_, sys_b = sedov(48, cuda, scheme)
    dt0 = torch.tensor([cfg.dt], device=cuda, dtype=torch.float32)
    sg = StepGraph(sys_a, integ, step, cfg, sch, dt=dt0, warmup=warm)
    assert sg.launches_per_step > 20
    sg.replay(steps)
    torch.cuda.synchronize()
    sg.check()
    A = sg.system.state
    assert torch.equal(A.positions, sg.inputs.state.positions), "the graph copies its result into its inputs"
    ops.release_device_lists()
    params = ws.make_params(cfg, sch)
    dt = dt0.clone()
    with ops.device_decided_lists():
        for _ in range(warm + steps):
            dt = ops.cfl_dt(params, sys_b.state.supports, sys_b.state.internalEnergies, dt_prev=dt)
            sys_b = integ.function(state=sys_b, f=step, dt=dt, config=cfg, compParams=sch).state
    B = sys_b.state
    assert torch.equal(sg.dt, dt) or abs(float(sg.dt) - float(dt)) <= 1e-6 * abs(float(dt))
    for name in ("positions", "velocities", "internalEnergies", "densities", "supports", "alphas"):
        assert_close(getattr(A, name).cpu().numpy(), getattr(B, name).cpu().numpy(), 1e-5, 1e-6, name)
    sg.release()


def test_device_list_overflow_reported(cuda):
    cfg, sch, _, _, system = sedov(64, cuda)
    params = ws.make_params(cfg, sch)
    S = system.state
    old = ops.DEVICE_LIST_HEADROOM
    ops.DEVICE_LIST_HEADROOM = 0.3
    try:
        nb = ops.device_lists_for(S.positions, S.supports, params, cfg.verletScale)
        adj = nb.update(S.positions, S.supports, params)
        ops._lists(params, adj, True)
        torch.cuda.synchronize()
        cnt = adj.numNeighbors.long()
        end = adj.neighborOffsets.long() + cnt
        assert bool(((end <= nb.capacity) | (cnt == 0)).all()), "rows are cut to the list"
        assert int(cnt.sum()) <= nb.capacity
        with pytest.raises(RuntimeError, match="more than"):
            nb.check()
    finally:
        ops.DEVICE_LIST_HEADROOM = old


def test_recorded_update_rebuilds_only_when_stale(cuda):
    """sph_neighbors_update recorded in a CUDA graph (the rebuild is a conditional node):
    a replay after a move across the skin rebuilds the rows, one after a small move keeps
    them, and the rewritten interacting rows equal a fresh build's in both cases."""
    cfg, sch, _, _, system = sedov(64, cuda)
    params = ws.make_params(cfg, sch)
    S = system.state
    n = S.positions.shape[0]
    x, H = S.positions.clone(), S.supports.clone()
    nb = ops.device_lists_for(x, H, params, cfg.verletScale)
    device_pairs(nb, x, H, params)                      # the first call (outside a recording) builds
    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):
        device_pairs(nb, x, H, params)
    torch.cuda.current_stream(cuda).wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        adj = nb.update(x, H, params)
        ops._lists(params, adj, True)
    gen = torch.Generator(device=cuda).manual_seed(5)
    skin = float((cfg.verletScale - 1.0) * H.min())
    for scale, rebuilt in ((4.0, True), (0.05, False), (4.0, True)):
        x_prev0 = nb.x0.clone()
        x.copy_(wrap(x + scale * skin * (torch.rand(x.shape, generator=gen, device=cuda) - 0.5)))
        g.replay()
        torch.cuda.synchronize()
        if rebuilt:
            assert torch.equal(nb.x0, x), "a replay after a move across the skin must rebuild"
        else:
            assert torch.equal(nb.x0, x_prev0), "a replay after a small move must keep the rows"
        assert np.array_equal(interacting_pairs(adj, n), fresh_pairs(x, H, params, cfg.verletScale, n))
    nb.check()


def _graph_vs_device_eager(cuda, cfg, sch, integ, step, sys_a, sys_b, warm, steps, rtol, atol):
    """Replays of a recorded step against the same steps issued eagerly with device-decided
    lists, from the same initial state."""
    dt0 = torch.tensor([cfg.dt], device=cuda, dtype=torch.float32)
    sg = StepGraph(sys_a, integ, step, cfg, sch, dt=dt0, warmup=warm)
    sg.replay(steps)
    torch.cuda.synchronize()
    sg.check()
    A = sg.system.state
    ops.release_device_lists()
    params = ws.make_params(cfg, sch)
    dt = dt0.clone()
    with ops.device_decided_lists():
        for _ in range(warm + steps):
            dt = ops.cfl_dt(params, sys_b.state.supports, sys_b.state.internalEnergies, dt_prev=dt)
            sys_b = integ.function(state=sys_b, f=step, dt=dt, config=cfg, compParams=sch).state
    B = sys_b.state
    for name in ("positions", "velocities", "internalEnergies", "densities", "supports"):
        assert_close(getattr(A, name).cpu().numpy(), getattr(B, name).cpu().numpy(), rtol, atol, name)
    sg.release()


def test_graph_replay_3d(cuda):
    from tests.test_gpu_sedov3d import sedov3d
    cfg, sch, integ, step, sys_a = sedov3d(16, cuda)
    *_, sys_b = sedov3d(16, cuda)
    _graph_vs_device_eager(cuda, cfg, sch, integ, step, sys_a, sys_b, 2, 3, 1e-5, 1e-6)


def test_graph_replay_rk4(cuda):
    cfg, sch, integ, step, sys_a = sedov(32, cuda)
    *_, sys_b = sedov(32, cuda)
    integ4 = ws.getIntegrator(ws.IntegrationSchemeType.rungeKutta4)
    _graph_vs_device_eager(cuda, cfg, sch, integ4, step, sys_a, sys_b, 2, 3, 1e-5, 1e-6)
