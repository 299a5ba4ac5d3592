"""CPU tests of the oracle itself: kernel functions, neighbour search, CRK reproducing
conditions, switch algebra and the conservation properties of a full step."""
import numpy as np
import pytest
from scipy.integrate import quad

from oracle import oracle
from oracle.steps import CRKSPHOracle, SWITCH_CULLEN
from tests.cases import assert_close, make_params, make_particles
from warpsph_b200 import core

KERNELS = [core.KernelFunctions.Wendland2, core.KernelFunctions.Wendland4, core.KernelFunctions.Wendland6]


@pytest.fixture(scope="module")
def o64():
    return oracle.get("f64")


@pytest.fixture(scope="module")
def o32():
    return oracle.get("f32")


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_b7_kernel(o64, dim):
    """The degree-7 B-spline: unit integral, the spline's values at its knots, derivatives
    against finite differences across the polynomial switch at q = 1/4, and the kernel
    scale table (1D and 2D read from the reference notebooks' printed time steps; their
    ratio is the quintic spline's sqrt(d I_(d-1)/I_(d+1)) ratio, which also gives 3D)."""
    kernel = core.KernelFunctions.B7
    surf = {1: lambda r: 2.0, 2: lambda r: 2 * np.pi * r, 3: lambda r: 4 * np.pi * r * r}[dim]
    W = lambda r: o64.kernel_eval(kernel.value, dim, np.array([r]), 1.0)[0][0]
    assert abs(quad(lambda r: W(r) * surf(r), 0, 1, epsabs=1e-13, points=[0.25, 0.5, 0.75])[0] - 1.0) < 1e-9
    C = core.kernel_constants(kernel, dim)[0]
    tp = lambda a, q: max(a - q, 0.0) ** 7
    for q in (0.0, 0.1, 0.25, 0.4, 0.5, 0.75, 0.9):
        want = C * (tp(1, q) - 8 * tp(0.75, q) + 28 * tp(0.5, q) - 56 * tp(0.25, q))
        assert abs(W(q) - want) < 1e-12 * C
    r = np.concatenate([np.linspace(0.01, 0.99, 97), [0.2499, 0.25, 0.2501]])
    H = 0.7
    _, dWdr, dWdH = o64.kernel_eval(kernel.value, dim, r, H)
    e = 1e-6
    Wp, _, _ = o64.kernel_eval(kernel.value, dim, r + e, H)
    Wm, _, _ = o64.kernel_eval(kernel.value, dim, r - e, H)
    assert_close(dWdr, (Wp - Wm) / (2 * e), 1e-6, 1e-6, "dW/dr")
    Hp, _, _ = o64.kernel_eval(kernel.value, dim, r, H + e)
    Hm, _, _ = o64.kernel_eval(kernel.value, dim, r, H - e)
    assert_close(dWdH, (Hp - Hm) / (2 * e), 1e-6, 1e-6, "dW/dH")
    s1, s2, s3 = (core.sphKernelScale(kernel, d) for d in (1, 2, 3))
    assert abs(s2 / s1 - np.sqrt(2868 / 2771)) < 1e-7 and abs(s3 / s1 - np.sqrt(15 / 14)) < 1e-9


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_kernel_normalisation_and_derivatives(o64, kernel, dim):
    surf = {1: lambda r: 2.0, 2: lambda r: 2 * np.pi * r, 3: lambda r: 4 * np.pi * r * r}[dim]
    W = lambda r: o64.kernel_eval(kernel.value, dim, np.array([r]), 1.0)[0][0]
    assert abs(quad(lambda r: W(r) * surf(r), 0, 1, epsabs=1e-13)[0] - 1.0) < 1e-9
    # kernel scale H/h = 1/(2 sigma) (Dehnen & Aly 2012 Table 1) from the second moment
    m2 = quad(lambda r: r * r * W(r) * surf(r), 0, 1, epsabs=1e-13)[0]
    assert abs(1 / (2 * np.sqrt(m2 / dim)) - core.sphKernelScale(kernel, dim)) < 1e-8
    r = np.linspace(0.01, 0.99, 97)
    H = 0.7
    _, dWdr, dWdH = o64.kernel_eval(kernel.value, dim, r, H)
    e = 1e-6
    Wp, _, _ = o64.kernel_eval(kernel.value, dim, r + e, H)
    Wm, _, _ = o64.kernel_eval(kernel.value, dim, r - e, H)
    assert_close(dWdr, (Wp - Wm) / (2 * e), 1e-6, 1e-6, "dW/dr")
    Wp, _, _ = o64.kernel_eval(kernel.value, dim, r, H + e)
    Wm, _, _ = o64.kernel_eval(kernel.value, dim, r, H - e)
    assert_close(dWdH, (Wp - Wm) / (2 * e), 1e-6, 1e-6, "dW/dH")
    Wo, _, _ = o64.kernel_eval(kernel.value, dim, np.array([1.0, 1.5]), 1.0)
    assert np.all(Wo == 0)


def brute_force(x, H, vs, L, periodic):
    d = x[:, None, :].astype(np.float32) - x[None, :, :].astype(np.float32)
    if periodic:
        hl = np.float32(0.5 * L)
        d = np.where(d > hl, d - np.float32(L), np.where(d < -hl, d + np.float32(L), d))
    r2 = np.zeros(d.shape[:2], np.float32)
    for a in range(x.shape[1]):
        r2 = (r2 + d[..., a] * d[..., a]).astype(np.float32)
    R = (np.float32(vs) * np.maximum(H[:, None], H[None, :])).astype(np.float32)
    return r2 < (R * R).astype(np.float32)


@pytest.mark.parametrize("dim,n_side", [(1, 300), (2, 30), (3, 11)])
@pytest.mark.parametrize("periodic", [True, False])
def test_neighbor_list_matches_brute_force(o32, dim, n_side, periodic):
    cfg, sch, p = make_params(dim, periodic=periodic)
    P = make_particles(dim, n_side, periodic=periodic, seed=dim)
    x, H = P["positions"], P["supports"]
    nb = o32.neighbors(p, x, H, 1 << 16, partition=False)
    ref = brute_force(x, H, p.verlet_scale, 1.0, periodic)
    pos = np.argsort(nb["sort_index"])
    assert np.array_equal(np.sort(nb["sort_index"]), np.arange(len(H)))
    # permutation sorted by (key, index)
    keys = nb["sorted_keys"].astype(np.int64)
    order = np.lexsort((nb["sort_index"], keys))
    assert np.array_equal(order, np.arange(len(H)))
    for i in range(len(H)):
        row = nb["list"][nb["offsets"][i]: nb["offsets"][i] + nb["counts"][i]]
        assert set(row.tolist()) == set(np.nonzero(ref[i])[0].tolist()), i
        # canonical order: cells contiguous, ascending sorted position inside a cell
        ck = nb["sorted_keys"][pos[row]]
        change = np.nonzero(np.diff(ck.astype(np.int64)))[0]
        assert len(set(ck.tolist())) == len(change) + 1, "each stencil cell appears once"
        for seg in np.split(pos[row], change + 1):
            assert np.all(np.diff(seg) > 0)
        assert i in row
    # super-symmetric lists are symmetric
    assert ref.sum() == nb["nnz"]
    # the library's layout: every row a stable partition of the walk-order row, the
    # entries with fl(sqrt(r^2)) / max(H_i, H_j) < 1 first
    part = o32.neighbors(p, x, H, 1 << 16)
    assert np.array_equal(part["offsets"], nb["offsets"]) and np.array_equal(part["counts"], nb["counts"])
    for i in range(len(H)):
        row = nb["list"][nb["offsets"][i]: nb["offsets"][i] + nb["counts"][i]]
        d = (x[i] - x[row]).astype(np.float32)
        if periodic:
            d = np.where(d > 0.5, d - np.float32(1.0), np.where(d < -0.5, d + np.float32(1.0), d)).astype(np.float32)
        r2 = d[:, 0] * d[:, 0]
        for a in range(1, dim):
            r2 = (r2 + d[:, a] * d[:, a]).astype(np.float32)
        inter = (np.sqrt(r2, dtype=np.float32) / np.maximum(H[i], H[row])) < np.float32(1.0)
        want = np.concatenate([row[inter], row[~inter]])
        got = part["list"][part["offsets"][i]: part["offsets"][i] + part["counts"][i]]
        assert np.array_equal(got, want), i
        assert part["inter_counts"][i] == inter.sum()


def test_neighbor_small_periodic_grid_deduplicates(o32):
    # fewer than three cells per axis: the periodic stencil wraps onto itself
    cfg, sch, p = make_params(2, periodic=True)
    rng = np.random.default_rng(3)
    x = (rng.random((64, 2)) - 0.5).astype(np.float32)
    H = np.full(64, 0.3, np.float32)
    nb = o32.neighbors(p, x, H, 4096)
    ref = brute_force(x, H, p.verlet_scale, 1.0, True)
    assert nb["grid"][0] <= 2
    for i in range(64):
        row = nb["list"][nb["offsets"][i]: nb["offsets"][i] + nb["counts"][i]]
        assert len(row) == len(set(row.tolist())) == ref[i].sum()


def test_neighbor_particles_outside_nonperiodic_domain(o32):
    cfg, sch, p = make_params(2, periodic=False)
    rng = np.random.default_rng(4)
    x = (rng.random((500, 2)) * 1.6 - 0.8).astype(np.float32)   # some outside [-0.5, 0.5]
    H = np.full(500, 0.05, np.float32)
    nb = o32.neighbors(p, x, H, 1 << 14)
    ref = brute_force(x, H, p.verlet_scale, 1.0, False)
    for i in range(500):
        row = nb["list"][nb["offsets"][i]: nb["offsets"][i] + nb["counts"][i]]
        assert set(row.tolist()) == set(np.nonzero(ref[i])[0].tolist())


def test_neighbor_empty_input(o32):
    cfg, sch, p = make_params(2)
    nb = o32.neighbors(p, np.zeros((0, 2), np.float32), np.zeros(0, np.float32), 1024)
    assert nb["nnz"] == 0


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_crk_reproduces_linear_fields(o64, dim):
    """Frontiere et al. 2017 reproducing conditions: sum_j V_j W^R_ij = 1 and
    sum_j V_j W^R_ij x_ij = 0, so the CRK gradient of a linear field is exact."""
    n_side = {1: 200, 2: 24, 3: 10}[dim]
    cfg, sch, p = make_params(dim, periodic=False)
    P = make_particles(dim, n_side, periodic=False, seed=7, h_spread=0.05)
    x, H, m = [P[k].astype(np.float64) for k in ("positions", "supports", "masses")]
    nb = o64.neighbors(p, x, H, 1 << 16)
    V = o64.crk_volume(p, x, H, nb)
    A, B, gA, gB, rho = o64.crk_factors(p, x, H, m, V, nb)
    M = np.arange(1, dim * dim + 1, dtype=np.float64).reshape(dim, dim) / 7.0
    v = x @ M.T + 0.3
    c = np.ones(len(H))
    G, drho, _, _ = o64.grad_v(p, x, H, m, rho, V, A, B, gA, gB, v, c, nb, cullen=False)
    interior = np.all(np.abs(x) < 0.5 - 1.6 * H.max(), axis=1)
    assert interior.sum() > 5
    assert_close(G[interior], np.broadcast_to(M, G[interior].shape), 1e-9, 1e-9, "CRK gradient of a linear field")


def test_crk_singular_moment_fallback(o64):
    """An isolated pair has a singular second moment in 2D: zeroth-order correction."""
    cfg, sch, p = make_params(2, periodic=False)
    x = np.array([[0.0, 0.0], [0.01, 0.0], [0.3, 0.3]])
    H = np.full(3, 0.05)
    m = np.ones(3)
    nb = o64.neighbors(p, x, H, 4096)
    V = o64.crk_volume(p, x, H, nb)
    A, B, gA, gB, rho = o64.crk_factors(p, x, H, m, V, nb)
    assert np.all(np.isfinite(A)) and np.all(B == 0) and np.all(gB == 0)


def test_full_step_conserves_mass_momentum_energy(o64):
    """Compatible energy: total energy and momentum are conserved to round-off."""
    cfg, sch, p = make_params(2)
    P = make_particles(2, 24, seed=11)
    st = {k: v.astype(np.float64) for k, v in P.items()}
    n = len(st["masses"])
    st.update(densities=np.ones(n), divergence=np.zeros(n), alpha0s=np.ones(n), alphas=np.ones(n))
    orc = CRKSPHOracle(p, "f64", switch=SWITCH_CULLEN)
    E = lambda s: np.sum(s["masses"] * (s["internalEnergies"] + 0.5 * np.sum(s["velocities"] ** 2, 1)))
    mom = lambda s: np.sum(s["masses"][:, None] * s["velocities"], 0)
    E0, p0 = E(st), mom(st)
    for _ in range(3):
        st, _, _ = orc.step(st, 2e-4, "rungeKutta2")
    assert abs(E(st) - E0) / E0 < 1e-12
    assert np.max(np.abs(mom(st) - p0)) < 1e-12 * np.sum(st["masses"])


def test_mlp_oracle_gradient_matches_finite_differences():
    """The MLP oracle's analytic gradient (float64, no BF16 rounding) against central
    differences of its loss, on every parameter block."""
    from oracle import mlp
    rng = np.random.default_rng(1)
    theta = mlp.init_params(3).astype(np.float64)
    theta[mlp.NPARAM - 1] = 0.3
    x = rng.standard_normal((40, 8))
    t = rng.standard_normal(40)
    g, _ = mlp.grad(theta, x, t, bf=False)
    loss = lambda th: np.mean((mlp.forward(th, x, bf=False)[0] - t) ** 2)
    idx = np.concatenate([rng.choice(np.arange(a, b), 12, replace=False) for a, b in
                          [(0, 512), (512, 576), (576, 4672), (4672, 4736), (4736, 8832), (8832, 8896), (8896, 8960)]] + [[8960]])
    for k in idx:
        e = np.zeros_like(theta)
        e[k] = 1e-6
        fd = (loss(theta + e) - loss(theta - e)) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_mlp_oracle_bf16_rounding():
    from oracle import mlp
    a = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3, 3.0e38], np.float32)
    b = mlp.bf16(a)
    assert b[0] == 1.0 and b[1] == 1.0 and b[2] == np.float32(1.0078125)   # ties to even, then round up
    assert np.all(np.abs(b - a) <= np.abs(a) * 2 ** -8)
