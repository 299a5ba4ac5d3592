"""GPU kernels (through the C ABI) against the CPU oracle on identical seeded inputs.

Integer/indexing work is compared bit for bit; floating-point outputs with the
tolerances written at each assertion (FP32 GPU vs FP32 oracle: differences come
only from FMA contraction and operation order; vs the FP64 oracle: FP32 rounding)."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle
from oracle.steps import cell_capacity_for
from tests.cases import assert_close, make_params, make_particles
from warpsph_b200 import _capi, core, ops
from warpsph_b200.enumTypes import EnergyScheme

pytestmark = pytest.mark.gpu

CASES = [(1, 400), (2, 40), (3, 14)]


def to_gpu(P, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in P.items()}


def nb_numpy(adj):
    return dict(offsets=adj.neighborOffsets.cpu().numpy(), counts=adj.numNeighbors.cpu().numpy(),
                list=adj.neighborList.cpu().numpy())


@pytest.mark.parametrize("dim,n_side", CASES)
@pytest.mark.parametrize("periodic", [True, False])
def test_neighbors_bit_exact(cuda, dim, n_side, periodic):
    cfg, sch, p = make_params(dim, periodic=periodic)
    P = make_particles(dim, n_side, periodic=periodic, seed=10 + dim)
    G = to_gpu(P, cuda)
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    ref = oracle.get("f32").neighbors(p, P["positions"], P["supports"], cell_capacity_for(len(P["supports"]), dim))
    assert adj.nnz == ref["nnz"]
    assert np.array_equal(adj.sortIndex.cpu().numpy(), ref["sort_index"])
    assert np.array_equal(adj.sortedKeys.cpu().numpy().view(np.uint32), ref["sorted_keys"])
    assert np.array_equal(adj.grid.cpu().numpy(), ref["grid"])
    assert np.array_equal(adj.neighborOffsets.cpu().numpy(), ref["offsets"])
    assert np.array_equal(adj.numNeighbors.cpu().numpy(), ref["counts"])
    assert np.array_equal(adj.neighborList.cpu().numpy(), ref["list"])
    i, j = adj.i.cpu().numpy(), adj.j.cpu().numpy()
    assert np.array_equal(j, ref["list"]) and np.array_equal(np.bincount(i, minlength=len(ref["counts"])), ref["counts"])


@pytest.mark.parametrize("dim,n_side", [(1, 12), (1, 20), (2, 9), (2, 12), (3, 8)])
def test_neighbors_bit_exact_small_periodic_grids(cuda, dim, n_side):
    """One or two cells along a periodic axis: a cell is reached through two periodic
    images, and every pair must still be tested at its minimum image."""
    cfg, sch, p = make_params(dim)
    P = make_particles(dim, n_side, seed=30 + dim, jitter=0.4, h_spread=0.15)
    G = to_gpu(P, cuda)
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    ref = oracle.get("f32").neighbors(p, P["positions"], P["supports"], cell_capacity_for(len(P["supports"]), dim))
    assert ref["grid"][:dim].min() < 3, ref["grid"]
    assert np.array_equal(adj.grid.cpu().numpy(), ref["grid"])
    assert adj.nnz == ref["nnz"]
    assert np.array_equal(adj.neighborOffsets.cpu().numpy(), ref["offsets"])
    assert np.array_equal(adj.numNeighbors.cpu().numpy(), ref["counts"])
    assert np.array_equal(adj.neighborList[: adj.nnz].cpu().numpy(), ref["list"])
    # brute force: every pair within verlet_scale * max(H_i, H_j) at its minimum image
    x, H = P["positions"], P["supports"]
    d = x[:, None, :] - x[None, :, :]
    d = np.where(d > 0.5, d - 1.0, np.where(d < -0.5, d + 1.0, d)).astype(np.float32)
    r2 = (d.astype(np.float64) ** 2).sum(-1)
    R = float(p.verlet_scale) * np.maximum(H[:, None], H[None, :]).astype(np.float64)
    assert abs(int((r2 < R * R).sum()) - adj.nnz) <= 4   # FP32 rounding at r = R


@pytest.mark.parametrize("dim,n_side", CASES)
def test_interacting_list_is_exact_subset(cuda, dim, n_side):
    """The interacting list holds exactly the Verlet entries with fl(sqrt(r^2))/max(H_i,H_j) < 1
    (same float operations as the list builder), in Verlet order, with their entry index."""
    cfg, sch, p = make_params(dim)
    P = make_particles(dim, n_side, seed=20 + dim)
    G = to_gpu(P, cuda)
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    x, H = P["positions"], P["supports"]
    offs, cnt, lst = (a.cpu().numpy() for a in (adj.neighborOffsets, adj.numNeighbors, adj.neighborList))
    i = np.repeat(np.arange(len(H)), cnt)
    d = (x[i] - x[lst]).astype(np.float32)
    hl = np.float32(0.5)
    d = np.where(d > hl, d - np.float32(1.0), np.where(d < -hl, d + np.float32(1.0), d)).astype(np.float32)
    r2 = np.zeros(len(lst), np.float32)
    for a in range(dim):
        r2 = (r2 + d[:, a] * d[:, a]).astype(np.float32)
    Hm = np.maximum(H[i], H[lst])
    keep = (np.sqrt(r2).astype(np.float32) / Hm).astype(np.float32) < np.float32(1.0)
    icnt = adj.interCounts.cpu().numpy()
    assert adj.interNnz == int(keep.sum()) == int(icnt.sum())
    assert np.array_equal(icnt, np.bincount(i[keep], minlength=len(H)))
    # every row: its interacting entries first, the rest after them
    pos_in_row = np.arange(len(lst)) - np.repeat(offs, cnt)
    assert np.array_equal(keep, pos_in_row < np.repeat(icnt, cnt))


def test_neighbors_capacity_overflow_is_recovered(cuda):
    cfg, sch, p = make_params(2)
    P = make_particles(2, 30, seed=5)
    G = to_gpu(P, cuda)
    from warpsph_b200 import ops as _ops
    _ops._nb_cache.cap_hint[(cuda.index or 0, 900, 2)] = 16   # force an overflow on the first attempt
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    ref = oracle.get("f32").neighbors(p, P["positions"], P["supports"], cell_capacity_for(900, 2))
    assert adj.nnz == ref["nnz"] and np.array_equal(adj.neighborList.cpu().numpy(), ref["list"])
    assert np.array_equal(adj.interCounts.cpu().numpy(), ref["inter_counts"])


def test_neighbors_reject_nonpositive_support(cuda):
    cfg, sch, p = make_params(2)
    P = make_particles(2, 10, seed=5)
    G = to_gpu(P, cuda)
    H = G["supports"].clone()
    H[3] = 0.0
    with pytest.raises(RuntimeError, match="finite and positive"):
        ops.buildVerletList(G["positions"], H, p, p.verlet_scale)


def test_neighbors_reuse_unchanged_prior(cuda):
    cfg, sch, p = make_params(2)
    G = to_gpu(make_particles(2, 12, seed=1), cuda)
    a = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    assert ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale, a) is a
    x2 = G["positions"].clone()
    assert ops.buildVerletList(x2, G["supports"], p, p.verlet_scale, a) is not a


def pipeline_inputs(dim, n_side, dev, seed=0, kernel=core.KernelFunctions.Wendland4, periodic=True, **kw):
    cfg, sch, p = make_params(dim, kernel=kernel, periodic=periodic, **kw)
    P = make_particles(dim, n_side, periodic=periodic, seed=seed)
    G = to_gpu(P, dev)
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    return cfg, sch, p, P, G, adj


@pytest.mark.parametrize("dim,n_side", CASES)
@pytest.mark.parametrize("kernel", [core.KernelFunctions.Wendland2, core.KernelFunctions.Wendland4])
def test_density_and_adaptive_support(cuda, dim, n_side, kernel):
    cfg, sch, p, P, G, adj = pipeline_inputs(dim, n_side, cuda, kernel=kernel)
    nb = nb_numpy(adj)
    for precision, tol in (("f32", 2e-6), ("f64", 2e-6)):
        o = oracle.get(precision)
        for mode in (core.SupportScheme.Gather, core.SupportScheme.Scatter, core.SupportScheme.SuperSymmetric,
                     core.SupportScheme.KernelMeanSymmetric, core.SupportScheme.Symmetric):
            rho = ops.density(p, G["positions"], G["supports"], G["masses"], adj, mode).cpu().numpy()
            ref = o.density(p, ops._SUPPORT[mode], P["positions"], P["supports"], P["masses"], nb)
            assert_close(rho, ref, tol, tol, f"density {mode} {precision}")
    hb = ops.minmax(G["supports"])
    rho, Hn, ratio = ops.adaptive_h_iter(p, G["positions"], G["supports"], G["masses"], adj, hb)
    r_rho, r_H, r_ratio = oracle.get("f32").adaptive_h_iter(p, P["positions"], P["supports"], P["masses"], nb, hb.cpu().numpy())
    assert_close(rho.cpu().numpy(), r_rho, 2e-6, 2e-6, "adaptive rho")
    assert_close(Hn.cpu().numpy(), r_H, 1e-5, 1e-5, "adaptive H")
    assert np.array_equal(hb.cpu().numpy(), np.array([P["supports"].min(), P["supports"].max()], np.float32))


@pytest.mark.parametrize("dim,n_side", CASES)
def test_crk_pipeline(cuda, dim, n_side):
    cfg, sch, p, P, G, adj = pipeline_inputs(dim, n_side, cuda, seed=3)
    nb = nb_numpy(adj)
    o32, o64 = oracle.get("f32"), oracle.get("f64")
    x, H, m, v, u = (P[k] for k in ("positions", "supports", "masses", "velocities", "internalEnergies"))
    # CRK volume and coefficients
    V = ops.crk_volume(p, G["positions"], G["supports"], adj)
    assert_close(V.cpu().numpy(), o32.crk_volume(p, x, H, nb), 2e-6, 2e-6, "V")
    Vn = V.cpu().numpy()
    crk, rho = ops.crk_factors(p, G["positions"], G["supports"], G["masses"], V, adj)
    rA, rB, rgA, rgB, rrho = o64.crk_factors(p, x, H, m, Vn, nb)
    assert_close(crk.A.cpu().numpy(), rA, 1e-4, 1e-4, "A")
    assert_close(crk.B.cpu().numpy(), rB, 1e-3, 1e-3, "B")
    assert_close(crk.gradA.cpu().numpy(), rgA, 1e-3, 1e-3, "gradA")
    assert_close(crk.gradB.cpu().numpy(), rgB, 2e-3, 2e-3, "gradB")
    assert_close(rho.cpu().numpy(), rrho, 1e-5, 1e-5, "CRK rho")
    # EOS
    A_, Pr, c = ops.eos_ideal_gas(p, G["internalEnergies"], rho)
    rA_, rP, rc = o32.eos(p, u, rho.cpu().numpy())
    assert_close(Pr.cpu().numpy(), rP, 1e-6, 1e-6, "P")
    assert_close(c.cpu().numpy(), rc, 1e-6, 1e-6, "c")
    assert_close(A_.cpu().numpy(), rA_, 1e-5, 1e-5, "A(entropy)")
    # velocity gradient + Cullen divergence + v_sig (inputs from the GPU so errors do not compound)
    cn = {k: t.cpu().numpy() for k, t in dict(A=crk.A, B=crk.B, gA=crk.gradA, gB=crk.gradB, rho=rho, c=c, P=Pr).items()}
    Gv, drho, div, vs = ops.grad_v(p, G["positions"], G["supports"], G["masses"], rho, V, crk, G["velocities"], c, adj, True,
                                   want_vsig=True)
    rG, rdrho, rdiv, rvs = o32.grad_v(p, x, H, m, cn["rho"], Vn, cn["A"], cn["B"], cn["gA"], cn["gB"], v, cn["c"], nb, True)
    assert_close(Gv.cpu().numpy(), rG, 1e-4, 1e-4, "DvDx")
    assert_close(drho.cpu().numpy(), rdrho, 1e-4, 1e-4, "drhodt")
    assert_close(div.cpu().numpy(), rdiv, 1e-4, 1e-4, "Cullen div")
    assert_close(vs.cpu().numpy(), rvs, 1e-6, 1e-6, "v_sig")
    # Cullen switch
    div_prev = torch.from_numpy(rdiv * 0.9 + 0.01).to(cuda)
    a0 = torch.full_like(rho, 0.5)
    al, R, _ = ops.switch_cullen(p, G["positions"], G["supports"], G["masses"], rho, div, div_prev, vs, a0, 1e-3, adj, want_R=True)
    # the same switch computing v_sig itself over the Verlet list
    al2, R2, vs2 = ops.switch_cullen(p, G["positions"], G["supports"], G["masses"], rho, div, div_prev, None, a0, 1e-3, adj,
                                     want_R=True, v=G["velocities"], c=c, want_vsig=True)
    assert_close(vs2.cpu().numpy(), rvs, 1e-6, 1e-6, "v_sig in the Cullen pass")
    assert_close(al2.cpu().numpy(), al.cpu().numpy(), 1e-6, 1e-6, "alphas with internal v_sig")
    ral, rR = o32.switch_cullen(p, x, H, m, cn["rho"], div.cpu().numpy(), div_prev.cpu().numpy(), vs.cpu().numpy(),
                                np.full(len(H), 0.5, np.float32), 1e-3, nb)
    assert_close(R.cpu().numpy(), rR, 1e-5, 1e-5, "R")
    assert_close(al.cpu().numpy(), ral, 1e-4, 1e-4, "alphas")
    bal = ops.switch_balsara(p, Gv, c)
    assert_close(bal.cpu().numpy(), o32.switch_balsara(p, Gv.cpu().numpy(), cn["c"]), 1e-5, 1e-5, "Balsara")
    # fused accel + dudt with pair arrays
    Gn = Gv.cpu().numpy()
    dvdt, dudt, ap, av = ops.crk_accel_dudt(p, G["positions"], G["supports"], G["masses"], rho, V, crk, G["velocities"], c, Pr,
                                            Gv, adj)
    rdv, rdu, rap, rav = o32.crk_accel_dudt(p, x, H, m, cn["rho"], Vn, cn["A"], cn["B"], cn["gA"], cn["gB"], v, cn["c"], cn["P"],
                                            Gn, nb)
    assert_close(ap.cpu().numpy(), rap, 1e-4, 1e-4, "ap_ij")
    assert_close(av.cpu().numpy(), rav, 1e-3, 1e-3, "av_ij")
    assert_close(dvdt.cpu().numpy(), rdv, 1e-3, 1e-3, "dvdt")
    assert_close(dudt.cpu().numpy(), rdu, 1e-3, 1e-3, "dudt")
    # against the FP64 oracle too (FP32 rounding only)
    r64 = o64.crk_accel_dudt(p, x, H, m, cn["rho"], Vn, cn["A"], cn["B"], cn["gA"], cn["gB"], v, cn["c"], cn["P"], Gn, nb)
    assert_close(dvdt.cpu().numpy(), r64[0], 2e-3, 2e-3, "dvdt vs f64")
    # balance, all energy schemes
    for es in EnergyScheme:
        p.energy_scheme = es.value
        f = ops.compsph_balance(p, G["masses"], rho, Pr, G["internalEnergies"], G["velocities"], dvdt, 1e-3, adj, ap, av)
        rf = o32.balance(p, m, cn["rho"], cn["P"], u, v, dvdt.cpu().numpy(), 1e-3, nb, ap.cpu().numpy(), av.cpu().numpy())
        fg = f.cpu().numpy()
        mism = np.mean(np.abs(fg - rf) > 1e-4)
        # the partition is discontinuous in sign(dE); entries where dE rounds across zero may flip
        assert mism < 2e-3, (es, mism)
        # skipping the entries past each row's interacting prefix (ap = av = 0 there) gives the
        # same f_ij, bit for bit, as reading them
        assert adj.interCounts is not None and adj._pending is None
        f_full = torch.empty_like(f)
        scratch = torch.empty(G["masses"].shape[0] * (int(p.dim) + 1), device=cuda)
        dtt = torch.tensor([1e-3], device=cuda)
        rc = _capi.lib().sph_compsph_balance(C.byref(p), G["masses"].shape[0], G["masses"].data_ptr(), rho.data_ptr(), Pr.data_ptr(),
                                             G["internalEnergies"].data_ptr(), G["velocities"].data_ptr(), dvdt.data_ptr(),
                                             dtt.data_ptr(), adj.neighborOffsets.data_ptr(), adj.numNeighbors.data_ptr(),
                                             adj.neighborList.data_ptr(), None, ap.data_ptr(), av.data_ptr(), scratch.data_ptr(),
                                             f_full.data_ptr(), _capi.stream_ptr(cuda))
        assert rc == 0
        assert torch.equal(f_full, f), es


def test_kahan_option_matches(cuda):
    cfg, sch, p, P, G, adj = pipeline_inputs(2, 32, cuda, seed=9, kahan=True)
    V = ops.crk_volume(p, G["positions"], G["supports"], adj)
    crk, rho = ops.crk_factors(p, G["positions"], G["supports"], G["masses"], V, adj)
    _, Pr, c = ops.eos_ideal_gas(p, G["internalEnergies"], rho)
    Gv, *_ = ops.grad_v(p, G["positions"], G["supports"], G["masses"], rho, V, crk, G["velocities"], c, adj, False)
    dv_k, du_k, _, _ = ops.crk_accel_dudt(p, G["positions"], G["supports"], G["masses"], rho, V, crk, G["velocities"], c, Pr, Gv, adj,
                                          pair_arrays=False)
    p.kahan = 0
    dv, du, _, _ = ops.crk_accel_dudt(p, G["positions"], G["supports"], G["masses"], rho, V, crk, G["velocities"], c, Pr, Gv, adj,
                                      pair_arrays=False)
    nb = nb_numpy(adj)
    cn = {k: t.cpu().numpy() for k, t in dict(A=crk.A, B=crk.B, gA=crk.gradA, gB=crk.gradB, rho=rho, c=c, P=Pr, G=Gv, V=V).items()}
    r64 = oracle.get("f64").crk_accel_dudt(p, P["positions"], P["supports"], P["masses"], cn["rho"], cn["V"], cn["A"], cn["B"],
                                           cn["gA"], cn["gB"], P["velocities"], cn["c"], cn["P"], cn["G"], nb)
    e_k = np.abs(dv_k.cpu().numpy() - r64[0]).max()
    e_p = np.abs(dv.cpu().numpy() - r64[0]).max()
    assert e_k <= e_p * 1.5 + 1e-7


@pytest.mark.parametrize("dim,n_side", CASES)
def test_prior_list_refresh(cuda, dim, n_side):
    """A still-valid prior list (small displacement and support change) is kept and its
    rows reordered for the new positions: per row the same Verlet set as before, its
    interacting prefix the same j set as a fresh build's, in the prior row order.  A large
    displacement rebuilds (the result then equals the oracle's list bit for bit)."""
    cfg, sch, p = make_params(dim)
    P = make_particles(dim, n_side, seed=90 + dim)
    G = to_gpu(P, cuda)
    adj0 = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    rng = np.random.default_rng(5)
    H = P["supports"]
    x1 = (P["positions"] + (0.02 * H[:, None] * rng.standard_normal(P["positions"].shape)).astype(np.float32)).astype(np.float32)
    x1 = ((x1 + 0.5) % 1.0 - 0.5).astype(np.float32)
    H1 = (H * (1 + 0.05 * (rng.random(len(H)) - 0.5))).astype(np.float32)
    adj1 = ops.buildVerletList(torch.from_numpy(x1).to(cuda), torch.from_numpy(H1).to(cuda), p, p.verlet_scale, adj0)
    assert adj1.neighborList.data_ptr() == adj0.neighborList.data_ptr(), "valid prior list must be kept"
    fresh = ops.buildVerletList(torch.from_numpy(x1).to(cuda), torch.from_numpy(H1).to(cuda), p, p.verlet_scale)
    assert adj1.interCounts is None                    # rows reordered on first use by a pass
    lst0 = adj0.neighborList.cpu().numpy().copy()
    ops._lists(p, adj1, True)
    assert adj1.neighborList.data_ptr() != adj0.neighborList.data_ptr(), "the prior rows must stay untouched"
    assert np.array_equal(adj0.neighborList.cpu().numpy(), lst0)
    o, cnt = adj1.neighborOffsets.cpu().numpy(), adj1.numNeighbors.cpu().numpy()
    l1, c1 = adj1.neighborList.cpu().numpy(), adj1.interCounts.cpu().numpy()
    l2, c2 = fresh.neighborList.cpu().numpy(), fresh.interCounts.cpu().numpy()
    o2 = fresh.neighborOffsets.cpu().numpy()
    assert int(adj1._inter_nnz_dev.item()) == fresh.interNnz == int(c1.sum())
    for i in range(len(H)):
        row0 = lst0[o[i]: o[i] + cnt[i]]
        row1 = l1[o[i]: o[i] + cnt[i]]
        assert sorted(row1.tolist()) == sorted(row0.tolist()), i
        pre1, pre2 = row1[: c1[i]], l2[o2[i]: o2[i] + c2[i]]
        assert set(pre1.tolist()) == set(pre2.tolist()), i
        where = {j: k for k, j in enumerate(row0.tolist())}
        assert np.all(np.diff([where[j] for j in pre1.tolist()]) > 0)          # prior order kept in the prefix
    # beyond the skin: rebuilt, identical to the oracle
    x2 = (((P["positions"] + 0.5 * H.max()) + 0.5) % 1.0 - 0.5).astype(np.float32)
    adj2 = ops.buildVerletList(torch.from_numpy(x2).to(cuda), G["supports"], p, p.verlet_scale, adj0)
    assert adj2.neighborList.data_ptr() != adj0.neighborList.data_ptr()
    ref = oracle.get("f32").neighbors(p, x2, H, cell_capacity_for(len(H), dim))
    assert np.array_equal(adj2.neighborList.cpu().numpy(), ref["list"])
    assert np.array_equal(adj2.interCounts.cpu().numpy(), ref["inter_counts"])


@pytest.mark.parametrize("dim,n_side", CASES)
def test_prior_list_rewrite_fused_with_volume(cuda, dim, n_side):
    """The CRK volume of a kept list whose rows await their rewrite comes from the fused
    pass (sph_neighbors_refresh_volume): the rewritten rows and interacting counts equal
    the plain rewrite's bit for bit, and the volumes equal the standalone volume pass on
    those rows to FP32 rounding (the fused sum runs in the row's original order)."""
    cfg, sch, p = make_params(dim)
    P = make_particles(dim, n_side, seed=70 + dim)
    G = to_gpu(P, cuda)
    adj0 = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    rng = np.random.default_rng(8)
    H = P["supports"]
    x1 = (P["positions"] + (0.02 * H[:, None] * rng.standard_normal(P["positions"].shape)).astype(np.float32)).astype(np.float32)
    x1 = torch.from_numpy(((x1 + 0.5) % 1.0 - 0.5).astype(np.float32)).to(cuda)
    H1 = torch.from_numpy((H * (1 + 0.05 * (rng.random(len(H)) - 0.5))).astype(np.float32)).to(cuda)
    fused = ops.buildVerletList(x1, H1, p, p.verlet_scale, adj0)
    plain = ops.buildVerletList(x1, H1, p, p.verlet_scale, adj0)
    assert fused._pending is not None and plain._pending is not None
    V_fused = ops.crk_volume(p, x1, H1, fused)
    assert fused._pending is None
    ops._lists(p, plain, True)
    V_plain = ops.crk_volume(p, x1, H1, plain)
    assert torch.equal(fused.neighborList, plain.neighborList)
    assert torch.equal(fused.interCounts, plain.interCounts)
    assert int(fused._inter_nnz_dev.item()) == int(plain._inter_nnz_dev.item())
    assert torch.allclose(V_fused, V_plain, rtol=2e-6, atol=0)


def _hopkins_both(p, P, G, adj, dev):
    nb = nb_numpy(adj)
    rho = ops.density(p, G["positions"], G["supports"], G["masses"], adj, core.SupportScheme.Gather)
    n = rho.shape[0]
    a0 = np.linspace(0.2, 1.5, n).astype(np.float32)
    gpu = ops.switch_hopkins_terms(p, G["positions"], G["supports"], G["masses"], rho, G["velocities"],
                                   torch.from_numpy(a0).to(dev), adj)
    ref = oracle.get("f64").switch_hopkins_terms(p, P["positions"], P["supports"], P["masses"], rho.cpu().numpy(),
                                                 P["velocities"], a0, nb)
    return [t.cpu().numpy() for t in gpu], ref


@pytest.mark.parametrize("dim,n_side", CASES)
def test_hopkins_corrected_gradient(cuda, dim, n_side):
    """correctVelocityGradient: moment matrix and FP64 one-sided Jacobi pseudo-inverse on
    the GPU against the FP64 oracle (LAPACK SVD pseudo-inverse, the same cutoff)."""
    cfg, sch, p, P, G, adj = pipeline_inputs(dim, n_side, cuda)
    (al0, div0, s20, _), _ = _hopkins_both(p, P, G, adj, cuda)
    p.correct_velocity_gradient = 1
    (al, div, s2, R), (r_al, r_div, r_s2, r_R) = _hopkins_both(p, P, G, adj, cuda)
    assert_close(div, r_div, 2e-4, 2e-5, f"corrected divergence {dim}D")
    assert_close(s2, r_s2, 1e-3, 1e-5, f"corrected |S|^2 {dim}D")
    assert_close(R, r_R, 2e-4, 2e-5, f"R {dim}D")
    assert_close(al, r_al, 1e-3, 1e-4, f"alphas {dim}D")
    assert np.abs(div - div0).max() > 1e-3 * np.abs(div0).max(), "the flag did not reach the kernel"


def test_hopkins_corrected_gradient_rank_deficient(cuda):
    """Particles on the x axis of a 2D domain: M has an exactly zero singular value, which
    the pseudo-inverse drops, so only the xx component of the gradient survives."""
    cfg, sch, p = make_params(2, periodic=False)
    n, dx = 256, 1.0 / 256
    x = np.zeros((n, 2), np.float32)
    x[:, 0] = ((np.arange(n) + 0.5) * dx - 0.5).astype(np.float32)
    rng = np.random.default_rng(3)
    v = np.stack([np.sin(2 * np.pi * x[:, 0]), np.cos(2 * np.pi * x[:, 0])], 1).astype(np.float32)
    v += (0.05 * rng.standard_normal(v.shape)).astype(np.float32)
    P = dict(positions=x, supports=np.full(n, 4 * dx, np.float32), masses=np.full(n, dx, np.float32), velocities=v)
    G = to_gpu(P, cuda)
    adj = ops.buildVerletList(G["positions"], G["supports"], p, p.verlet_scale)
    p.correct_velocity_gradient = 1
    (al, div, s2, R), (r_al, r_div, r_s2, r_R) = _hopkins_both(p, P, G, adj, cuda)
    assert np.isfinite(div).all() and np.isfinite(s2).all()
    assert_close(div, r_div, 2e-4, 2e-5, "corrected divergence on a line")
    assert_close(s2, r_s2, 1e-3, 1e-5, "corrected |S|^2 on a line")
    # traceless symmetric part of diag(g, 0): |S|^2 = g^2 / 2 with g the divergence
    assert_close(s2, 0.5 * div.astype(np.float64) ** 2, 1e-4, 1e-6, "|S|^2 of a rank-one gradient")
