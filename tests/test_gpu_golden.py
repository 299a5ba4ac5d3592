"""The CUDA kernels (through the C ABI) against the golden vectors produced by the
reference's own Python source (tests/golden/make_golden.py).  The GPU replaces
repeated divisions by reciprocal multiplications and sums pairs in a different order,
so the tolerances are relative to each field's magnitude (stated per assertion)."""
from pathlib import Path

import numpy as np
import pytest
import torch

from tests.cases import assert_close, make_params
from warpsph_b200 import core, ops
from warpsph_b200.core import AdjacencyList, CRKState
from warpsph_b200.enumTypes import EnergyScheme

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "crk_pair_golden.npz"


@pytest.fixture(scope="module")
def G(cuda):
    g = dict(np.load(GOLD))
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in g.items()}, g


def adjacency(t):
    n = t["offsets"].shape[0]
    return AdjacencyList(neighborOffsets=t["offsets"], numNeighbors=t["counts"], neighborList=t["list"], numRows=n, numCols=n,
                         nnz=int(t["list"].shape[0]))


def test_gpu_golden_accel_dudt(G):
    t, g = G
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    crk = CRKState(A=t["A"], B=t["B"], gradA=t["gA"], gradB=t["gB"])
    dvdt, dudt, ap, av = ops.crk_accel_dudt(p, t["x"], t["H"], t["m"], t["rho"], t["V"], crk, t["v"], t["c"], t["P"], t["G"],
                                            adjacency(t))
    assert_close(ap.cpu().numpy(), g["ap"], 1e-4, 1e-5, "ap_ij vs reference accel.py (GPU)")
    assert_close(av.cpu().numpy(), g["av"], 1e-4, 1e-5, "av_ij vs reference accel.py (GPU)")
    assert_close(dvdt.cpu().numpy(), g["accel"], 1e-4, 1e-5, "dv/dt vs reference accel.py (GPU)")
    assert_close(dudt.cpu().numpy(), g["dudt"], 1e-4, 1e-5, "du/dt vs reference dudt.py (GPU)")


def test_gpu_golden_balance_vsig_eos_switch(G):
    t, g = G
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    adj = adjacency(t)
    dt = float(g["balance_dt"][0])
    for es in EnergyScheme:
        p.energy_scheme = es.value
        f = ops.compsph_balance(p, t["m"], t["rho"], t["P"], t["u"], t["v"], t["dvdt_guess"], dt, adj, t["ap"], t["av"])
        mism = np.mean(np.abs(f.cpu().numpy() - g["f_ij"][es.value]) > 1e-5)
        assert mism < 2e-3, (es, mism)   # dE rounding across zero can flip the branch of a few entries
    A, P, c = ops.eos_ideal_gas(p, t["u"], t["rho"])
    assert_close(P.cpu().numpy(), g["eos_P"], 1e-6, 1e-7, "P vs reference idealGas.py (GPU)")
    assert_close(c.cpu().numpy(), g["eos_c"], 1e-6, 1e-7, "c vs reference idealGas.py (GPU)")
    al, R, vs = ops.switch_cullen(p, t["x"], t["H"], t["m"], t["rho"], t["div"], t["cullen_div_prev"], None, t["cullen_alpha0"],
                                  1e-3, adj, want_R=True, v=t["v"], c=t["c"], want_vsig=True)
    assert_close(vs.cpu().numpy(), g["vsig"], 1e-5, 1e-6, "v_sig vs reference wp_vsig.py (GPU)")
    assert_close(R.cpu().numpy(), g["cullen_R"], 1e-4, 1e-5, "R vs reference CullenDehnen2010.py (GPU)")
    assert_close(al.cpu().numpy(), g["cullen_alpha"], 1e-4, 1e-5, "alpha vs reference CullenDehnen2010.py (GPU)")
    dtv = ops.cfl_dt(p, t["H"], t["u"], dt_prev=1e-4)
    assert abs(float(dtv.item()) - g["cfl_dt_grow"][0]) <= 1e-6 * g["cfl_dt_grow"][0]


@pytest.mark.parametrize("scheme", [EnergyScheme.CRK, EnergyScheme.PdV])
def test_gpu_golden_compatible_energy(G, scheme):
    t, g = G
    cfg, sch, p = make_params(2, kernel=core.KernelFunctions.Wendland4)
    p.energy_scheme = scheme.value
    adj = adjacency(t)
    stages = [(t["multistep_dvdt"][s].contiguous(), adj, t["f_ij"][5 if s == 0 else 0].contiguous(),
               (t["ap"] * (1 + 0.1 * s)).contiguous(), (t["av"] * (1 - 0.1 * s)).contiguous()) for s in range(2)]
    u, du = ops.finalize_compatible_energy(p, [0.5, 0.5], float(g["balance_dt"][0]), t["v"], t["u"], stages)
    assert_close(du.cpu().numpy(), g[f"multistep_du_{scheme.name}"], 1e-4, 1e-5, f"du vs reference multistep.py ({scheme.name}, GPU)")
