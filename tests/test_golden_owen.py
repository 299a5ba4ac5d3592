"""The Owen adaptive support on the CPU: the library's n_h(psi_H) table against the
reference's own table generator, and the oracle's support iteration against the
reference's psi0 pair body, table lookup and support update (tests/golden/owen_golden.npz,
made by tests/golden/make_golden.py --which owen from modules/adaptiveSupport/wp_psi.py,
wp_psi0.py, owenLUT.py and optimalSupportOwen.py)."""
from pathlib import Path

import numpy as np
import pytest

import warpsph_b200 as ws
from oracle import oracle
from tests.cases import assert_close, make_params
from warpsph_b200.owen import owen_table

GOLD = Path(__file__).resolve().parent / "golden" / "owen_golden.npz"


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


@pytest.mark.parametrize("kernel,dim", [(1, 1), (2, 2), (2, 3)])
def test_owen_table_matches_reference_generator(gold, kernel, dim):
    nh, psiH = owen_table(ws.KernelFunctions(kernel), dim)
    assert len(nh) == 4096 and nh[0] == 2.0 and abs(nh[-1] - 6.0) < 1e-5
    assert np.all(np.diff(psiH) > 0), "psi_H must increase with n_h for the lookup"
    sel = gold[f"owen_lut_sel_k{kernel}_d{dim}"]
    np.testing.assert_array_equal(nh[sel], gold[f"owen_lut_nh_k{kernel}_d{dim}"])
    assert_close(psiH[sel], gold[f"owen_lut_psiH_k{kernel}_d{dim}"], 1e-6, 1e-7, "psi_H table vs reference wp_psi.py")


def test_owen_iteration_matches_reference(gold):
    g = gold
    cfg, sch, p = make_params(2, kernel=ws.KernelFunctions.Wendland4)
    nh, psiH = owen_table(ws.KernelFunctions.Wendland4, 2)
    nb = dict(offsets=g["owen_offsets"], counts=g["owen_counts"], list=g["owen_list"])
    H = g["owen_H"]
    hb = np.array([H.min(), H.max()], np.float32)
    psi0, psi0H, Hn, ratio = oracle.get("f32").owen_iter(p, g["owen_x"], H, nb, nh, psiH, float(g["owen_target"][0]), hb)
    assert_close(psi0, g["owen_psi0"], 1e-6, 1e-7, "psi0 vs reference wp_psi0.py")
    assert_close(psi0H, g["owen_psi0H"], 1e-6, 1e-7, "psi0_H vs reference wp_psi0.py")
    assert_close(Hn, g["owen_Hnew"], 1e-6, 1e-7, "new support vs reference optimalSupportOwen.py")
    assert_close(ratio, Hn / H, 1e-6, 1e-7, "ratio")
    assert np.abs(g["owen_Hnew"] / H - 1).max() > 1e-3          # the update actually moves the supports
