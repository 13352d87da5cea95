"""The oracle reproduces the committed golden fixtures (guards drift)."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.structures_adapter import end_bases, make_sampler
from tests.cases import CASES
from tests.conftest import golden, relerr


@pytest.mark.parametrize("name", [k for k, v in CASES.items() if "pq_z" in v])
def test_oracle_pq_matches_golden(name):
    case = CASES[name]
    g = golden(name)
    s = make_sampler(case["desc"])
    for k, z in enumerate(case["pq_z"]):
        P, Q = s.sample(z)
        assert relerr(P, g["P"][k]) < 1e-13
        assert relerr(Q, g["Q"][k]) < 1e-13


@pytest.mark.parametrize("name", ["pillar_rcwa", "asym_diff", "pillar_redheffer", "asym_redheffer"])
def test_oracle_smatrix_matches_golden(name):
    case = CASES[name]
    d = case["desc"]
    g = golden(name)
    s = make_sampler(d)
    e0, e1 = end_bases(d, s)
    if case["method"] == "rcwa":
        S = O.rcwa_compute(s, d["z0"], d["z1"], case["N"], end0=e0, end1=e1)
    elif case["method"] == "differential":
        S = O.differential_compute(s, d["z0"], d["z1"], case["N"], end0=e0, end1=e1)
    else:
        S = O.redheffer_compute(s, d["z0"], d["z1"], pe=case["pe"], end0=e0, end1=e1)
        assert S.N == int(g["N"])
    F = S.fourier_blocks()
    for k in F:
        assert relerr(F[k], g["F_" + k]) < 1e-11


def test_oracle_stack_adjoint_matches_golden():
    """The layer-stack forward and its pixel / thickness gradients reproduce
    the committed fixture (guards the adjoint oracle against drift)."""
    from oracle.stack_adjoint import Stack, order_index, stack_backward, stack_forward
    g = golden("stack_small")
    st = Stack(0.633, 3, 3, 0.6, 0.6, list(g["layers"]), [0.15, 0.2], eps_in=1.0, eps_out=2.085)
    R, T, tp = stack_forward(st)
    assert np.abs(R - g["R"]).max() < 1e-13 and np.abs(T - g["T"]).max() < 1e-13
    wT = np.zeros(9)
    wT[order_index(3, 3, 1, 0)] = 1.0
    gr, gt = stack_backward(st, tp, np.zeros(9), wT, want_thick=True)
    assert relerr(np.array(gr), g["grad"]) < 1e-11
    assert relerr(gt, g["grad_thick"]) < 1e-11
