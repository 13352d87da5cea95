"""GPU P,Q assembly (Fourier/Toeplitz/Li rule, periodic and PML) vs the oracle."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.structures_adapter import make_sampler
from tests.cases import CASES
from tests.conftest import golden, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("name", [k for k, v in CASES.items() if "pq_z" in v])
def test_pq_matches_golden(ctx, name):
    case = CASES[name]
    g = golden(name)
    P, Q = ctx.sample_pq(case["desc"], case["pq_z"])
    for k in range(len(case["pq_z"])):
        assert relerr(P[k], g["P"][k]) < TOL
        assert relerr(Q[k], g["Q"][k]) < TOL


def test_pq_full_size_pillar_raster(ctx):
    # 11x11 orders on the 256x256 raster (the config-2 cell)
    from varrcwa_b200 import structures as st
    d = st.pillar_config2()
    s = make_sampler(d)
    P, Q = ctx.sample_pq(d, [0.3])
    Po, Qo = s.sample(0.3)
    assert relerr(P[0], Po) < TOL and relerr(Q[0], Qo) < TOL


def test_wave_solve_basis_invariants(ctx):
    g = golden("pillar_pq")
    P, Q = g["P"][0], g["Q"][0]
    W, V, gam = ctx.wave_solve(P, Q)
    PQ = P @ Q
    assert np.abs(PQ @ W - W * (gam * gam)[None, :]).max() < 1e-12 * np.abs(PQ).max()
    assert np.abs(V - (Q @ W) / gam[None, :]).max() < 1e-12 * np.abs(V).max()
    # same propagation constants as zgeev + the reference branch rule
    _, _, go = O.wave_equation_solve(P, Q)
    assert max(np.abs(go - x).min() for x in gam) < 1e-10 * np.abs(go).max()
    assert np.all(gam.imag >= -1e-12 * np.abs(gam).max())
