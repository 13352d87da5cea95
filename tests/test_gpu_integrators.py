"""GPU parity of the integrators (varRCWA, RCWA, differential) and of the
per-order powers against the CPU oracle.

S-matrix blocks are compared in the Fourier (plane-wave) basis
(W1 Tuu W0^-1, ...), which does not depend on the eigenvector ordering,
phase or the choice of basis inside degenerate eigenspaces.  Adaptive runs
are compared on the oracle's segmentation (replay); where the structure has
no degenerate modes the device's own adaptive tree is compared too."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.structures_adapter import end_bases, make_sampler
from tests.cases import CASES
from tests.conftest import fourier_blocks, golden, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-9  # relative, S-matrix blocks and order powers


def _check_blocks(r, g):
    assert r["status"] == 0
    F = fourier_blocks(r)
    for k in F:
        assert relerr(F[k], g["F_" + k]) < TOL, k


def test_rcwa_matches_oracle(ctx):
    case = CASES["pillar_rcwa"]
    r = ctx.rcwa([case["desc"]], case["N"])[0]
    _check_blocks(r, golden("pillar_rcwa"))
    assert r["N"] == case["N"]


def test_differential_matches_oracle(ctx):
    case = CASES["asym_diff"]
    r = ctx.differential([case["desc"]], case["N"])[0]
    _check_blocks(r, golden("asym_diff"))


@pytest.mark.parametrize("name", ["taper_redheffer", "pillar_redheffer", "asym_redheffer", "pml_redheffer"])
def test_redheffer_replay_matches_oracle(ctx, name):
    g = golden(name)
    r = ctx.redheffer_segments([CASES[name]["desc"]], [g["cuts"]])[0]
    assert r["N"] == len(g["cuts"]) - 1
    _check_blocks(r, g)


def test_redheffer_adaptive_tree_matches_oracle(ctx):
    # no degenerate modes: the error estimate is basis-independent, so the
    # device reproduces the oracle's accept/reject decisions
    name = "asym_redheffer"
    case = CASES[name]
    g = golden(name)
    r = ctx.redheffer([case["desc"]], pe=case["pe"])[0]
    tree = {(round(a, 12), round(b, 12)): (e, acc) for (a, b, e, acc) in ctx.tree(0)}
    pe = case["pe"]
    for a, b, e, acc in g["nodes"]:
        key = (round(a, 12), round(b, 12))
        assert key in tree, key
        eg, accg = tree[key]
        assert abs(eg - e) <= 1e-6 * max(e, pe)
        if abs(e / pe - 1.0) > 1e-6:
            assert accg == bool(acc)
    assert r["N"] == int(g["N"])
    _check_blocks(r, g)


def test_order_powers_rcwa(ctx):
    case = CASES["pillar_rcwa"]
    g = golden("pillar_rcwa")
    for side in (0, 1):
        p = ctx.order_powers([case["desc"]], method="rcwa", nslices=case["N"], side=side)[0]
        assert p["status"] == 0
        for pol in (0, 1):
            R, T = p["R"][pol], p["T"][pol]
            assert relerr(R, g[f"R_{side}_{pol}"]) < TOL
            assert relerr(T, g[f"T_{side}_{pol}"]) < TOL
            assert abs(R.sum() + T.sum() - 1.0) < 1e-10  # lossless


def test_order_powers_varrcwa_replay(ctx):
    # powers from the device adaptive run vs the oracle's on the same tree
    name = "asym_redheffer"
    case = CASES[name]
    g = golden(name)
    p = ctx.order_powers([case["desc"]], method="redheffer", pe=case["pe"], side=1)[0]
    for pol in (0, 1):
        assert relerr(p["R"][pol], g[f"R_1_{pol}"]) < TOL
        assert relerr(p["T"][pol], g[f"T_1_{pol}"]) < TOL


def test_batched_uneven_sizes_match_single_calls(ctx):
    from varrcwa_b200 import structures as st
    descs = [st.pillar_cell(3000 + i, norders=o, npix=16, lam=0.5 + 0.03 * i) for i, o in enumerate([3, 5, 3, 7])]
    batch = ctx.redheffer(descs, pe=1e-2)
    for d, rb in zip(descs, batch):
        r1 = ctx.redheffer([d], pe=1e-2)[0]
        assert rb["N"] == r1["N"]
        for k in ("Tuu", "Tdd", "Rud", "Rdu"):
            assert np.allclose(rb[k], r1[k], rtol=0, atol=1e-13 * np.abs(r1[k]).max())


def test_invalid_arguments_are_rejected(ctx):
    from varrcwa_b200.capi import VrcError
    d = dict(CASES["asym_redheffer"]["desc"])
    d["nx"] = 4  # even harmonic count
    with pytest.raises(VrcError) as e:
        ctx.redheffer([d], pe=1e-2)
    assert e.value.status == 1
    with pytest.raises(VrcError):
        ctx.redheffer([CASES["asym_redheffer"]["desc"]], pe=-1.0)


def test_lanes_match_one_engine(ctx, monkeypatch):
    """A call on many cells is split over concurrent engines (lanes); every
    cell's arithmetic is the same as on one engine, so results agree bit for
    bit, in call order, with the trees kept per cell."""
    from varrcwa_b200 import structures as st
    cells = [st.pillar_cell(2100 + i, norders=3, lam=0.532, npix=32) for i in range(8)]
    out = {}
    for lanes in ("1", "3"):
        monkeypatch.setenv("VRC_LANES", lanes)
        out[lanes] = (ctx.order_powers(cells, method="redheffer", pe=1e-2, side=1),
                      ctx.redheffer(cells, pe=1e-2), [ctx.tree(c) for c in range(len(cells))])
    for a, b in zip(out["1"][0], out["3"][0]):
        assert np.array_equal(a["R"], b["R"]) and np.array_equal(a["T"], b["T"])
    for a, b in zip(out["1"][1], out["3"][1]):
        for k in ("Tdd", "Tuu", "Rud", "Rdu"):
            assert np.array_equal(a[k], b[k])
        assert a["N"] == b["N"]
    assert out["1"][2] == out["3"][2]


def test_planar_gds_cell_matches_oracle(ctx):
    """A planar (GDS-style) taper seen from above: per-z cross-sections with
    a varying number of x cells, PML on all four sides.  P, Q against the
    oracle's GDSIISampler restatement, then adaptive varRCWA against the
    oracle replayed on the device's tree."""
    from oracle.structures_adapter import make_sampler
    from varrcwa_b200 import structures as st
    d = st.planar_taper(norders=(7, 3))
    zs = [0.3, 0.5, 1.7, 2.9, 4.5, 4.6]
    P, Q = ctx.sample_pq(d, zs)
    s = make_sampler(d)
    for k, z in enumerate(zs):
        oP, oQ = s.sample(z)
        assert relerr(P[k], oP) < 1e-12 and relerr(Q[k], oQ) < 1e-12, z
    r = ctx.redheffer([d], pe=1e-2)[0]
    assert r["status"] == 0 and r["N"] >= 1
    leaves = sorted((a, b) for (a, b, e, acc) in ctx.tree(0) if acc)
    cuts = [leaves[0][0]] + [b for (_, b) in leaves]
    S = O.redheffer_segments(s, d["z0"], d["z1"], cuts)
    F, G = fourier_blocks(r), S.fourier_blocks()
    for k in F:
        assert relerr(F[k], G[k]) < TOL, k
