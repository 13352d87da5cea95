"""Checks at the benchmark configurations' full sizes (GPU), through
properties that do not need the oracle to run at that size, plus one
full-size replay against the oracle.

* config 2 (11x11 orders, n = 242, 256x256 raster) and the largest config-3
  truncation (15x15, n = 450): lossless RCWA conserves energy,
  |sum R + sum T - 1| < 1e-10 for both polarisations and both sides;
* config 2 adaptive varRCWA: the device's own tree replayed in the oracle
  gives the same Fourier-basis S-matrix blocks (1e-9 relative);
* a batch solved in one call equals the same cells solved one per call."""
import numpy as np
import pytest

from tests.conftest import fourier_blocks, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("norders,nslices", [(11, 6), (15, 3)])
def test_full_size_rcwa_conserves_energy(ctx, norders, nslices):
    from varrcwa_b200 import structures as st
    d = st.pillar_cell(3100 + norders, norders=norders, lam=0.55, npix=256)
    for side in (0, 1):
        p = ctx.order_powers([d], method="rcwa", nslices=nslices, side=side)[0]
        assert p["status"] == 0
        for pol in (0, 1):
            assert abs(p["R"][pol].sum() + p["T"][pol].sum() - 1.0) < 1e-10, (side, pol)


def test_full_size_varrcwa_matches_oracle_on_device_tree(ctx):
    from oracle import varrcwa_oracle as O
    from oracle.structures_adapter import end_bases, make_sampler
    from varrcwa_b200 import structures as st
    d = st.pillar_config2(seed=2000)
    r = ctx.redheffer([d], pe=1e-2)[0]
    assert r["status"] == 0
    cuts = sorted({a for (a, b, e, acc) in ctx.tree(0) if acc} | {d["z1"]})
    assert len(cuts) - 1 == r["N"]
    s = make_sampler(d)
    e0, e1 = end_bases(d, s)
    S = O.redheffer_segments(s, d["z0"], d["z1"], cuts, end0=e0, end1=e1)
    F, G = fourier_blocks(r), S.fourier_blocks()
    for k in F:
        assert relerr(F[k], G[k]) < 1e-9, k


def test_full_size_batch_equals_single_calls(ctx):
    from varrcwa_b200.replicas import make_cells
    cells = make_cells("c2", 3, 0, 256)
    pb = ctx.order_powers(cells, method="redheffer", pe=1e-2, side=1)
    for d, b in zip(cells, pb):
        p1 = ctx.order_powers([d], method="redheffer", pe=1e-2, side=1)[0]
        for pol in (0, 1):
            assert np.array_equal(b["R"][pol], p1["R"][pol]) and np.array_equal(b["T"][pol], p1["T"][pol])


def test_config1_taper_at_its_tolerance(ctx):
    # config 1 at full size: 41 orders (n = 82), pe = 1e-6, thousands of
    # segments.  The oracle replay of that tree takes minutes on the CPU, so
    # the full-size run is checked against the device's plain RCWA with
    # N = 1000 and 4000 slices: the transmission blocks converge to the
    # varRCWA result at the slab method's second order.  (Parity with the
    # oracle on the same structure is tested at pe = 1e-4.)
    from varrcwa_b200 import structures as st
    d = st.taper_2d()
    r = ctx.redheffer([d], pe=1e-6)[0]
    assert r["status"] == 0 and r["n"] == 82 and r["N"] > 1000
    F = fourier_blocks(r)
    err = {}
    for N in (1000, 4000):
        G = fourier_blocks(ctx.rcwa([d], N)[0])
        err[N] = max(relerr(F[k], G[k]) for k in ("Tuu", "Tdd"))
    assert err[4000] < 1e-5
    assert err[4000] < err[1000] / 8  # O(1/N^2) convergence onto the varRCWA result
