"""Stacks of sections on the GPU (vrc_chain, vrc_chain_order_powers,
vrc_chain_fields): a pillar section, a z-uniform pixel layer and another
pillar section between a substrate and air, each solved by adaptive
varRCWA, against the oracle's chain of the same sections replayed on the
device's segmentations (oracle/chain.py): Fourier-basis blocks, per-order
powers and the transverse fields at every interface to 1e-9, energy
conserved to 1e-10."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.chain import chain_amplitudes, chain_sections
from oracle.structures_adapter import end_bases, make_sampler
from tests.conftest import fourier_blocks, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _stack():
    from varrcwa_b200 import structures as st
    d1 = st.pillar_cell(2000, norders=5, lam=0.532, npix=32)
    d1.update(z1=0.3, end1=None)  # substrate below
    eps = np.where((np.arange(32)[None, :] - 16) ** 2 + (np.arange(32)[:, None] - 16) ** 2 < 81, 4.0, 1.0)
    lay = dict(kind="pixels", lam=0.532, nx=5, ny=5, pml=False, Lx=0.4, Ly=0.4, z0=0.3, z1=0.42, end0=None,
               end1=None, eps=eps.astype(np.complex128))
    d3 = st.pillar_cell(2001, norders=5, lam=0.532, npix=32)
    d3.update(z0=0.42, z1=1.0, end0=None)  # air above
    return [d1, lay, d3]


def test_chain_matches_oracle_blocks_powers_and_fields(ctx):
    ds = _stack()
    r = ctx.chain(ds, pe=1e-2)
    assert r["status"] == 0
    Ss = []
    for k, d in enumerate(ds):
        leaves = sorted((a, b) for (a, b, e, acc) in ctx.tree(k) if acc)
        cuts = [leaves[0][0]] + [b for (_, b) in leaves]
        s = make_sampler(d)
        e0, e1 = end_bases(d, s)
        Ss.append(O.redheffer_segments(s, d["z0"], d["z1"], cuts, end0=e0, end1=e1))
    T, _, _ = chain_sections(Ss)
    F, G = fourier_blocks(r), T.fourier_blocks()
    for k in F:
        assert relerr(F[k], G[k]) < TOL, k
    p = ctx.chain_order_powers(side=1)
    s0 = make_sampler(ds[0])
    for pol, (px, py) in enumerate(((1.0, 0.0), (0.0, 1.0))):
        R, Tr = O.order_powers(T, s0, ds[-1]["end1"], ds[0]["end0"], px, py, side="top")
        assert relerr(p["R"][pol], R) < TOL and relerr(p["T"][pol], Tr) < TOL
        # perturbative varRCWA sections (pe = 1e-2) conserve flux only to the
        # method's accuracy, the same for the oracle; stacks of z-uniform
        # sections conserve it to 1e-10 (test_oracle_chain.py)
        assert abs(p["R"][pol].sum() + p["T"][pol].sum() - (R.sum() + Tr.sum())) < 1e-9
        assert abs(p["R"][pol].sum() + p["T"][pol].sum() - 1.0) < 1e-3
    # interface fields for an incident entrance mode: the transverse E field
    # on a grid over the period does not depend on any basis choice
    n = r["W0"].shape[0]
    m = n // 2
    c_dev = np.linalg.solve(r["W0"], T.W0[:, 3])  # the oracle's entrance mode 3 in the device basis
    amps, img = ctx.chain_fields(c_dev, 8, 8)
    c_or = np.zeros(n, np.complex128)
    c_or[3] = 1.0
    oamps = chain_amplitudes(Ss, c_or)
    oW = [Ss[0].W0] + [S.W1 for S in Ss]
    sm = make_sampler(ds[0])
    alpha, beta = np.diag(sm.Kx).real, np.diag(sm.Ky).real
    xs, ys = 0.4 * np.arange(8) / 8, 0.4 * np.arange(8) / 8
    ph = np.exp(1j * (alpha[:, None, None] * xs[None, None, :] + beta[:, None, None] * ys[None, :, None]))
    for j in range(len(ds) + 1):
        e = oW[j] @ (oamps[j, 0] + oamps[j, 1])
        ex, ey = np.tensordot(e[:m], ph, axes=(0, 0)), np.tensordot(e[m:], ph, axes=(0, 0))
        assert relerr(img[j, 0], ex) < TOL and relerr(img[j, 1], ey) < TOL, j
    # entrance and exit amplitudes in the device's own end bases
    assert relerr(r["W0"] @ (amps[0, 0] + amps[0, 1]), oW[0] @ (oamps[0, 0] + oamps[0, 1])) < TOL
    assert relerr(r["W1"] @ amps[-1, 0], oW[-1] @ oamps[-1, 0]) < TOL
