"""Stacks of sections in the oracle (oracle/chain.py), pinned by known
answers: a cell cut into two sections at a segment boundary equals the whole
cell, and the internal amplitudes of a lossless periodic stack carry the
same z-power flux through every interface, equal to the transmitted power."""
import numpy as np

from oracle import varrcwa_oracle as O
from oracle.chain import chain_amplitudes, chain_sections
from oracle.structures_adapter import end_bases, make_sampler
from tests.cases import CASES


def _flux(W, V, ap, am):
    m = W.shape[0] // 2
    e, h = W @ (ap + am), V @ (ap - am)
    return float(np.real(np.vdot(h[m:], e[:m]) - np.vdot(h[:m], e[m:])))


def test_two_sections_equal_the_whole_cell():
    d = dict(CASES["asym_redheffer"]["desc"], end0=None, end1=None)
    s = make_sampler(d)
    cuts = [0.0, 0.3, 0.75, 1.1, 1.5]
    S = O.redheffer_segments(s, 0.0, 1.5, cuts)
    T, _, _ = chain_sections([O.redheffer_segments(s, 0.0, 0.75, cuts[:3]),
                              O.redheffer_segments(s, 0.75, 1.5, cuts[2:])])
    F, G = S.fourier_blocks(), T.fourier_blocks()
    for k in F:
        assert np.linalg.norm(F[k] - G[k]) <= 1e-12 * np.linalg.norm(F[k]), k


def test_interface_flux_is_conserved_in_a_lossless_stack():
    """Three z-uniform pixel sections (exact: a z-invariant section's
    perturbation vanishes) with half-spaces: the z-power flux of the fields
    W (a+ + a-), V (a+ - a-) is the same at every interface and equals the
    transmitted flux."""
    def layer(z0, z1, radius, eps_in, end0=None, end1=None):
        g = np.arange(16) - 7.5
        eps = np.where(g[None, :] ** 2 + g[:, None] ** 2 < radius ** 2, eps_in, 1.0).astype(np.complex128)
        return dict(kind="pixels", lam=0.532, nx=3, ny=3, pml=False, Lx=0.4, Ly=0.4, z0=z0, z1=z1, eps=eps,
                    end0=end0, end1=end1)
    ds = [layer(0.0, 0.2, 5.0, 5.8, end0=2.13), layer(0.2, 0.3, 7.0, 3.0), layer(0.3, 0.55, 3.0, 5.8, end1=1.0)]
    Ss = []
    for d in ds:
        s = make_sampler(d)
        e0, e1 = end_bases(d, s)
        Ss.append(O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-3, end0=e0, end1=e1))
        assert Ss[-1].N == 1
    n = Ss[0].W0.shape[0]
    c = np.zeros(n, np.complex128)
    c[4] = 1.0  # a propagating mode of the entrance medium
    amps = chain_amplitudes(Ss, c)
    Ws = [Ss[0].W0] + [S.W1 for S in Ss]
    Vs = [Ss[0].V0] + [S.V1 for S in Ss]
    fl = [_flux(W, V, a[0], a[1]) for W, V, a in zip(Ws, Vs, amps)]
    T, _, _ = chain_sections(Ss)
    trn = _flux(T.W1, T.V1, T.Tuu @ c, np.zeros(n))
    assert abs(fl[0]) > 0.1
    assert max(abs(f - trn) for f in fl) <= 1e-10 * abs(fl[0]), (fl, trn)
