"""Geometric-parameter gradient of an adaptive varRCWA cell on its fixed
segmentation (oracle/segments_adjoint.py): the frozen-basis first-order
adjoint against central differences of the oracle's forward on the same cuts,
for a control knot inside the cell (the end cross-sections unchanged)."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.segments_adjoint import (end_bases_adjoint, end_basis_derivative, fourier_transmission_adjoint,
                                     segments_block_adjoints, segments_forward, segments_gradient)
from oracle.structures_adapter import make_sampler
from varrcwa_b200 import structures as st


@pytest.fixture(autouse=True, scope="module")
def _one_blas_thread():
    # the matrices here are small (n <= 50): threaded BLAS only adds overhead
    from threadpoolctl import threadpool_limits
    with threadpool_limits(1):
        yield


def _cell(knot):
    """Config-1 style taper (11 orders) whose right core edge has a middle
    control knot at z = L/2 of value `knot` (the ends stay at w0, w1)."""
    d = dict(st.taper_2d(norders=11))
    (i1, zs1, v1), (i2, zs2, v2) = d["xrules"]
    L = zs2[-1]
    d["xrules"] = [(i1, [0.0, 0.5 * L, L], [v1[0], 0.5 * (v1[0] + v1[1]), v1[1]]),
                   (i2, [0.0, 0.5 * L, L], [v2[0], knot, v2[1]])]
    return d


def test_interior_knot_gradient_matches_central_differences():
    knot, pe = 1.05, 1e-4
    d = _cell(knot)
    s = make_sampler(d)
    cuts = O.tree_cuts(O.redheffer_compute(s, d["z0"], d["z1"], pe=pe).nodes)
    fw = segments_forward(s, cuts)
    k = 5  # centre harmonic of the first polarisation block (nx = 11, ny = 1)
    J, gS = fourier_transmission_adjoint(fw, k)
    h = 1e-6
    sp, sm = make_sampler(_cell(knot + h)), make_sampler(_cell(knot - h))

    def dsample(z):
        Pp, Qp = sp.sample(z)
        Pm, Qm = sm.sample(z)
        return (Pp - Pm) / (2 * h), (Qp - Qm) / (2 * h)

    g = segments_gradient(fw, gS, dsample)

    def objective(kv):
        f = segments_forward(make_sampler(_cell(kv)), cuts)
        return fourier_transmission_adjoint(f, k)[0]

    hf = 1e-5
    fd = (objective(knot + hf) - objective(knot - hf)) / (2 * hf)
    # the frozen-basis gradient is the first-order derivative of the exact
    # propagation; it differs from the discrete forward's by the segments'
    # truncation (1.8e-6 at pe = 1e-6, 5.7e-6 here)
    assert abs(g - fd) <= 2e-5 * abs(fd), (g, fd)
    assert abs(J - objective(knot)) < 1e-14


def _cell_end(kv, which):
    """The taper with an off-centre middle knot; knot `which` (0: z0, 2: z1)
    of the right core edge takes the value kv."""
    d = dict(st.taper_2d(norders=11))
    (i1, zs1, v1), (i2, zs2, v2) = d["xrules"]
    L = zs2[-1]
    v = [v2[0], 0.5 * (v2[0] + v2[1]) + 0.05, v2[1]]
    v[which] = kv
    d["xrules"] = [(i1, [0.0, 0.5 * L, L], [v1[0], 0.5 * (v1[0] + v1[1]), v1[1]]), (i2, [0.0, 0.5 * L, L], v)]
    return d


@pytest.mark.parametrize("which", [0, 2])
def test_end_knot_gradient_with_end_basis_terms(which):
    """A knot that moves an end cross-section: the segment terms plus the
    derivative through that end's eigenbasis meet central differences."""
    base = st.taper_2d(norders=11)["xrules"][1][2]
    kv = (base[1] if which == 2 else base[0]) + 0.02
    d = _cell_end(kv, which)
    s = make_sampler(d)
    cuts = O.tree_cuts(O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-5).nodes)
    fw = segments_forward(s, cuts)
    k = 5
    J, gS, gW0o, gW1o = fourier_transmission_adjoint(fw, k, want_bases=True)
    _, gfirst = segments_block_adjoints(fw, gS, want_first=True)
    gends = end_bases_adjoint(fw, gS, gfirst, gW0o, gW1o)
    h = 1e-6
    sp, sm = make_sampler(_cell_end(kv + h, which)), make_sampler(_cell_end(kv - h, which))

    def dsample(z):
        Pp, Qp = sp.sample(z)
        Pm, Qm = sm.sample(z)
        return (Pp - Pm) / (2 * h), (Qp - Qm) / (2 * h)

    dW0, dV0 = end_basis_derivative(sp, sm, d["z0"], fw["b0"], h)
    dW1, dV1 = end_basis_derivative(sp, sm, d["z1"], fw["b1"], h)
    g = segments_gradient(fw, gS, dsample, end_terms=(gends, (dW0, dV0, dW1, dV1)))

    def objective(v):
        f = segments_forward(make_sampler(_cell_end(v, which)), cuts)
        return fourier_transmission_adjoint(f, k)[0]

    hf = 1e-5
    fd = (objective(kv + hf) - objective(kv - hf)) / (2 * hf)
    assert abs(g - fd) <= 2e-5 * abs(fd), (g, fd)


def _waveguide(widths):
    """PML waveguide mode converter (5 x 5 orders, six width control points
    over 3 um): the widths move both core edges."""
    d = dict(st.waveguide_pml(5000, norders=5, ncontrol=6, length=3.0))
    zs = d["xrules"][0][1]
    cx = 2.0
    w = np.asarray(widths, dtype=float)
    d["xrules"] = [(2, zs, cx - 0.5 * w), (3, zs, cx + 0.5 * w)]
    d["x"] = np.array(d["x"])
    d["x"][2], d["x"][3] = cx - 0.5 * w[0], cx + 0.5 * w[0]
    return d


@pytest.mark.parametrize("k", [2, 5])
def test_mode_conversion_gradient_pml_waveguide(k):
    """Config-5 style objective: power from the entrance's leading mode into
    another mode of the exit basis, flux normalised, with respect to a width
    control point (interior, and the exit one that moves the end basis)."""
    from oracle.segments_adjoint import H, mode_conversion_adjoint
    w = np.array(st.waveguide_pml(5000, norders=5, ncontrol=6, length=3.0)["widths"])
    d = _waveguide(w)
    s = make_sampler(d)
    cuts = O.tree_cuts(O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-4).nodes)
    fw = segments_forward(s, cuts)
    i0 = int(np.argmax(fw["b0"].gam.real))
    i1 = int(np.argsort(-fw["b1"].gam.real)[1])
    L, gS, gW0o, gV0o, gW1o, gV1o = mode_conversion_adjoint(fw, i0, i1)
    _, gfirst = segments_block_adjoints(fw, gS, want_first=True)
    gends = end_bases_adjoint(fw, gS, gfirst, gW0o, gW1o, gV0o, gV1o)
    h = 1e-6
    wp, wm = w.copy(), w.copy()
    wp[k] += h
    wm[k] -= h
    sp, sm = make_sampler(_waveguide(wp)), make_sampler(_waveguide(wm))

    def dsample(z):
        Pp, Qp = sp.sample(z)
        Pm, Qm = sm.sample(z)
        return (Pp - Pm) / (2 * h), (Qp - Qm) / (2 * h)

    dW0, dV0 = end_basis_derivative(sp, sm, d["z0"], fw["b0"], h)
    dW1, dV1 = end_basis_derivative(sp, sm, d["z1"], fw["b1"], h)
    g = segments_gradient(fw, gS, dsample, end_terms=(gends, (dW0, dV0, dW1, dV1)))

    def objective(widths):
        f = segments_forward(make_sampler(_waveguide(widths)), cuts)
        j0 = int(np.argmax(np.abs(H(f["b0"].W) @ fw["b0"].W[:, i0])))
        j1 = int(np.argmax(np.abs(H(f["b1"].W) @ fw["b1"].W[:, i1])))
        return mode_conversion_adjoint(f, j0, j1)[0]

    hf = 1e-5
    wp, wm = w.copy(), w.copy()
    wp[k] += hf
    wm[k] -= hf
    fd = (objective(wp) - objective(wm)) / (2 * hf)
    assert abs(g - fd) <= 1e-5 * abs(fd), (g, fd)


def test_checkpointed_reverse_pass_equals_full_tape():
    """Keeping only every 7th chain state and recomputing blocks on the way
    back gives the same per-segment adjoints as the full tape."""
    from oracle.segments_adjoint import segments_block_adjoints_checkpointed
    d = _cell(1.05)
    s = make_sampler(d)
    cuts = O.tree_cuts(O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-3).nodes)
    fw = segments_forward(s, cuts)
    _, gS = fourier_transmission_adjoint(fw, 5)
    full = segments_block_adjoints(fw, gS)
    ck = segments_block_adjoints_checkpointed(make_sampler(d), cuts, lambda f: fourier_transmission_adjoint(f, 5)[1], 7)
    assert len(full) == len(ck) == len(cuts) - 1
    for a, b in zip(full, ck):
        for x, y in zip(a, b):
            assert np.abs(x - y).max() <= 1e-12 * max(np.abs(x).max(), 1e-300)


def test_node_adjoints_are_the_transpose_of_the_segment_formula():
    from oracle.segments_adjoint import first_order_blocks, node_adjoints
    rng = np.random.default_rng(7)
    n = 12
    W = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    V = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    gam = rng.uniform(0.5, 2.0, n) + 1j * rng.uniform(0.0, 0.3, n)
    basis = O.Basis(W, V, gam)
    dP3 = [rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) for _ in range(3)]
    dQ3 = [rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) for _ in range(3)]
    g = [rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) for _ in range(4)]
    k0, a, b = 4.0, 0.3, 0.45
    lhs = sum(np.real(np.vdot(gi, di)) for gi, di in zip(g, first_order_blocks(basis, k0, a, b, dP3, dQ3)))
    rhs = sum(np.real(np.vdot(gp, dp) + np.vdot(gq, dq))
              for (gp, gq), dp, dq in zip(node_adjoints(basis, k0, a, b, g), dP3, dQ3))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_eig_adjoint_matches_central_differences_of_a_gauge_invariant_objective():
    """L = |(W diag(e^{i gam d}) W^-1)[k, k]|^2 + Re tr(V W^-1 C) does not
    depend on how the eigenvectors are scaled; its (P, Q) gradient from
    eig_adjoint against central differences."""
    from oracle.segments_adjoint import H, eig_adjoint
    d = _waveguide(np.array(st.waveguide_pml(5000, norders=5, ncontrol=6, length=3.0)["widths"]))
    s = make_sampler(d)
    P, Q = s.sample(0.7)
    rng = np.random.default_rng(3)
    n = P.shape[0]
    Cm = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    dd, k = 0.37, 4

    def obj(P_, Q_):
        W, V, gam = O.wave_equation_solve(P_, Q_)
        Wi = np.linalg.inv(W)
        T = W @ (np.exp(1j * gam * dd)[:, None] * Wi)
        return float(abs(T[k, k]) ** 2 + np.real(np.trace(V @ Wi @ Cm))), (W, V, gam)

    L, (W, V, gam) = obj(P, Q)
    Wi = np.linalg.inv(W)
    X = np.exp(1j * gam * dd)
    T = W @ (X[:, None] * Wi)
    gT = np.zeros((n, n), np.complex128)
    gT[k, k] = 2.0 * T[k, k]
    # T = W X W^-1 (X = diag(e^{i gam d})), and tr(V W^-1 C)
    gX = np.diag(H(W) @ gT @ H(Wi)).copy()
    gWi = H(W * X[None, :]) @ gT + H(Cm @ V)  # from T and from V W^-1 C
    gW = gT @ H(X[:, None] * Wi) - H(Wi) @ gWi @ H(Wi)
    gV = H(Wi @ Cm)
    ggam = np.conj(1j * dd * X) * gX  # T's explicit dependence on gam
    gP, gQ = eig_adjoint(P, Q, W, V, gam, gW, gV, ggam=ggam)
    for _ in range(3):
        dP = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        dQ = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        h = 1e-6 * np.linalg.norm(P) / np.linalg.norm(dP)
        fd = (obj(P + h * dP, Q + h * dQ)[0] - obj(P - h * dP, Q - h * dQ)[0]) / (2 * h)
        ad = float(np.real(np.vdot(gP, dP) + np.vdot(gQ, dQ)))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-3 * abs(L)), (ad, fd)


def test_knot_gradient_matches_parameter_gradient_and_central_differences():
    """The knot-level gradient (node adjoints, coordinate differences, the
    analytic end-basis adjoint) chained to the widths of the converter equals
    central differences of the objective on the same cuts."""
    from oracle.segments_adjoint import H, knot_gradient, mode_conversion_adjoint
    w = np.array(st.waveguide_pml(5000, norders=5, ncontrol=6, length=3.0)["widths"])
    d = _waveguide(w)
    s = make_sampler(d)
    cuts = O.tree_cuts(O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-4).nodes)
    fw = segments_forward(s, cuts)
    i0 = int(np.argmax(fw["b0"].gam.real))
    i1 = int(np.argsort(-fw["b1"].gam.real)[1])
    L, gS, gW0o, gV0o, gW1o, gV1o = mode_conversion_adjoint(fw, i0, i1)
    gl, gr = knot_gradient(d, cuts, gS, gW0o, gV0o, gW1o, gV1o)
    gw = -0.5 * gl + 0.5 * gr  # x_left = cx - w/2, x_right = cx + w/2

    def objective(widths):
        f = segments_forward(make_sampler(_waveguide(widths)), cuts)
        j0 = int(np.argmax(np.abs(H(f["b0"].W) @ fw["b0"].W[:, i0])))
        j1 = int(np.argmax(np.abs(H(f["b1"].W) @ fw["b1"].W[:, i1])))
        return mode_conversion_adjoint(f, j0, j1)[0]

    hf = 1e-5
    for k in (0, 2, 5):
        wp, wm = w.copy(), w.copy()
        wp[k] += hf
        wm[k] -= hf
        fd = (objective(wp) - objective(wm)) / (2 * hf)
        assert abs(gw[k] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gw).max()), (k, gw[k], fd)
