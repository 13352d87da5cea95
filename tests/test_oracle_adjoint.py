"""The oracle's layer-stack forward and adjoint: the forward against the
oracle's RCWA integrator, the adjoint against central finite differences
(also through a homogeneous layer, whose eigenvalues are degenerate)."""
import numpy as np
import pytest

from oracle.stack_adjoint import Stack, order_index, stack_backward, stack_forward
from varrcwa_b200.structures import smooth_pixels
from oracle.varrcwa_oracle import homogeneous_basis, order_powers, rcwa_compute

LAM, PER = 0.633, 0.6


def _stack(layers, thick, nx=3):
    return Stack(LAM, nx, nx, PER, PER, layers, thick, eps_in=1.0, eps_out=2.085)


def _objective(st, wR, wT):
    R, T, _ = stack_forward(st)
    return float(np.dot(wR, R) + np.dot(wT, T))


def _fd_check(layers, thick, picks, wR, wT, h=1e-4, nx=3):
    st = _stack(layers, thick, nx)
    _, _, tp = stack_forward(st)
    g = stack_backward(st, tp, wR, wT)
    gmax = max(np.abs(a).max() for a in g)
    for (l, i, j) in picks:
        vals = []
        for s in (1.0, -1.0):
            lay = [a.copy() for a in layers]
            lay[l][i, j] += s * h
            vals.append(_objective(_stack(lay, thick, nx), wR, wT))
        fd = (vals[0] - vals[1]) / (2 * h)
        # central difference with h = 1e-4: truncation ~1e-9 of the gradient scale
        assert abs(fd - g[l][i, j]) <= 1e-6 * gmax, (l, i, j, fd, g[l][i, j])
    return g


def test_stack_forward_matches_rcwa_integrator():
    layers = [smooth_pixels(4000 + l, 8, 8, sigma=1.0) for l in range(3)]
    st = _stack(layers, [0.15] * 3)
    R, T, _ = stack_forward(st)
    smp = st.sampler()
    S = rcwa_compute(smp, 0.0, 0.45, 3, end0=homogeneous_basis(smp, 1.0), end1=homogeneous_basis(smp, 2.085))
    R2, T2 = order_powers(S, smp, 1.0, 2.085, 1.0, 0.0, side="bottom")
    assert np.abs(R - R2).max() < 1e-11 and np.abs(T - T2).max() < 1e-11
    assert abs(R.sum() + T.sum() - 1.0) < 1e-10


def test_adjoint_matches_central_differences():
    layers = [smooth_pixels(4100 + l, 8, 8, sigma=1.0) for l in range(2)]
    wT = np.zeros(9)
    wT[order_index(3, 3, 1, 0)] = 1.0
    rng = np.random.default_rng(7)
    picks = [(int(rng.integers(2)), int(rng.integers(8)), int(rng.integers(8))) for _ in range(6)]
    _fd_check(layers, [0.15, 0.15], picks, np.zeros(9), wT)


def test_adjoint_reflection_and_transmission_weights():
    layers = [smooth_pixels(4200, 6, 8, sigma=1.0)]
    wR = np.linspace(0.1, 0.9, 9)
    wT = np.linspace(1.0, -1.0, 9)
    _fd_check(layers, [0.2], [(0, 0, 0), (0, 3, 5), (0, 7, 1)], wR, wT)


def test_adjoint_through_degenerate_eigenvalues():
    layers = [smooth_pixels(4001, 8, 8, sigma=1.0), np.full((8, 8), 4.0)]
    st = _stack(layers, [0.15, 0.2])
    _, _, tp = stack_forward(st)
    gam = np.sort_complex(tp.bases[1].gam)
    assert np.min(np.abs(np.diff(gam))) < 1e-12  # the homogeneous layer is degenerate
    wT = np.zeros(9)
    wT[order_index(3, 3, 1, 0)] = 1.0
    _fd_check(layers, [0.15, 0.2], [(1, 0, 0), (1, 3, 5), (0, 2, 2)], np.zeros(9), wT)


@pytest.mark.parametrize("seed", [1, 2])
def test_smooth_pixels_range(seed):
    p = smooth_pixels(seed, 64, 64)
    assert p.shape == (64, 64) and p.min() >= 2.085 and p.max() <= 12.11
    assert p.max() - p.min() > 5.0


def test_thickness_gradient_matches_central_differences():
    layers = [smooth_pixels(4600 + l, 8, 8, sigma=1.0) for l in range(3)]
    thick = [0.12, 0.2, 0.15]
    wR = np.linspace(0.2, 0.0, 9)
    wT = np.zeros(9)
    wT[order_index(3, 3, 1, 0)] = 1.0
    st = _stack(layers, thick)
    _, _, tp = stack_forward(st)
    _, gt = stack_backward(st, tp, wR, wT, want_thick=True)
    # fourth-order central differences: the objective oscillates with the
    # thickness on the scale k0 / gamma ~ 0.03 um, so a second-order stencil
    # would need h ~ 1e-6 and meet rounding there
    h = 1e-4
    for l in range(3):
        vals = []
        for s in (2.0, 1.0, -1.0, -2.0):
            t2 = list(thick)
            t2[l] += s * h
            vals.append(_objective(_stack(layers, t2), wR, wT))
        fd = (8.0 * (vals[1] - vals[2]) - (vals[0] - vals[3])) / (12.0 * h)
        assert abs(fd - gt[l]) <= 1e-7 * np.abs(gt).max(), (l, fd, gt[l])


def test_internal_fields_conserve_flux():
    """The amplitudes at every interface carry the same z-power flux,
    Re sum(ex conj(hy) - ey conj(hx)) over the harmonics, equal to the
    transmitted power (lossless stack), and the field images are the
    harmonic sums on the period grid."""
    from oracle.stack_adjoint import stack_fields
    layers = [smooth_pixels([5000, l], 8, 8, sigma=1.0) for l in range(3)]
    st = Stack(LAM, 3, 3, PER, PER, layers, [0.15, 0.1, 0.2], eps_in=1.0, eps_out=2.085)
    R, T, tp = stack_forward(st)
    amps, e, h, f = stack_fields(st, tp, 6, 5)
    m = 9
    flux = [np.real(np.vdot(h[j, m:], e[j, :m]) - np.vdot(h[j, :m], e[j, m:])) for j in range(4)]
    assert np.ptp(flux) < 1e-12 and abs(flux[0] - T.sum()) < 1e-12 and abs(1 - R.sum() - flux[0]) < 1e-12
    assert f.shape == (4, 2, 5, 6)
    # the centre pixel-free check: the mean of Ex over the period is the zero harmonic
    k0 = (3 * (3 - 1)) // 2 + (3 - 1) // 2
    np.testing.assert_allclose(f[:, 0].mean(axis=(1, 2)), e[:, k0], rtol=0, atol=1e-13)
