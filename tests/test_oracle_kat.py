"""Known-answer tests pinning the CPU oracle (no GPU needed)."""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.structures_adapter import end_bases, make_sampler
from varrcwa_b200 import structures as st


def _slab(eps, nx=3, ny=3, lam=0.532):
    x = np.array([0.0, 0.15, 0.4])
    y = np.array([0.0, 0.2, 0.4])
    E = np.full((2, 2), eps, dtype=np.complex128)
    return O.VarLayerSampler(lam, nx, ny, x, y, E, enable_pml=False)


def test_homogeneous_pq_is_diagonal():
    # K2: homogeneous medium -> P Q = k0^2 (k0^2 eps - alpha^2 - beta^2) I
    s = _slab(2.13)
    P, Q = s.sample(0.0)
    a, b = O.alpha_beta(3, 3, 0.4, 0.4)
    k0 = s.k0
    d = k0 * k0 * (k0 * k0 * 2.13 - a * a - b * b)
    PQ = P @ Q
    assert np.abs(PQ - np.diag(np.concatenate([d, d]))).max() < 1e-9 * np.abs(PQ).max()


def test_z_invariant_varrcwa_is_pure_phase():
    # K1: z-invariant structure -> one segment, S = diag(exp(i gam dz / k0))
    s = _slab(5.8)
    S = O.redheffer_compute(s, 0.0, 0.3, pe=1e-3)
    assert S.N == 1
    ph = np.exp(1j * S.gam1 * 0.3 / s.k0)
    assert np.abs(S.Tuu - np.diag(ph)).max() < 1e-12
    assert np.abs(S.Rdu).max() < 1e-12 and np.abs(S.Rud).max() < 1e-12


@pytest.mark.parametrize("side", ["bottom", "top"])
def test_thin_film_fresnel(side):
    # analytic thin film between two half-spaces at normal incidence
    lam, d = 0.532, 0.2
    e1, e2, e3 = 2.13, 5.8, 1.0
    s = _slab(e2, lam=lam)
    b1, b3 = O.homogeneous_basis(s, e1), O.homogeneous_basis(s, e3)
    S = O.redheffer_compute(s, 0.0, d, pe=1e-3, end0=b1, end1=b3)
    n1, n2, n3 = np.sqrt([e1, e2, e3])
    if side == "top":
        n1, n3 = n3, n1
    k0 = 2 * np.pi / lam
    r12, r23 = (n1 - n2) / (n1 + n2), (n2 - n3) / (n2 + n3)
    t12, t23 = 2 * n1 / (n1 + n2), 2 * n2 / (n2 + n3)
    p = np.exp(1j * n2 * k0 * d)
    r = (r12 + r23 * p * p) / (1 + r12 * r23 * p * p)
    t = t12 * t23 * p / (1 + r12 * r23 * p * p)
    ein, eout = (e1, e3) if side == "bottom" else (e3, e1)
    R, T = O.order_powers(S, s, ein, eout, 1.0, 0.0, side=side)
    assert abs(R.sum() - abs(r) ** 2) < 1e-12
    assert abs(T.sum() - abs(t) ** 2 * n3 / n1) < 1e-12


def test_rcwa_energy_conservation_grating():
    # K3: lossless periodic grating, plain RCWA conserves energy exactly
    d = st.pillar_cell(2001, norders=5, lam=0.532, npix=32)
    s = make_sampler(d)
    e0, e1 = end_bases(d, s)
    S = O.rcwa_compute(s, d["z0"], d["z1"], 3, end0=e0, end1=e1)
    for side, (ein, eout) in (("bottom", (d["end0"], d["end1"])), ("top", (d["end1"], d["end0"]))):
        for pol in ((1.0, 0.0), (0.0, 1.0)):
            R, T = O.order_powers(S, s, ein, eout, *pol, side=side)
            assert abs(R.sum() + T.sum() - 1.0) < 1e-10


def test_z_invariant_varrcwa_equals_rcwa():
    d = st.pillar_cell(2002, norders=3, lam=0.532, npix=16)
    d["r1"] = d["r0"]
    s = make_sampler(d)
    e0, e1 = end_bases(d, s)
    A = O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-3, end0=e0, end1=e1).fourier_blocks()
    B = O.rcwa_compute(s, d["z0"], d["z1"], 1, end0=e0, end1=e1).fourier_blocks()
    for k in A:
        assert np.linalg.norm(A[k] - B[k]) <= 1e-10 * np.linalg.norm(B[k])


def test_varrcwa_converges_to_rcwa():
    # K4: tightening pe moves varRCWA towards a fine RCWA reference
    d = dict(st.taper_2d(norders=7, length=1.0))
    s = make_sampler(d)
    ref = O.rcwa_compute(s, 0.0, 1.0, 256).fourier_blocks()["Tuu"]
    errs = []
    for pe in (1e-2, 1e-4):
        F = O.redheffer_compute(s, 0.0, 1.0, pe=pe).fourier_blocks()["Tuu"]
        errs.append(np.abs(F - ref).max())
    assert errs[1] < errs[0]
    assert errs[1] < 1e-3


def test_refill_matches_sorted_geometry():
    # crossing coordinates refilled in painter's order equal the explicit
    # sorted geometry for the Laurent (e33) coefficients
    x = np.array([0.0, 0.3, 1.1, 0.8, 1.6, 2.0])
    y = np.array([0.0, 1.0])
    f = np.array([[2.0, 3.0, 4.0, 5.0, 2.0]], dtype=np.complex128)
    F = O.fourier_solve_2d(x, y, f, 3, 1, O.CONTINUOUS_XY)
    assert np.all(np.isfinite(F))


def test_pml_factors_without_pml_regions_are_identity():
    # Zero-width PML regions (l0 = l1, r0 = r1, b0 = b1, u0 = u1) leave the
    # coordinate unstretched: Fx = Fy = I exactly.
    nx = ny = 5
    Lx, Ly = 4.0, 2.0
    gamma = 1.0 / (1.0 - 1.0j)
    Fx, Fy = O.pml_factors(nx, ny, gamma, 0.0, 0.0, Ly, Ly, 0.0, 0.0, Lx, Lx, Lx, Ly)
    assert np.abs(Fx - np.eye(nx * ny)).max() < 1e-12
    assert np.abs(Fy - np.eye(nx * ny)).max() < 1e-12


def test_pml_factors_damp_with_complex_stretch():
    # With PML regions the stretch factor of the DC term has a negative
    # imaginary part proportional to the PML width (absorbing layers).
    nx = ny = 3
    x = np.array([0.0, 0.5, 1.5, 2.5, 3.5, 4.0])
    y = np.array([0.0, 0.5, 0.9, 1.1, 1.5, 2.0])
    gamma = 1.0 / (1.0 - 1.0j)
    Fx, Fy = O.pml_factors(nx, ny, gamma, y[0], y[1], y[-2], y[-1], x[0], x[1], x[-2], x[-1], 4.0, 2.0)
    assert np.all(np.isfinite(Fx)) and np.all(np.isfinite(Fy))
    c = (nx * ny) // 2
    assert Fx[c, c].imag != 0.0 and Fy[c, c].imag != 0.0


@pytest.mark.parametrize("method", ["redheffer", "rcwa"])
def test_z_mirror_symmetry(method):
    """A structure symmetric under z -> L - z between identical half-spaces:
    the up- and down-going blocks coincide in the Fourier basis (Tuu = Tdd,
    Rdu = Rud), for varRCWA (its trisection tree and Simpson segments are
    mirror symmetric) and for RCWA."""
    L = 2.0
    zs = np.linspace(0.0, L, 9)
    w = 0.4 + 0.5 * 4.0 * zs * (L - zs) / L ** 2      # symmetric width profile
    c = 0.75
    x = np.array([0.0, c - 0.2, c + 0.2, 1.5])
    eps = np.array([[2.085, 12.11, 2.085]], dtype=np.complex128)
    s = O.VarLayerSampler(1.55, 7, 1, x, np.array([0.0, 1.0]), eps, enable_pml=False)
    s.add_x_rule(1, lambda z: float(np.interp(z, zs, c - 0.5 * w)))
    s.add_x_rule(2, lambda z: float(np.interp(z, zs, c + 0.5 * w)))
    e = O.homogeneous_basis(s, 2.085)
    if method == "redheffer":
        S = O.redheffer_compute(s, 0.0, L, pe=1e-4, end0=e, end1=e)
    else:
        S = O.rcwa_compute(s, 0.0, L, 12, end0=e, end1=e)
    F = S.fourier_blocks()
    scale = np.linalg.norm(F["Tuu"])
    assert np.linalg.norm(F["Tuu"] - F["Tdd"]) <= 1e-10 * scale
    assert np.linalg.norm(F["Rdu"] - F["Rud"]) <= 1e-10 * scale
