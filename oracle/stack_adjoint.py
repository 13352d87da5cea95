"""CPU restatement of the layer-stack forward solve and its adjoint.

TEST INFRASTRUCTURE ONLY: the GPU path never imports this module; tests and
the benchmark's CPU baseline use it as the checker.

Structure: L z-uniform layers, each a uniform pixel raster of permittivity
on a (Lx, Ly) period, between a homogeneous medium eps_in (below, z0) and
eps_out (above).  Layer l spans thickness d_l.

Forward (the Redheffer chain of src/core/RedhefferIntegrator.cpp:174-277 for
a piecewise-constant structure): for a z-uniform layer the perturbative
segment of RedhefferIntegrator.cpp:317-399 has zero perturbation, so the
layer's S-matrix in its own eigenbasis is (tdd, tuu, rud, rdu) =
(X, X, 0, 0), X = diag(exp(i gamma d / k0)).  Each layer is re-expressed at
its left end in the previous layer's basis (RedhefferIntegrator.cpp:253-262),
star-multiplied (:267-277), and the chain's right end is finally moved to the
exit medium (:211-223).  P, Q follow Layer::waveEqnCoeff
(src/rcwa/Layer.cpp:36-171) on the pixel grid; per-order powers follow
RCWASolver::scatterPlaneWave (src/rcwa/RCWASolver.cpp:1636-1733).

Adjoint: with every basis held fixed (a fixed basis re-expresses the same
S-matrix exactly), a perturbation (dP, dQ) of layer l changes only that
layer's own-basis blocks, by the first-order term of the perturbative
segment with the z-integrals done exactly instead of by Simpson's rule:

    dtuu = dtdd = K_E o (W^-1 dP V + V^-1 dQ W)
    drud = drdu = -K_D o (W^-1 dP V - V^-1 dQ W)
    K_E[i,j] = i/(2 k0) * int_0^d exp(i (g_i (d - z) + g_j z) / k0) dz
    K_D[i,j] = i/(2 k0) * int_0^d exp(i (g_i + g_j) z / k0) dz

(divided differences of exponentials; equal or nearly equal eigenvalues take
the series form, so degenerate modes need no special treatment).  The
adjoint of the star-product chain, the projections and the Toeplitz
assembly (Laurent rule for e33, Li's inverse rule for e11 / e22,
src/rcwa/FourierSolver2D.cpp:43-349) is written out step by step below.

Complex gradients use the convention dL = Re(sum(conj(G) * dZ)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from .varrcwa_oracle import (
    PI, Basis, RasterSampler, fourier_matrix_1d, fourier_solve_2d, homogeneous_basis, k_matrices,
    project_left, project_right, star_right, toeplitz_dense, wave_equation_solve, wave_eqn_coeff,
    DISCONTINUOUS_X, DISCONTINUOUS_Y, CONTINUOUS_XY,
)


def H(a):
    return a.conj().T


@dataclass
class Stack:
    lam: float
    nx: int
    ny: int
    Lx: float
    Ly: float
    layers: List[np.ndarray]          # each (npy, npx) permittivity raster
    thick: List[float]
    eps_in: complex = 1.0
    eps_out: complex = 1.0

    def sampler(self):
        z = np.concatenate([[0.0], np.cumsum(self.thick)])
        layers = self.layers

        def raster(zq):
            i = int(np.searchsorted(z, zq, side="right") - 1)
            return layers[min(max(i, 0), len(layers) - 1)]

        return RasterSampler(self.lam, self.nx, self.ny, self.Lx, self.Ly, raster, enable_pml=False)


def _phi(x):
    """(exp(x) - 1) / x for complex x, series near 0."""
    x = np.asarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    small = np.abs(x) < 0.1
    xs = x[small]
    s = np.ones_like(xs)
    term = np.ones_like(xs)
    for k in range(2, 12):
        term = term * xs / k
        s = s + term
    out[small] = s
    xl = x[~small]
    out[~small] = np.expm1(xl) / xl
    return out


def kernels_ED(gam, d, k0):
    """K_E, K_D of the exact first-order layer perturbation."""
    gi = gam[:, None]
    gj = gam[None, :]
    c = 1j / (2.0 * k0)
    # int_0^d exp(i(gi(d-z)+gj z)/k0) dz = exp(i gi d/k0) d phi(i (gj-gi) d/k0)
    KE = c * np.exp(1j * gi * d / k0) * d * _phi(1j * (gj - gi) * d / k0)
    KD = c * d * _phi(1j * (gi + gj) * d / k0)
    return KE, KD


@dataclass
class Tape:
    P: list = field(default_factory=list)
    Q: list = field(default_factory=list)
    bases: list = field(default_factory=list)
    segs: list = field(default_factory=list)      # projected layer blocks
    AB: list = field(default_factory=list)        # (A, B, Minv) of each left projection
    prefix: list = field(default_factory=list)    # S before each star product
    Sc: list = None                               # chain before the right projection
    ABr: tuple = None
    S: list = None                                # final blocks
    e0: Basis = None
    e1: Basis = None
    c: np.ndarray = None


def _proj_mats(basis: Basis, leftW, leftV):
    invW_W0 = basis.solveW(leftW)
    invV_V0 = basis.solveV(leftV)
    return 0.5 * (invW_W0 + invV_V0), 0.5 * (invW_W0 - invV_V0)


def stack_forward(st: Stack, px=1.0, py=0.0):
    """S-matrix of the stack and per-order (REF, TRN) for incidence from
    eps_in (side "bottom"), flux-normalised.  Returns (REF, TRN, tape)."""
    smp = st.sampler()
    k0 = smp.k0
    n = smp.ndim
    tp = Tape()
    x, y = smp.x, smp.y
    for eps in st.layers:
        P, Q = wave_eqn_coeff(x, y, eps, smp.Kx, smp.Ky, smp.lam, st.nx, st.ny)
        tp.P.append(P)
        tp.Q.append(Q)
        tp.bases.append(Basis(*wave_equation_solve(P, Q)))
    e0 = homogeneous_basis(smp, st.eps_in)
    e1 = homogeneous_basis(smp, st.eps_out)
    tp.e0, tp.e1 = e0, e1
    I = np.eye(n, dtype=np.complex128)
    Z = np.zeros((n, n), np.complex128)
    S = [I.copy(), I.copy(), Z.copy(), Z.copy()]
    leftW, leftV = e0.W, e0.V
    for b, d in zip(tp.bases, st.thick):
        X = np.diag(np.exp(1j * b.gam * d / k0))
        A, B = _proj_mats(b, leftW, leftV)
        seg = project_left([X, X.copy(), Z, Z], b, leftW, leftV)
        tp.AB.append((A, B, np.linalg.inv(A)))
        tp.segs.append(seg)
        tp.prefix.append(S)
        S = star_right(S, seg)
        leftW, leftV = b.W, b.V
    tp.Sc = S
    last = tp.bases[-1]
    Ar = 0.5 * (np.linalg.solve(last.W, e1.W) + np.linalg.solve(last.V, e1.V))
    Br = 0.5 * (np.linalg.solve(last.W, e1.W) - np.linalg.solve(last.V, e1.V))
    Mr = Ar - S[2] @ Br
    tp.ABr = (Ar, Br, np.linalg.inv(Mr))
    S = project_right(S, last.W, last.V, e1.W, e1.V)
    tp.S = S
    REF, TRN, c = _powers(st, smp, S, e0, e1, px, py)
    tp.c = c
    return REF, TRN, tp


def _powers(st, smp, S, e0, e1, px, py, want=False):
    m = st.nx * st.ny
    k0 = smp.k0
    alpha = np.diag(smp.Kx).copy()
    beta = np.diag(smp.Ky).copy()
    delta = np.zeros(m, dtype=np.complex128)
    delta[(st.ny * (st.nx - 1)) // 2 + (st.ny - 1) // 2] = 1.0
    s = np.concatenate([px * delta, py * delta])
    c = np.linalg.solve(e0.W, s)
    rxy = e0.W @ (S[3] @ c)
    txy = e1.W @ (S[1] @ c)
    kz_r = -np.sqrt(k0 * k0 * st.eps_in - alpha * alpha - beta * beta + 0j)
    kz_t = np.sqrt(k0 * k0 * st.eps_out - alpha * alpha - beta * beta + 0j)
    norm = math.sqrt(np.real(st.eps_in)) * k0

    def pw(v, kz):
        vx, vy = v[:m], v[m:]
        vz = (alpha * vx + beta * vy) / kz
        return np.abs(kz.real) * (np.abs(vx) ** 2 + np.abs(vy) ** 2 + np.abs(vz) ** 2) / norm

    return pw(rxy, kz_r), pw(txy, kz_t), c


# ---------------------------------------------------------------------------
# Adjoint
# ---------------------------------------------------------------------------
def _powers_adjoint(st, smp, S, e0, e1, c, wR, wT):
    """dL/d(Rdu), dL/d(Tuu) for L = sum wR*REF + wT*TRN."""
    m = st.nx * st.ny
    k0 = smp.k0
    alpha = np.diag(smp.Kx).copy()
    beta = np.diag(smp.Ky).copy()
    kz_r = -np.sqrt(k0 * k0 * st.eps_in - alpha * alpha - beta * beta + 0j)
    kz_t = np.sqrt(k0 * k0 * st.eps_out - alpha * alpha - beta * beta + 0j)
    norm = math.sqrt(np.real(st.eps_in)) * k0

    def gvec(v, kz, w):
        vx, vy = v[:m], v[m:]
        ux, uy = alpha / kz, beta / kz
        vz = ux * vx + uy * vy
        a = w * np.abs(kz.real) / norm
        return np.concatenate([2 * a * (vx + np.conj(ux) * vz), 2 * a * (vy + np.conj(uy) * vz)])

    rxy = e0.W @ (S[3] @ c)
    txy = e1.W @ (S[1] @ c)
    gr = gvec(rxy, kz_r, np.asarray(wR, dtype=np.float64))
    gt = gvec(txy, kz_t, np.asarray(wT, dtype=np.float64))
    Rdu_b = np.outer(H(e0.W) @ gr, np.conj(c))
    Tuu_b = np.outer(H(e1.W) @ gt, np.conj(c))
    return Rdu_b, Tuu_b


def project_right_adjoint(S, ABr, Sn, G):
    """Reverse of project_right (RedhefferIntegrator.cpp:211-223) with respect
    to S, the projection matrices held fixed.  S = (Tdd, Tuu, Rud, Rdu) before,
    Sn after; G = adjoints of Sn.  Returns adjoints of S."""
    Tdd, Tuu, Rud, Rdu = S
    Tdd_n, Tuu_n, Rud_n, Rdu_n = Sn
    gTdd_n, gTuu_n, gRud_n, gRdu_n = G
    A, B, Minv = ABr
    gRdu = gRdu_n
    gTdd = gRdu_n @ H(B @ Tuu_n) + gTdd_n @ H(B @ Rud_n + A)
    TB = Tdd @ B
    gTuu_n2 = gTuu_n + H(TB) @ gRdu_n
    gRud_n2 = gRud_n + H(TB) @ gTdd_n
    gTuu = H(Minv) @ gTuu_n2
    gY = H(Minv) @ gRud_n2
    gM = -gTuu @ H(Tuu_n) - gY @ H(Rud_n)
    gRud = gY @ H(A) - gM @ H(B)
    return [gTdd, gTuu, gRud, gRdu]


def star_adjoint(S, s, G):
    """Reverse of star_right (RedhefferIntegrator.cpp:267-277) with respect to
    both operands.  Returns (adjoints of S, adjoints of s)."""
    Tdd, Tuu, Rud, Rdu = S
    tdd, tuu, rud, rdu = s
    gTdd_n, gTuu_n, gRud_n, gRdu_n = G
    n = Tdd.shape[0]
    I = np.eye(n)
    C1 = np.linalg.inv(I - rdu @ Rud)
    C1r = C1 @ rdu
    C2 = I + Rud @ C1r
    X1 = Tdd @ rdu
    X2 = C2 @ Tuu
    Y = C1 @ tdd
    Zm = Rud @ Y
    # Rdu_n = Rdu + X1 X2
    gRdu = gRdu_n.copy()
    gX1 = gRdu_n @ H(X2)
    gTdd = gX1 @ H(rdu)
    grdu = H(Tdd) @ gX1
    # Tuu_n = tuu C2 Tuu and the X2 = C2 Tuu part of Rdu_n
    U = H(X1) @ gRdu_n + H(tuu) @ gTuu_n
    gC2 = U @ H(Tuu)
    gTuu = H(C2) @ U
    gtuu = gTuu_n @ H(X2) + gRud_n @ H(Zm)
    # Tdd_n = Tdd Y,  Rud_n = rud + tuu Rud Y
    grud = gRud_n.copy()
    gTdd = gTdd + gTdd_n @ H(Y)
    gZ = H(tuu) @ gRud_n
    gRud = gZ @ H(Y)
    gY = H(Tdd) @ gTdd_n + H(Rud) @ gZ
    gC1 = gY @ H(tdd)
    gtdd = H(C1) @ gY
    # C2 = I + Rud C1 rdu
    gRud = gRud + gC2 @ H(C1r)
    gC1 = gC1 + H(Rud) @ gC2 @ H(rdu)
    grdu = grdu + H(Rud @ C1) @ gC2
    # C1 = (I - rdu Rud)^-1
    gN = -H(C1) @ gC1 @ H(C1)
    grdu = grdu - gN @ H(Rud)
    gRud = gRud - H(rdu) @ gN
    return [gTdd, gTuu, gRud, gRdu], [gtdd, gtuu, grud, grdu]


def project_left_adjoint(s, ABM, sn, G):
    """Reverse of project_left (RedhefferIntegrator.cpp:253-262) with respect
    to the segment blocks s, the projection matrices (A, B, M^-1) fixed."""
    tdd, tuu, rud, rdu = s
    tdd_n, tuu_n, rud_n, rdu_n = sn
    gtdd_n, gtuu_n, grud_n, grdu_n = G
    A, B, Minv = ABM
    gtuu = gtuu_n @ H(A + B @ rdu_n) + grud_n @ H(B @ tdd_n)
    tB = tuu @ B
    grdu_n2 = grdu_n + H(tB) @ gtuu_n
    gtdd_n2 = gtdd_n + H(tB) @ grud_n
    grud = grud_n
    gtdd = H(Minv) @ gtdd_n2
    gY = H(Minv) @ grdu_n2
    gM = -gtdd @ H(tdd_n) - gY @ H(rdu_n)
    grdu = gY @ H(A) - gM @ H(B)
    return [gtdd, gtuu, grud, grdu]


def layer_pq_adjoint(basis: Basis, d, k0, gs):
    """Own-basis block adjoints of one z-uniform layer -> (dL/dP, dL/dQ)."""
    KE, KD = kernels_ED(basis.gam, d, k0)
    gA = np.conj(KE) * (gs[0] + gs[1])
    gB = -np.conj(KD) * (gs[2] + gs[3])
    Wi = np.linalg.inv(basis.W)
    Vi = np.linalg.inv(basis.V)
    gP = H(Wi) @ (gA + gB) @ H(basis.V)
    gQ = H(Vi) @ (gA - gB) @ H(basis.W)
    return gP, gQ


def assembly_adjoint(st: Stack, eps, gP, gQ):
    """dL/d(pixel permittivity) of one layer from dL/dP, dL/dQ (real pixels:
    the real part of the complex gradient).  Adjoint of Layer::waveEqnCoeff
    and FourierSolver2D::solve on a uniform pixel grid."""
    nx, ny = st.nx, st.ny
    m = nx * ny
    x = np.linspace(0.0, st.Lx, eps.shape[1] + 1)
    y = np.linspace(0.0, st.Ly, eps.shape[0] + 1)
    Kx, Ky = k_matrices(nx, ny, x, y, False)
    al = np.diag(Kx).real
    be = np.diag(Ky).real
    k0 = 2 * PI / st.lam
    f = np.asarray(eps, dtype=np.complex128)
    # Q blocks: Q10 = -Ky Ky + k0^2 fe11, Q01 = Kx Kx - k0^2 fe22
    g11 = k0 * k0 * gQ[m:, :m]
    g22 = -k0 * k0 * gQ[:m, m:]
    # P blocks through F = fe33^-1 [Kx Ky]
    gF2 = al[:, None] * gP[:m, :m] + be[:, None] * gP[m:, :m]
    gF1 = -al[:, None] * gP[:m, m:] - be[:, None] * gP[m:, m:]
    fe33 = fourier_solve_2d(x, y, f, nx, ny, CONTINUOUS_XY)
    G = H(np.linalg.inv(fe33))
    g33 = -G @ (gF1 * al[None, :] + gF2 * be[None, :]) @ G
    dx, dy = x[-1] - x[0], y[-1] - y[0]
    Ex = fourier_matrix_1d(x, dx, 2 * nx - 1)
    Ey = fourier_matrix_1d(y, dy, 2 * ny - 1)
    # e33: four = Ex f^T Ey^T gathered block-Toeplitz
    gfour = np.zeros((2 * nx - 1, 2 * ny - 1), np.complex128)
    mi = np.repeat(np.arange(nx), ny)
    ni = np.tile(np.arange(ny), nx)
    di = nx - 1 + mi[:, None] - mi[None, :]
    dj = ny - 1 + ni[:, None] - ni[None, :]
    np.add.at(gfour, (di, dj), g33)
    gf = (H(Ex) @ gfour @ np.conj(Ey)).T  # (npy, npx)
    inv = 1.0 / f
    # e11: sum over y strips r of kron(inv(Toep(Ex inv[r])), Toep(Ey[:, r]))
    g11_4 = g11.reshape(nx, ny, nx, ny)
    for r in range(f.shape[0]):
        C = toeplitz_dense(Ey[:, r])
        T = np.linalg.inv(toeplitz_dense(Ex @ inv[r]))
        gT = np.einsum("acbd,cd->ab", g11_4, np.conj(C))
        gTo = -H(T) @ gT @ H(T)
        gv = np.zeros(2 * nx - 1, np.complex128)
        a = np.arange(nx)[:, None]
        b = np.arange(nx)[None, :]
        np.add.at(gv, nx - 1 + a - b, gTo)
        ginv = H(Ex) @ gv
        gf[r] += np.conj(-inv[r] ** 2) * ginv
    # e22: sum over x columns i of kron(Toep(Ex[:, i]), inv(Toep(Ey inv[:, i])))
    g22_4 = g22.reshape(nx, ny, nx, ny)
    for i in range(f.shape[1]):
        C = toeplitz_dense(Ex[:, i])
        T = np.linalg.inv(toeplitz_dense(Ey @ inv[:, i]))
        gT = np.einsum("acbd,ab->cd", g22_4, np.conj(C))
        gTo = -H(T) @ gT @ H(T)
        gv = np.zeros(2 * ny - 1, np.complex128)
        a = np.arange(ny)[:, None]
        b = np.arange(ny)[None, :]
        np.add.at(gv, ny - 1 + a - b, gTo)
        ginv = H(Ey) @ gv
        gf[:, i] += np.conj(-inv[:, i] ** 2) * ginv
    return gf.real


def stack_backward(st: Stack, tp: Tape, wR, wT, want_pq=False, want_thick=False):
    """Gradient of L = sum_k wR[k] REF[k] + wT[k] TRN[k] with respect to every
    pixel of every layer.  Returns a list of (npy, npx) real arrays (and the
    per-layer (dL/dP, dL/dQ) when want_pq, and dL/d(thickness) per layer when
    want_thick: a layer's own-basis blocks depend on its thickness only
    through X = diag(exp(i gamma d / k0)), dX/dd = (i gamma / k0) X)."""
    smp = st.sampler()
    k0 = smp.k0
    n = smp.ndim
    Zn = np.zeros((n, n), np.complex128)
    gRdu, gTuu = _powers_adjoint(st, smp, tp.S, tp.e0, tp.e1, tp.c, wR, wT)
    G = [Zn, gTuu, Zn, gRdu]
    G = project_right_adjoint(tp.Sc, tp.ABr, tp.S, G)
    grads, pq = [None] * len(st.layers), [None] * len(st.layers)
    gthick = np.zeros(len(st.layers))
    for l in range(len(st.layers) - 1, -1, -1):
        b = tp.bases[l]
        d = st.thick[l]
        X = np.diag(np.exp(1j * b.gam * d / k0))
        G, gseg = star_adjoint(tp.prefix[l], tp.segs[l], G)
        gown = project_left_adjoint([X, X, Zn, Zn], tp.AB[l], tp.segs[l], gseg)
        dX = (1j * b.gam / k0) * np.diag(X)
        gthick[l] = float(np.real(np.sum(np.conj(np.diag(gown[0]) + np.diag(gown[1])) * dX)))
        gP, gQ = layer_pq_adjoint(b, d, k0, gown)
        pq[l] = (gP, gQ)
        grads[l] = assembly_adjoint(st, st.layers[l], gP, gQ)
    out = [grads]
    if want_pq:
        out.append(pq)
    if want_thick:
        out.append(gthick)
    return out[0] if len(out) == 1 else tuple(out)


def order_index(nx, ny, ox, oy):
    """Index of diffraction order (ox, oy) in the per-order power vectors."""
    return ny * (ox + (nx - 1) // 2) + (oy + (ny - 1) // 2)


# ---------------------------------------------------------------------------
# Internal amplitudes and fields (the role of RCWASolver::
# evaluateIntermediateField, src/rcwa/RCWASolver.cpp:1373-1480)
# ---------------------------------------------------------------------------
def stack_fields(st: Stack, tp: Tape, ngx=0, ngy=0):
    """Up- and down-going amplitudes at every interface j = 0..L of the
    stack for the forward's incidence, and the transverse fields there.

    Interface j is the top of region j-1 (region -1: the entrance medium,
    region L: the exit medium); amplitudes are in that region's eigenbasis
    (j = 0: entrance medium, incident c and reflected; j = L: exit medium,
    transmitted and nothing incoming).  For 0 < j < L, with S_L the chain of
    layers 0..j-1 and S_R the rest (layers j..L-1 and the exit) whose left
    end is in the basis of layer j-1:
        a+ = (I - Rud_L Rdu_R)^-1 Tuu_L c,   a- = Rdu_R a+.
    Transverse harmonics: e = W (a+ + a-), h = V (a+ - a-) (E and H of the
    interface matching of RedhefferIntegrator.cpp:253-262).  Returns
    (amps (L+1, 2, n), e (L+1, n), h (L+1, n), fields (L+1, 2, ngy, ngx) of
    Ex, Ey on the period when ngx, ngy > 0)."""
    L = len(st.layers)
    n = tp.S[0].shape[0]
    m = n // 2
    I = np.eye(n, dtype=np.complex128)
    Z = np.zeros((n, n), np.complex128)
    c = tp.c
    last = tp.bases[-1]
    # exit interface as a zero-thickness S-matrix: left end in the last
    # layer's basis, right end in the exit medium's
    SR = project_right([I.copy(), I.copy(), Z.copy(), Z.copy()], last.W, last.V, tp.e1.W, tp.e1.V)
    suffix = [None] * (L + 1)
    suffix[L] = SR
    for j in range(L - 1, 0, -1):
        suffix[j] = star_right(tp.segs[j], suffix[j + 1])
    amps = np.zeros((L + 1, 2, n), np.complex128)
    bases_W = [tp.e0.W] + [b.W for b in tp.bases[:-1]] + [tp.e1.W]
    bases_V = [tp.e0.V] + [b.V for b in tp.bases[:-1]] + [tp.e1.V]
    amps[0, 0] = c
    amps[0, 1] = tp.S[3] @ c
    for j in range(1, L):
        SL = tp.prefix[j]
        SRj = suffix[j]
        ap = np.linalg.solve(I - SL[2] @ SRj[3], SL[1] @ c)
        amps[j, 0] = ap
        amps[j, 1] = SRj[3] @ ap
    amps[L, 0] = tp.S[1] @ c
    e = np.array([bases_W[j] @ (amps[j, 0] + amps[j, 1]) for j in range(L + 1)])
    h = np.array([bases_V[j] @ (amps[j, 0] - amps[j, 1]) for j in range(L + 1)])
    fields = None
    if ngx > 0 and ngy > 0:
        smp = st.sampler()
        alpha = np.diag(smp.Kx).real
        beta = np.diag(smp.Ky).real
        xs = st.Lx * np.arange(ngx) / ngx
        ys = st.Ly * np.arange(ngy) / ngy
        ph = np.exp(1j * (alpha[:, None, None] * xs[None, None, :] + beta[:, None, None] * ys[None, :, None]))
        fields = np.zeros((L + 1, 2, ngy, ngx), np.complex128)
        for j in range(L + 1):
            fields[j, 0] = np.tensordot(e[j, :m], ph, axes=(0, 0))
            fields[j, 1] = np.tensordot(e[j, m:], ph, axes=(0, 0))
    return amps, e, h, fields
