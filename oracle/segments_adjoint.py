"""CPU restatement of a geometric-parameter gradient for adaptive varRCWA
cells on a fixed segmentation (the accepted leaves of the adaptive tree).

TEST INFRASTRUCTURE ONLY: the GPU path never imports this module.  It states
the algorithm the device adjoint of adaptive cells is to follow and pins it
against central differences of the oracle's own forward on the same cuts.

Forward: redheffer_segments (the trisecting integrator's accepted segments,
src/core/RedhefferIntegrator.cpp:174-399), each segment the first-order
perturbative S-matrix in the eigenbasis of its midpoint sample, its left end
re-expressed in the previous segment's basis, star-multiplied, the right end
moved to the end basis.

Gradient: every basis is held fixed (a fixed basis re-expresses the same
operator exactly), so a parameter reaches the S-matrix through the samples
P(z), Q(z) inside each segment only, and to first order by the segment
formula itself applied to dP/dtheta, dQ/dtheta at its three Simpson nodes
(the reference sample included: the basis is frozen, the sample moves).
The chain is reversed with respect to the segment blocks (star products and
projections, as for layer stacks).  dP/dtheta of a sample is taken here by
central differences of the sampler (assembly only, no eigen-solve).

A parameter that moves an end cross-section also moves the end basis the
result is expressed in (the semi-infinite continuation of that section):
end_bases_adjoint reverses the two end projections and the objective with
respect to the end bases (W, V), to be contracted with dW/dtheta, dV/dtheta of
the end eigen-decompositions (end_basis_derivative: central differences
with the eigenvectors' order and phase aligned to the unperturbed basis).
"""
from __future__ import annotations

import numpy as np

from . import varrcwa_oracle as O
from .stack_adjoint import H, project_left_adjoint, project_right_adjoint, star_adjoint


def segments_forward(sampler, cuts):
    """redheffer_segments with the quantities the reverse pass needs."""
    k0 = sampler.k0
    cuts = list(cuts)
    P0, Q0 = sampler.sample(cuts[0])
    b0 = O.Basis(*O.wave_equation_solve(P0, Q0))
    P1, Q1 = sampler.sample(cuts[-1])
    b1 = O.Basis(*O.wave_equation_solve(P1, Q1))
    n = P0.shape[0]
    I = np.eye(n, dtype=np.complex128)
    Z = np.zeros((n, n), np.complex128)
    S = [I.copy(), I.copy(), Z.copy(), Z.copy()]
    leftW, leftV = b0.W, b0.V
    tape = []
    Pa, Qa = P0, Q0
    for a, b in zip(cuts[:-1], cuts[1:]):
        Pm, Qm = sampler.sample(0.5 * (a + b))
        Pb, Qb = (P1, Q1) if b == cuts[-1] else sampler.sample(b)
        bm = O.Basis(*O.wave_equation_solve(Pm, Qm))
        seg, _ = O.perturbation_segment(Pm, Qm, bm, k0, a, b, (Pa, Pm, Pb), (Qa, Qm, Qb))
        invW, invV = bm.solveW(leftW), bm.solveV(leftV)
        A, B = 0.5 * (invW + invV), 0.5 * (invW - invV)
        segp = O.project_left(seg, bm, leftW, leftV)
        tape.append(dict(a=a, b=b, basis=bm, seg=seg, segp=segp,
                         ABM=(A, B, np.linalg.inv(A - seg[3] @ B)), prefix=S))
        S = O.star_right(S, segp)
        leftW, leftV = bm.W, bm.V
        Pa, Qa = Pb, Qb
    Sc = S
    Ar = 0.5 * (np.linalg.solve(leftW, b1.W) + np.linalg.solve(leftV, b1.V))
    Br = 0.5 * (np.linalg.solve(leftW, b1.W) - np.linalg.solve(leftV, b1.V))
    S = O.project_right(Sc, leftW, leftV, b1.W, b1.V)
    return dict(tape=tape, Sc=Sc, S=S, ABr=(Ar, Br, np.linalg.inv(Ar - Sc[2] @ Br)), b0=b0, b1=b1, k0=k0)


def first_order_blocks(basis, k0, a, b, dP3, dQ3):
    """The segment formula (RedhefferIntegrator.cpp:343-396) applied to
    perturbations dP3, dQ3 at (a, midpoint, b) in a fixed basis: the
    segment's own-basis blocks' first-order change."""
    W, V, gam = basis.W, basis.V, basis.gam
    dA, dB = [], []
    for dP, dQ in zip(dP3, dQ3):
        x = basis.solveW(dP @ V)
        y = basis.solveV(dQ @ W)
        dA.append(x + y)
        dB.append(x - y)
    dz = b - a
    ph = np.exp(1j * 0.5 * dz / k0 * gam)
    pf = np.exp(1j * dz / k0 * gam)
    c = 1j * dz / (12 * k0)
    tuu = c * (pf[:, None] * dA[0] + 4.0 * ph[:, None] * dA[1] * ph[None, :] + dA[2] * pf[None, :])
    rud = -c * (pf[:, None] * dB[0] * pf[None, :] + 4.0 * ph[:, None] * dB[1] * ph[None, :] + dB[2])
    rdu = -c * (dB[0] + 4.0 * ph[:, None] * dB[1] * ph[None, :] + pf[:, None] * dB[2] * pf[None, :])
    tdd = c * (dA[0] * pf[None, :] + 4.0 * ph[:, None] * dA[1] * ph[None, :] + pf[:, None] * dA[2])
    return [tdd, tuu, rud, rdu]


def segments_block_adjoints(fw, gS, want_first=False):
    """Own-basis block adjoints of every segment from the adjoints gS of the
    final blocks (Tdd, Tuu, Rud, Rdu); with want_first also the adjoints of
    the first segment's projected blocks (for the entrance-basis term)."""
    G = project_right_adjoint(fw["Sc"], fw["ABr"], fw["S"], gS)
    out = [None] * len(fw["tape"])
    first = None
    for j in range(len(fw["tape"]) - 1, -1, -1):
        t = fw["tape"][j]
        G, gsegp = star_adjoint(t["prefix"], t["segp"], G)
        out[j] = project_left_adjoint(t["seg"], t["ABM"], t["segp"], gsegp)
        if j == 0:
            first = gsegp
    return (out, first) if want_first else out


def _proj_left_ab_adjoint(s, ABM, sn, G):
    """Reverse of project_left with respect to its projection matrices A, B
    (segment blocks s fixed)."""
    tdd, tuu, rud, rdu = s
    tdd_n, tuu_n, rud_n, rdu_n = sn
    gtdd_n, gtuu_n, grud_n, grdu_n = G
    A, B, Minv = ABM
    tB = tuu @ B
    gA = H(tuu) @ gtuu_n
    gB = H(tuu) @ gtuu_n @ H(rdu_n) + H(tuu) @ grud_n @ H(tdd_n)
    grdu_n2 = grdu_n + H(tB) @ gtuu_n
    gtdd_n2 = gtdd_n + H(tB) @ grud_n
    gY = H(Minv) @ grdu_n2
    gM = -H(Minv) @ gtdd_n2 @ H(tdd_n) - gY @ H(rdu_n)
    gA = gA + H(rdu) @ gY + gM
    gB = gB - gY - H(rdu) @ gM
    return gA, gB


def _proj_right_ab_adjoint(S, ABr, Sn, G):
    """Reverse of project_right with respect to its projection matrices."""
    Tdd, Tuu, Rud, Rdu = S
    Tdd_n, Tuu_n, Rud_n, Rdu_n = Sn
    gTdd_n, gTuu_n, gRud_n, gRdu_n = G
    A, B, Minv = ABr
    TB = Tdd @ B
    gTuu_n2 = gTuu_n + H(TB) @ gRdu_n
    gRud_n2 = gRud_n + H(TB) @ gTdd_n
    gB = H(Tdd) @ gRdu_n @ H(Tuu_n) + H(Tdd) @ gTdd_n @ H(Rud_n)
    gA = H(Tdd) @ gTdd_n
    gY = H(Minv) @ gRud_n2
    gM = -H(Minv) @ gTuu_n2 @ H(Tuu_n) - gY @ H(Rud_n)
    gA = gA + H(Rud) @ gY + gM
    gB = gB - gY - H(Rud) @ gM
    return gA, gB


def end_bases_adjoint(fw, gS, gsegp_first, gW0_obj=None, gW1_obj=None, gV0_obj=None, gV1_obj=None):
    """dL/d(W0, V0, W1, V1) of the end bases through the entrance projection
    of the first segment and the exit projection (plus explicit objective
    terms).  A = (L_W^-1 W + L_V^-1 V) / 2, B = (L_W^-1 W - L_V^-1 V) / 2."""
    t0 = fw["tape"][0]
    gA, gB = _proj_left_ab_adjoint(t0["seg"], t0["ABM"], t0["segp"], gsegp_first)
    bm = t0["basis"]
    Wi, Vi = np.linalg.inv(bm.W), np.linalg.inv(bm.V)
    gW0 = 0.5 * H(Wi) @ (gA + gB)
    gV0 = 0.5 * H(Vi) @ (gA - gB)
    gA, gB = _proj_right_ab_adjoint(fw["Sc"], fw["ABr"], fw["S"], gS)
    last = fw["tape"][-1]["basis"]
    Wi, Vi = np.linalg.inv(last.W), np.linalg.inv(last.V)
    gW1 = 0.5 * H(Wi) @ (gA + gB)
    gV1 = 0.5 * H(Vi) @ (gA - gB)
    if gW0_obj is not None:
        gW0 = gW0 + gW0_obj
    if gW1_obj is not None:
        gW1 = gW1 + gW1_obj
    if gV0_obj is not None:
        gV0 = gV0 + gV0_obj
    if gV1_obj is not None:
        gV1 = gV1 + gV1_obj
    return gW0, gV0, gW1, gV1


def end_basis_derivative(sampler_p, sampler_m, z, ref, h):
    """dW/dtheta, dV/dtheta of the eigenbasis at z by central differences of
    the sampler, each perturbed basis's columns matched to `ref` by overlap
    and their phases aligned (the zgeev normalisation fixes each column only
    up to a phase, which the S-matrix's end projections absorb)."""
    out = []
    for smp in (sampler_p, sampler_m):
        P, Q = smp.sample(z)
        W, V, _ = O.wave_equation_solve(P, Q)
        idx = np.argmax(np.abs(H(ref.W) @ W), axis=1)
        W, V = W[:, idx], V[:, idx]
        ph = np.array([np.vdot(W[:, i], ref.W[:, i]) for i in range(W.shape[1])])
        ph = ph / np.abs(ph)
        out.append((W * ph[None, :], V * ph[None, :]))
    return (out[0][0] - out[1][0]) / (2 * h), (out[0][1] - out[1][1]) / (2 * h)


def segments_gradient(fw, gS, dsample, end_terms=None):
    """dL/dtheta for one parameter: gS are the adjoints of the final blocks,
    dsample(z) -> (dP/dtheta, dQ/dtheta) at a sample position.  end_terms:
    optional ((gW0, gV0, gW1, gV1), (dW0, dV0, dW1, dV1)) for a parameter that
    moves an end cross-section."""
    gsegs = segments_block_adjoints(fw, gS)
    grad = 0.0
    if end_terms is not None:
        for g, dv in zip(*end_terms):
            grad += float(np.real(np.vdot(g, dv)))
    for t, g in zip(fw["tape"], gsegs):
        a, b = t["a"], t["b"]
        dd = [dsample(a), dsample(0.5 * (a + b)), dsample(b)]
        ds = first_order_blocks(t["basis"], fw["k0"], a, b, [x[0] for x in dd], [x[1] for x in dd])
        grad += sum(float(np.real(np.vdot(gi, di))) for gi, di in zip(g, ds))
    return grad


def fourier_transmission_adjoint(fw, k, want_bases=False):
    """Adjoint of L = |(W1 Tuu W0^-1)[k, k]|^2 (power of Fourier harmonic k
    carried through) with respect to the final Tuu; other blocks zero.  With
    want_bases also the explicit dL/dW0 and dL/dW1 of the Fourier mapping."""
    n = fw["S"][0].shape[0]
    W0i = np.linalg.inv(fw["b0"].W)
    Tuu = fw["S"][1]
    Tf = fw["b1"].W @ Tuu @ W0i
    gTf = np.zeros((n, n), np.complex128)
    gTf[k, k] = 2.0 * Tf[k, k]
    Z = np.zeros((n, n), np.complex128)
    out = (float(abs(Tf[k, k]) ** 2), [Z, H(fw["b1"].W) @ gTf @ H(W0i), Z, Z.copy()])
    if not want_bases:
        return out
    gW1 = gTf @ H(Tuu @ W0i)
    gW0 = -H(W0i) @ H(fw["b1"].W @ Tuu) @ gTf @ H(W0i)
    return out + (gW0, gW1)


def mode_flux(W, V, j):
    """z-power flux of mode j of a basis: Re sum(e_x conj(h_y) - e_y conj(h_x))
    over the harmonics, e = W[:, j], h = V[:, j] (the interface fields'
    flux, conserved across interfaces of lossless stacks)."""
    m = W.shape[0] // 2
    e, h = W[:, j], V[:, j]
    return float(np.real(np.vdot(h[m:], e[:m]) - np.vdot(h[:m], e[m:])))


def mode_conversion_adjoint(fw, i0, i1):
    """L = |Tuu[i1, i0]|^2 f1 / f0: power carried from mode i0 of the entrance
    basis into mode i1 of the exit basis, f the modes' fluxes.  Returns
    (L, adjoints of the final blocks, dL/dW0, dL/dV0, dL/dW1, dL/dV1 of the
    explicit flux terms)."""
    b0, b1 = fw["b0"], fw["b1"]
    n = b0.W.shape[0]
    m = n // 2
    T = fw["S"][1][i1, i0]
    f0, f1 = mode_flux(b0.W, b0.V, i0), mode_flux(b1.W, b1.V, i1)
    L = float(abs(T) ** 2 * f1 / f0)
    Z = np.zeros((n, n), np.complex128)
    gTuu = Z.copy()
    gTuu[i1, i0] = 2.0 * T * f1 / f0
    gS = [Z, gTuu, Z.copy(), Z.copy()]

    def flux_grads(W, V, j, c):
        gW, gV = Z.copy(), Z.copy()
        gW[:m, j] = c * V[m:, j]
        gW[m:, j] = -c * V[:m, j]
        gV[:m, j] = -c * W[m:, j]
        gV[m:, j] = c * W[:m, j]
        return gW, gV

    gW1, gV1 = flux_grads(b1.W, b1.V, i1, abs(T) ** 2 / f0)
    gW0, gV0 = flux_grads(b0.W, b0.V, i0, -abs(T) ** 2 * f1 / f0 ** 2)
    return L, gS, gW0, gV0, gW1, gV1


def segments_block_adjoints_checkpointed(sampler, cuts, gS_of, every):
    """The reverse pass of segments_block_adjoints with the forward's
    per-segment data kept only at checkpoints: the chain state before every
    `every`-th segment is stored (memory ~ (K / every) chain states), and each
    block of segments is recomputed from its checkpoint on the way back
    (about one extra forward in total).  gS_of(fw_final) gives the final
    blocks' adjoints.  Returns the per-segment own-basis block adjoints."""
    cuts = list(cuts)
    K = len(cuts) - 1
    k0 = sampler.k0
    P0, Q0 = sampler.sample(cuts[0])
    b0 = O.Basis(*O.wave_equation_solve(P0, Q0))
    P1, Q1 = sampler.sample(cuts[-1])
    b1 = O.Basis(*O.wave_equation_solve(P1, Q1))
    n = P0.shape[0]
    I = np.eye(n, dtype=np.complex128)
    Z = np.zeros((n, n), np.complex128)

    def run(j0, j1, S, leftW, leftV, keep):
        """Segments j0..j1-1 from chain state S (left basis leftW, leftV)."""
        tape = []
        for j in range(j0, j1):
            a, b = cuts[j], cuts[j + 1]
            Pa, Qa = (P0, Q0) if j == 0 else sampler.sample(a)
            Pm, Qm = sampler.sample(0.5 * (a + b))
            Pb, Qb = (P1, Q1) if j == K - 1 else sampler.sample(b)
            bm = O.Basis(*O.wave_equation_solve(Pm, Qm))
            seg, _ = O.perturbation_segment(Pm, Qm, bm, k0, a, b, (Pa, Pm, Pb), (Qa, Qm, Qb))
            invW, invV = bm.solveW(leftW), bm.solveV(leftV)
            A, B = 0.5 * (invW + invV), 0.5 * (invW - invV)
            segp = O.project_left(seg, bm, leftW, leftV)
            if keep:
                tape.append(dict(seg=seg, segp=segp, ABM=(A, B, np.linalg.inv(A - seg[3] @ B)), prefix=S))
            S = O.star_right(S, segp)
            leftW, leftV = bm.W, bm.V
        return S, leftW, leftV, tape

    # forward: chain states at the checkpoints only
    checkpoints = {}
    S, lW, lV = [I.copy(), I.copy(), Z.copy(), Z.copy()], b0.W, b0.V
    for j0 in range(0, K, every):
        checkpoints[j0] = (S, lW, lV)
        S, lW, lV, _ = run(j0, min(j0 + every, K), S, lW, lV, keep=False)
    Sc = S
    Ar = 0.5 * (np.linalg.solve(lW, b1.W) + np.linalg.solve(lV, b1.V))
    Br = 0.5 * (np.linalg.solve(lW, b1.W) - np.linalg.solve(lV, b1.V))
    Sf = O.project_right(Sc, lW, lV, b1.W, b1.V)
    fw_final = dict(Sc=Sc, S=Sf, ABr=(Ar, Br, np.linalg.inv(Ar - Sc[2] @ Br)), b0=b0, b1=b1, k0=k0)
    G = project_right_adjoint(Sc, fw_final["ABr"], Sf, gS_of(fw_final))
    out = [None] * K
    for j0 in sorted(checkpoints, reverse=True):
        S, lW, lV = checkpoints[j0]
        _, _, _, tape = run(j0, min(j0 + every, K), S, lW, lV, keep=True)
        for jj in range(len(tape) - 1, -1, -1):
            t = tape[jj]
            G, gsegp = star_adjoint(t["prefix"], t["segp"], G)
            out[j0 + jj] = project_left_adjoint(t["seg"], t["ABM"], t["segp"], gsegp)
    return out


def node_adjoints(basis, k0, a, b, gseg):
    """Adjoint of first_order_blocks with respect to its perturbations: for a
    segment's own-basis block adjoints gseg = (gtdd, gtuu, grud, grdu), the
    (dL/dP, dL/dQ) at its three Simpson nodes (a, midpoint, b), so that
    Re <gseg, first_order_blocks(dP3, dQ3)> = sum_k Re <gP_k, dP_k> + Re <gQ_k, dQ_k>."""
    gtdd, gtuu, grud, grdu = gseg
    gam = basis.gam
    dz = b - a
    ph = np.exp(1j * 0.5 * dz / k0 * gam)
    pf = np.exp(1j * dz / k0 * gam)
    c = 1j * dz / (12 * k0)
    cc = np.conj(c)
    P2 = np.conj(ph)[:, None] * np.conj(ph)[None, :]
    F = np.conj(pf)
    gA = [cc * (F[:, None] * gtuu + gtdd * F[None, :]),
          4.0 * cc * P2 * (gtuu + gtdd),
          cc * (gtuu * F[None, :] + F[:, None] * gtdd)]
    gB = [-cc * (F[:, None] * grud * F[None, :] + grdu),
          -4.0 * cc * P2 * (grud + grdu),
          -cc * (grud + F[:, None] * grdu * F[None, :])]
    Wi, Vi = np.linalg.inv(basis.W), np.linalg.inv(basis.V)
    out = []
    for ga, gb in zip(gA, gB):
        gx, gy = ga + gb, ga - gb
        out.append((H(Wi) @ gx @ H(basis.V), H(Vi) @ gy @ H(basis.W)))
    return out


def eig_adjoint(P, Q, W, V, gam, gW, gV, ggam=None, eta=None):
    """Adjoint of the eigen step W, gam, V = wave_equation_solve(P, Q)
    (src/rcwa/WaveEquationSolver.cpp:24-37: A = P Q = W diag(gam^2) W^-1,
    V = Q W diag(1/gam)) with respect to (P, Q), for cotangents gW, gV and
    optionally ggam.

    Eigenvector part: dW = W C with C_ij = (W^-1 dA W)_ij / (lam_j - lam_i)
    off the diagonal.  Its diagonal (each column's scale and phase) is left
    out, which is exact for objectives that do not depend on how the modes
    are normalised (Fourier-basis S-matrix blocks, flux-normalised modal
    powers).  Degenerate pairs are guarded by a Lorentzian broadening of
    1 / (lam_j - lam_i): conj(d) / (|d|^2 + eta^2), eta = 1e-12 max|lam|
    by default."""
    lam = gam * gam
    n = W.shape[0]
    if eta is None:
        eta = 1e-12 * float(np.abs(lam).max())
    Wi = np.linalg.inv(W)
    # V = Q W G^-1: cotangents of Q, W and gam
    gQ = gV @ H(W / gam[None, :])
    gWt = gW + H(Q) @ gV / np.conj(gam)[None, :]
    ggam_t = -np.sum(np.conj(V) * gV, axis=0) / np.conj(gam)
    if ggam is not None:
        ggam_t = ggam_t + ggam
    glam = ggam_t / np.conj(2.0 * gam)
    M = H(W) @ gWt
    d = lam[None, :] - lam[:, None]  # lam_j - lam_i
    Fm = M * d / (np.abs(d) ** 2 + eta * eta)
    Fm[np.arange(n), np.arange(n)] = glam
    gA = H(Wi) @ Fm @ H(W)
    gP = gA @ H(Q)
    gQ = gQ + H(P) @ gA
    return gP, gQ


def rule_weights(zs, z, spline=False):
    """d x(z) / d vals[k] of a coordinate rule through knots zs: the
    piecewise-linear hat functions (clamped outside), or the natural cubic
    spline's cardinal functions (the spline is linear in its values)."""
    from .structures_adapter import _pwl, natural_spline_eval
    ev = natural_spline_eval if spline else _pwl
    K = len(zs)
    return np.array([ev(zs, np.eye(K)[k], z) for k in range(K)])


def knot_gradient(desc, cuts, gS, gW0=None, gV0=None, gW1=None, gV1=None, h=1e-6, fw=None):
    """dL/d(knot values) of every coordinate rule of a grid cell (x rules
    first, then y rules, each rule's knots in order), for cotangents gS of the
    final blocks and optional explicit cotangents of the end bases: the
    algorithm of the device backward.

    Per segment the own-basis block adjoints (segments_block_adjoints) are
    turned into (dL/dP, dL/dQ) at its Simpson nodes (node_adjoints); the end
    bases' cotangents (projections and explicit terms) into (dL/dP, dL/dQ) at
    z0 and z1 (eig_adjoint).  At every node each moving coordinate's
    dP/dx, dQ/dx is a central difference of the sampler (+-h on that
    coordinate alone), contracted to dL/dx(z) and spread over the rule's knots
    by d x(z) / d vals.  fw: the forward replay on these cuts when the caller
    already has it (segments_forward of the same cell)."""
    from .structures_adapter import make_sampler
    s = make_sampler(desc)
    if fw is None:
        fw = segments_forward(s, cuts)
    gsegs, gfirst = segments_block_adjoints(fw, gS, want_first=True)
    spline = bool(desc.get("spline"))
    rules = [(0, r) for r in desc.get("xrules", [])] + [(1, r) for r in desc.get("yrules", [])]

    def shifted(axis, idx, dlt):
        d = dict(desc)
        key = "x" if axis == 0 else "y"
        rk = "xrules" if axis == 0 else "yrules"
        d[rk] = [(i, zs, np.asarray(v, float) + (dlt if i == idx else 0.0)) for (i, zs, v) in desc.get(rk, [])]
        base = np.array(desc[key], dtype=float)
        base[idx] += dlt
        d[key] = base
        return make_sampler(d)

    pert = {(ax, r[0]): (shifted(ax, r[0], h), shifted(ax, r[0], -h)) for ax, r in rules}
    out = [np.zeros(len(r[1])) for _, r in rules]

    def contract(z, gP, gQ):
        for q, (ax, (idx, zs, _)) in enumerate(rules):
            sp, sm = pert[(ax, idx)]
            Pp, Qp = sp.sample(z)
            Pm, Qm = sm.sample(z)
            dLdx = float(np.real(np.vdot(gP, (Pp - Pm) / (2 * h)) + np.vdot(gQ, (Qp - Qm) / (2 * h))))
            out[q] += dLdx * rule_weights(zs, z, spline)

    k0 = fw["k0"]
    for t, g in zip(fw["tape"], gsegs):
        a, b = t["a"], t["b"]
        for z, (gP, gQ) in zip((a, 0.5 * (a + b), b), node_adjoints(t["basis"], k0, a, b, g)):
            contract(z, gP, gQ)
    if desc.get("end0") is None and desc.get("end1") is None:
        Z = np.zeros_like(gS[0])
        e = end_bases_adjoint(fw, gS, gfirst, *(x if x is not None else Z for x in (gW0, gW1, gV0, gV1)))
        for z, b, (gW, gV) in ((cuts[0], fw["b0"], e[0:2]), (cuts[-1], fw["b1"], e[2:4])):
            P, Q = s.sample(z)
            gP, gQ = eig_adjoint(P, Q, b.W, b.V, b.gam, gW, gV)
            contract(z, gP, gQ)
    return out
