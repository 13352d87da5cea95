"""Objectives of S-matrix results and their cotangents, for the
forward/backward pair of adaptive cells (Context.redheffer_forward /
redheffer_backward).

The backward takes the cotangents of the forward's outputs (the blocks and
the end bases, convention dL = Re sum conj(g) dX); an objective is any
function of those outputs, evaluated on the host where it costs O(n^2).
"""
from __future__ import annotations

import numpy as np


def mode_flux(W, V, j):
    """z-power flux of mode j: Re sum(e_x conj(h_y) - e_y conj(h_x)) over the
    harmonics, e = W[:, j] (Ex then Ey harmonics), h = V[:, j]."""
    m = W.shape[0] // 2
    e, h = W[:, j], V[:, j]
    return float(np.real(np.vdot(h[m:], e[:m]) - np.vdot(h[:m], e[m:])))


def mode_conversion(r, i0, i1):
    """Power carried from mode i0 of the entrance basis into mode i1 of the
    exit basis, normalised by the two modes' fluxes:
    L = |Tuu[i1, i0]|^2 f1 / f0 (independent of how the modes are scaled).
    r: a result dict of the forward.  Returns (L, gS, gB) with gS = (gTdd,
    gTuu, gRud, gRdu) and gB = (gW0, gV0, gW1, gV1)."""
    n = r["Tuu"].shape[0]
    m = n // 2
    T = r["Tuu"][i1, i0]
    f0 = mode_flux(r["W0"], r["V0"], i0)
    f1 = mode_flux(r["W1"], r["V1"], i1)
    L = float(abs(T) ** 2 * f1 / f0)
    Z = np.zeros((n, n), np.complex128)
    gTuu = Z.copy()
    gTuu[i1, i0] = 2.0 * T * f1 / f0

    def flux_grads(W, V, j, c):
        gW, gV = Z.copy(), Z.copy()
        gW[:m, j] = c * V[m:, j]
        gW[m:, j] = -c * V[:m, j]
        gV[:m, j] = -c * W[m:, j]
        gV[m:, j] = c * W[:m, j]
        return gW, gV

    gW1, gV1 = flux_grads(r["W1"], r["V1"], i1, abs(T) ** 2 / f0)
    gW0, gV0 = flux_grads(r["W0"], r["V0"], i0, -abs(T) ** 2 * f1 / f0 ** 2)
    return L, (Z, gTuu, Z.copy(), Z.copy()), (gW0, gV0, gW1, gV1)
