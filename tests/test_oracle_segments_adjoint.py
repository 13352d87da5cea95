"""Geometric-parameter gradient of an adaptive varRCWA cell on its fixed
segmentation (oracle/segments_adjoint.py): the frozen-basis first-order
adjoint against central differences of the oracle's forward on the same cuts,
for a control knot inside the cell (the end cross-sections unchanged)."""
import numpy as np

from oracle import varrcwa_oracle as O
from oracle.segments_adjoint import fourier_transmission_adjoint, segments_forward, segments_gradient
from oracle.structures_adapter import make_sampler
from varrcwa_b200 import structures as st


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
