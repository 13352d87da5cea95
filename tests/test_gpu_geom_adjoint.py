"""Gradients of adaptive varRCWA cells with respect to geometric parameters
on the GPU (vrc_redheffer_forward / vrc_redheffer_backward): the config-5
objective -- power converted from the entrance's leading mode into another
exit mode, flux normalised -- of a PML waveguide converter whose core width
follows control points (piecewise-linear and natural cubic spline rules),
with respect to every control point.

* against the oracle's knot gradient (oracle/segments_adjoint.py:
  knot_gradient) on the device's segmentation: 1e-8 of the gradient scale;
* against central differences of the device's own forward on the same cuts
  (widths +-1e-4): 1e-6 of the gradient scale.  The gradient holds every
  segment's reference basis fixed, while the perturbative segment formula
  depends on that basis at the level of its own error, so the two differ by
  a bias that falls with the tolerance: the oracle on the same cells gives
  2.7e-5 (spline) and 1.7e-6 (linear) of the scale at pe = 1e-4, 9.4e-7 and
  1.5e-7 at 1e-5, 6.2e-7 and 1.5e-8 at 1e-6; the cells here run at pe =
  1e-6 (about 630 segments);
* checkpointed reverse passes (a checkpoint every 1, 2, and about sqrt(K)
  segments) equal the full tape to 1e-12;
* a batch of cells of different segment counts equals its cells one per call.
"""
import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.segments_adjoint import H, knot_gradient, mode_conversion_adjoint, segments_forward
from oracle.structures_adapter import make_sampler
from varrcwa_b200 import objectives
from varrcwa_b200 import structures as st

pytestmark = pytest.mark.gpu


def _waveguide(widths, spline=False, norders=5, length=3.0):
    d = dict(st.waveguide_pml(5000, norders=norders, ncontrol=len(widths), length=length))
    zs = d["xrules"][0][1]
    cx = 2.0
    w = np.asarray(widths, dtype=float)
    d["xrules"] = [(2, zs, cx - 0.5 * w), (3, zs, cx + 0.5 * w)]
    d["x"] = np.array(d["x"])
    d["x"][2], d["x"][3] = cx - 0.5 * w[0], cx + 0.5 * w[0]
    d["spline"] = spline
    return d


def _cuts(ctx):
    leaves = sorted((a, b) for (a, b, e, acc) in ctx.tree(0) if acc)
    return [leaves[0][0]] + [b for (_, b) in leaves]


def _modes(r):
    return int(np.argmax(r["gam0"].real)), int(np.argsort(-r["gam1"].real)[1])


@pytest.mark.parametrize("spline", [False, True])
def test_cell_gradient_matches_oracle_and_central_differences(ctx, spline):
    w = np.array(st.waveguide_pml(5000, norders=5, ncontrol=6, length=3.0)["widths"])
    d = _waveguide(w, spline)
    r = ctx.redheffer_forward([d], pe=1e-6)[0]
    assert r["status"] == 0 and r["N"] >= 3
    cuts = _cuts(ctx)
    i0, i1 = _modes(r)
    L, gS, gB = objectives.mode_conversion(r, i0, i1)
    gl, gr = ctx.redheffer_backward([gS], [gB])[0]
    gw = -0.5 * gl + 0.5 * gr  # x_left = cx - w/2, x_right = cx + w/2
    scale = np.abs(gw).max()
    assert scale > 0
    # the oracle on the same cuts, same modes, same coordinate step
    fw = segments_forward(make_sampler(d), cuts)
    j0 = int(np.argmax(fw["b0"].gam.real))
    j1 = int(np.argsort(-fw["b1"].gam.real)[1])
    Lo, gSo, gW0o, gV0o, gW1o, gV1o = mode_conversion_adjoint(fw, j0, j1)
    assert abs(L - Lo) <= 1e-9 * abs(Lo)
    ol, orr = knot_gradient(d, cuts, gSo, gW0o, gV0o, gW1o, gV1o, h=1e-6 * 4.0)
    gwo = -0.5 * ol + 0.5 * orr
    assert np.abs(gw - gwo).max() <= 1e-8 * np.abs(gwo).max(), np.abs(gw - gwo).max() / np.abs(gwo).max()

    # central differences of the device forward on the same segmentation
    def objective(widths):
        rp = ctx.redheffer_segments([_waveguide(widths, spline)], [cuts])[0]
        k0 = int(np.argmax(np.abs(H(rp["W0"]) @ r["W0"][:, i0])))
        k1 = int(np.argmax(np.abs(H(rp["W1"]) @ r["W1"][:, i1])))
        return objectives.mode_conversion(rp, k0, k1)[0]

    hf = 1e-4
    for k in range(len(w)):
        wp, wm = w.copy(), w.copy()
        wp[k] += hf
        wm[k] -= hf
        fd = (objective(wp) - objective(wm)) / (2 * hf)
        assert abs(gw[k] - fd) <= 1e-6 * scale, (k, gw[k], fd)


def test_checkpointed_reverse_equals_full_tape(ctx):
    w = np.array(st.waveguide_pml(5001, norders=3, ncontrol=8, length=4.0)["widths"])
    d = _waveguide(w, norders=3, length=4.0)
    r = ctx.redheffer_forward([d], pe=1e-4)[0]
    K = r["N"]
    assert K >= 6
    L, gS, gB = objectives.mode_conversion(r, *_modes(r))
    full = np.concatenate(ctx.redheffer_backward([gS], [gB], every=K)[0])
    for every in (1, 2, 0):
        g = np.concatenate(ctx.redheffer_backward([gS], [gB], every=every)[0])
        assert np.abs(g - full).max() <= 1e-12 * np.abs(full).max(), every


def test_batch_of_cells_equals_single_calls(ctx):
    ds = [_waveguide(np.array(st.waveguide_pml(5010 + i, norders=3, ncontrol=5, length=2.0 + i)["widths"]),
                     norders=3, length=2.0 + i) for i in range(3)]
    rs = ctx.redheffer_forward(ds, pe=1e-4)
    cot = [objectives.mode_conversion(r, *_modes(r)) for r in rs]
    gb = ctx.redheffer_backward([c[1] for c in cot], [c[2] for c in cot])
    for d, r, c, g in zip(ds, rs, cot, gb):
        r1 = ctx.redheffer_forward([d], pe=1e-4)[0]
        assert r1["N"] == r["N"]
        g1 = ctx.redheffer_backward([c[1]], [c[2]])[0]
        for a, b in zip(g, g1):
            assert np.abs(a - b).max() <= 1e-11 * max(np.abs(b).max(), 1e-300)
