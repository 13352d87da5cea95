"""Layer-stack forward and adjoint on the GPU: per-order powers and pixel
gradients against the oracle (oracle/stack_adjoint.py), and the gradient
against central finite differences computed on the device as one batch of
perturbed stacks."""
import numpy as np
import pytest

from oracle.stack_adjoint import Stack, order_index, stack_backward, stack_forward
from varrcwa_b200.structures import smooth_pixels

pytestmark = pytest.mark.gpu

LAM, PER = 0.633, 0.6


@pytest.fixture(scope="module")
def ctx():
    from varrcwa_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def _desc(layers, thick, nx, eps_in=1.0, eps_out=2.085):
    return dict(lam=LAM, Lx=PER, Ly=PER, nx=nx, ny=nx, layers=layers, thick=thick, eps_in=eps_in, eps_out=eps_out)


def _oracle(d):
    st = Stack(d["lam"], d["nx"], d["ny"], d["Lx"], d["Ly"], d["layers"], d["thick"], d["eps_in"], d["eps_out"])
    return st, stack_forward(st)


def _weights(nx, C=1):
    m = nx * nx
    wT = np.zeros((C, m))
    wT[:, order_index(nx, nx, 1, 0)] = 1.0
    wR = np.zeros((C, m))
    wR[:, order_index(nx, nx, 0, 0)] = 0.25
    return wR, wT


def test_small_stack_matches_oracle(ctx):
    layers = [smooth_pixels(4100 + l, 8, 8, sigma=1.0) for l in range(2)]
    d = _desc(layers, [0.15, 0.2], 3)
    R, T, st = ctx.stack_forward([d])
    assert st[0] == 0
    ost, (oR, oT, tp) = _oracle(d)
    # per-order powers: 1e-9 relative to the incident power
    assert np.abs(R[0] - oR).max() < 1e-9 and np.abs(T[0] - oT).max() < 1e-9
    wR, wT = _weights(3)
    g = ctx.stack_backward(wR, wT)[0]
    og = np.array(stack_backward(ost, tp, wR[0], wT[0]))
    assert np.abs(g - og).max() <= 1e-9 * np.abs(og).max()


def test_config4_metagrating_matches_oracle(ctx):
    """Config 4 shape: 600 nm period, 633 nm, 9x9 orders (n = 162), four
    150 nm layers of 64 x 64 freeform pixels; objective T(+1, 0)."""
    layers = [smooth_pixels(4000 + l, 64, 64) for l in range(4)]
    d = _desc(layers, [0.15] * 4, 9)
    R, T, st = ctx.stack_forward([d])
    assert st[0] == 0
    ost, (oR, oT, tp) = _oracle(d)
    assert abs(R[0].sum() + T[0].sum() - 1.0) < 1e-10  # lossless
    assert np.abs(R[0] - oR).max() < 1e-9 and np.abs(T[0] - oT).max() < 1e-9
    m = 81
    wT = np.zeros((1, m))
    wT[0, order_index(9, 9, 1, 0)] = 1.0
    g = ctx.stack_backward(np.zeros((1, m)), wT)[0]
    og = np.array(stack_backward(ost, tp, np.zeros(m), wT[0]))
    assert g.shape == (4, 64, 64)
    assert np.abs(g - og).max() <= 1e-8 * np.abs(og).max()


def test_gradient_matches_device_central_differences(ctx):
    """64 random pixels of a config-4 stack against fourth-order central
    differences, (8 (f(h) - f(-h)) - (f(2h) - f(-2h))) / (12 h): 256
    perturbed stacks solved as one batch on the device.  The forward solve's
    rounding differs between neighbouring inputs by ~1e-11 of T (eigen-solver
    paths), so h = 1e-3 with an O(h^4) stencil keeps both truncation and
    rounding below 1e-6 of the gradient scale (h = 1e-6 would amplify the
    rounding to ~1e-5)."""
    layers = [smooth_pixels(4300 + l, 64, 64) for l in range(4)]
    d = _desc(layers, [0.15] * 4, 9)
    m = 81
    wT = np.zeros((1, m))
    wT[0, order_index(9, 9, 1, 0)] = 1.0
    ctx.stack_forward([d])
    g = ctx.stack_backward(np.zeros((1, m)), wT)[0]
    rng = np.random.default_rng(11)
    picks = [(int(rng.integers(4)), int(rng.integers(64)), int(rng.integers(64))) for _ in range(64)]
    h = 1e-3
    steps = (2.0, 1.0, -1.0, -2.0)
    batch = []
    for (l, i, j) in picks:
        for s in steps:
            lay = [a.copy() for a in layers]
            lay[l][i, j] += s * h
            batch.append(_desc(lay, [0.15] * 4, 9))
    _, T, st = ctx.stack_forward(batch)
    assert (st == 0).all()
    k = order_index(9, 9, 1, 0)
    f = T[:, k].reshape(len(picks), 4)
    fd = (8.0 * (f[:, 1] - f[:, 2]) - (f[:, 0] - f[:, 3])) / (12.0 * h)
    ad = np.array([g[l, i, j] for (l, i, j) in picks])
    assert np.abs(fd - ad).max() <= 1e-6 * np.abs(g).max(), np.abs(fd - ad).max() / np.abs(g).max()
    # per pixel: every picked pixel whose gradient is above 1% of the largest
    # carries a relative error below 1e-4 (the absolute bound above, divided
    # by the floor), and the floor leaves most picks in the check
    big = np.abs(ad) >= 1e-2 * np.abs(g).max()
    assert big.sum() >= len(picks) // 2, big.sum()
    rel = np.abs(fd - ad)[big] / np.abs(ad)[big]
    assert rel.max() <= 1e-4, rel.max()


def test_batch_equals_single_and_degenerate_layer(ctx):
    nx = 3
    a = _desc([smooth_pixels(4400, 8, 8, sigma=1.0), np.full((8, 8), 4.0)], [0.15, 0.2], nx)
    b = _desc([smooth_pixels(4401, 8, 8, sigma=1.0), smooth_pixels(4402, 8, 8, sigma=1.0)], [0.1, 0.3], nx,
              eps_in=1.5, eps_out=2.0)
    wR, wT = _weights(nx, 2)
    R2, T2, _ = ctx.stack_forward([a, b])
    g2 = ctx.stack_backward(wR, wT)
    for i, d in enumerate((a, b)):
        R1, T1, _ = ctx.stack_forward([d])
        g1 = ctx.stack_backward(wR[i:i + 1], wT[i:i + 1])
        assert np.abs(R1[0] - R2[i]).max() < 1e-13 and np.abs(T1[0] - T2[i]).max() < 1e-13
        assert np.abs(g1[0] - g2[i]).max() <= 1e-12 * np.abs(g1).max()
        ost, (_, _, tp) = _oracle(d)
        og = np.array(stack_backward(ost, tp, wR[i], wT[i]))
        assert np.abs(g2[i] - og).max() <= 1e-9 * np.abs(og).max()


def test_stack_lanes_match_one_engine(ctx, monkeypatch):
    """Seven stacks dealt over three concurrent engines: forward powers and
    gradients equal those of one engine, in call order."""
    nx = 3
    ds = [_desc([smooth_pixels(4500 + 2 * i, 8, 8, sigma=1.0), smooth_pixels(4501 + 2 * i, 8, 8, sigma=1.0)],
                [0.1 + 0.02 * i, 0.2], nx) for i in range(7)]
    wR, wT = _weights(nx, 7)
    wT = wT * np.arange(1, 8)[:, None]
    out = {}
    for lanes in ("1", "3"):
        monkeypatch.setenv("VRC_LANES", lanes)
        R, T, st = ctx.stack_forward(ds)
        out[lanes] = (R, T, st, ctx.stack_backward(wR, wT))
    for a, b in zip(out["1"], out["3"]):
        assert np.array_equal(a, b)


def test_thickness_gradient(ctx):
    """dL/d(layer thickness) against the oracle and against fourth-order
    central differences solved on the device in one batch."""
    nx = 3
    layers = [smooth_pixels(4700 + l, 8, 8, sigma=1.0) for l in range(3)]
    thick = [0.12, 0.2, 0.15]
    wR, wT = _weights(nx)
    ctx.stack_forward([_desc(layers, thick, nx)])
    _, gt = ctx.stack_backward(wR, wT, want_thick=True)
    ost, (_, _, tp) = _oracle(_desc(layers, thick, nx))
    _, ogt = stack_backward(ost, tp, wR[0], wT[0], want_thick=True)
    assert np.abs(gt[0] - ogt).max() <= 1e-9 * np.abs(ogt).max()
    h = 1e-4
    batch = []
    for l in range(3):
        for s in (2.0, 1.0, -1.0, -2.0):
            t2 = list(thick)
            t2[l] += s * h
            batch.append(_desc(layers, t2, nx))
    R, T, st = ctx.stack_forward(batch)
    assert (st == 0).all()
    L = (R * wR[0]).sum(axis=1) + (T * wT[0]).sum(axis=1)
    f = L.reshape(3, 4)
    fd = (8.0 * (f[:, 1] - f[:, 2]) - (f[:, 0] - f[:, 3])) / (12.0 * h)
    assert np.abs(fd - gt[0]).max() <= 1e-6 * np.abs(gt).max()


def test_fifteen_orders_stack_matches_oracle(ctx):
    """15 x 15 orders (n = 450): the pixel adjoint keeps its Toeplitz-diagonal
    sums in global scratch and runs with fewer warps per CTA."""
    nx = 15
    layers = [smooth_pixels(4800 + l, 16, 16, sigma=1.5) for l in range(2)]
    d = _desc(layers, [0.15, 0.1], nx)
    R, T, st = ctx.stack_forward([d])
    assert st[0] == 0
    ost, (oR, oT, tp) = _oracle(d)
    assert np.abs(R[0] - oR).max() < 1e-9 and np.abs(T[0] - oT).max() < 1e-9
    m = nx * nx
    wT = np.zeros((1, m))
    wT[0, order_index(nx, nx, 1, 0)] = 1.0
    g = ctx.stack_backward(np.zeros((1, m)), wT)[0]
    og = np.array(stack_backward(ost, tp, np.zeros(m), wT[0]))
    assert np.abs(g - og).max() <= 1e-8 * np.abs(og).max()


@pytest.mark.parametrize("lanes", ["1", "3"])
def test_internal_fields_match_oracle(ctx, monkeypatch, lanes):
    """Transverse E images at every interface (basis invariant) against the
    oracle, for stacks solved on one and on three lanes."""
    from oracle.stack_adjoint import stack_fields
    monkeypatch.setenv("VRC_LANES", lanes)
    nx = 3
    ds = [_desc([smooth_pixels([5100, i, l], 8, 8, sigma=1.0) for l in range(3)], [0.15, 0.1 + 0.02 * i, 0.2], nx)
          for i in range(6)]
    ctx.stack_forward(ds)
    amps, img = ctx.stack_fields(8, 6)
    assert amps.shape == (6, 4, 2, 18) and img.shape == (6, 4, 2, 6, 8)
    for i, d in enumerate(ds):
        ost, (_, oT, tp) = _oracle(d)
        _, _, _, of = stack_fields(ost, tp, 8, 6)
        assert np.abs(img[i] - of).max() <= 1e-9 * np.abs(of).max()
        # entrance: the incident amplitudes are c = W0^-1 s, the exit has nothing incoming
        assert np.abs(amps[i, -1, 1]).max() == 0.0
