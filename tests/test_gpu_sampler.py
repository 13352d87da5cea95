"""Caller-sampler cells (VRC_GEOM_SAMPLER) through the C ABI: the engine's
integrators driven by a sampler callback of the caller instead of the
engine's own Fourier-Toeplitz assembly, the way a LayerSampler subclass
drives the reference's integrators (src/core/LayerSampler.h:49-55).

Here the callback is the oracle's sampler of a structure that the engine
can also assemble itself, so the two routes must agree: P, Q to 1e-12, and
the integrators (replayed on fixed cuts) and the per-order powers with
half-space ends to 1e-9 relative."""
import ctypes

import numpy as np
import pytest

from oracle import varrcwa_oracle as O
from oracle.structures_adapter import end_bases, make_sampler
from tests.cases import CASES
from tests.conftest import fourier_blocks, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _sampler_cell(d, device=False):
    s = make_sampler(d)
    cell = dict(kind="sampler", lam=d["lam"], nx=d["nx"], ny=d["ny"], z0=d["z0"], z1=d["z1"],
                end0=d.get("end0"), end1=d.get("end1"))
    if d.get("Lx"):
        cell.update(Lx=d["Lx"], Ly=d["Ly"])
    if device:
        # the device callback copies the oracle's matrices into the engine's
        # device buffers on the engine's stream (cudaMemcpyAsync of the CUDA
        # runtime the library itself loaded), from pageable host copies that
        # must outlive the transfer: the stream is synchronised before return
        rt = ctypes.CDLL("libcudart.so.12")
        rt.cudaMemcpyAsync.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                       ctypes.c_void_p]
        rt.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]
        n = 2 * d["nx"] * d["ny"]

        def sample_device(z, P_ptr, Q_ptr, stream):
            P, Q = s.sample(z)
            for M, ptr in ((P, P_ptr), (Q, Q_ptr)):
                buf = np.ascontiguousarray(M.T)  # column-major bytes
                if rt.cudaMemcpyAsync(ptr, buf.ctypes.data, n * n * 16, 1, stream) != 0:
                    return 3
                # pageable source: wait before the buffer goes out of scope
                if rt.cudaStreamSynchronize(stream) != 0:
                    return 4
            return 0

        cell["sample_device"] = sample_device
    else:
        cell["sample"] = s.sample
    return cell, s


@pytest.mark.parametrize("device", [False, True])
def test_sampler_cell_pq_and_integrators_match_engine_assembly(ctx, device):
    d = CASES["asym_redheffer"]["desc"]
    cell, s = _sampler_cell(dict(d, end0=None, end1=None), device=device)
    zs = [0.0, 0.37, 1.5]
    P, Q = ctx.sample_pq(cell, zs)
    for k, z in enumerate(zs):
        oP, oQ = s.sample(z)
        assert relerr(P[k], oP) < 1e-15 and relerr(Q[k], oQ) < 1e-15  # the callback's own matrices
    cuts = [0.0, 0.2, 0.55, 0.9, 1.5]
    a = ctx.redheffer_segments([cell], [cuts])[0]
    S = O.redheffer_segments(s, 0.0, 1.5, cuts)
    F, G = fourier_blocks(a), S.fourier_blocks()
    for k in F:
        assert relerr(F[k], G[k]) < TOL, k
    for name, N in (("rcwa", 6), ("differential", 3)):
        r = getattr(ctx, name)([cell], N)[0]
        ref = (O.rcwa_compute if name == "rcwa" else O.differential_compute)(s, 0.0, 1.5, N)
        F, G = fourier_blocks(r), ref.fourier_blocks()
        for k in F:
            assert relerr(F[k], G[k]) < TOL, (name, k)
    # the adaptive run: a structure without degenerate modes, so the device
    # reproduces the oracle's tree from the callback's samples
    r = ctx.redheffer([cell], pe=1e-3)[0]
    So = O.redheffer_compute(s, 0.0, 1.5, pe=1e-3)
    assert r["status"] == 0 and r["N"] == So.N
    F, G = fourier_blocks(r), So.fourier_blocks()
    for k in F:
        assert relerr(F[k], G[k]) < TOL, k


def test_sampler_cell_order_powers_with_half_spaces(ctx):
    from varrcwa_b200 import structures as st
    d = st.pillar_cell(2000, norders=5, lam=0.532, npix=32)
    cell, s = _sampler_cell(d)
    p = ctx.order_powers([cell], method="rcwa", nslices=4, side=1)[0]
    e0, e1 = end_bases(d, s)
    S = O.rcwa_compute(s, d["z0"], d["z1"], 4, end0=e0, end1=e1)
    for pol, (px, py) in enumerate(((1.0, 0.0), (0.0, 1.0))):
        R, T = O.order_powers(S, s, d["end1"], d["end0"], px, py, side="top")
        assert relerr(p["R"][pol], R) < TOL and relerr(p["T"][pol], T) < TOL
        assert abs(p["R"][pol].sum() + p["T"][pol].sum() - 1.0) < 1e-10


def test_failing_sampler_is_reported(ctx):
    from varrcwa_b200.capi import VrcError
    d = CASES["asym_redheffer"]["desc"]
    cell, _ = _sampler_cell(dict(d, end0=None, end1=None))

    def bad(z):
        raise RuntimeError("no sample")

    cell["sample"] = bad
    with pytest.raises(VrcError) as e:
        ctx.redheffer([cell], pe=1e-2)
    assert e.value.status == 1
