"""vrc_eig_noalloc: the eigensolver entry point that allocates no device
memory, for callers that cannot let a library call cudaMalloc (their own
memory pool owns the device, or an allocation's implicit synchronisation is
not acceptable).  Its scratch is a fixed area inside the library.

Checked through the C-ABI against vrc_eig (the allocating entry point) on
the same matrices, twice in a row, so that the second call runs on the
scratch left by the first.  The test buffers are allocated by torch here,
in the test; the entry point itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _dev(a, torch):
    # column-major device copy: the C-order transpose has the column-major bytes
    return torch.from_numpy(np.ascontiguousarray(a.T)).to("cuda")


@pytest.mark.parametrize("n", [40, 242])
def test_eig_noalloc_matches_eig_twice(ctx, n):
    import torch

    from varrcwa_b200 import capi

    L = capi.lib()
    rng = np.random.default_rng(11 + n)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        lam_ref, W_ref = ctx.eig(A)
        dA = _dev(A, torch)
        dW = torch.full((n, n), complex("nan"), dtype=torch.complex128, device="cuda")
        dlam = torch.full((n,), complex("nan"), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        st = L.vrc_eig_noalloc(n, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dW.data_ptr()),
                               ctypes.c_void_p(dlam.data_ptr()), ctypes.c_void_p(stream))
        assert st == capi.VRC_OK, call
        W = dW.cpu().numpy().T
        lam = dlam.cpu().numpy()
        assert np.all(np.isfinite(W)) and np.all(np.isfinite(lam))
        assert np.abs(lam - lam_ref).max() <= TOL * np.abs(lam_ref).max(), call
        assert np.abs(W - W_ref).max() <= TOL, call
        # the input is left untouched
        assert np.array_equal(dA.cpu().numpy().T, A)


def test_eig_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    from varrcwa_b200 import capi

    L = capi.lib()
    assert L.vrc_eig_noalloc(257, None, None, None, None) == capi.VRC_EINVAL
    assert L.vrc_eig_noalloc(1, None, None, None, None) == capi.VRC_EINVAL
