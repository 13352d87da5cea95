"""vrc_eig_noalloc: the eigensolver entry point that allocates no device
memory, for callers that cannot let a library call cudaMalloc (their own
memory pool owns the device, or an allocation's implicit synchronisation is
not acceptable).  Its scratch is a fixed area inside the library.

Checked through the C-ABI, twice in a row (so that the second call runs on
the scratch left by the first):
* against vrc_eig (the allocating entry point) on the same matrices,
  eigenvalues matched (their order may differ) at the eigensolver tests'
  tolerance and the normalised eigenvectors to 1e-10;
* directly: the residual ||A W - W diag(lam)|| and the eigenvalues against
  numpy's (LAPACK zgeev), unit-norm columns;
* that a warmed-up call leaves the device's free memory and torch's
  allocator untouched (it allocates nothing).
The test buffers are allocated by torch here, in the test; the entry point
itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    # column-major device copy: the C-order transpose has the column-major bytes
    return torch.from_numpy(np.ascontiguousarray(a.T)).to("cuda")


def _call(L, torch, dA, dW, dlam, n):
    stream = torch.cuda.current_stream().cuda_stream
    return L.vrc_eig_noalloc(n, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dW.data_ptr()),
                             ctypes.c_void_p(dlam.data_ptr()), ctypes.c_void_p(stream))


def _match_eigs(lam, ref):
    """Greedy nearest matching of two eigenvalue lists; max distance."""
    ref = list(ref)
    worst = 0.0
    for x in lam:
        d = np.abs(np.asarray(ref) - x)
        k = int(np.argmin(d))
        worst = max(worst, float(d[k]))
        ref.pop(k)
    return worst


@pytest.mark.parametrize("n", [40, 242])
def test_eig_noalloc_matches_eig_twice(ctx, n):
    import torch

    from varrcwa_b200 import capi

    L = capi.lib()
    rng = np.random.default_rng(11 + n)
    for call in range(2):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        lam_ref, W_ref = ctx.eig(A)
        dA = _dev(A, torch)
        dW = torch.full((n, n), complex("nan"), dtype=torch.complex128, device="cuda")
        dlam = torch.full((n,), complex("nan"), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        assert _call(L, torch, dA, dW, dlam, n) == capi.VRC_OK, call
        W = dW.cpu().numpy().T
        lam = dlam.cpu().numpy()
        assert np.all(np.isfinite(W)) and np.all(np.isfinite(lam))
        # the allocating entry point may order the eigenvalues differently
        # (its Hessenberg reduction is blocked for larger n): match them, then
        # the unit, largest-component-real eigenvector columns
        scale = np.abs(A).max()
        order = []
        free = list(range(n))
        for x in lam:
            k = min(free, key=lambda q: abs(lam_ref[q] - x))
            order.append(k)
            free.remove(k)
        assert np.abs(lam - lam_ref[order]).max() <= 1e-12 * scale * n, call
        assert np.abs(W - W_ref[:, order]).max() <= 1e-10, call
        # directly: A W = W diag(lam), unit columns, eigenvalues of LAPACK's zgeev
        scale = np.linalg.norm(A, 2)
        res = np.linalg.norm(A @ W - W * lam[None, :], 2)
        assert res <= 1e-12 * n * scale, (call, res / scale)
        assert np.allclose(np.linalg.norm(W, axis=0), 1.0, rtol=0, atol=1e-13)
        assert _match_eigs(lam, np.linalg.eigvals(A)) <= 1e-11 * scale, call
        # the input is left untouched
        assert np.array_equal(dA.cpu().numpy().T, A)


def test_eig_noalloc_allocates_nothing(ctx):
    import torch

    from varrcwa_b200 import capi

    L = capi.lib()
    n = 128
    A = np.random.default_rng(5).standard_normal((n, n)) + 0j
    dA = _dev(A, torch)
    dW = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    dlam = torch.zeros((n,), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    assert _call(L, torch, dA, dW, dlam, n) == capi.VRC_OK  # warm-up: scratch lookup, kernel attributes
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = torch.cuda.memory_stats()
    for _ in range(3):
        assert _call(L, torch, dA, dW, dlam, n) == capi.VRC_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = torch.cuda.memory_stats()
    assert free1 == free0
    for k in ("allocation.all.allocated", "reserved_bytes.all.current", "segment.all.allocated"):
        assert stats1.get(k, 0) == stats0.get(k, 0), k


def test_eig_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    from varrcwa_b200 import capi

    L = capi.lib()
    assert L.vrc_eig_noalloc(257, None, None, None, None) == capi.VRC_EINVAL
    assert L.vrc_eig_noalloc(1, None, None, None, None) == capi.VRC_EINVAL
