"""GPU parity of the batched kernels (GEMM, inverse, eigensolver) through the C-ABI."""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu
rng = np.random.default_rng(7)


def _rand(b, n):
    return rng.standard_normal((b, n, n)) + 1j * rng.standard_normal((b, n, n))


@pytest.mark.parametrize("n", [1, 5, 64, 82, 98, 162, 242, 450])
def test_zgemm(ctx, n):
    A, B = _rand(3, n), _rand(3, n)
    assert relerr(ctx.zgemm(A, B), A @ B) < 1e-14


@pytest.mark.parametrize("n", [2, 21, 82, 242, 450])
def test_zinv(ctx, n):
    A = _rand(2, n)
    Ai, st = ctx.zinv(A)
    assert np.all(st == 0)
    # forward error relative to the conditioning
    for k in range(2):
        assert relerr(Ai[k], np.linalg.inv(A[k])) < 1e-12 * np.linalg.cond(A[k])


def test_zinv_singular_reports_status(ctx):
    A = _rand(1, 6)
    A[0, :, 3] = 0.0
    _, st = ctx.zinv(A)
    assert st[0] == 4  # VRC_ESINGULAR


@pytest.mark.parametrize("n", [3, 20, 82, 162, 242, 338, 450])
def test_eig_random(ctx, n):
    A = _rand(1, n)[0]
    lam, W = ctx.eig(A)
    scale = np.abs(A).max()
    assert np.abs(A @ W - W * lam[None, :]).max() < 1e-12 * scale * n
    ref = np.linalg.eigvals(A)
    assert max(np.abs(ref - l).min() for l in lam) < 1e-12 * scale * n
    assert np.abs(np.linalg.norm(W, axis=0) - 1).max() < 1e-13


def test_eig_diagonal_and_degenerate(ctx):
    d = np.array([3.0, 1.0, 3.0, -2.0, 1.0 + 1j, 3.0], dtype=np.complex128)
    lam, W = ctx.eig(np.diag(d))
    assert np.allclose(np.sort_complex(lam), np.sort_complex(d), atol=1e-14)
    assert np.linalg.matrix_rank(W) == len(d)


def test_eig_batched_equals_single(ctx):
    A = _rand(4, 40)
    lam_b, W_b = ctx.eig(A)
    for k in range(4):
        lam, W = ctx.eig(A[k])
        assert np.array_equal(lam, lam_b[k]) and np.array_equal(W, W_b[k])


@pytest.mark.parametrize("n", [82, 98, 162])
def test_zgemm_tiles_identical(ctx, n, monkeypatch):
    """The 32 x 32 and 64 x 64 tiles accumulate every element over k in the
    same order: their products agree bit for bit (so the engine's tile
    autotuning cannot change results)."""
    A, B = _rand(70, n), _rand(70, n)
    out = {}
    for tile in ("64", "32"):
        monkeypatch.setenv("VRC_GEMM_TILE", tile)
        out[tile] = ctx.zgemm(A, B)
    assert np.array_equal(out["64"], out["32"])
    assert relerr(out["32"], A @ B) < 1e-14


@pytest.mark.parametrize("mode", ["2", "1"])
def test_gemm_bulk_staging_bit_identical(ctx, mode, monkeypatch):
    """The 64 x 64 tile with its operands staged by bulk copies
    (VRC_GEMM_BULK=2: two CTAs per SM, 1: one) computes the same products bit
    for bit as the 16-byte cp.async staging: square products with ragged
    edges (n = 242 = 3 x 64 + 50, k = 30 x 8 + 2), and the eigensolver, whose
    blocked Hessenberg reduction multiplies rectangular and conjugate-
    transposed operands."""
    A, B = _rand(16, 242), _rand(16, 242)
    E = _rand(3, 242)
    monkeypatch.setenv("VRC_GEMM_TILE", "64")
    monkeypatch.delenv("VRC_GEMM_BULK", raising=False)
    ref = ctx.zgemm(A, B)
    lam0, W0 = ctx.eig(E)
    monkeypatch.setenv("VRC_GEMM_BULK", mode)
    out = ctx.zgemm(A, B)
    lam1, W1 = ctx.eig(E)
    assert np.array_equal(out, ref)
    assert relerr(out, A @ B) < 1e-14
    assert np.array_equal(lam1, lam0) and np.array_equal(W1, W0)
