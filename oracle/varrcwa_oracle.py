"""CPU restatement of the varRCWA reference path (numpy, complex128).

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may
import it.  The product path (``varrcwa_b200``) never calls into it.

Parity status: **parity unpinned**.  The reference ships no golden vectors and
no assertions (its ``src/tests/*.cpp`` drivers write ground-truth files at run
time), and its CPU build needs Eigen, MKL/LAPACKE and TBB, none of which is
present, so it cannot be compiled to produce vectors.  This restatement is
pinned instead by analytic known-answer tests (homogeneous media, z-invariant
structures, energy conservation, Fresnel interfaces) in ``tests/``.

Each function cites the reference file:line it restates (paths relative to
the reference project root).  Third-party arithmetic used by the reference:
Eigen (GEMM, PartialPivLU, BDCSVD) and MKL ``LAPACKE_zgeev``; here numpy's
LAPACK (OpenBLAS) stands in: ``numpy.linalg.eig`` is ``zgeev`` with the same
right-eigenvector convention, ``numpy.linalg.solve``/``inv`` are
``zgetrf/zgetrs`` (Eigen PartialPivLU), and the BDCSVD least-squares solve of
a square nonsingular ``fe33`` is replaced by an LU solve (identical up to
rounding).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg

PI = 3.1415926535897932  # src/rcwa/defns.h:25 (double precision pi)

# Fourier solver options, src/rcwa/FourierSolver2D.h:7-12
CONTINUOUS_XY = 0
DISCONTINUOUS_X = 1
DISCONTINUOUS_Y = 2


# ---------------------------------------------------------------------------
# Math helpers
# ---------------------------------------------------------------------------
def sinc(x):
    """sin(pi x)/(pi x), 1 at 0.  src/rcwa/MathFunction.h:6-9"""
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    nz = x != 0.0
    out[nz] = np.sin(PI * x[nz]) / (PI * x[nz])
    return out


def toeplitz_dense(vec: np.ndarray) -> np.ndarray:
    """T[r, c] = vec[n-1 + r - c].  src/rcwa/ToeplitzMatrixXcs.cpp:8-38"""
    n = (vec.shape[0] + 1) // 2
    r = np.arange(n)[:, None]
    c = np.arange(n)[None, :]
    return vec[n - 1 + r - c]


def block_toeplitz_dense(mat: np.ndarray) -> np.ndarray:
    """F[(m,n),(j,l)] = mat[nx-1+m-j, ny-1+n-l], row index m*ny+n.
    src/rcwa/BlockToeplitzMatrixXcs.cpp:5-53"""
    nx = (mat.shape[0] + 1) // 2
    ny = (mat.shape[1] + 1) // 2
    m = np.repeat(np.arange(nx), ny)
    n = np.tile(np.arange(ny), nx)
    di = nx - 1 + m[:, None] - m[None, :]
    dj = ny - 1 + n[:, None] - n[None, :]
    return mat[di, dj]


# ---------------------------------------------------------------------------
# 1D Fourier solver (closed-form coefficients of piecewise-constant f)
# ---------------------------------------------------------------------------
def fourier_matrix_1d(x: np.ndarray, d: float, M: int) -> np.ndarray:
    """E[i, j] so that Ff = E @ f.  Row i <-> harmonic m = i - (M-1)/2.
    Cell j spans [x[j], x[j+1]] (unsorted coordinates allowed: negative width).
    src/rcwa/FourierSolver1D.cpp:11-41"""
    x = np.asarray(x, dtype=np.float64)
    x0 = x[:-1]
    x1 = x[1:]
    m = (np.arange(M) - (M - 1) // 2).astype(np.float64)[:, None]
    w = (x1 - x0)[None, :]
    E = np.where(
        m == 0,
        (w / d) + 0j,
        (1.0 / d) * np.exp(-1j * (m * PI * (x1 + x0)[None, :] / d)) * sinc(m * w / d) * w,
    )
    return E


def fourier_solve_1d(x, d, f, M):
    """FourierSolver1D::solve, src/rcwa/FourierSolver1D.cpp:11-41"""
    return fourier_matrix_1d(x, d, M) @ np.asarray(f, dtype=np.complex128)


def reorder_index(x: np.ndarray) -> np.ndarray:
    """FourierSolver1D::reorder, src/rcwa/FourierSolver1D.cpp:145-154.
    The reference uses (unstable) std::sort; ties are ordered stably here."""
    return np.argsort(np.asarray(x), kind="stable")


def refill(x: np.ndarray, f: np.ndarray, rindex: np.ndarray) -> np.ndarray:
    """Painter's-order refill for crossed coordinates.
    src/rcwa/FourierSolver1D.cpp:156-193"""
    f = np.asarray(f, dtype=np.complex128)
    newf = f.copy()
    need = any(rindex[i] != i for i in range(len(rindex) - 1))
    if need:
        for i in range(f.shape[-1]):
            if x[i] >= x[i + 1]:
                continue
            for j in range(newf.shape[-1]):
                if rindex[i] <= j and rindex[i + 1] >= j + 1:
                    newf[..., j] = f[..., i]
    return newf


# ---------------------------------------------------------------------------
# 2D Fourier solver (Laurent rule for e33, Li inverse rule for e11/e22)
# ---------------------------------------------------------------------------
def fourier_solve_2d(x, y, f, nx, ny, opt) -> np.ndarray:
    """FourierSolver2D::solve, src/rcwa/FourierSolver2D.cpp:12-351.
    f has shape (len(y)-1, len(x)-1): rows are y-strips, columns x-cells."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    f = np.asarray(f, dtype=np.complex128)
    dx = x[-1] - x[0]
    dy = y[-1] - y[0]
    index = reorder_index(x)
    rindex = np.empty_like(index)
    rindex[index] = np.arange(len(index))
    newf = refill(x, f, rindex)
    # strip y-Fourier factors: fY1_i = FT_y(indicator of strip i), (2ny-1) coeffs
    Ey = fourier_matrix_1d(y, dy, 2 * ny - 1)  # (2ny-1, nstrips)
    if opt == DISCONTINUOUS_X:  # :43-144
        Ex = fourier_matrix_1d(x, dx, 2 * nx - 1)
        Ff = np.zeros((nx * ny, nx * ny), dtype=np.complex128)
        for i in range(len(y) - 1):
            finv = Ex @ (1.0 / newf[i])
            tinv = np.linalg.inv(toeplitz_dense(finv))
            Ff += np.kron(tinv, toeplitz_dense(Ey[:, i]))
        return Ff
    if opt == DISCONTINUOUS_Y:  # :145-249
        Eyf = Ey
        xs = x[index]
        Exs = fourier_matrix_1d(xs, dx, 2 * nx - 1)  # cells in sorted order
        Ff = np.zeros((nx * ny, nx * ny), dtype=np.complex128)
        for i in range(len(x) - 1):
            finv = Eyf @ (1.0 / newf[:, i])
            tinv = np.linalg.inv(toeplitz_dense(finv))
            Ff += np.kron(toeplitz_dense(Exs[:, i]), tinv)
        return Ff
    if opt == CONTINUOUS_XY:  # :250-349
        Ex = fourier_matrix_1d(x, dx, 2 * nx - 1)
        four = Ex @ newf.T @ Ey.T  # (2nx-1, 2ny-1)
        return block_toeplitz_dense(four)
    raise ValueError(opt)


# ---------------------------------------------------------------------------
# K matrices (periodic or PML boundaries)
# ---------------------------------------------------------------------------
def alpha_beta(nx, ny, Lx, Ly):
    """Diagonals alpha, beta; index ny*i + j.  src/core/LayerSampler.cpp:9-32"""
    Nx = (nx - 1) // 2
    Ny = (ny - 1) // 2
    i = np.repeat(np.arange(nx), ny)
    j = np.tile(np.arange(ny), nx)
    alpha = (2 * PI / Lx) * (i - Nx).astype(np.float64)
    beta = (2 * PI / Ly) * (j - Ny).astype(np.float64)
    return alpha.astype(np.complex128), beta.astype(np.complex128)


def pml_solve_1d(b0, b1, L, gamma, n, coeff):
    """PMLSolver1D::solve, src/rcwa/PMLSolver1D.cpp:15-30"""
    def expipi(v):
        return np.exp(1j * PI * v)

    bm = (b1 - b0) / L
    bp = (b1 + b0) / L
    s = lambda v: float(sinc(np.array(v)))
    r = 4.0 * s(n * bm - 0.5) * expipi(-(n * bp + coeff * 0.5))
    r += 8.0 * expipi(-(n * bp)) * s(n * bm)
    r += -2.0 * gamma * expipi(-(n * bp)) * s(n * bm)
    r += 4.0 * s(n * bm + 0.5) * expipi(-(n * bp - coeff * 0.5))
    r += gamma * s(n * bm - 1.0) * expipi(-(n * bp + coeff * 1.0))
    r += gamma * s(n * bm + 1.0) * expipi(-(n * bp - coeff * 1.0))
    r *= bm / 16.0
    return r


def pml_factors(nx, ny, gamma, b0, b1, u0, u1, l0, l1, r0, r1, Lx, Ly):
    """Block-Toeplitz PML stretch factors Fx, Fy (dense).
    src/core/LayerSampler.cpp:34-111"""
    nPx, nPy = 2 * nx - 1, 2 * ny - 1
    maxPx, maxPy = (nPx - 1) // 2, (nPy - 1) // 2
    fyy = np.zeros(nPy, dtype=np.complex128)
    for i in range(nPy):
        n = i - maxPy
        v = (u0 - b1) / Ly * float(sinc(np.array(n * (u0 - b1) / Ly))) / np.exp(
            1j * PI * (n * (b1 + u0) / Ly))
        v += pml_solve_1d(b0, b1, Ly, gamma, n, 1.0)
        v += pml_solve_1d(u0, u1, Ly, gamma, n, -1.0)
        fyy[i] = v
    fxx = np.zeros(nPx, dtype=np.complex128)
    for i in range(nPx):
        m = i - maxPx
        v = (r0 - l1) * float(sinc(np.array(m * (r0 - l1) / Lx))) / Lx / np.exp(
            1j * (PI * m * (l1 + r0) / Lx))
        v += pml_solve_1d(l0, l1, Lx, gamma, m, 1.0)
        v += pml_solve_1d(r0, r1, Lx, gamma, m, -1.0)
        fxx[i] = v
    fyx = np.zeros(nPx, dtype=np.complex128)
    for i in range(nPx):
        m = i - maxPx
        if m == 0:
            fyx[i] = r1 - l0
        else:
            fyx[i] = (np.exp(-2j * PI / Lx * m * r1) - np.exp(-2j * PI / Lx * m * l0)) * (
                1j * Lx * Lx / (m * 2 * PI))
    fxy = np.zeros(nPy, dtype=np.complex128)
    for i in range(nPy):
        n = i - maxPy
        if n == 0:
            fxy[i] = u1 - b0
        else:
            fxy[i] = (np.exp(-2j * PI / Ly * n * u1) - np.exp(-2j * PI / Ly * n * b0)) * (
                1j * Ly * Ly / (2 * n * PI))
    fy = (1.0 / Lx) * np.outer(fyx, fyy)
    fx = (1.0 / Ly) * np.outer(fxx, fxy)
    return block_toeplitz_dense(fx), block_toeplitz_dense(fy)


def k_matrices(nx, ny, x, y, enable_pml):
    """Kx, Ky (dense, m x m).  src/core/LayerSampler.cpp:114-144 with the
    simulation region of src/core/VarLayerSampler.cpp:23-39."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    Lx = x[-1] - x[0]
    Ly = y[-1] - y[0]
    alpha, beta = alpha_beta(nx, ny, Lx, Ly)
    if enable_pml:
        gamma = 1.0 / (1.0 - 1.0j)
        Fx, Fy = pml_factors(nx, ny, gamma, y[0], y[1], y[-2], y[-1],
                             x[0], x[1], x[-2], x[-1], Lx, Ly)
        return Fx * alpha[None, :], Fy * beta[None, :]
    return np.diag(alpha), np.diag(beta)


# ---------------------------------------------------------------------------
# P, Q assembly
# ---------------------------------------------------------------------------
def wave_eqn_coeff(x, y, eps, Kx, Ky, lam, nx, ny):
    """Layer::waveEqnCoeff, src/rcwa/Layer.cpp:36-171 (no derivatives).
    Returns (P, Q), each n x n with n = 2*nx*ny."""
    fe11 = fourier_solve_2d(x, y, eps, nx, ny, DISCONTINUOUS_X)
    fe22 = fourier_solve_2d(x, y, eps, nx, ny, DISCONTINUOUS_Y)
    fe33 = fourier_solve_2d(x, y, eps, nx, ny, CONTINUOUS_XY)
    m = nx * ny
    # BDCSVD(fe33).solve(K) (Layer.cpp:84-86): LU solve of the square system
    F = np.linalg.solve(fe33, np.concatenate([Kx, Ky], axis=1))
    F1h, F2h = F[:, :m], F[:, m:]
    k0 = 2 * PI / lam
    k02 = k0 * k0
    I = np.eye(m)
    P = np.empty((2 * m, 2 * m), dtype=np.complex128)
    P[:m, :m] = Kx @ F2h
    P[:m, m:] = -Kx @ F1h + k02 * I
    P[m:, :m] = Ky @ F2h - k02 * I
    P[m:, m:] = -Ky @ F1h
    Q = np.empty_like(P)
    Q[:m, :m] = -Kx @ Ky
    Q[:m, m:] = Kx @ Kx - k02 * fe22
    Q[m:, :m] = -Ky @ Ky + k02 * fe11
    Q[m:, m:] = Ky @ Kx
    return P, Q


# ---------------------------------------------------------------------------
# Eigen step
# ---------------------------------------------------------------------------
def gamma_sqrt(lam_: np.ndarray) -> np.ndarray:
    """GammaSqrtOp, src/rcwa/WaveEquationSolver.cpp:8-22"""
    g = np.sqrt(lam_.astype(np.complex128))
    g = np.where(g.imag < 0, -g, g)
    flip = (np.abs(g.imag) < np.abs(g.real)) & (g.real < 0)
    return np.where(flip, -g, g)


def wave_equation_solve(P, Q):
    """WaveEquationSolver::solve, src/rcwa/WaveEquationSolver.cpp:24-37
    (zgeev right vectors, src/rcwa/MKLEigenSolver.hpp:45-55)."""
    PQ = P @ Q
    lam_, W = np.linalg.eig(PQ)
    gam = gamma_sqrt(lam_)
    V = (Q @ W) * (1.0 / gam)[None, :]
    return W, V, gam


@dataclass
class Basis:
    """Eigen basis of one z-sample: E-field modes W, H-field modes V, gamma."""
    W: np.ndarray
    V: np.ndarray
    gam: np.ndarray

    def solveW(self, rhs):
        """W^{-1} rhs through a cached partial-pivot LU (Eigen PartialPivLU)."""
        if not hasattr(self, "_luW"):
            self._luW = scipy.linalg.lu_factor(self.W, check_finite=False)
        return scipy.linalg.lu_solve(self._luW, rhs, check_finite=False)

    def solveV(self, rhs):
        if not hasattr(self, "_luV"):
            self._luV = scipy.linalg.lu_factor(self.V, check_finite=False)
        return scipy.linalg.lu_solve(self._luV, rhs, check_finite=False)


# ---------------------------------------------------------------------------
# Samplers
# ---------------------------------------------------------------------------
class VarLayerSampler:
    """Tensor-grid sampler with moving coordinates.
    src/core/VarLayerSampler.cpp:10-69, src/core/LayerSampler.h:31-55."""

    def __init__(self, lam, nx, ny, x, y, eps, enable_pml=True):
        self.lam = float(lam)
        self.nx, self.ny = int(nx), int(ny)
        self.x = np.asarray(x, dtype=np.float64).copy()
        self.y = np.asarray(y, dtype=np.float64).copy()
        self.eps = np.asarray(eps, dtype=np.complex128).copy()
        self.enable_pml = bool(enable_pml)
        self.xrules: Dict[int, Callable[[float], float]] = {}
        self.yrules: Dict[int, Callable[[float], float]] = {}
        self.Kx, self.Ky = k_matrices(self.nx, self.ny, self.x, self.y, self.enable_pml)
        self.n_samples = 0

    @property
    def k0(self):
        return 2 * PI / self.lam

    @property
    def ndim(self):
        return 2 * self.nx * self.ny

    def add_x_rule(self, layout, rule):
        self.xrules[int(layout)] = rule

    def add_y_rule(self, layout, rule):
        self.yrules[int(layout)] = rule

    def geometry(self, z):
        x = self.x.copy()
        y = self.y.copy()
        for i, f in self.xrules.items():
            x[i] = f(z)
        for i, f in self.yrules.items():
            y[i] = f(z)
        return x, y, self.eps

    def sample(self, z):
        self.n_samples += 1
        x, y, eps = self.geometry(z)
        return wave_eqn_coeff(x, y, eps, self.Kx, self.Ky, self.lam, self.nx, self.ny)


class RasterSampler:
    """Uniform pixel-grid sampler: eps(z) is a (ny_pix, nx_pix) raster on a
    fixed uniform grid (a tensor grid whose eps table changes with z)."""

    def __init__(self, lam, nx, ny, Lx, Ly, raster_fn, enable_pml=False):
        self.lam = float(lam)
        self.nx, self.ny = int(nx), int(ny)
        self.raster_fn = raster_fn
        r0 = raster_fn(0.0)
        self.x = np.linspace(0.0, Lx, r0.shape[1] + 1)
        self.y = np.linspace(0.0, Ly, r0.shape[0] + 1)
        self.enable_pml = enable_pml
        self.Kx, self.Ky = k_matrices(self.nx, self.ny, self.x, self.y, enable_pml)
        self.n_samples = 0

    @property
    def k0(self):
        return 2 * PI / self.lam

    @property
    def ndim(self):
        return 2 * self.nx * self.ny

    def geometry(self, z):
        return self.x, self.y, self.raster_fn(z)

    def sample(self, z):
        self.n_samples += 1
        x, y, eps = self.geometry(z)
        return wave_eqn_coeff(x, y, eps, self.Kx, self.Ky, self.lam, self.nx, self.ny)


def homogeneous_basis(sampler, eps_val) -> Basis:
    """Eigen basis of a homogeneous medium eps_val with the sampler's K and
    harmonics (the reference solves such layers through Layer::solve,
    src/rcwa/Layer.cpp:173-190)."""
    nx, ny = sampler.nx, sampler.ny
    x = np.array([sampler.x[0], sampler.x[-1]])
    y = np.array([sampler.y[0], sampler.y[-1]])
    eps = np.array([[eps_val]], dtype=np.complex128)
    P, Q = wave_eqn_coeff(x, y, eps, sampler.Kx, sampler.Ky, sampler.lam, nx, ny)
    return Basis(*wave_equation_solve(P, Q))


# ---------------------------------------------------------------------------
# S-matrix building blocks
# ---------------------------------------------------------------------------
def star_right(S, s):
    """Redheffer star product accumulating s to the right of S (in place).
    src/core/RedhefferIntegrator.cpp:267-277"""
    Tdd, Tuu, Rud, Rdu = S
    tdd, tuu, rud, rdu = s
    n = Tdd.shape[0]
    C1 = np.linalg.inv(np.eye(n) - rdu @ Rud)
    C2 = np.eye(n) + Rud @ C1 @ rdu
    Rdu_n = Rdu + Tdd @ rdu @ C2 @ Tuu
    Tdd_n = Tdd @ C1 @ tdd
    Rud_n = rud + tuu @ Rud @ C1 @ tdd
    Tuu_n = tuu @ C2 @ Tuu
    return [Tdd_n, Tuu_n, Rud_n, Rdu_n]


def project_left(s, basis: Basis, leftW, leftV):
    """Re-express the left end of segment s (in basis `basis`) in the basis
    (leftW, leftV).  src/core/RedhefferIntegrator.cpp:253-262"""
    tdd, tuu, rud, rdu = s
    invW_W0 = basis.solveW(leftW)
    invV_V0 = basis.solveV(leftV)
    A = 0.5 * (invW_W0 + invV_V0)
    B = 0.5 * (invW_W0 - invV_V0)
    M = A - rdu @ B
    rdu_n = np.linalg.solve(M, rdu @ A - B)
    tdd_n = np.linalg.solve(M, tdd)
    rud_n = tuu @ B @ tdd_n + rud
    tuu_n = tuu @ A + tuu @ B @ rdu_n
    return [tdd_n, tuu_n, rud_n, rdu_n]


def project_right(S, leftW, leftV, W1, V1):
    """Re-express the right end of S from basis (leftW, leftV) to (W1, V1).
    src/core/RedhefferIntegrator.cpp:211-223"""
    Tdd, Tuu, Rud, Rdu = S
    invW0_W = np.linalg.solve(leftW, W1)
    invV0_V = np.linalg.solve(leftV, V1)
    A = 0.5 * (invW0_W + invV0_V)
    B = 0.5 * (invW0_W - invV0_V)
    M = A - Rud @ B
    Tuu_n = np.linalg.solve(M, Tuu)
    Rud_n = np.linalg.solve(M, Rud @ A - B)
    Rdu_n = Rdu + Tdd @ B @ Tuu_n
    Tdd_n = Tdd @ (B @ Rud_n + A)
    return [Tdd_n, Tuu_n, Rud_n, Rdu_n]


def project_left_end(S, W1, V1, W0, V0):
    """Final left-end projection of the RCWA / differential integrators:
    segment chain expressed in (W1, V1) on both ends, left end moved to
    (W0, V0).  src/core/RCWAIntegrator.cpp:73-86"""
    Tdd, Tuu, Rud, Rdu = S
    invW1_W0 = np.linalg.solve(W1, W0)
    invV1_V0 = np.linalg.solve(V1, V0)
    A = 0.5 * (invW1_W0 + invV1_V0)
    B = 0.5 * (invW1_W0 - invV1_V0)
    M = A - Rdu @ B
    Rdu_n = np.linalg.solve(M, Rdu @ A - B)
    Tdd_n = np.linalg.solve(M, Tdd)
    Rud_n = Tuu @ B @ Tdd_n + Rud
    Tuu_n = Tuu @ (B @ Rdu_n + A)
    return [Tdd_n, Tuu_n, Rud_n, Rdu_n]


def perturbation_segment(Pr, Qr, basis: Basis, k0, z0, z1, P3, Q3):
    """Simpson-rule first-order perturbative segment S-matrix and its error
    estimate.  src/core/RedhefferIntegrator.cpp:317-399.
    P3/Q3 = samples at (z0, (z0+z1)/2, z1).  Returns ([tdd,tuu,rud,rdu], err)."""
    W, V, gam = basis.W, basis.V, basis.gam
    dA, dB = [], []
    for Pk, Qk in zip(P3, Q3):
        x = basis.solveW((Pk - Pr) @ V)
        yv = basis.solveV((Qk - Qr) @ W)
        dA.append(x + yv)
        dB.append(x - yv)
    dz = z1 - z0
    ph = np.exp(1j * 0.5 * dz / k0 * gam)
    pf = np.exp(1j * dz / k0 * gam)
    c = 1j * dz / (6 * 2 * k0)
    tuu = c * (pf[:, None] * dA[0] + 4.0 * ph[:, None] * dA[1] * ph[None, :] + dA[2] * pf[None, :])
    err = np.abs(tuu).max()
    tuu[np.diag_indices_from(tuu)] += pf
    rud = -c * (pf[:, None] * dB[0] * pf[None, :] + 4.0 * ph[:, None] * dB[1] * ph[None, :] + dB[2])
    err = max(err, np.abs(rud).max())
    rdu = -c * (dB[0] + 4.0 * ph[:, None] * dB[1] * ph[None, :] + pf[:, None] * dB[2] * pf[None, :])
    err = max(err, np.abs(rdu).max())
    tdd = c * (dA[0] * pf[None, :] + 4.0 * ph[:, None] * dA[1] * ph[None, :] + pf[:, None] * dA[2])
    err = max(err, np.abs(tdd).max())
    tdd[np.diag_indices_from(tdd)] += pf
    return [tdd, tuu, rud, rdu], float(err)


def rcwa_slab(P, Q, k0, wz, W0, V0):
    """Uniform slab S-matrix expressed in (W0, V0) on both sides.
    dtmm::RCWAScatterMatrix::compute, src/rcwa/RCWAScatterMatrix.cpp:26-85.
    Returns (tuu, rud); the slab is symmetric: tdd = tuu, rdu = rud
    (src/rcwa/RCWAScatterMatrix.h:44-47)."""
    W, V, gam = wave_equation_solve(P, Q)
    X = np.exp(1j * gam * (wz / k0))
    F0 = np.linalg.solve(W, W0)
    G0 = np.linalg.solve(V, V0)
    A = F0 + G0
    B = F0 - G0
    invAB = np.linalg.solve(A, B)
    invAXA = np.linalg.solve(A, X[:, None] * A)
    invAXB = np.linalg.solve(A, X[:, None] * B)
    I = np.eye(P.shape[0])
    M = I - invAXB @ invAXB
    Rud = np.linalg.solve(M, invAXB @ invAXA - invAB)
    Tuu = np.linalg.solve(M, invAXA - invAXB @ invAB)
    return Tuu, Rud


# ---------------------------------------------------------------------------
# Integrators
# ---------------------------------------------------------------------------
@dataclass
class SMatrix:
    Tdd: np.ndarray
    Tuu: np.ndarray
    Rud: np.ndarray
    Rdu: np.ndarray
    W0: np.ndarray
    V0: np.ndarray
    gam0: np.ndarray
    W1: np.ndarray
    V1: np.ndarray
    gam1: np.ndarray
    N: int = 0
    n_eig: int = 0
    n_samples: int = 0
    nodes: List[Tuple[float, float, float, bool]] = field(default_factory=list)

    def blocks(self):
        return [self.Tdd, self.Tuu, self.Rud, self.Rdu]

    def fourier_blocks(self):
        """Basis-invariant view: blocks mapped to the Fourier E-field basis.
        Tuu: z0 -> z1, Tdd: z1 -> z0, Rdu: z0 -> z0, Rud: z1 -> z1."""
        W0i = np.linalg.inv(self.W0)
        W1i = np.linalg.inv(self.W1)
        return {
            "Tuu": self.W1 @ self.Tuu @ W0i,
            "Tdd": self.W0 @ self.Tdd @ W1i,
            "Rdu": self.W0 @ self.Rdu @ W0i,
            "Rud": self.W1 @ self.Rud @ W1i,
        }


def redheffer_compute(sampler, z0, z1, pe=1e-2, end0: Optional[Basis] = None,
                      end1: Optional[Basis] = None, max_depth=40) -> SMatrix:
    """Adaptive varRCWA, trisecting scheme.
    RedhefferIntegrator::compute + recursive_solve,
    src/core/RedhefferIntegrator.cpp:174-314 (the active #else branch).

    end0/end1 optionally replace the structure's own end bases (W0,V0 at z0,
    W1,V1 at z1) by other media (e.g. homogeneous half-spaces); None keeps the
    reference behaviour."""
    k0 = sampler.k0
    P0, Q0 = sampler.sample(z0)
    b0 = Basis(*wave_equation_solve(P0, Q0))
    P1, Q1 = sampler.sample(z1)
    b1 = Basis(*wave_equation_solve(P1, Q1))
    n_eig = 3
    zm = 0.5 * (z0 + z1)
    Pm, Qm = sampler.sample(zm)
    bm = Basis(*wave_equation_solve(Pm, Qm))
    e0 = end0 if end0 is not None else b0
    e1 = end1 if end1 is not None else b1
    n = P0.shape[0]
    state = {
        "S": [np.eye(n, dtype=np.complex128), np.eye(n, dtype=np.complex128),
              np.zeros((n, n), np.complex128), np.zeros((n, n), np.complex128)],
        "leftW": e0.W, "leftV": e0.V, "N": 0, "n_eig": n_eig, "nodes": [],
    }

    def recurse(Pr, Qr, basis, a, b, Pa, Pmid, Pb, Qa, Qmid, Qb, depth):
        seg, err = perturbation_segment(Pr, Qr, basis, k0, a, b, (Pa, Pmid, Pb), (Qa, Qmid, Qb))
        accepted = err <= pe or depth >= max_depth
        state["nodes"].append((a, b, err, bool(accepted)))
        if accepted:
            state["N"] += 1
            seg = project_left(seg, basis, state["leftW"], state["leftV"])
            state["leftW"], state["leftV"] = basis.W, basis.V
            state["S"] = star_right(state["S"], seg)
            return
        zm0 = 2.0 / 3.0 * a + 1.0 / 3.0 * b
        zm1 = 1.0 / 3.0 * a + 2.0 / 3.0 * b
        Pt, Qt = sampler.sample(0.5 * (a + zm0))
        Pk, Qk = sampler.sample(zm0)
        bt = Basis(*wave_equation_solve(Pt, Qt))
        state["n_eig"] += 1
        recurse(Pt, Qt, bt, a, zm0, Pa, Pt, Pk, Qa, Qt, Qk, depth + 1)
        Pt2, Qt2 = sampler.sample(zm1)
        recurse(Pr, Qr, basis, zm0, zm1, Pk, Pmid, Pt2, Qk, Qmid, Qt2, depth + 1)
        Pk2, Qk2 = sampler.sample(0.5 * (zm1 + b))
        bk = Basis(*wave_equation_solve(Pk2, Qk2))
        state["n_eig"] += 1
        recurse(Pk2, Qk2, bk, zm1, b, Pt2, Pk2, Pb, Qt2, Qk2, Qb, depth + 1)

    ns0 = getattr(sampler, "n_samples", 0)
    recurse(Pm, Qm, bm, z0, z1, P0, Pm, P1, Q0, Qm, Q1, 0)
    S = project_right(state["S"], state["leftW"], state["leftV"], e1.W, e1.V)
    return SMatrix(*S, e0.W, e0.V, e0.gam, e1.W, e1.V, e1.gam, N=state["N"],
                   n_eig=state["n_eig"], n_samples=getattr(sampler, "n_samples", 0) - ns0 + 3,
                   nodes=state["nodes"])


def redheffer_segments(sampler, z0, z1, cuts: Sequence[float],
                       end0: Optional[Basis] = None, end1: Optional[Basis] = None) -> SMatrix:
    """Non-adaptive varRCWA over explicit segment boundaries z0=c_0<...<c_K=z1,
    each segment with its own midpoint reference (the GPU reference's
    compute_direct(N) is the uniform case, src/gpu/RedhefferIntegratorGPU.cpp:361-412)."""
    k0 = sampler.k0
    cuts = list(cuts)
    P0, Q0 = sampler.sample(z0)
    b0 = Basis(*wave_equation_solve(P0, Q0))
    P1, Q1 = sampler.sample(z1)
    b1 = Basis(*wave_equation_solve(P1, Q1))
    e0 = end0 if end0 is not None else b0
    e1 = end1 if end1 is not None else b1
    n = P0.shape[0]
    S = [np.eye(n, dtype=np.complex128), np.eye(n, dtype=np.complex128),
         np.zeros((n, n), np.complex128), np.zeros((n, n), np.complex128)]
    leftW, leftV = e0.W, e0.V
    Pa, Qa = P0, Q0
    nodes = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        Pm, Qm = sampler.sample(0.5 * (a + b))
        Pb, Qb = (P1, Q1) if b == cuts[-1] else sampler.sample(b)
        bm = Basis(*wave_equation_solve(Pm, Qm))
        seg, err = perturbation_segment(Pm, Qm, bm, k0, a, b, (Pa, Pm, Pb), (Qa, Qm, Qb))
        nodes.append((a, b, err, True))
        seg = project_left(seg, bm, leftW, leftV)
        leftW, leftV = bm.W, bm.V
        S = star_right(S, seg)
        Pa, Qa = Pb, Qb
    S = project_right(S, leftW, leftV, e1.W, e1.V)
    return SMatrix(*S, e0.W, e0.V, e0.gam, e1.W, e1.V, e1.gam, N=len(cuts) - 1,
                   n_eig=len(cuts) + 1, nodes=nodes)


def tree_cuts(nodes) -> List[float]:
    """Segment boundaries of the accepted leaves of an adaptive run, in order."""
    leaves = [(a, b) for (a, b, _, acc) in nodes if acc]
    return [leaves[0][0]] + [b for (_, b) in leaves]


def rcwa_compute(sampler, z0, z1, N, end0: Optional[Basis] = None,
                 end1: Optional[Basis] = None) -> SMatrix:
    """Plain RCWA with N midpoint slices.  RCWAIntegrator::compute,
    src/core/RCWAIntegrator.cpp:20-87."""
    k0 = sampler.k0
    P1, Q1 = sampler.sample(z1)
    b1 = Basis(*wave_equation_solve(P1, Q1))
    e1 = end1 if end1 is not None else b1
    n = P1.shape[0]
    S = [np.eye(n, dtype=np.complex128), np.eye(n, dtype=np.complex128),
         np.zeros((n, n), np.complex128), np.zeros((n, n), np.complex128)]
    dz = (z1 - z0) / float(N)
    for i in range(N):
        z = z0 + (i + 0.5) * dz
        P, Q = sampler.sample(z)
        tuu, rud = rcwa_slab(P, Q, k0, dz, e1.W, e1.V)
        S = star_right(S, [tuu, tuu, rud, rud])
    P0, Q0 = sampler.sample(z0)
    b0 = Basis(*wave_equation_solve(P0, Q0))
    e0 = end0 if end0 is not None else b0
    S = project_left_end(S, e1.W, e1.V, e0.W, e0.V)
    return SMatrix(*S, e0.W, e0.V, e0.gam, e1.W, e1.V, e1.gam, N=N, n_eig=N + 2)


def differential_compute(sampler, z0, z1, N, end0: Optional[Basis] = None,
                         end1: Optional[Basis] = None) -> SMatrix:
    """Differential method, N slices of a 2nd-order propagator.
    DifferentialIntegrator::compute, src/core/DifferentialIntegrator.cpp:21-134."""
    k0 = sampler.k0
    P1_, Q1_ = sampler.sample(z1)
    b1 = Basis(*wave_equation_solve(P1_, Q1_))
    e1 = end1 if end1 is not None else b1
    W1, V1 = e1.W, e1.V
    n = P1_.shape[0]
    I = np.eye(n)
    S = [np.eye(n, dtype=np.complex128), np.eye(n, dtype=np.complex128),
         np.zeros((n, n), np.complex128), np.zeros((n, n), np.complex128)]
    dz = (z1 - z0) / float(N)
    P0, Q0 = sampler.sample(z0)
    for i in range(N):
        zl = z0 + i * dz
        zr = z0 + (i + 1) * dz
        zm = 0.5 * (zl + zr)
        P1, Q1 = sampler.sample(zm)
        P2, Q2 = sampler.sample(zr)
        a2 = dz * dz / (6.0 * k0 * k0)
        b2 = dz * dz / (4.0 * k0 * k0)
        h2 = dz * dz / (2.0 * k0 * k0)
        L11 = I - a2 * (P1 @ Q0 + P1 @ Q1 + P2 @ Q1 - b2 * (P2 @ Q1 @ P1 @ Q0))
        L12 = (1j * dz / (6.0 * k0)) * (P0 + 4.0 * P1 + P2 - h2 * (P1 @ Q1 @ P0 + P2 @ Q1 @ P1))
        L21 = (1j * dz / (6.0 * k0)) * (Q0 + 4.0 * Q1 + Q2 - h2 * (Q1 @ P1 @ Q0 + Q2 @ P1 @ Q1))
        L22 = I - a2 * (Q1 @ P0 + Q1 @ P1 + Q2 @ P1 - b2 * (Q2 @ P1 @ Q1 @ P0))
        iW_L11 = np.linalg.solve(W1, L11)
        iW_L12 = np.linalg.solve(W1, L12)
        iV_L21 = np.linalg.solve(V1, L21)
        iV_L22 = np.linalg.solve(V1, L22)
        A11 = 0.5 * (iW_L11 + iV_L21)
        A12 = 0.5 * (iW_L12 + iV_L22)
        A21 = 0.5 * (iW_L11 - iV_L21)
        A22 = 0.5 * (iW_L12 - iV_L22)
        T11 = A11 @ W1 + A12 @ V1
        T12 = A11 @ W1 - A12 @ V1
        T21 = A21 @ W1 + A22 @ V1
        T22 = A21 @ W1 - A22 @ V1
        tdd = np.linalg.inv(T22)
        rud = T12 @ tdd
        rdu = -np.linalg.solve(T22, T21)
        tuu = T11 + T12 @ rdu
        S = star_right(S, [tdd, tuu, rud, rdu])
        P0, Q0 = P2, Q2
    Pz0, Qz0 = sampler.sample(z0)
    b0 = Basis(*wave_equation_solve(Pz0, Qz0))
    e0 = end0 if end0 is not None else b0
    S = project_left_end(S, W1, V1, e0.W, e0.V)
    return SMatrix(*S, e0.W, e0.V, e0.gam, e1.W, e1.V, e1.gam, N=N, n_eig=2)


# ---------------------------------------------------------------------------
# Per-order diffraction power
# ---------------------------------------------------------------------------
def order_powers(S: SMatrix, sampler, eps_in, eps_out, px, py, side="bottom",
                 flux_norm=True):
    """Per-order reflected / transmitted power for a unit plane wave at
    normal incidence.  RCWASolver::scatterPlaneWave + generatePlaneWave,
    src/rcwa/RCWASolver.cpp:1622-1733, src/rcwa/Layer.cpp:339-366.

    Block naming is R_{out,in}: Rdu reflects an up-going wave at z0 into a
    down-going one, Rud reflects a down-going wave at z1 (this follows the
    star product, src/core/RedhefferIntegrator.cpp:274-277).
    side="bottom": incidence from the z0 medium (eps_in) upward; reflection
    by Rdu, transmission by Tuu into the z1 medium (eps_out).
    side="top": incidence from the z1 medium downward (Rud, Tdd), the
    reference's own choice (RCWASolver.cpp:1650-1651).
    flux_norm=True normalises both powers by the incident medium (so that
    R+T = 1 for lossless structures); False divides TRN by sqrt(eps_out) as
    the reference does (RCWASolver.cpp:1733)."""
    nx, ny = sampler.nx, sampler.ny
    m = nx * ny
    k0 = sampler.k0
    alpha = np.diag(sampler.Kx).copy()
    beta = np.diag(sampler.Ky).copy()
    if side == "bottom":
        Win, Wout, R, T = S.W0, S.W1, S.Rdu, S.Tuu
    else:
        Win, Wout, R, T = S.W1, S.W0, S.Rud, S.Tdd
    delta = np.zeros(m, dtype=np.complex128)
    delta[(ny * (nx - 1)) // 2 + (ny - 1) // 2] = 1.0
    s = np.concatenate([px * delta, py * delta])
    c = np.linalg.solve(Win, s)
    rxy = Win @ (R @ c)
    txy = Wout @ (T @ c)
    rx, ry = rxy[:m], rxy[m:]
    tx, ty = txy[:m], txy[m:]
    kz_r = -np.sqrt(k0 * k0 * eps_in - alpha * alpha - beta * beta + 0j)
    kz_t = np.sqrt(k0 * k0 * eps_out - alpha * alpha - beta * beta + 0j)
    rz = (alpha * rx + beta * ry) / kz_r
    tz = (alpha * tx + beta * ty) / kz_t
    r = np.abs(rx) ** 2 + np.abs(ry) ** 2 + np.abs(rz) ** 2
    t = np.abs(tx) ** 2 + np.abs(ty) ** 2 + np.abs(tz) ** 2
    REF = np.abs(kz_r.real) * r / (math.sqrt(np.real(eps_in)) * k0)
    norm_t = math.sqrt(np.real(eps_in)) if flux_norm else math.sqrt(np.real(eps_out))
    TRN = np.abs(kz_t.real) * t / (norm_t * k0)
    return REF, TRN
