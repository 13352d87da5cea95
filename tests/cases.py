"""Small seeded structures shared by the golden-fixture generator and the
parity tests (one per benchmark family and geometry kind)."""
from __future__ import annotations

import numpy as np

from varrcwa_b200 import structures as st


def _taper_short():
    d = st.taper_2d(norders=11, length=2.0)
    return d


def _pillar(npix=16, nord=3, seed=2000):
    d = st.pillar_cell(seed, norders=nord, lam=0.532, npix=npix)
    return d


def _asym_grid():
    """Off-centre rectangular core in a 2D-periodic cell (no mirror symmetry),
    one edge moving linearly with z."""
    x = np.array([0.0, 0.13, 0.41, 0.62, 1.0])
    y = np.array([0.0, 0.21, 0.35, 0.8])
    c, s, t = 2.085, 12.11, 4.0
    eps = np.array([[c, c, c, c],
                    [c, s, t, c],
                    [c, c, c, c]], dtype=np.complex128)
    return dict(kind="grid", lam=1.3, nx=5, ny=3, pml=False, x=x, y=y, eps=eps,
                xrules=[(2, [0.0, 1.5], [0.41, 0.55])], z0=0.0, z1=1.5, end0=2.085, end1=1.0)


def _cross_grid():
    """Coordinates that cross (x[2] > x[3]): exercises the painter's-order
    refill (src/rcwa/FourierSolver1D.cpp:156-193)."""
    x = np.array([0.0, 0.3, 1.1, 0.8, 1.6, 2.0])
    y = np.array([0.0, 0.5, 1.0])
    eps = np.array([[2.0, 3.0, 4.0, 5.0, 2.0],
                    [2.0, 6.0, 2.5, 3.5, 2.0]], dtype=np.complex128)
    return dict(kind="grid", lam=1.55, nx=5, ny=3, pml=False, x=x, y=y, eps=eps, z0=0.0, z1=1.0,
                end0=None, end1=None)


def _pml_short(nord=5):
    d = st.waveguide_pml(1, norders=nord, ncontrol=8, length=2.0)
    return d


CASES = {
    "taper_pq": dict(desc=st.taper_2d(), pq_z=[0.0, 3.7]),
    "pillar_pq": dict(desc=_pillar(npix=32, nord=5), pq_z=[0.1, 0.45]),
    "pml_pq": dict(desc=_pml_short(), pq_z=[0.0, 1.3]),
    "cross_pq": dict(desc=_cross_grid(), pq_z=[0.0]),
    "planar_pq": dict(desc=st.planar_taper(norders=(5, 3)), pq_z=[0.3, 2.9]),
    "taper_redheffer": dict(desc=_taper_short(), method="redheffer", pe=1e-4),
    "pillar_rcwa": dict(desc=_pillar(), method="rcwa", N=4),
    "pillar_redheffer": dict(desc=_pillar(), method="redheffer", pe=1e-2),
    "asym_redheffer": dict(desc=_asym_grid(), method="redheffer", pe=1e-3),
    "asym_diff": dict(desc=_asym_grid(), method="differential", N=4),
    "pml_redheffer": dict(desc=_pml_short(3), method="redheffer", pe=1e-2),
}
