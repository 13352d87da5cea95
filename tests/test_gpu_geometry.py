"""Device geometry of tensor-grid cells: the moving coordinates' rules
(piecewise-linear and natural cubic spline z-rules, VarLayerSampler::addXRule,
src/core/VarLayerSampler.cpp:42-69) evaluated per sample on the device, the
sorted coordinates and the painter's-order refill where coordinates cross
(src/rcwa/FourierSolver1D.cpp:145-193), against the host evaluation of the
same rules (VRC_HOST_GEOMETRY) and against the oracle."""
import numpy as np
import pytest

from oracle.structures_adapter import make_sampler
from tests.cases import CASES
from tests.conftest import relerr
from varrcwa_b200 import structures as st

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _both(ctx, desc, zs, monkeypatch):
    monkeypatch.delenv("VRC_HOST_GEOMETRY", raising=False)
    Pd, Qd = ctx.sample_pq(desc, zs)
    monkeypatch.setenv("VRC_HOST_GEOMETRY", "1")
    Ph, Qh = ctx.sample_pq(desc, zs)
    monkeypatch.delenv("VRC_HOST_GEOMETRY", raising=False)
    return Pd, Qd, Ph, Qh


def _crossing_rules(spline=False):
    """A moving coordinate that crosses its neighbour half way along z (x[2]
    from 0.7 to 1.1 past x[3] = 0.9), and a second one through four knots."""
    x = np.array([0.0, 0.3, 0.7, 0.9, 1.6, 2.0])
    y = np.array([0.0, 0.5, 1.0])
    eps = np.array([[2.0, 3.0, 4.0, 5.0, 2.0],
                    [2.0, 6.0, 2.5, 3.5, 2.0]], dtype=np.complex128)
    return dict(kind="grid", lam=1.55, nx=5, ny=3, pml=False, x=x, y=y, eps=eps, z0=0.0, z1=1.0,
                xrules=[(2, [0.0, 1.0], [0.7, 1.1]), (4, [0.0, 0.3, 0.6, 1.0], [1.6, 1.5, 1.7, 1.55])],
                spline=spline, end0=None, end1=None)


DESCS = {"crossing_rules": _crossing_rules, "crossing_spline": lambda: _crossing_rules(True), "taper": lambda: CASES["taper_pq"]["desc"],
         "asym_grid": lambda: CASES["asym_redheffer"]["desc"], "pml_linear": lambda: CASES["pml_pq"]["desc"]}


@pytest.mark.parametrize("name", list(DESCS))
def test_device_rules_match_host_rules(ctx, name, monkeypatch):
    d = DESCS[name]()
    zs = np.linspace(d["z0"], d["z1"], 7)
    Pd, Qd, Ph, Qh = _both(ctx, d, zs, monkeypatch)
    s = make_sampler(d)
    for k, z in enumerate(zs):
        assert relerr(Pd[k], Ph[k]) < TOL and relerr(Qd[k], Qh[k]) < TOL
        Po, Qo = s.sample(z)
        assert relerr(Pd[k], Po) < TOL and relerr(Qd[k], Qo) < TOL


def test_device_spline_rules_match_host(ctx, monkeypatch):
    # the PML mode converter with spline width rules (config-5 geometry) at 5x5 orders
    d = st.waveguide_pml(5000, norders=5, ncontrol=12, length=3.0, spline=True)
    zs = np.linspace(d["z0"], d["z1"], 9)
    Pd, Qd, Ph, Qh = _both(ctx, d, zs, monkeypatch)
    s = make_sampler(d)
    for k, z in enumerate(zs):
        assert relerr(Pd[k], Ph[k]) < TOL and relerr(Qd[k], Qh[k]) < TOL
        Po, Qo = s.sample(z)
        assert relerr(Pd[k], Po) < TOL and relerr(Qd[k], Qo) < TOL
