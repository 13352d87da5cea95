"""Build oracle samplers from structure descriptor dicts (test infrastructure).

The descriptor format is plain data (see the package's ``structures``
module); this adapter only evaluates it with the oracle's samplers."""
from __future__ import annotations

import numpy as np

from . import varrcwa_oracle as O


def _pwl(zs, vals, z):
    zs = np.asarray(zs, dtype=np.float64)
    vals = np.asarray(vals, dtype=np.float64)
    if z <= zs[0]:
        return float(vals[0])
    if z >= zs[-1]:
        return float(vals[-1])
    k = int(np.searchsorted(zs, z, side="right")) - 1
    t = (z - zs[k]) / (zs[k + 1] - zs[k])
    return float((1.0 - t) * vals[k] + t * vals[k + 1])


def _pillar_raster(d, z):
    npx, npy, Lx, Ly = d["npx"], d["npy"], d["Lx"], d["Ly"]
    xc = (np.arange(npx) + 0.5) * (Lx / npx) - 0.5 * Lx
    yc = (np.arange(npy) + 0.5) * (Ly / npy) - 0.5 * Ly
    t = 0.0 if d["z1"] == d["z0"] else (z - d["z0"]) / (d["z1"] - d["z0"])
    r = d["r0"] + (d["r1"] - d["r0"]) * t
    inside = (xc[None, :] ** 2 + yc[:, None] ** 2) <= r * r
    return np.where(inside, d["eps_in"], d["eps_out"]).astype(np.complex128)


def make_sampler(d):
    kind = d["kind"]
    if kind == "grid":
        s = O.VarLayerSampler(d["lam"], d["nx"], d["ny"], d["x"], d["y"], d["eps"],
                              enable_pml=d["pml"])
        ev = natural_spline_eval if d.get("spline") else _pwl
        for (i, zs, vals) in d.get("xrules", []):
            s.add_x_rule(i, lambda z, zs=zs, vals=vals, ev=ev: ev(zs, vals, z))
        for (j, zs, vals) in d.get("yrules", []):
            s.add_y_rule(j, lambda z, zs=zs, vals=vals, ev=ev: ev(zs, vals, z))
        return s
    if kind == "pillar":
        return O.RasterSampler(d["lam"], d["nx"], d["ny"], d["Lx"], d["Ly"],
                               lambda z: _pillar_raster(d, z), enable_pml=d["pml"])
    if kind == "pixels":
        eps = np.asarray(d["eps"], dtype=np.complex128)
        return O.RasterSampler(d["lam"], d["nx"], d["ny"], d["Lx"], d["Ly"],
                               lambda z: eps, enable_pml=d["pml"])
    if kind == "planar":
        from .planar_sampler import PlanarSampler
        return PlanarSampler(d["lam"], d["nx"], d["ny"], d["polys"], d.get("shift", (0.0, 0.0, 0.0)),
                             d.get("pml_w", (0.5, 0.5, 0.5, 0.5)), d.get("space", (1.5, 1.5, 1.08, 1.0)),
                             d.get("thickness", 0.22), d["eps_bg"], d["eps_dev"])
    raise ValueError(kind)


def end_bases(d, sampler):
    e0 = None if d.get("end0") is None else O.homogeneous_basis(sampler, d["end0"])
    e1 = None if d.get("end1") is None else O.homogeneous_basis(sampler, d["end1"])
    return e0, e1


def natural_spline_eval(zs, vals, z):
    """Natural cubic spline through (zs, vals) at z, constant beyond the end
    knots (the clamping of the piecewise-linear rules).  Second derivatives
    from the tridiagonal system of the natural end conditions."""
    zs = np.asarray(zs, dtype=np.float64)
    vals = np.asarray(vals, dtype=np.float64)
    if z <= zs[0]:
        return float(vals[0])
    if z >= zs[-1]:
        return float(vals[-1])
    K = len(zs)
    h = np.diff(zs)
    A = np.zeros((K, K))
    r = np.zeros(K)
    A[0, 0] = A[-1, -1] = 1.0
    for i in range(1, K - 1):
        A[i, i - 1] = h[i - 1]
        A[i, i] = 2.0 * (h[i - 1] + h[i])
        A[i, i + 1] = h[i]
        r[i] = 6.0 * ((vals[i + 1] - vals[i]) / h[i] - (vals[i] - vals[i - 1]) / h[i - 1])
    M2 = np.linalg.solve(A, r)
    k = min(int(np.searchsorted(zs, z, side="right")) - 1, K - 2)
    t = z - zs[k]
    hk = h[k]
    b = (vals[k + 1] - vals[k]) / hk - hk * (2.0 * M2[k] + M2[k + 1]) / 6.0
    return float(vals[k] + b * t + 0.5 * M2[k] * t * t + (M2[k + 1] - M2[k]) / (6.0 * hk) * t ** 3)
