"""Synthetic structure descriptors for the benchmark families.

A structure is a plain dict (numbers and numpy arrays only) that both the
device engine and the CPU oracle consume:

``kind = "grid"``
    Tensor grid with fixed permittivity table ``eps`` (shape
    ``(len(y)-1, len(x)-1)``: rows are y-strips, columns x-cells) whose
    coordinates ``x[i]``/``y[j]`` may move with z through piecewise-linear
    rules ``xrules = [(i, zs, vals), ...]`` (clamped outside ``zs``).  This is
    the reference's ``VarLayerSampler`` (src/core/VarLayerSampler.cpp:42-69).
``kind = "pillar"``
    Uniform ``npx x npy`` pixel raster of a circular pillar (``eps_in``) in
    ``eps_out`` whose radius varies linearly from ``r0`` at ``z0`` to ``r1`` at
    ``z1``; a pixel is inside when its centre is.
``kind = "pixels"``
    A z-invariant pixel raster ``eps`` on a uniform grid (one layer of a
    freeform stack).

Common keys: ``lam`` (wavelength), ``nx``/``ny`` (harmonics per axis, odd),
``pml`` (bool), ``z0``/``z1``, ``end0``/``end1`` (permittivity of homogeneous
half-spaces joined at z0/z1, or None to keep the structure's own end bases).
"""
from __future__ import annotations

import math

import numpy as np

EPS_SI_BENCH = 12.11
EPS_SIO2_BENCH = 2.085


def pwl(zs, vals, z):
    """Piecewise-linear, clamped rule evaluation."""
    zs = np.asarray(zs, dtype=np.float64)
    vals = np.asarray(vals, dtype=np.float64)
    if z <= zs[0]:
        return float(vals[0])
    if z >= zs[-1]:
        return float(vals[-1])
    k = int(np.searchsorted(zs, z, side="right")) - 1
    t = (z - zs[k]) / (zs[k + 1] - zs[k])
    return float((1.0 - t) * vals[k] + t * vals[k + 1])


def geometry(desc, z):
    """(x, y, eps) of a structure at height z (host-side evaluation)."""
    kind = desc["kind"]
    if kind == "grid":
        x = np.array(desc["x"], dtype=np.float64)
        y = np.array(desc["y"], dtype=np.float64)
        for (i, zs, vals) in desc.get("xrules", []):
            x[i] = pwl(zs, vals, z)
        for (j, zs, vals) in desc.get("yrules", []):
            y[j] = pwl(zs, vals, z)
        return x, y, np.asarray(desc["eps"], dtype=np.complex128)
    if kind == "pillar":
        npx, npy = desc["npx"], desc["npy"]
        Lx, Ly = desc["Lx"], desc["Ly"]
        x = np.linspace(0.0, Lx, npx + 1)
        y = np.linspace(0.0, Ly, npy + 1)
        return x, y, pillar_raster(desc, z)
    if kind == "pixels":
        eps = np.asarray(desc["eps"], dtype=np.complex128)
        x = np.linspace(0.0, desc["Lx"], eps.shape[1] + 1)
        y = np.linspace(0.0, desc["Ly"], eps.shape[0] + 1)
        return x, y, eps
    raise ValueError(kind)


def pillar_radius(desc, z):
    z0, z1 = desc["z0"], desc["z1"]
    t = 0.0 if z1 == z0 else (z - z0) / (z1 - z0)
    return desc["r0"] + (desc["r1"] - desc["r0"]) * t


def pillar_raster(desc, z):
    """Cell-centre in/out raster of the pillar at height z, shape (npy, npx)."""
    npx, npy = desc["npx"], desc["npy"]
    Lx, Ly = desc["Lx"], desc["Ly"]
    xc = (np.arange(npx) + 0.5) * (Lx / npx) - 0.5 * Lx
    yc = (np.arange(npy) + 0.5) * (Ly / npy) - 0.5 * Ly
    r = pillar_radius(desc, z)
    inside = (xc[None, :] ** 2 + yc[:, None] ** 2) <= r * r
    return np.where(inside, desc["eps_in"], desc["eps_out"]).astype(np.complex128)


# ---------------------------------------------------------------------------
# Benchmark families (seeded)
# ---------------------------------------------------------------------------
def taper_2d(lam=1.55, period=2.0, norders=41, w0=0.40, w1=1.00, length=10.0,
             eps_core=EPS_SI_BENCH, eps_clad=EPS_SIO2_BENCH):
    """2D (x-z) periodic taper: a core centred in the cell whose width tapers
    linearly from w0 to w1 over `length`; ny = 1 (TE/TM decoupled).  The two
    core edges are moving coordinates with linear z-rules (the reference's
    VarLayerSampler idiom, src/tests/test_cpu.cpp:139-176)."""
    c = 0.5 * period
    x = np.array([0.0, c - 0.5 * w0, c + 0.5 * w0, period])
    y = np.array([0.0, 1.0])
    eps = np.array([[eps_clad, eps_core, eps_clad]], dtype=np.complex128)
    return dict(kind="grid", lam=lam, nx=norders, ny=1, pml=False, x=x, y=y, eps=eps,
                xrules=[(1, [0.0, length], [c - 0.5 * w0, c - 0.5 * w1]),
                        (2, [0.0, length], [c + 0.5 * w0, c + 0.5 * w1])],
                z0=0.0, z1=length, end0=None, end1=None)


def pillar_cell(seed, norders=11, lam=None, npix=256, period=0.4, height=0.6,
                eps_pillar=5.8, eps_sub=2.13, eps_sup=1.0):
    """Tapered circular pillar unit cell; radius ~ U[60,140] nm at the base,
    sidewall angle ~ U[85,90] deg (radius shrinks linearly upward)."""
    rng = np.random.default_rng(seed)
    r0 = rng.uniform(0.060, 0.140)
    theta = rng.uniform(85.0, 90.0)
    lam_draw = rng.uniform(0.450, 0.650)
    if lam is None:
        lam = lam_draw
    r1 = r0 - height / math.tan(math.radians(theta))
    return dict(kind="pillar", lam=float(lam), nx=norders, ny=norders, pml=False,
                npx=npix, npy=npix, Lx=period, Ly=period, eps_in=eps_pillar,
                eps_out=eps_sup, r0=float(r0), r1=float(max(r1, 0.0)), z0=0.0, z1=height,
                end0=eps_sub, end1=eps_sup, theta=theta)


def pillar_config2(seed=2000, npix=256):
    """11x11 orders, 532 nm, 400 nm period, 600 nm pillar."""
    return pillar_cell(seed, norders=11, lam=0.532, npix=npix)


def pillar_config3(seed, npix=256):
    """Uneven batch member: orders ~ U{7,9,11,13,15}, lambda ~ U[450,650] nm."""
    rng = np.random.default_rng(seed + 7)
    norders = int(rng.choice([7, 9, 11, 13, 15]))
    return pillar_cell(seed, norders=norders, lam=None, npix=npix)


def waveguide_pml(seed, norders=21, ncontrol=64, length=20.0, cell=(4.0, 2.0),
                  pml=0.5, eps_core=EPS_SI_BENCH, eps_clad=EPS_SIO2_BENCH, lam=1.55,
                  core_h=0.22, spline=False):
    """Waveguide mode converter with PML on both lateral boundaries: the core
    width follows seeded control points, interpolated piecewise-linearly or
    (spline=True, config 5) by the natural cubic spline; the two core edges
    are the moving coordinates, cx -+ w(z) / 2."""
    rng = np.random.default_rng(seed)
    widths = rng.uniform(0.3, 1.2, size=ncontrol)
    zs = np.linspace(0.0, length, ncontrol)
    Lx, Ly = cell
    cx, cy = 0.5 * Lx, 0.5 * Ly
    x = np.array([0.0, pml, cx - 0.5 * widths[0], cx + 0.5 * widths[0], Lx - pml, Lx])
    y = np.array([0.0, pml, cy - 0.5 * core_h, cy + 0.5 * core_h, Ly - pml, Ly])
    c, s = eps_clad, eps_core
    eps = np.full((5, 5), c, dtype=np.complex128)
    eps[2, 2] = s
    return dict(kind="grid", lam=lam, nx=norders, ny=norders, pml=True, x=x, y=y, eps=eps,
                xrules=[(2, zs, cx - 0.5 * widths), (3, zs, cx + 0.5 * widths)],
                z0=0.0, z1=length, end0=None, end1=None, widths=widths, spline=bool(spline))


def converter_c5(seed, norders=21, ncontrol=64, length=20.0):
    """Config 5: 4 x 2 um cell, PML 0.5 um, Si core in SiO2, width over 20 um
    through 64 seeded control points U[0.3, 1.2] um, natural cubic spline,
    21 x 21 orders (n = 882)."""
    return waveguide_pml(seed, norders=norders, ncontrol=ncontrol, length=length, spline=True)


def smooth_pixels(seed, npx, npy, sigma=3.0, beta=8.0, lo=2.085, hi=12.11):
    """Freeform layer permittivity: seeded uniform noise, periodic Gaussian
    smoothing (sigma in pixels), sigmoid threshold (beta) of the standardised
    field, mapped to [lo, hi].  Returns an (npy, npx) real array."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, 1.0, (npy, npx))
    ky = np.fft.fftfreq(npy)[:, None]
    kx = np.fft.fftfreq(npx)[None, :]
    g = np.exp(-2.0 * (math.pi * sigma) ** 2 * (kx * kx + ky * ky))
    f = np.fft.ifft2(np.fft.fft2(u) * g).real
    f = (f - f.mean()) / (f.std() + 1e-30)
    t = 1.0 / (1.0 + np.exp(-beta * f))
    return lo + (hi - lo) * t


def metagrating_c4(seed=4000, npix=64, nlayers=4, norders=9):
    """Freeform metagrating of config 4: 600 nm square period, 633 nm, 9x9
    orders (n = 162; norders sets another truncation, e.g. 15 for the
    15x15-order comparison), four 150 nm layers of npix x npix pixels (smoothed
    thresholded noise in [2.085, 12.11], layer l seeded by (seed, l)).
    Incidence from air below; transmission into the SiO2 substrate (eps
    2.085), where the (+1, 0) order propagates (it is evanescent in air at
    this period)."""
    layers = [smooth_pixels([seed, l], npix, npix) for l in range(nlayers)]
    return dict(lam=0.633, Lx=0.6, Ly=0.6, nx=norders, ny=norders, layers=layers, thick=[0.15] * nlayers,
                eps_in=1.0, eps_out=2.085)


def planar_taper(w0=0.5, w1=1.2, length=4.0, lam=1.55, norders=(11, 5), thickness=0.22, eps_bg=EPS_SIO2_BENCH,
                 eps_dev=EPS_SI_BENCH, lead=0.5):
    """Planar (GDS-style) silicon taper seen from above: a straight lead of
    width w0, a linear taper to w1 over `length`, a straight lead of width w1
    (one polygon in the layout's (x, z) plane), in the device layer of the
    given thickness; integration over the taper (GDSIISampler's geometry)."""
    z0, z1 = lead, lead + length
    pts = [(-0.5 * w0, 0.0), (0.5 * w0, 0.0), (0.5 * w0, z0), (0.5 * w1, z1), (0.5 * w1, z1 + lead),
           (-0.5 * w1, z1 + lead), (-0.5 * w1, z1), (-0.5 * w0, z0)]
    return dict(kind="planar", lam=lam, nx=norders[0], ny=norders[1], pml=True, polys=[np.array(pts)],
                shift=(0.0, 0.0, 0.0), pml_w=(0.5, 0.5, 0.5, 0.5), space=(1.0, 1.0, 0.8, 0.8),
                thickness=thickness, eps_bg=eps_bg, eps_dev=eps_dev, z0=z0, z1=z1, end0=None, end1=None)


def gds_planar(polys, norders=(13, 11), lam=1.55, shift=(2.3647, 0.0, 0.0), z0=-1.63, z1=1.36,
               pml_w=(0.5, 0.5, 0.5, 0.5), space=(1.0, 1.3, 1.08, 1.0), thickness=0.22,
               eps_bg=1.445 ** 2, eps_dev=3.48 ** 2):
    """Planar device from GDSII polygons with the parameters of the
    reference's GDS driver (src/tests/test_gds_cpu.cpp:131-146: 1.55 um,
    x shift 2.3647, side PML 0.5 / 0.5 and spaces 1.0 / 1.3, the
    GDSIISampler defaults below and above, SiO2 / Si at 1.445^2 / 3.48^2,
    z in [-1.63, 1.36]).  The reference runs 25 x 21 harmonics (n = 1050);
    `norders` sets the truncation here."""
    return dict(kind="planar", lam=lam, nx=norders[0], ny=norders[1], pml=True,
                polys=[np.asarray(p, dtype=np.float64) for p in polys], shift=tuple(shift), pml_w=tuple(pml_w),
                space=tuple(space), thickness=thickness, eps_bg=eps_bg, eps_dev=eps_dev, z0=z0, z1=z1,
                end0=None, end1=None)
