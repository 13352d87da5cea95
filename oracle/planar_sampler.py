"""CPU restatement of GDSIISampler (src/core/GDSIISampler.cpp): a planar
device seen from above.

TEST INFRASTRUCTURE ONLY: the GPU path never imports this module.

The layout's polygons lie in the (x, z) plane, z being the propagation
coordinate.  At every z the cross-section is a tensor grid: x holds the
crossings of the polygon edges with the line y_layout = z between the spacer
and PML coordinates, y is fixed (PML, spacer, device layer, spacer, PML), and
the device strip holds the device material in every other x cell.  PML on
all four sides (the reference always enables it).
"""
from __future__ import annotations

import numpy as np

from .varrcwa_oracle import PI, k_matrices, wave_eqn_coeff


class PlanarSampler:
    def __init__(self, lam, nx, ny, polys, shift=(0.0, 0.0, 0.0), pml_w=(0.5, 0.5, 0.5, 0.5),
                 space=(1.5, 1.5, 1.08, 1.0), thickness=0.22, eps_bg=2.085, eps_dev=12.11):
        self.lam = float(lam)
        self.nx, self.ny = int(nx), int(ny)
        self.polys = [np.asarray(p, dtype=np.float64).reshape(-1, 2) for p in polys]
        self.shift = np.asarray(shift, dtype=np.float64)
        self.eps_bg, self.eps_dev = complex(eps_bg), complex(eps_dev)
        # assignSimulationRegion (GDSIISampler.cpp:48-88)
        allx = np.concatenate([p[:, 0] for p in self.polys])
        minX, maxX = allx.min() + self.shift[0], allx.max() + self.shift[0]
        lP, rP, bP, uP = pml_w
        ls, rs, bs, us = space
        b0 = self.shift[1]
        b1 = b0 + bP
        u0 = b1 + bs + thickness + us
        u1 = u0 + uP
        l1 = minX - ls
        l0 = l1 - lP
        r0 = maxX + rs
        r1 = r0 + rP
        self.xlim = np.array([l0, l1, r0, r1])
        # the constructor's y grid (GDSIISampler.cpp:35-42)
        self.y = np.array([b0, b1, b1 + bs, b1 + bs + thickness, u0, u1])
        self.x = self.xlim  # x[0], x[1], x[-2], x[-1] set the PML regions
        self.Kx, self.Ky = k_matrices(self.nx, self.ny, self.xlim, self.y, True)
        self.n_samples = 0

    @property
    def k0(self):
        return 2 * PI / self.lam

    @property
    def ndim(self):
        return 2 * self.nx * self.ny

    def section(self, z):
        """sampleLayout (GDSIISampler.cpp:90-140): x, eps (5 x (len(x) - 1))."""
        xs = []
        for p in self.polys:
            n = len(p)
            for i in range(n):
                x0, y0 = p[i]
                x1, y1 = p[(i + 1) % n]
                if (y0 <= z < y1) or (y1 <= z < y0):
                    h = y1 - y0
                    if abs(h) < 1e-12:
                        h += 2e-12
                    a = (z - y0) / h
                    xs.append((1 - a) * x0 + a * x1)
        xs.sort()
        x = np.concatenate([self.xlim[:2], np.asarray(xs, dtype=np.float64) + self.shift[0], self.xlim[2:]])
        eps = np.full((5, len(x) - 1), self.eps_bg, dtype=np.complex128)
        eps[2, 2:len(x) - 3:2] = self.eps_dev
        return x, eps

    def geometry(self, z):
        x, eps = self.section(z)
        return x, self.y, eps

    def sample(self, z):
        self.n_samples += 1
        x, y, eps = self.geometry(z)
        return wave_eqn_coeff(x, y, eps, self.Kx, self.Ky, self.lam, self.nx, self.ny)
