"""CPU restatement of stacks of sections (test infrastructure: the GPU path
never imports this module).

RCWASolver::solve (src/rcwa/RCWASolver.cpp:104-113) joins z-uniform layers:
each layer's S-matrix in its own modes, interfaces matching the transverse
fields of neighbouring layers, the chain star-multiplied.  Here every section
is an S-matrix of the oracle's integrators in the bases of its own end
cross-sections; a section's entrance is re-expressed in the previous
section's exit basis by project_left (RedhefferIntegrator.cpp:253-262, the
same field matching) and the chain star-multiplied (:267-277).  The internal
amplitudes follow RCWASolver::evaluateIntermediateField (:1373-1480) from the
prefix and suffix chains.
"""
from __future__ import annotations

import numpy as np

from . import varrcwa_oracle as O


def chain_sections(Ss):
    """Join section S-matrices (SMatrix, in order); returns (total SMatrix,
    projected section blocks, prefix chains)."""
    proj = [list(Ss[0].blocks())]
    for a, b in zip(Ss[:-1], Ss[1:]):
        proj.append(O.project_left(list(b.blocks()), O.Basis(b.W0, b.V0, b.gam0), a.W1, a.V1))
    prefix = [proj[0]]
    for p in proj[1:]:
        prefix.append(O.star_right(prefix[-1], p))
    f, l = Ss[0], Ss[-1]
    T = O.SMatrix(*prefix[-1], f.W0, f.V0, f.gam0, l.W1, l.V1, l.gam1)
    return T, proj, prefix


def chain_amplitudes(Ss, c):
    """Up- and down-going amplitudes at every interface (entrance of each
    section, then the exit) for incident entrance amplitudes c."""
    T, proj, prefix = chain_sections(Ss)
    S = len(Ss)
    n = len(c)
    I = np.eye(n)
    amps = np.zeros((S + 1, 2, n), np.complex128)
    amps[0, 0] = c
    amps[0, 1] = T.Rdu @ c
    amps[S, 0] = T.Tuu @ c
    suffix = [None] * S
    suffix[S - 1] = proj[S - 1]
    for j in range(S - 2, 0, -1):
        suffix[j] = O.star_right(proj[j], suffix[j + 1])
    for j in range(1, S):
        L, R = prefix[j - 1], suffix[j]
        ap = np.linalg.solve(I - L[2] @ R[3], L[1] @ c)
        amps[j, 0] = ap
        amps[j, 1] = R[3] @ ap
    return amps
