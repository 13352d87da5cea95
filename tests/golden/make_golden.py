"""Generate the golden fixtures of tests/golden/ with the CPU oracle.

The reference ships no numeric golden vectors (its drivers write ground
truth at run time and it cannot be built here), so these fixtures are the
oracle's outputs on small seeded structures of each benchmark family.  They
pin the oracle against drift (tests/test_golden_oracle.py) and give the GPU
parity tests fixed targets.

Run from the repository root:  python tests/golden/make_golden.py [names...]
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import varrcwa_oracle as O  # noqa: E402
from oracle.structures_adapter import end_bases, make_sampler  # noqa: E402
from tests.cases import CASES  # noqa: E402

OUT = Path(__file__).resolve().parent


def fourier(S):
    F = S.fourier_blocks()
    return {f"F_{k}": v for k, v in F.items()}


def stack_small():
    """A two-layer pixel stack: per-order powers and the pixel and thickness
    gradients of T(+1, 0) (oracle/stack_adjoint.py)."""
    from oracle.stack_adjoint import Stack, order_index, stack_backward, stack_forward
    from varrcwa_b200.structures import smooth_pixels
    layers = [smooth_pixels([4900, l], 8, 8, sigma=1.0) for l in range(2)]
    st = Stack(0.633, 3, 3, 0.6, 0.6, layers, [0.15, 0.2], eps_in=1.0, eps_out=2.085)
    R, T, tp = stack_forward(st)
    wT = np.zeros(9)
    wT[order_index(3, 3, 1, 0)] = 1.0
    g, gt = stack_backward(st, tp, np.zeros(9), wT, want_thick=True)
    return dict(layers=np.array(layers), R=R, T=T, grad=np.array(g), grad_thick=gt)


def main(names=None):
    if names is None or "stack_small" in names:
        data = stack_small()
        np.savez_compressed(OUT / "stack_small.npz", **data)
        print("stack_small", {k: v.shape for k, v in data.items()})
    for name, case in CASES.items():
        if names is not None and name not in names:
            continue
        d = case["desc"]
        s = make_sampler(d)
        e0, e1 = end_bases(d, s)
        data = {}
        if "pq_z" in case:
            Ps, Qs = [], []
            for z in case["pq_z"]:
                P, Q = s.sample(z)
                Ps.append(P)
                Qs.append(Q)
            data["P"] = np.array(Ps)
            data["Q"] = np.array(Qs)
            data["pq_z"] = np.array(case["pq_z"])
        method = case.get("method")
        if method == "redheffer":
            S = O.redheffer_compute(s, d["z0"], d["z1"], pe=case["pe"], end0=e0, end1=e1)
            nodes = np.array([(a, b, e, 1.0 if acc else 0.0) for (a, b, e, acc) in S.nodes])
            data["nodes"] = nodes
            data["cuts"] = np.array(O.tree_cuts(S.nodes))
            data["N"] = np.array(S.N)
        elif method == "rcwa":
            S = O.rcwa_compute(s, d["z0"], d["z1"], case["N"], end0=e0, end1=e1)
        elif method == "differential":
            S = O.differential_compute(s, d["z0"], d["z1"], case["N"], end0=e0, end1=e1)
        else:
            S = None
        if S is not None:
            data.update(fourier(S))
            data["gam0"] = S.gam0
            data["gam1"] = S.gam1
            if d.get("end0") is not None and d.get("end1") is not None:
                for side, (ein, eout) in ((0, (d["end0"], d["end1"])), (1, (d["end1"], d["end0"]))):
                    for p, (px, py) in enumerate(((1.0, 0.0), (0.0, 1.0))):
                        R, T = O.order_powers(S, s, ein, eout, px, py, side="bottom" if side == 0 else "top")
                        data[f"R_{side}_{p}"] = R
                        data[f"T_{side}_{p}"] = T
        np.savez_compressed(OUT / f"{name}.npz", **data)
        print(name, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    # optional fixture names: regenerate only those
    main(sys.argv[1:] or None)
