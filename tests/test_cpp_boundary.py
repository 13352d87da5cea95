"""The C ABI from C++: tests/cpp/shim_check.cpp, a C++ program built here
with g++ against include/vrc.h and include/vrc_integrators.hpp (the
reference's RedhefferIntegrator / RCWAIntegrator / DifferentialIntegrator
classes over the ABI), driven by a caller-defined sampler as a LayerSampler
subclass of the reference would be.

* CPU: the program compiles warning-free and links against libvrc.so.
* GPU: run with the sampler's host sample() and with its sampleOnGPU(), the
  three integrators agree with the oracle on the same sampler (adaptive run
  replayed on the device tree) in the Fourier basis to 1e-9, and the host
  and device sampling paths give identical results.
"""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import relerr

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "shim_check.cpp"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def _build(out_dir: Path) -> Path:
    exe = out_dir / "shim_check"
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", str(ROOT / "include"), "-I", str(CUDA / "include"), str(SRC), "-o", str(exe),
           "-L", str(ROOT / "varrcwa_b200"), "-lvrc", "-L", str(CUDA / "lib64"), "-lcudart",
           f"-Wl,-rpath,{ROOT / 'varrcwa_b200'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_cpp_caller_compiles_against_the_headers(tmp_path):
    from varrcwa_b200 import capi
    capi.lib()  # the library is current and present
    exe = _build(tmp_path)
    syms = subprocess.run(["nm", "-D", "--undefined-only", str(exe)], capture_output=True, text=True).stdout
    for s in ("vrc_create", "vrc_redheffer", "vrc_rcwa", "vrc_differential", "vrc_get_tree"):
        assert s in syms, s


class LinearPQ:
    """The oracle's view of the C++ sampler: P, Q linear in z between two
    sampled end matrices."""

    def __init__(self, lam, za, zb, P0, P1, Q0, Q1):
        self.lam, self.za, self.zb = lam, za, zb
        self.P0, self.P1, self.Q0, self.Q1 = P0, P1, Q0, Q1
        self.k0 = 2 * np.pi / lam

    def sample(self, z):
        t = (z - self.za) / (self.zb - self.za)
        return self.P0 + t * (self.P1 - self.P0), self.Q0 + t * (self.Q1 - self.Q0)


def _fourier(blocks):
    Tdd, Tuu, Rud, Rdu, W0, W1 = blocks
    W0i, W1i = np.linalg.inv(W0), np.linalg.inv(W1)
    return {"Tuu": W1 @ Tuu @ W0i, "Tdd": W0 @ Tdd @ W1i, "Rdu": W0 @ Rdu @ W0i, "Rud": W1 @ Rud @ W1i}


@pytest.mark.gpu
def test_cpp_integrators_match_oracle_host_and_device_sampling(tmp_path):
    from oracle import varrcwa_oracle as O
    from oracle.structures_adapter import make_sampler
    from tests.cases import CASES
    d = CASES["asym_redheffer"]["desc"]  # off-centre core, one moving edge, n = 30
    grid = make_sampler(d)
    za, zb = 0.0, 1.5
    P0, Q0 = grid.sample(za)
    P1, Q1 = grid.sample(zb)
    n = P0.shape[0]
    lam, z0, z1, pe, nr, nd = d["lam"], 0.0, 1.5, 1e-3, 8, 4
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.array([lam, za, zb, z0, z1], dtype=np.float64).tobytes())
        for M in (P0, P1, Q0, Q1):
            f.write(np.ascontiguousarray(M.T).tobytes())  # column-major
    exe = _build(tmp_path)
    outs = {}
    for mode in ("host", "device"):
        out = tmp_path / f"out_{mode}.bin"
        r = subprocess.run([str(exe), str(inp), str(out), mode, str(pe), str(nr), str(nd)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
        raw = out.read_bytes()
        N, neig = np.frombuffer(raw[:8], dtype=np.int32)
        ncut = int(np.frombuffer(raw[8:12], dtype=np.int32)[0])
        cuts = np.frombuffer(raw[12:12 + 8 * ncut], dtype=np.float64)
        mats = np.frombuffer(raw[12 + 8 * ncut:], dtype=np.complex128).reshape(3, 6, n, n).transpose(0, 1, 3, 2)
        outs[mode] = (int(N), int(neig), cuts, mats)
    (N, neig, cuts, mats), dev = outs["host"], outs["device"]
    assert N == len(cuts) - 1 >= 2 and neig >= N
    assert N == dev[0] and np.array_equal(cuts, dev[2]) and np.array_equal(mats, dev[3])
    s = LinearPQ(lam, za, zb, P0, P1, Q0, Q1)
    refs = [O.redheffer_segments(s, z0, z1, list(cuts)), O.rcwa_compute(s, z0, z1, nr),
            O.differential_compute(s, z0, z1, nd)]
    for k, (S, blocks) in enumerate(zip(refs, mats)):
        F, G = _fourier(blocks), S.fourier_blocks()
        for name in F:
            assert relerr(F[name], G[name]) < 1e-9, (k, name)
