"""ctypes binding of the C-ABI declared in ``include/vrc.h``.

The shared library is the in-tree ``libvrc.so`` built by ``build.py``; there
is no fallback: if it is missing or no CUDA device is present, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libvrc.so"

VRC_OK, VRC_EINVAL, VRC_ECUDA, VRC_ENOMEM, VRC_ESINGULAR, VRC_ENOCONV, VRC_ENONFINITE, VRC_ETIMEOUT, \
    VRC_EDEPTH, VRC_ENODEV = range(10)
GEOM_GRID, GEOM_PILLAR, GEOM_PIXELS, GEOM_PLANAR, GEOM_SAMPLER = 0, 1, 2, 3, 4

# Every function declared in include/vrc.h.
EXPORTS = [
    "vrc_create", "vrc_destroy", "vrc_last_error", "vrc_status_string", "vrc_get_timing", "vrc_sample_pq",
    "vrc_wave_solve", "vrc_eig", "vrc_redheffer", "vrc_redheffer_segments", "vrc_get_tree", "vrc_rcwa",
    "vrc_differential", "vrc_order_powers", "vrc_zgemm", "vrc_zinv", "vrc_set_profiling",
    "vrc_get_kernel_stats", "vrc_eig_noalloc", "vrc_stack_forward", "vrc_stack_backward", "vrc_gds_read",
    "vrc_planar_section", "vrc_stack_fields", "vrc_redheffer_forward", "vrc_redheffer_backward",
    "vrc_chain", "vrc_chain_order_powers", "vrc_chain_fields",
]


class VrcComplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class VrcRule(C.Structure):
    _fields_ = [("index", C.c_int), ("nknots", C.c_int), ("zs", C.POINTER(C.c_double)),
                ("vals", C.POINTER(C.c_double)), ("interp", C.c_int)]


GEOM_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double))


class VrcCell(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("pml", C.c_int), ("lam", C.c_double),
        ("z0", C.c_double), ("z1", C.c_double),
        ("ncx", C.c_int), ("ncy", C.c_int), ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
        ("eps", C.POINTER(VrcComplex)),
        ("n_xrules", C.c_int), ("xrules", C.POINTER(VrcRule)), ("n_yrules", C.c_int),
        ("yrules", C.POINTER(VrcRule)),
        ("geometry_fn", GEOM_FN), ("geometry_user", C.c_void_p),
        ("Lx", C.c_double), ("Ly", C.c_double), ("npx", C.c_int), ("npy", C.c_int),
        ("eps_in", VrcComplex), ("eps_out", VrcComplex), ("r0", C.c_double), ("r1", C.c_double),
        ("has_end0", C.c_int), ("has_end1", C.c_int), ("eps_end0", VrcComplex), ("eps_end1", VrcComplex),
        ("npoly", C.c_int), ("poly_start", C.POINTER(C.c_int)), ("poly_xz", C.POINTER(C.c_double)),
        ("shift", C.c_double * 3), ("pml_w", C.c_double * 4), ("space", C.c_double * 4), ("thickness", C.c_double),
        ("eps_background", VrcComplex), ("eps_device", VrcComplex),
        ("sample", C.c_void_p), ("sample_device", C.c_void_p), ("sample_user", C.c_void_p),
    ]


CP = C.POINTER(VrcComplex)


class VrcResult(C.Structure):
    _fields_ = [("Tdd", CP), ("Tuu", CP), ("Rud", CP), ("Rdu", CP), ("W0", CP), ("V0", CP), ("gam0", CP),
                ("W1", CP), ("V1", CP), ("gam1", CP), ("status", C.c_int), ("n", C.c_int), ("N", C.c_int),
                ("n_eig", C.c_int), ("n_samples", C.c_int), ("n_nodes", C.c_int)]


class VrcStack(C.Structure):
    _fields_ = [("lam", C.c_double), ("Lx", C.c_double), ("Ly", C.c_double), ("nx", C.c_int), ("ny", C.c_int),
                ("npx", C.c_int), ("npy", C.c_int), ("nlayers", C.c_int), ("eps", C.POINTER(C.c_double)),
                ("thick", C.POINTER(C.c_double)), ("eps_in", VrcComplex), ("eps_out", VrcComplex)]


class VrcTiming(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("launches", C.c_longlong)]


class VrcKernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_double), ("launches", C.c_longlong), ("flops", C.c_double),
                ("bytes", C.c_double), ("busy_ms", C.c_double)]


class VrcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"vrc status {status}: {msg}")
        self.status = status


_lib = None


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m varrcwa_b200.build`")
    from . import build as _build
    if _build.CSRC.exists() and not _build.is_current():
        raise RuntimeError(f"{LIB_PATH} was built from other sources than the tree's: "
                           "run `python -m varrcwa_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    L.vrc_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.vrc_destroy.argtypes = [vp]
    L.vrc_destroy.restype = None
    L.vrc_last_error.argtypes = [vp]
    L.vrc_last_error.restype = C.c_char_p
    L.vrc_status_string.argtypes = [C.c_int]
    L.vrc_status_string.restype = C.c_char_p
    L.vrc_get_timing.argtypes = [vp, C.POINTER(VrcTiming)]
    L.vrc_sample_pq.argtypes = [vp, C.POINTER(VrcCell), C.c_int, C.POINTER(C.c_double), CP, CP]
    L.vrc_wave_solve.argtypes = [vp, C.c_int, C.c_int, CP, CP, CP, CP, CP]
    L.vrc_eig.argtypes = [vp, C.c_int, C.c_int, CP, CP, CP]
    L.vrc_redheffer.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_double, C.c_int, C.POINTER(VrcResult)]
    L.vrc_redheffer_segments.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.POINTER(C.c_int),
                                         C.POINTER(C.POINTER(C.c_double)), C.POINTER(VrcResult)]
    L.vrc_get_tree.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.vrc_rcwa.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_int, C.POINTER(VrcResult)]
    L.vrc_differential.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_int, C.POINTER(VrcResult)]
    L.vrc_order_powers.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.vrc_zgemm.argtypes = [vp, C.c_int, C.c_int, CP, CP, CP]
    L.vrc_zinv.argtypes = [vp, C.c_int, C.c_int, CP, C.POINTER(C.c_int)]
    L.vrc_set_profiling.argtypes = [vp, C.c_int]
    L.vrc_get_kernel_stats.argtypes = [vp, C.c_int, C.POINTER(VrcKernelStat)]
    L.vrc_eig_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    DP = C.POINTER(C.c_double)
    L.vrc_stack_forward.argtypes = [vp, C.c_int, C.POINTER(VrcStack), C.c_double, C.c_double, DP, DP,
                                    C.POINTER(C.c_int)]
    L.vrc_stack_backward.argtypes = [vp, DP, DP, DP, DP]
    IP = C.POINTER(C.c_int)
    L.vrc_stack_fields.argtypes = [vp, C.c_int, C.c_int, CP, CP]
    L.vrc_gds_read.argtypes = [C.c_char_p, C.c_double, IP, IP, IP, DP, C.c_int, C.c_int]
    L.vrc_planar_section.argtypes = [C.POINTER(VrcCell), C.c_double, C.c_int, DP, DP, CP]
    L.vrc_redheffer_forward.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_double, C.c_int,
                                        C.POINTER(VrcResult)]
    L.vrc_redheffer_backward.argtypes = [vp, CP, CP, C.c_int, DP]
    L.vrc_chain.argtypes = [vp, C.c_int, C.POINTER(VrcCell), C.c_int, C.c_double, C.c_int, C.c_int,
                            C.POINTER(VrcResult)]
    L.vrc_chain_order_powers.argtypes = [vp, C.c_int, C.c_int, DP, DP]
    L.vrc_chain_fields.argtypes = [vp, CP, C.c_int, C.c_int, CP, CP]
    _lib = L
    return L


def _cptr(a: np.ndarray):
    assert a.dtype == np.complex128 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(CP)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vc(z) -> VrcComplex:
    z = complex(z)
    return VrcComplex(z.real, z.imag)


SAMPLE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, C.POINTER(VrcComplex), C.POINTER(VrcComplex))
SAMPLE_DEVICE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, C.POINTER(VrcComplex), C.POINTER(VrcComplex),
                               C.c_void_p)


class _CellPack:
    """A VrcCell plus the numpy buffers it points to (kept alive)."""

    def __init__(self, d: dict):
        self.keep = []
        c = VrcCell()
        kind = {"grid": GEOM_GRID, "pillar": GEOM_PILLAR, "pixels": GEOM_PIXELS, "planar": GEOM_PLANAR,
                "sampler": GEOM_SAMPLER}[d["kind"]]
        c.kind = kind
        c.nx, c.ny = int(d["nx"]), int(d["ny"])
        c.pml = 1 if d.get("pml") else 0
        c.lam = float(d["lam"])
        c.z0, c.z1 = float(d.get("z0", 0.0)), float(d.get("z1", 0.0))
        if kind == GEOM_PILLAR:
            c.Lx, c.Ly = float(d["Lx"]), float(d["Ly"])
            c.npx, c.npy = int(d["npx"]), int(d["npy"])
            c.eps_in, c.eps_out = _vc(d["eps_in"]), _vc(d["eps_out"])
            c.r0, c.r1 = float(d["r0"]), float(d["r1"])
        elif kind == GEOM_SAMPLER:
            # d["sample"](z) -> (P, Q) as n x n arrays (host callback), or
            # d["sample_device"](z, P_ptr, Q_ptr, stream) filling device buffers
            n = 2 * c.nx * c.ny
            c.Lx, c.Ly = float(d.get("Lx", 0.0)), float(d.get("Ly", 0.0))
            if d.get("sample_device") is not None:
                fdev = d["sample_device"]

                def dcb(user, z, P, Q, stream):
                    try:
                        return int(fdev(z, C.cast(P, C.c_void_p).value, C.cast(Q, C.c_void_p).value, stream) or 0)
                    except Exception:  # noqa: BLE001 - reported to the engine as a failed sample
                        return 1

                f = SAMPLE_DEVICE_FN(dcb)
                c.sample_device = C.cast(f, C.c_void_p)
            else:
                fhost = d["sample"]

                def hcb(user, z, P, Q):
                    try:
                        Pm, Qm = fhost(z)
                        for src, dst in ((Pm, P), (Qm, Q)):
                            a = np.ctypeslib.as_array(C.cast(dst, C.POINTER(C.c_double)), shape=(n * n * 2,))
                            # column-major: the bytes of the C-order transpose
                            a[:] = np.ascontiguousarray(np.asarray(src, dtype=np.complex128).T).view(np.float64).ravel()
                        return 0
                    except Exception:  # noqa: BLE001 - reported to the engine as a failed sample
                        return 1

                f = SAMPLE_FN(hcb)
                c.sample = C.cast(f, C.c_void_p)
            self.keep.append(f)
        elif kind == GEOM_PLANAR:
            polys = [np.ascontiguousarray(p, dtype=np.float64).reshape(-1, 2) for p in d["polys"]]
            start = np.ascontiguousarray(np.cumsum([0] + [len(p) for p in polys]), dtype=np.int32)
            xz = np.ascontiguousarray(np.concatenate(polys).reshape(-1))
            self.keep += [start, xz]
            c.npoly = len(polys)
            c.poly_start = start.ctypes.data_as(C.POINTER(C.c_int))
            c.poly_xz = _dptr(xz)
            for name, default in (("shift", (0.0, 0.0, 0.0)), ("pml_w", (0.5, 0.5, 0.5, 0.5)),
                                  ("space", (1.5, 1.5, 1.08, 1.0))):
                for q, v in enumerate(d.get(name, default)):
                    getattr(c, name)[q] = float(v)
            c.thickness = float(d.get("thickness", 0.22))
            c.eps_background, c.eps_device = _vc(d["eps_bg"]), _vc(d["eps_dev"])
        else:
            eps = np.ascontiguousarray(d["eps"], dtype=np.complex128)
            if kind == GEOM_PIXELS:
                x = np.linspace(0.0, d["Lx"], eps.shape[1] + 1)
                y = np.linspace(0.0, d["Ly"], eps.shape[0] + 1)
            else:
                x = np.ascontiguousarray(d["x"], dtype=np.float64)
                y = np.ascontiguousarray(d["y"], dtype=np.float64)
            self.keep += [eps, x, y]
            c.ncx, c.ncy = len(x), len(y)
            c.x, c.y = _dptr(x), _dptr(y)
            c.eps = eps.ctypes.data_as(CP)
            for name in ("xrules", "yrules"):
                rules = d.get(name, [])
                arr = (VrcRule * max(1, len(rules)))()
                for k, (idx, zs, vals) in enumerate(rules):
                    zs = np.ascontiguousarray(zs, dtype=np.float64)
                    vals = np.ascontiguousarray(vals, dtype=np.float64)
                    self.keep += [zs, vals]
                    arr[k] = VrcRule(int(idx), len(zs), _dptr(zs), _dptr(vals), 1 if d.get("spline") else 0)
                self.keep.append(arr)
                setattr(c, "n_" + name, len(rules))
                setattr(c, name, C.cast(arr, C.POINTER(VrcRule)))
            if d.get("geometry_fn") is not None:
                fn = d["geometry_fn"]
                ncx, ncy = c.ncx, c.ncy

                def cb(user, z, xp, yp):
                    xa = np.ctypeslib.as_array(xp, shape=(ncx,))
                    ya = np.ctypeslib.as_array(yp, shape=(ncy,))
                    fn(z, xa, ya)

                cfn = GEOM_FN(cb)
                self.keep.append(cfn)
                c.geometry_fn = cfn
        if d.get("end0") is not None:
            c.has_end0, c.eps_end0 = 1, _vc(d["end0"])
        if d.get("end1") is not None:
            c.has_end1, c.eps_end1 = 1, _vc(d["end1"])
        self.cell = c


def gds_read(path, unit: float = 1e-6) -> List[np.ndarray]:
    """BOUNDARY / BOX polygons of the first structure of a GDSII file, each an
    (npoints, 2) array of (x, y) in units of `unit` metres (the C reader)."""
    L = lib()
    npoly, npts = C.c_int(0), C.c_int(0)
    st = L.vrc_gds_read(str(path).encode(), float(unit), C.byref(npoly), C.byref(npts), None, None, 0, 0)
    if st != 0:
        raise VrcError(st, L.vrc_status_string(st).decode())
    start = np.zeros(npoly.value + 1, dtype=np.int32)
    xz = np.zeros(2 * max(npts.value, 1))
    st = L.vrc_gds_read(str(path).encode(), float(unit), C.byref(npoly), C.byref(npts),
                        start.ctypes.data_as(C.POINTER(C.c_int)), _dptr(xz), npoly.value, npts.value)
    if st != 0:
        raise VrcError(st, L.vrc_status_string(st).decode())
    return [xz[2 * start[p]:2 * start[p + 1]].reshape(-1, 2).copy() for p in range(npoly.value)]


def planar_section(desc: dict, z: float):
    """Cross-section of a planar cell at z: (x, y, eps (5, len(x) - 1))."""
    L = lib()
    pack = _CellPack(desc)
    n = L.vrc_planar_section(C.byref(pack.cell), float(z), 0, None, None, None)
    if n < 0:
        raise VrcError(-n, L.vrc_status_string(-n).decode())
    x = np.zeros(n)
    y = np.zeros(6)
    eps = np.zeros((5, n - 1), dtype=np.complex128)
    n2 = L.vrc_planar_section(C.byref(pack.cell), float(z), n, _dptr(x), _dptr(y), eps.ctypes.data_as(CP))
    if n2 != n:
        raise VrcError(1, "planar section size changed")
    return x, y, eps


class Context:
    """One engine context on a CUDA device."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        st = L.vrc_create(int(device), C.byref(h))
        if st != VRC_OK:
            raise VrcError(st, L.vrc_status_string(st).decode())
        self.h = h
        self.L = L

    def close(self):
        if self.h:
            self.L.vrc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != VRC_OK:
            raise VrcError(st, self.L.vrc_last_error(self.h).decode())

    def timing(self) -> Dict[str, float]:
        t = VrcTiming()
        self._check(self.L.vrc_get_timing(self.h, C.byref(t)))
        return {"device_ms": t.device_ms, "launches": int(t.launches)}

    def set_profiling(self, on: bool = True):
        self._check(self.L.vrc_set_profiling(self.h, 1 if on else 0))

    def kernel_stats(self) -> Dict[str, dict]:
        cnt = self.L.vrc_get_kernel_stats(self.h, 0, None)
        if cnt < 0:
            raise VrcError(-cnt, self.L.vrc_last_error(self.h).decode())
        arr = (VrcKernelStat * max(cnt, 1))()
        self.L.vrc_get_kernel_stats(self.h, cnt, arr)
        return {arr[i].name.decode(): {"ms": arr[i].ms, "launches": int(arr[i].launches), "flops": arr[i].flops,
                                       "bytes": arr[i].bytes, "busy_ms": arr[i].busy_ms} for i in range(cnt)}

    # ---- assembly / eigen ----
    def sample_pq(self, desc: dict, zs: Sequence[float]):
        pk = _CellPack(desc)
        n = 2 * desc["nx"] * desc["ny"]
        z = np.ascontiguousarray(zs, dtype=np.float64)
        P = np.zeros((len(z), n, n), dtype=np.complex128)
        Q = np.zeros_like(P)
        self._check(self.L.vrc_sample_pq(self.h, C.byref(pk.cell), len(z), _dptr(z), _cptr(P), _cptr(Q)))
        # C-ABI matrices are column-major: stored block b is P[b].T in C order
        return np.ascontiguousarray(P.transpose(0, 2, 1)), np.ascontiguousarray(Q.transpose(0, 2, 1))

    def wave_solve(self, P: np.ndarray, Q: np.ndarray):
        P = np.asarray(P, dtype=np.complex128)
        Q = np.asarray(Q, dtype=np.complex128)
        single = P.ndim == 2
        if single:
            P, Q = P[None], Q[None]
        b, n = P.shape[0], P.shape[1]
        Pc = np.ascontiguousarray(P.transpose(0, 2, 1))
        Qc = np.ascontiguousarray(Q.transpose(0, 2, 1))
        W = np.zeros_like(Pc)
        V = np.zeros_like(Pc)
        g = np.zeros((b, n), dtype=np.complex128)
        self._check(self.L.vrc_wave_solve(self.h, b, n, _cptr(Pc), _cptr(Qc), _cptr(W), _cptr(V), _cptr(g)))
        W = W.transpose(0, 2, 1)
        V = V.transpose(0, 2, 1)
        return (W[0], V[0], g[0]) if single else (W, V, g)

    def eig(self, A: np.ndarray):
        A = np.asarray(A, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A = A[None]
        b, n = A.shape[0], A.shape[1]
        Ac = np.ascontiguousarray(A.transpose(0, 2, 1))
        W = np.zeros_like(Ac)
        lam = np.zeros((b, n), dtype=np.complex128)
        self._check(self.L.vrc_eig(self.h, b, n, _cptr(Ac), _cptr(W), _cptr(lam)))
        W = W.transpose(0, 2, 1)
        return (lam[0], W[0]) if single else (lam, W)

    def zgemm(self, A: np.ndarray, B: np.ndarray):
        A = np.asarray(A, dtype=np.complex128)
        B = np.asarray(B, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A, B = A[None], B[None]
        b, n = A.shape[0], A.shape[1]
        Ac = np.ascontiguousarray(A.transpose(0, 2, 1))
        Bc = np.ascontiguousarray(B.transpose(0, 2, 1))
        Cc = np.zeros_like(Ac)
        self._check(self.L.vrc_zgemm(self.h, b, n, _cptr(Ac), _cptr(Bc), _cptr(Cc)))
        Cm = Cc.transpose(0, 2, 1)
        return Cm[0] if single else Cm

    def zinv(self, A: np.ndarray):
        A = np.asarray(A, dtype=np.complex128)
        single = A.ndim == 2
        if single:
            A = A[None]
        b, n = A.shape[0], A.shape[1]
        Ac = np.ascontiguousarray(A.transpose(0, 2, 1))
        st = np.zeros(b, dtype=np.int32)
        self._check(self.L.vrc_zinv(self.h, b, n, _cptr(Ac), st.ctypes.data_as(C.POINTER(C.c_int))))
        Ai = Ac.transpose(0, 2, 1)
        return (Ai[0], int(st[0])) if single else (Ai, st)

    # ---- integrators ----
    def _results(self, descs, want_blocks=True):
        res = (VrcResult * len(descs))()
        bufs = []
        for i, d in enumerate(descs):
            n = 2 * d["nx"] * d["ny"]
            if want_blocks:
                arrs = {k: np.zeros((n, n), dtype=np.complex128) for k in
                        ("Tdd", "Tuu", "Rud", "Rdu", "W0", "V0", "W1", "V1")}
                arrs["gam0"] = np.zeros(n, dtype=np.complex128)
                arrs["gam1"] = np.zeros(n, dtype=np.complex128)
                for k, a in arrs.items():
                    setattr(res[i], k, _cptr(a))
                bufs.append(arrs)
            else:
                bufs.append({})
        return res, bufs

    @staticmethod
    def _unpack(res, bufs) -> List[dict]:
        out = []
        for i, arrs in enumerate(bufs):
            r = {k: (v.T.copy() if v.ndim == 2 else v) for k, v in arrs.items()}
            r.update(status=res[i].status, n=res[i].n, N=res[i].N, n_eig=res[i].n_eig,
                     n_samples=res[i].n_samples, n_nodes=res[i].n_nodes)
            out.append(r)
        return out

    def redheffer(self, descs: List[dict], pe: float = 1e-2, max_depth: int = 40, blocks=True):
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        res, bufs = self._results(descs, blocks)
        self._check(self.L.vrc_redheffer(self.h, len(descs), cells, float(pe), int(max_depth), res))
        return self._unpack(res, bufs)

    def redheffer_forward(self, descs: List[dict], pe: float = 1e-2, max_depth: int = 40):
        """redheffer() that keeps the cells and segmentations for redheffer_backward."""
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        res, bufs = self._results(descs, True)
        self._check(self.L.vrc_redheffer_forward(self.h, len(descs), cells, float(pe), int(max_depth), res))
        self._grad_packs = packs  # geometry callbacks stay alive for the backward
        self._grad_descs = descs
        return self._unpack(res, bufs)

    def redheffer_backward(self, gS, gB=None, every: int = 0):
        """Gradient of the last redheffer_forward's cells with respect to their
        rule knots.  gS: per cell (gTdd, gTuu, gRud, gRdu), gB: per cell
        (gW0, gV0, gW1, gV1) or None (n x n arrays).  Returns per cell a list of
        arrays, dL/d vals of each x rule then each y rule."""
        descs = self._grad_descs

        def pack(mats_per_cell):
            return np.ascontiguousarray(np.concatenate(
                [np.stack([np.asarray(m, dtype=np.complex128).T for m in ms]).reshape(-1) for ms in mats_per_cell]))

        S = pack(gS)
        B = pack(gB) if gB is not None else None
        sizes = [[len(r[1]) for r in d.get("xrules", [])] + [len(r[1]) for r in d.get("yrules", [])] for d in descs]
        g = np.zeros(sum(sum(z) for z in sizes))
        self._check(self.L.vrc_redheffer_backward(self.h, _cptr(S), _cptr(B) if B is not None else None, int(every),
                                                  _dptr(g)))
        out, off = [], 0
        for z in sizes:
            per = []
            for k in z:
                per.append(g[off:off + k].copy())
                off += k
            out.append(per)
        return out

    def redheffer_segments(self, descs: List[dict], cuts: List[Sequence[float]], blocks=True):
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        cut_arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in cuts]
        ncuts = (C.c_int * len(descs))(*[len(c) for c in cut_arrs])
        cptrs = (C.POINTER(C.c_double) * len(descs))(*[_dptr(c) for c in cut_arrs])
        res, bufs = self._results(descs, blocks)
        self._check(self.L.vrc_redheffer_segments(self.h, len(descs), cells, ncuts, cptrs, res))
        return self._unpack(res, bufs)

    def tree(self, cell: int = 0):
        cnt = self.L.vrc_get_tree(self.h, cell, 0, None, None, None, None)
        if cnt < 0:
            raise VrcError(-cnt, "no tree")
        a = np.zeros(cnt)
        b = np.zeros(cnt)
        e = np.zeros(cnt)
        acc = np.zeros(cnt, dtype=np.int32)
        self.L.vrc_get_tree(self.h, cell, cnt, _dptr(a), _dptr(b), _dptr(e),
                            acc.ctypes.data_as(C.POINTER(C.c_int)))
        return [(float(a[i]), float(b[i]), float(e[i]), bool(acc[i])) for i in range(cnt)]

    def rcwa(self, descs: List[dict], N: int, blocks=True):
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        res, bufs = self._results(descs, blocks)
        self._check(self.L.vrc_rcwa(self.h, len(descs), cells, int(N), res))
        return self._unpack(res, bufs)

    def differential(self, descs: List[dict], N: int, blocks=True):
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        res, bufs = self._results(descs, blocks)
        self._check(self.L.vrc_differential(self.h, len(descs), cells, int(N), res))
        return self._unpack(res, bufs)

    def order_powers(self, descs: List[dict], method: str = "redheffer", pe: float = 1e-2, max_depth: int = 40,
                     nslices: int = 10, side: int = 1, flux_norm: bool = True):
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        total = sum(2 * d["nx"] * d["ny"] for d in descs)
        R = np.zeros(total)
        T = np.zeros(total)
        st = np.zeros(len(descs), dtype=np.int32)
        meth = {"redheffer": 0, "rcwa": 1, "differential": 2}[method]
        self._check(self.L.vrc_order_powers(self.h, len(descs), cells, meth, float(pe), int(max_depth),
                                            int(nslices), int(side), 1 if flux_norm else 0, _dptr(R), _dptr(T),
                                            st.ctypes.data_as(C.POINTER(C.c_int))))
        out = []
        off = 0
        for i, d in enumerate(descs):
            m = d["nx"] * d["ny"]
            out.append({"R": R[off:off + 2 * m].reshape(2, m), "T": T[off:off + 2 * m].reshape(2, m),
                        "status": int(st[i])})
            off += 2 * m
        return out

    # ---- stacks of sections ----
    def chain(self, descs: List[dict], method: str = "redheffer", pe: float = 1e-2, max_depth: int = 40,
              nslices: int = 10):
        """Sections (each a structure on its own z-range) solved and joined in
        order; returns the stack's result dict (blocks, entrance and exit bases)."""
        packs = [_CellPack(d) for d in descs]
        cells = (VrcCell * len(descs))(*[p.cell for p in packs])
        res, bufs = self._results(descs[:1], True)
        meth = {"redheffer": 0, "rcwa": 1, "differential": 2}[method]
        self._check(self.L.vrc_chain(self.h, len(descs), cells, meth, float(pe), int(max_depth), int(nslices), res))
        self._chain = (len(descs), 2 * descs[0]["nx"] * descs[0]["ny"], descs[0]["nx"] * descs[0]["ny"])
        return self._unpack(res, bufs)[0]

    def chain_order_powers(self, side: int = 1, flux_norm: bool = True):
        _, _, m = self._chain
        R = np.zeros(2 * m)
        T = np.zeros(2 * m)
        self._check(self.L.vrc_chain_order_powers(self.h, int(side), 1 if flux_norm else 0, _dptr(R), _dptr(T)))
        return {"R": R.reshape(2, m), "T": T.reshape(2, m)}

    def chain_fields(self, c, ngx: int = 0, ngy: int = 0):
        """Interface amplitudes (S+1, 2, n) for incident entrance amplitudes c,
        and Ex / Ey images (S+1, 2, ngy, ngx) when ngx, ngy > 0."""
        S, n, _ = self._chain
        c = np.ascontiguousarray(c, dtype=np.complex128)
        amps = np.zeros((S + 1, 2, n), dtype=np.complex128)
        img = np.zeros((S + 1, 2, ngy, ngx), dtype=np.complex128) if ngx > 0 else None
        self._check(self.L.vrc_chain_fields(self.h, _cptr(c), int(ngx), int(ngy), amps.ctypes.data_as(CP),
                                            img.ctypes.data_as(CP) if img is not None else None))
        return amps, img

    # ---- layer stacks: forward and adjoint ----
    def stack_forward(self, stacks: List[dict], px: float = 1.0, py: float = 0.0):
        """Per-order (REF, TRN) of a batch of pixel-layer stacks.  Each stack is a
        dict with lam, Lx, Ly, nx, ny, layers (list of (npy, npx) real arrays),
        thick (list), eps_in, eps_out.  Returns (REF, TRN, status) with REF and
        TRN of shape (nstacks, nx*ny); keeps the state for stack_backward."""
        keep = []
        arr = (VrcStack * len(stacks))()
        for i, d in enumerate(stacks):
            eps = np.ascontiguousarray(np.stack([np.asarray(a, dtype=np.float64) for a in d["layers"]]))
            thick = np.ascontiguousarray(np.asarray(d["thick"], dtype=np.float64))
            keep += [eps, thick]
            L_, npy, npx = eps.shape
            arr[i] = VrcStack(float(d["lam"]), float(d["Lx"]), float(d["Ly"]), int(d["nx"]), int(d["ny"]), npx, npy,
                              L_, _dptr(eps), _dptr(thick), _vc(d.get("eps_in", 1.0)), _vc(d.get("eps_out", 1.0)))
        m = stacks[0]["nx"] * stacks[0]["ny"]
        REF = np.zeros((len(stacks), m))
        TRN = np.zeros((len(stacks), m))
        st = np.zeros(len(stacks), dtype=np.int32)
        self._check(self.L.vrc_stack_forward(self.h, len(stacks), arr, float(px), float(py), _dptr(REF), _dptr(TRN),
                                             st.ctypes.data_as(C.POINTER(C.c_int))))
        self._stack_shape = (len(stacks), len(stacks[0]["layers"]), *np.asarray(stacks[0]["layers"][0]).shape)
        self._stack_m = m
        return REF, TRN, st

    def stack_backward(self, wR: np.ndarray, wT: np.ndarray, want_thick: bool = False):
        """dL/d(pixel) of L = sum wR*REF + wT*TRN for the last stack_forward,
        shape (nstacks, nlayers, npy, npx); with want_thick also dL/d(layer
        thickness), shape (nstacks, nlayers)."""
        shape = self._stack_shape
        wR = np.ascontiguousarray(np.broadcast_to(np.asarray(wR, dtype=np.float64), (shape[0], wR.shape[-1])))
        wT = np.ascontiguousarray(np.broadcast_to(np.asarray(wT, dtype=np.float64), (shape[0], wT.shape[-1])))
        g = np.zeros(shape)
        gt = np.zeros(shape[:2])
        self._check(self.L.vrc_stack_backward(self.h, _dptr(wR), _dptr(wT), _dptr(g), _dptr(gt)))
        return (g, gt) if want_thick else g

    def stack_fields(self, ngx: int = 0, ngy: int = 0):
        """Amplitudes (nstacks, nlayers+1, 2, n) at every interface of the last
        stack_forward and, with ngx, ngy > 0, Ex / Ey images
        (nstacks, nlayers+1, 2, ngy, ngx) over the period."""
        C_, L_ = self._stack_shape[:2]
        n = 2 * self._stack_m
        amps = np.zeros((C_, L_ + 1, 2, n), dtype=np.complex128)
        img = np.zeros((C_, L_ + 1, 2, ngy, ngx), dtype=np.complex128) if ngx > 0 else None
        self._check(self.L.vrc_stack_fields(self.h, int(ngx), int(ngy), amps.ctypes.data_as(CP),
                                            img.ctypes.data_as(CP) if img is not None else None))
        return amps, img
