"""GDSII input and the planar-device sampler (GDSIISampler): the C reader
against a file written here, and the C cross-sections against the oracle's.
No GPU needed (the reader and the sections are host code behind the C ABI)."""
import math
import struct

import numpy as np
import pytest

from oracle.planar_sampler import PlanarSampler
from varrcwa_b200 import capi
from varrcwa_b200 import structures as st


def _real8(v):
    """GDSII 8-byte real: sign, excess-64 base-16 exponent, 56-bit mantissa."""
    if v == 0:
        return bytes(8)
    sign = 0x80 if v < 0 else 0
    v = abs(v)
    e = 0
    while v >= 1.0:
        v /= 16.0
        e += 1
    while v < 1.0 / 16.0:
        v *= 16.0
        e -= 1
    mant = int(round(v * (1 << 56)))
    if mant >= 1 << 56:
        mant >>= 4
        e += 1
    return bytes([sign | (e + 64)]) + mant.to_bytes(7, "big")


def _rec(rtype, dtype, payload=b""):
    return struct.pack(">HBB", 4 + len(payload), rtype, dtype) + payload


def _xy(points):
    return _rec(0x10, 0x03, b"".join(struct.pack(">ii", int(x), int(y)) for x, y in points))


def _write_gds(path, first, second, dbu_m=1e-9):
    """Library with two structures; `first` is a list of (kind, points)."""
    b = _rec(0x00, 0x02, struct.pack(">h", 600))
    b += _rec(0x01, 0x02, bytes(24))
    b += _rec(0x02, 0x06, b"LIB\0")
    b += _rec(0x03, 0x05, _real8(dbu_m / 1e-6) + _real8(dbu_m))
    for name, elems in ((b"TOP\0", first), (b"OTHER\0", second)):
        b += _rec(0x05, 0x02, bytes(24)) + _rec(0x06, 0x06, name)
        for kind, pts in elems:
            if kind == "boundary":
                b += _rec(0x08, 0x00) + _rec(0x0D, 0x02, struct.pack(">h", 1)) + _rec(0x0E, 0x02, struct.pack(">h", 0))
                b += _xy(list(pts) + [pts[0]]) + _rec(0x11, 0x00)
            elif kind == "box":
                b += _rec(0x2D, 0x00) + _rec(0x0D, 0x02, struct.pack(">h", 2)) + _rec(0x2E, 0x02, struct.pack(">h", 0))
                b += _xy(list(pts) + [pts[0]]) + _rec(0x11, 0x00)
            elif kind == "path":
                b += _rec(0x09, 0x00) + _rec(0x0D, 0x02, struct.pack(">h", 3)) + _rec(0x0E, 0x02, struct.pack(">h", 0))
                b += _rec(0x0F, 0x03, struct.pack(">i", 100)) + _xy(pts) + _rec(0x11, 0x00)
        b += _rec(0x07, 0x00)
    b += _rec(0x04, 0x00)
    path.write_bytes(b)


def test_real8_encoding_roundtrip():
    # the encoder above against the format's definition
    for v in (1e-3, 1e-9, 1.0, 0.5, 123.456):
        raw = _real8(v)
        e = (raw[0] & 0x7F) - 64
        m = int.from_bytes(raw[1:], "big")
        assert math.isclose(m / (1 << 56) * 16.0 ** e, v, rel_tol=1e-15)


def test_gds_reader_reads_first_structure_polygons(tmp_path):
    taper = [(-250, 0), (250, 0), (600, 4000), (-600, 4000)]
    box = [(2000, 0), (3000, 0), (3000, 500), (2000, 500)]
    _write_gds(tmp_path / "t.gds", [("boundary", taper), ("path", [(0, 0), (0, 1000)]), ("box", box)],
               [("boundary", [(0, 0), (10, 0), (10, 10)])])
    polys = capi.gds_read(tmp_path / "t.gds")  # micrometres
    assert len(polys) == 2  # the path and the second structure are skipped
    np.testing.assert_allclose(polys[0], np.array(taper) * 1e-3, rtol=0, atol=1e-15)
    np.testing.assert_allclose(polys[1], np.array(box) * 1e-3, rtol=0, atol=1e-15)
    nm = capi.gds_read(tmp_path / "t.gds", unit=1e-9)
    np.testing.assert_allclose(nm[0], np.array(taper, dtype=float), rtol=1e-14)


def test_gds_reader_rejects_malformed_files(tmp_path):
    (tmp_path / "bad.gds").write_bytes(struct.pack(">HBB", 2, 0, 0) + b"xx")
    with pytest.raises(capi.VrcError):
        capi.gds_read(tmp_path / "bad.gds")
    with pytest.raises(capi.VrcError):
        capi.gds_read(tmp_path / "missing.gds")


@pytest.mark.parametrize("z", [0.0, 0.25, 0.5, 1.3, 2.5, 4.5, 4.75, 5.0, -0.1, 9.0])
def test_planar_section_matches_oracle(z):
    d = st.planar_taper()
    x, y, eps = capi.planar_section(d, z)
    o = PlanarSampler(d["lam"], d["nx"], d["ny"], d["polys"], d["shift"], d["pml_w"], d["space"], d["thickness"],
                      d["eps_bg"], d["eps_dev"])
    ox, oeps = o.section(z)
    np.testing.assert_array_equal(x, ox)
    np.testing.assert_array_equal(y, o.y)
    np.testing.assert_array_equal(eps, oeps)


def test_planar_section_two_polygons_and_shift():
    d = st.planar_taper()
    d["polys"] = [d["polys"][0], np.array([(2.0, 0.5), (2.6, 0.5), (2.6, 3.0), (2.0, 3.0)])]
    d["shift"] = (0.3, -0.2, 0.0)
    x, y, eps = capi.planar_section(d, 1.0)
    assert len(x) == 4 + 4  # four crossings at z = 1
    assert (eps[2, 2::2][: (len(x) - 4) // 2] == d["eps_dev"]).all()
    o = PlanarSampler(d["lam"], d["nx"], d["ny"], d["polys"], d["shift"], d["pml_w"], d["space"], d["thickness"],
                      d["eps_bg"], d["eps_dev"])
    ox, oeps = o.section(1.0)
    np.testing.assert_array_equal(x, ox)
    np.testing.assert_array_equal(eps, oeps)


def test_planar_straight_waveguide_known_answer():
    """A z-invariant planar device (one straight strip): the oracle's varRCWA
    accepts the whole range as one segment, and its S-matrix equals a single
    RCWA slab of the same cross-section (the z-invariance known answer on the
    GDSIISampler path)."""
    from oracle import varrcwa_oracle as O
    from oracle.structures_adapter import make_sampler
    d = st.planar_taper(w0=0.5, w1=0.5, length=1.0, norders=(5, 3))
    s = make_sampler(d)
    S = O.redheffer_compute(s, d["z0"], d["z1"], pe=1e-8)
    assert S.N == 1
    R = O.rcwa_compute(s, d["z0"], d["z1"], 1)
    F, G = S.fourier_blocks(), R.fourier_blocks()
    scale = np.linalg.norm(G["Tuu"])  # the reflections vanish (own end bases)
    for k in F:
        assert np.linalg.norm(F[k] - G[k]) <= 1e-9 * scale, k


def test_gds_reader_units_negative_coordinates_and_skipped_elements(tmp_path):
    """Database unit 0.1 nm, negative coordinates, TEXT and SREF elements
    (skipped) between polygons."""
    tri = [(-12345, -6789), (40000, -6789), (0, 55555)]
    lib = _rec(0x00, 0x02, struct.pack(">h", 600)) + _rec(0x01, 0x02, bytes(24)) + _rec(0x02, 0x06, b"L\0")
    lib += _rec(0x03, 0x05, _real8(1e-10 / 1e-6) + _real8(1e-10))
    lib += _rec(0x05, 0x02, bytes(24)) + _rec(0x06, 0x06, b"T\0")
    lib += _rec(0x0C, 0x00) + _rec(0x0D, 0x02, struct.pack(">h", 5)) + _rec(0x16, 0x02, struct.pack(">h", 0))
    lib += _xy([(1, 2)]) + _rec(0x19, 0x06, b"hi") + _rec(0x11, 0x00)            # TEXT
    lib += _rec(0x0A, 0x00) + _rec(0x12, 0x06, b"X\0") + _xy([(0, 0)]) + _rec(0x11, 0x00)  # SREF
    lib += _rec(0x08, 0x00) + _rec(0x0D, 0x02, struct.pack(">h", 1)) + _rec(0x0E, 0x02, struct.pack(">h", 0))
    lib += _xy(tri + [tri[0]]) + _rec(0x11, 0x00)
    lib += _rec(0x07, 0x00) + _rec(0x04, 0x00)
    (tmp_path / "u.gds").write_bytes(lib)
    polys = capi.gds_read(tmp_path / "u.gds")
    assert len(polys) == 1
    np.testing.assert_allclose(polys[0], np.array(tri) * 1e-4, rtol=1e-15, atol=1e-18)
