"""The reference's own GDSII fixture (`contour_extract.gds`, shipped at the
root of the reference and driven by src/tests/test_gds_cpu.cpp:131-146),
copied unchanged to tests/golden/.

* The C reader (vrc_gds_read) against an independent parse of the stream
  written here from the GDSII record definitions (HEADER ... ENDLIB,
  excess-64 reals, BOUNDARY XY lists closed by a repeated first point).
* The C cross-sections of the planar device (vrc_planar_section, the role of
  GDSIISampler::sampleLayout) against the oracle's restatement, bit for bit,
  with the driver's shift, PML and spacer widths, over its z-range.
No GPU needed: both are host code behind the C ABI."""
import struct
from pathlib import Path

import numpy as np
import pytest

from oracle.planar_sampler import PlanarSampler
from varrcwa_b200 import capi
from varrcwa_b200 import structures as st

GDS = Path(__file__).resolve().parent / "golden" / "contour_extract.gds"


def _real8(raw):
    sign = -1.0 if raw[0] & 0x80 else 1.0
    return sign * int.from_bytes(raw[1:8], "big") / float(1 << 56) * 16.0 ** ((raw[0] & 0x7F) - 64)


def _parse(path, unit=1e-6):
    """BOUNDARY / BOX polygons of the first structure, in `unit` metres."""
    b = Path(path).read_bytes()
    off, scale, polys, struct_no, kind = 0, None, [], 0, None
    while off + 4 <= len(b):
        ln, rt, _ = struct.unpack(">HBB", b[off:off + 4])
        if ln < 4:
            break
        pay = b[off + 4:off + ln]
        off += ln
        if rt == 0x03:  # UNITS: user units per db unit, metres per db unit
            scale = _real8(pay[8:16]) / unit
        elif rt == 0x05:
            struct_no += 1
        elif struct_no == 1 and rt in (0x08, 0x2D):  # BOUNDARY, BOX
            kind = "poly"
        elif struct_no == 1 and rt == 0x10 and kind == "poly":
            xy = np.array(struct.unpack(f">{len(pay) // 4}i", pay), dtype=np.float64).reshape(-1, 2) * scale
            if len(xy) > 1 and np.array_equal(xy[0], xy[-1]):
                xy = xy[:-1]
            polys.append(xy)
        elif rt == 0x11:
            kind = None
        elif rt == 0x04:
            break
    return polys


def test_reader_matches_independent_parse_of_reference_fixture():
    polys = capi.gds_read(GDS)
    ref = _parse(GDS)
    assert len(polys) == len(ref) == 8
    assert sum(len(p) for p in polys) == 1085
    for a, b in zip(polys, ref):
        np.testing.assert_allclose(a, b, rtol=1e-15, atol=1e-15)
    allp = np.concatenate(polys)
    # the layout spans the driver's integration range [-1.63, 1.36] in z
    assert allp[:, 1].min() < -1.63 and allp[:, 1].max() > 1.36


@pytest.mark.parametrize("z", np.linspace(-1.63, 1.36, 13).tolist() + [-1.0, 0.0, 0.5])
def test_contour_sections_match_oracle(z):
    d = st.gds_planar(capi.gds_read(GDS))
    x, y, eps = capi.planar_section(d, z)
    o = PlanarSampler(d["lam"], d["nx"], d["ny"], d["polys"], d["shift"], d["pml_w"], d["space"], d["thickness"],
                      d["eps_bg"], d["eps_dev"])
    ox, oeps = o.section(z)
    np.testing.assert_array_equal(x, ox)
    np.testing.assert_array_equal(y, o.y)
    np.testing.assert_array_equal(eps, oeps)
    # the driver's cell: the shift puts the layout's left edge (-0.8646 um)
    # 1.5 um (PML 0.5 + space 1.0) right of x = 1e-4
    assert x[0] == pytest.approx(1e-4, abs=1e-12) and len(x) >= 4
