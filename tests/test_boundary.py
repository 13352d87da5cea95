"""The C-ABI library builds, loads and exports every declared entry point
(no GPU needed: no compute call is made)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    txt = (ROOT / "include" / "vrc.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vrc_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from varrcwa_b200 import build
    lib = build.build()
    L = ctypes.CDLL(str(lib))
    missing = [s for s in _declared() if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_header():
    from varrcwa_b200 import capi
    assert sorted(capi.EXPORTS) == _declared()


def test_status_strings_and_invalid_context():
    from varrcwa_b200 import capi
    L = capi.lib()
    assert L.vrc_status_string(0) == b"ok"
    assert L.vrc_status_string(4) == b"singular matrix"
    # null context is rejected without touching a device
    assert L.vrc_redheffer(None, 0, None, 1e-2, 10, None) == capi.VRC_EINVAL


def test_no_device_is_reported_not_hidden():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from varrcwa_b200 import capi
    h = ctypes.c_void_p()
    assert capi.lib().vrc_create(0, ctypes.byref(h)) == capi.VRC_ENODEV
    with pytest.raises(capi.VrcError):
        capi.Context(0)
