"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re

from conftest import ROOT
from sloth_b200 import _capi


def _declared():
    hdr = open(os.path.join(ROOT, "include", "sloth_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(sloth_[a-z0-9_]+)\s*\(", hdr)))


def test_header_matches_binding():
    assert _declared() == sorted(_capi.EXPORTED_SYMBOLS)


def test_library_exports_every_symbol():
    lib = _capi.load()
    for name in _declared():
        assert hasattr(lib, name), name


def test_no_device_calls_are_safe():
    lib = _capi.load()
    assert lib.sloth_abi_version() == 3
    assert "sm_100" in _capi.strerror(_capi.SLOTH_ERR_UNSUPPORTED_DEVICE)
    assert _capi.strerror(12345) == "unknown error code"
    # size queries need no device
    g = _capi.grid_desc((4, 5, 6), (0, 0, 0), (1e-3, 1e-3, 1e-3))
    assert lib.sloth_grid_bytes(g, 4) == 4 * 5 * 6 * 16
    assert lib.sloth_grid_bytes(g, 8) == 4 * 5 * 6 * 32
    assert lib.sloth_grid_bytes(g, 2) == 0
    bad = _capi.grid_desc((1, 5, 6), (0, 0, 0), (1e-3, 1e-3, 1e-3))
    assert lib.sloth_grid_bytes(bad, 4) == 0
    assert lib.sloth_trace_workspace_bytes(10) >= 3 * 40
    # argument validation happens before any CUDA call
    p = _capi.SlothTraceParams()
    out = _capi.SlothTraceOutputs()
    rc = lib.sloth_trace_f32(g, None, p, None, 10, out, None, 0, None)
    assert rc == _capi.SLOTH_ERR_INVALID_ARGUMENT      # omega = 0
    assert lib.sloth_trace_f32(None, None, p, None, 10, out, None, 0, None) == _capi.SLOTH_ERR_NULL_POINTER
