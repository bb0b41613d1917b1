"""The ctypes structs of the binding (sloth_b200/_capi.py) have the sizes and
field offsets that a C compiler gives the same structs in
include/sloth_b200.h: a small C program prints sizeof and offsetof for every
field the binding declares, and the two must agree exactly."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT
from sloth_b200 import _capi

STRUCTS = ["SlothGridDesc", "SlothTraceParams", "SlothTraceOutputs", "SlothServerConfig", "SlothServerStats",
           "SlothOptic", "SlothDetectorParams", "SlothBeamParams", "SlothImageParams"]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_the_c_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sloth_b200.h"', "int main(void) {"]
    expected = {}
    for name in STRUCTS:
        cls = getattr(_capi, name)
        expected[(name, "")] = _capi.ctypes.sizeof(cls)
        lines.append(f'    printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            expected[(name, field)] = getattr(cls, field).offset
            lines.append(f'    printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if not line.strip():
            continue
        key, value = line.rsplit(" ", 1)
        name, _, field = key.partition(".")
        got[(name, field)] = int(value)
    assert got == expected


def _stub():
    import importlib.util
    spec = importlib.util.spec_from_file_location("sloth_b200_ctypes", os.path.join(ROOT, "include", "sloth_b200_ctypes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_side_stub_structs_match_the_binding():
    """The ctypes stub a SLOTH maintainer adds (include/sloth_b200_ctypes.py)
    declares the same struct layouts as the package's binding."""
    ns = _stub()
    for stub_name, name in (("GridDesc", "SlothGridDesc"), ("TraceParams", "SlothTraceParams"),
                            ("TraceOutputs", "SlothTraceOutputs")):
        a, b = getattr(ns, stub_name), getattr(_capi, name)
        assert _capi.ctypes.sizeof(a) == _capi.ctypes.sizeof(b), stub_name
        assert [f for f, _ in a._fields_] == [f for f, _ in b._fields_], stub_name
        for f, _ in a._fields_:
            assert getattr(a, f).offset == getattr(b, f).offset, (stub_name, f)


def test_reference_side_stub_loads_the_library():
    """The stub opens the built library and finds every entry point it declares
    (no compute call: no GPU is needed)."""
    lib = _stub().load(_capi.LIB_PATH)
    assert lib.sloth_trace_workspace_bytes(1000) > 0
    assert lib.sloth_strerror(0)
