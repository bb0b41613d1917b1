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


def test_integration_stub_structs_match_the_binding():
    """The ctypes stub that INTEGRATION.md shows a SLOTH maintainer declares
    the same struct layouts as the binding (its class definitions run here;
    the library loading lines do not)."""
    import re
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```python\n(.*?)```", text, flags=re.S)
    stub = next(b for b in blocks if "class TraceParams(Structure)" in b)
    import ast
    tree = ast.parse(stub)
    keep = [n for n in tree.body if isinstance(n, (ast.Import, ast.ImportFrom, ast.ClassDef))]
    ns = {}
    exec(compile(ast.Module(body=keep, type_ignores=[]), "INTEGRATION.md", "exec"), ns)
    for stub_name, name in (("GridDesc", "SlothGridDesc"), ("TraceParams", "SlothTraceParams"),
                            ("TraceOutputs", "SlothTraceOutputs")):
        a, b = ns[stub_name], getattr(_capi, name)
        assert _capi.ctypes.sizeof(a) == _capi.ctypes.sizeof(b), stub_name
        assert [f for f, _ in a._fields_] == [f for f, _ in b._fields_], stub_name
        for f, _ in a._fields_:
            assert getattr(a, f).offset == getattr(b, f).offset, (stub_name, f)
