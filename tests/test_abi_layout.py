"""CPU check of the boundary's struct layouts: the ctypes mirrors in
thegraphpartitioning_b200/_abi.py have the size and field offsets that a C
compiler gives the structs of include/gp_partition.h (a drift between the two
would corrupt every options, stats, trace or learned-report exchange)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from thegraphpartitioning_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "gp_options": _abi.GpOptions,
    "gp_stats": _abi.GpStats,
    "gp_trace_event": _abi.GpTraceEvent,
    "gp_learned_report": _abi.GpLearnedReport,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("layout")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gp_partition.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr   # a field named in _abi.py but absent from the header fails here
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    table = {}
    for line in out.splitlines():
        s, f, v = line.split()
        table[(s, f)] = int(v)
    return table


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_struct_matches_header(c_layout, cname):
    py = STRUCTS[cname]
    assert ctypes.sizeof(py) == c_layout[(cname, "size")], cname
    for field, _ in py._fields_:
        assert getattr(py, field).offset == c_layout[(cname, field)], f"{cname}.{field}"
