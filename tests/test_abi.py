"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every function that include/*.h declares (no compute calls: no GPU here)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(gp_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("gp_partition", "gp_partition_ex", "gp_partition_device", "gp_edge_cut_device",
                 "gp_last_error", "gp_default_options", "gp_release_workspace", "gp_version"):
        assert must in names


def test_library_exports_every_declared_symbol(gp):
    lib = gp.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", gp.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gp_\w+)", out))
    assert declared_functions() <= exported


def test_library_built_for_sm100a():
    """Every device object is compiled for sm_100a only (the GPU tests then
    launch its kernels, which fails on a library without sm_100a code)."""
    mk = open(os.path.join(ROOT, "thegraphpartitioning_b200", "csrc", "Makefile")).read()
    arch = re.search(r"^ARCH\s*:=\s*(.*)$", mk, flags=re.M).group(1).strip()
    assert arch == "-gencode arch=compute_100a,code=sm_100a"
    assert "$(NVCC) $(NVFLAGS) -c" in mk and "$(ARCH)" in re.search(r"^NVFLAGS\s*:=(.*)$", mk, flags=re.M).group(1)


def test_cli_built():
    import thegraphpartitioning_b200 as gp
    assert os.path.exists(gp.CLI_PATH)


def test_no_oracle_in_product():
    """The product package never imports or links the oracle."""
    pkg = os.path.join(ROOT, "thegraphpartitioning_b200")
    for path in glob.glob(os.path.join(pkg, "**", "*"), recursive=True):
        if path.endswith((".py", ".cu", ".cuh", ".cpp", ".h")) or os.path.basename(path) == "Makefile":
            text = open(path).read()
            assert "import oracle" not in text and "from oracle" not in text, path
            assert "libgp_oracle" not in text and "gpo_" not in text, path
