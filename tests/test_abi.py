"""CPU: the C-ABI library loads and exports every entry point include/dipl_bvh.h declares."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from diplodocus_b200 import _lib as L


def declared():
    src = open(os.path.join(ROOT, "include", "dipl_bvh.h")).read()
    return sorted(set(re.findall(r"DIPL_API\s+[\w\s\*]+?\b(dipl_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared() == sorted(L.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in declared():
        assert hasattr(lib, name), name


def test_library_exports_nothing_else():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    syms = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert {s for s in syms if s.startswith("dipl_")} == set(declared())


def test_version_and_status_strings_need_no_gpu():
    lib = L.load()
    assert lib.dipl_abi_version() == 2
    assert lib.dipl_status_string(0) == b"DIPL_OK"
    assert lib.dipl_status_string(4) == b"DIPL_ERR_TIMEOUT"


def test_desc_defaults():
    d = L.default_desc()
    assert (d.code_type, d.bv_type, d.layout, d.max_triangles_per_leaf, d.nn_search_radius, d.kdop_size) == \
        (0, 0, 0, 4, 16, 32)


def test_missing_library_fails_loudly(tmp_path):
    saved = L._lib
    try:
        L._lib = None
        with pytest.raises(FileNotFoundError):
            L.load(str(tmp_path / "nope.so"))
    finally:
        L._lib = saved
