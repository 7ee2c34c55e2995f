"""The C ABI library loads without a GPU, exports every function declared in
include/rgpu.h, and reports errors through status codes instead of crashing."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import rgpu

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "rgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("rg_create", "rg_destroy", "rg_sync_topology", "rg_upload_state", "rg_godunov_level",
                 "rg_set_unew", "rg_set_uold", "rg_download_state", "rg_last_error", "rg_courant_step"):
        assert must in names


def test_library_exports_every_declared_symbol(rgpu_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(rgpu.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (rg_\w+)$", out, flags=re.M))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert getattr(rgpu_lib, n)


def test_riemann_string_resolution_matches_reference(rgpu_lib):
    # HydroSolver.cpp:456-461: exact, case-sensitive names; anything else is LLF
    f = rgpu_lib.rg_riemann_from_string
    assert [f(s) for s in (b"hllc", b"hll", b"exact", b"acoustic", b"llf", b"HLLC", b"roe")] == [2, 1, 3, 4, 0, 0, 0]


def test_invalid_params_are_reported_not_raised(rgpu_lib):
    p = rgpu.make_params(2)  # ndim 2 is not built
    h = rgpu_lib.rg_create(C.byref(p), 0)
    assert h
    try:
        assert b"ndim" in rgpu_lib.rg_last_error(h)
        assert rgpu_lib.rg_set_unew(h, 1) != 0
        assert rgpu_lib.rg_godunov_level(None, 1, 0.1, 0.1) == rgpu.RG_ERR_ARG
    finally:
        rgpu_lib.rg_destroy(h)


def test_tree_and_plan_queries_report_misuse(rgpu_lib):
    """rg_tree_sizes and rg_level_plan_info: a null context is RG_ERR_ARG, a
    context without a tree or without a usable device an error status, a null
    output RG_ERR_ARG -- never a crash."""
    g, n = C.c_int(-7), C.c_int(-7)
    info = rgpu.rg_plan_info()
    assert rgpu_lib.rg_tree_sizes(None, C.byref(g), C.byref(n)) == rgpu.RG_ERR_ARG
    assert rgpu_lib.rg_level_plan_info(None, 1, C.byref(info)) == rgpu.RG_ERR_ARG
    p = rgpu.make_params(3)
    h = rgpu_lib.rg_create(C.byref(p), 0)
    assert h
    try:
        assert rgpu_lib.rg_tree_sizes(h, C.byref(g), C.byref(n)) != rgpu.RG_OK
        assert (g.value, n.value) == (-7, -7)
        assert rgpu_lib.rg_level_plan_info(h, 1, None) != rgpu.RG_OK
        assert rgpu_lib.rg_level_plan_info(h, 1, C.byref(info)) != rgpu.RG_OK
    finally:
        rgpu_lib.rg_destroy(h)
