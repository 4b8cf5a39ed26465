"""The C-ABI library loads and exports every entry point of include/dacti_gpu.h (no GPU needed)."""
import ctypes
import os
import re

from conftest import ROOT
from dacti_b200 import solver


def declared_functions():
    src = open(os.path.join(ROOT, "include", "dacti_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(dg_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    fns = declared_functions()
    assert "dg_create" in fns and "dg_step" in fns and "dg_destroy" in fns
    assert set(fns) == set(solver.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = solver.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = solver.load_library()
    h = ctypes.c_void_p()
    assert lib.dg_create(None, ctypes.byref(h)) == -1
    assert lib.dg_set_device(-1) == -1
    assert isinstance(lib.dg_last_error(None), bytes)


def test_stage_option_constants_mirror_the_header():
    src = open(os.path.join(ROOT, "include", "dacti_gpu.h")).read()
    vals = dict((k, int(v)) for k, v in re.findall(r"(DG_OPT_(?:ORDERED_LISTS|FACE_TILES))\s*=\s*(\d+)", src))
    assert vals == {"DG_OPT_ORDERED_LISTS": solver.OPT_ORDERED_LISTS, "DG_OPT_FACE_TILES": solver.OPT_FACE_TILES}
    assert solver.OPT_DEFAULT == solver.OPT_ORDERED_LISTS | solver.OPT_FACE_TILES
    lib = solver.load_library()
    assert lib.dg_set_options(None, solver.OPT_DEFAULT) == -1
