"""The C ABI: the library loads without a GPU and exports every function the header declares."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import fmm_b200 as F

HEADER = Path(__file__).resolve().parent.parent / "include" / "fmm_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(fmmgpu_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    assert "fmmgpu_fmm_build" in names and "fmmgpu_fmm_evaluate" in names and len(names) >= 15


def test_library_exports_every_declared_function():
    lib = C.CDLL(F._LIBPATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_function():
    lib = F.lib()
    for name in declared_functions():
        assert getattr(lib, name).restype is not None or name in ("fmmgpu_default_settings", "fmmgpu_fmm_destroy"), name


def test_direct_sum_argument_errors_reach_last_error():
    lib = F.lib()
    rc = lib.fmmgpu_direct_sum(4, None, None, 1, None, None, None, 0)
    assert rc == 1
    assert b"null buffer" in lib.fmmgpu_last_error()


def test_level_calls_need_an_evaluator():
    """A plan-only handle (no GPU needed) answers the level calls with an argument error."""
    x = np.random.default_rng(0).uniform(size=(500, 3))
    plan = F.FmmBuilder(3).max_points_per_leaf(16).plan(x)
    lib = F.lib()
    assert lib.fmmgpu_op_p2m(plan._h, 0) == 1
    assert b"plan-only" in lib.fmmgpu_last_error()
    assert lib.fmmgpu_op_begin_evaluation(plan._h, None) == 1


def _struct_fields(name):
    """(type, field) pairs of the header's `typedef struct { ... } name;`, in order."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = re.search(r"typedef struct \{([^}]*)\}\s*" + name + r";", text).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        if decl.startswith("const char*"):
            ctype, names = "const char*", decl[len("const char*"):]
        else:
            ctype, names = decl.split(None, 1)
        out += [(ctype, n.strip()) for n in names.split(",")]
    return out


@pytest.mark.parametrize("cname,pystruct", [("fmmgpu_settings", F.Settings), ("fmmgpu_info", F.Info)])
def test_python_structs_mirror_the_header(cname, pystruct):
    """The ctypes mirrors of the header's structs: the same fields in the same order with
    the same widths, so the library and the binding agree on the layout."""
    width = {"int": C.c_int, "int64_t": C.c_int64, "const char*": C.c_char_p}
    fields = _struct_fields(cname)
    assert [n for _, n in fields] == [n for n, _ in pystruct._fields_]
    for (ctype, n), (pn, pt) in zip(fields, pystruct._fields_):
        assert C.sizeof(width[ctype]) == C.sizeof(pt), (n, ctype, pt)
