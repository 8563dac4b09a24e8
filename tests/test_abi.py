"""The C ABI library loads and exports everything include/*.h declares;
host-side argument checking works without a GPU (no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from swehr_b200 import lib as swlib
from swehr_b200.params import SwehrParams, SwehrInputs, make_params, params_dict, REFERENCE_DEFAULTS
from swehr_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b(swehr_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = swlib.load()
    decl = declared_functions()
    assert len(decl) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", swlib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in decl if n not in exported]
    assert not missing, missing
    for n in decl:
        getattr(L, n)


def test_params_struct_and_defaults_match_reference():
    L = swlib.load()
    assert L.swehr_params_size() == C.sizeof(SwehrParams)
    assert L.swehr_abi_version() == 2
    p = SwehrParams()
    L.swehr_params_default(C.byref(p))
    d = params_dict(p)
    for k, v in REFERENCE_DEFAULTS.items():
        got = d["lambda_" if k == "lambda" else k]
        assert (list(got) == list(v)) if isinstance(v, (tuple, list)) else got == v, k


def test_status_strings():
    L = swlib.load()
    for s in range(9):
        assert L.swehr_status_str(s)
    assert b"CFL" in L.swehr_status_str(1)


def _inputs(case):
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (case.topo, case.rain, case.ds, case.pfrac)]
    ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
    return arrs, SwehrInputs(ptr[0], ptr[1], ptr[2], ptr[3], None)


@pytest.mark.parametrize("bad", [dict(nx=1), dict(sclass=0), dict(sclass=17), dict(rnum=0), dict(dx=0.0),
                                 dict(bndry=(2, 0, 0, 0)), dict(outlet_row=99)])
def test_create_rejects_bad_parameters(bad):
    L = swlib.load()
    case = W.tiny_case()
    kw = dict(case.params)
    kw.update(bad)
    p = make_params(**kw)
    keep, inp = _inputs(case)
    ctx = C.c_void_p()
    st = L.swehr_create(C.byref(p), C.byref(inp), 0, C.byref(ctx))
    assert st == 5 and not ctx.value
    assert L.swehr_last_error()


def test_create_without_device_or_with_bad_precision():
    L = swlib.load()
    case = W.tiny_case()
    p = case.make_params()
    keep, inp = _inputs(case)
    ctx = C.c_void_p()
    st = L.swehr_create(C.byref(p), C.byref(inp), 7, C.byref(ctx))
    assert st == 5
    st = L.swehr_create(C.byref(p), C.byref(inp), 0, C.byref(ctx))
    if st == 0:
        L.swehr_destroy(ctx)
    else:
        assert st == 7, L.swehr_last_error()


def test_null_arguments():
    L = swlib.load()
    assert L.swehr_advance(None, 1.0, 1, None) == 5
    assert L.swehr_read_field(None, 0, 0, None) == 5
    assert L.swehr_get_budget(None, None) == 5
    L.swehr_destroy(None)


def test_footprint_scales_with_cells_and_classes():
    L = swlib.load()
    a = L.swehr_footprint_bytes(4096, 4096, 7, 0)
    b = L.swehr_footprint_bytes(8192, 8192, 10, 0)
    assert 6e9 < a < 8e9
    assert b > 3.5 * a


def test_pool_entry_points_check_arguments_without_device():
    L = swlib.load()
    h = C.c_void_p()
    assert L.swehr_pool_create(7, 4, 0, 0, 8, C.byref(h)) == 5          # unknown precision
    assert L.swehr_pool_create(0, 0, 0, 0, 8, C.byref(h)) == 5          # max_classes
    assert L.swehr_pool_create(0, 4, 0, 0, 0, C.byref(h)) == 5          # max_scenarios
    assert L.swehr_pool_run(None, 1, None) == 5
    assert L.swehr_pool_release(None, 1) == 5
    L.swehr_pool_destroy(None)
    if not _has_device():
        assert L.swehr_pool_create(0, 4, 0, 0, 8, C.byref(h)) == 7      # no device
        assert not h.value


def _has_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_slab_entry_points_check_arguments_without_device():
    """Slab rows, budgets and solid masks are refused before any device call."""
    L = swlib.load()
    from swehr_b200.lib import CaseInputs
    case = W.tiny_case(nx=20, ny=9)
    inp = CaseInputs(case)
    h = C.c_void_p()
    for lo, hi in ((0, 5), (3, 21), (4, 4), (2, 10), (1, 19)):
        # outside 1..nx, a single row, or a neighbour left with one row
        assert L.swehr_slab_create(C.byref(inp.params), C.byref(inp.inputs), 0, lo, hi, C.byref(h)) == 5, (lo, hi)
        assert not h.value
    inb = CaseInputs(case, budget=True)
    assert L.swehr_slab_create(C.byref(inb.params), C.byref(inb.inputs), 0, 1, 10, C.byref(h)) == 5
    for f in ("swehr_slab_wave", "swehr_slab_update", "swehr_slab_pack", "swehr_slab_unpack"):
        assert getattr(L, f)(None) == 5
    assert L.swehr_slab_copy_halo(None, 0, None) == 5
    assert L.swehr_slab_reduce_local(None, 0) == 5
