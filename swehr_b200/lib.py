"""ctypes binding of libswehr.so (the C ABI in include/swehr.h).

The library is loaded from this package directory only; if it is missing
the import fails loudly -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .params import (SwehrParams, SwehrInputs, SwehrProgress, SwehrBudget, FIELD_NAMES, PER_CLASS_FIELDS,
                     STATUS, FP64)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswehr.so")

_lib = None


class SwehrError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"swehr status {status} ({STATUS.get(status, '?')}): {msg}")


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not found: build it with `python -m swehr_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_double
    L.swehr_params_default.argtypes = [vp]
    L.swehr_params_size.restype = C.c_size_t
    L.swehr_abi_version.restype = i32
    L.swehr_status_str.restype = C.c_char_p
    L.swehr_status_str.argtypes = [i32]
    L.swehr_last_error.restype = C.c_char_p
    L.swehr_create.restype = i32
    L.swehr_create.argtypes = [vp, vp, i32, C.POINTER(vp)]
    L.swehr_advance.restype = i32
    L.swehr_advance.argtypes = [vp, dbl, i64, vp]
    L.swehr_read_field.restype = i32
    L.swehr_read_field.argtypes = [vp, i32, i32, vp]
    L.swehr_write_field.restype = i32
    L.swehr_write_field.argtypes = [vp, i32, i32, vp]
    L.swehr_read_series.restype = i32
    L.swehr_read_series.argtypes = [vp, vp, vp, i64, vp]
    L.swehr_get_budget.restype = i32
    L.swehr_get_budget.argtypes = [vp, vp]
    L.swehr_set_timing.restype = i32
    L.swehr_set_timing.argtypes = [vp, i32]
    L.swehr_footprint_bytes.restype = C.c_size_t
    L.swehr_footprint_bytes.argtypes = [i32, i32, i32, i32]
    L.swehr_destroy.argtypes = [vp]
    L.swehr_cfl_noalloc.restype = i32
    L.swehr_cfl_noalloc.argtypes = [vp, vp, vp, vp, vp, i64, dbl, vp, vp]
    if L.swehr_params_size() != C.sizeof(SwehrParams):
        raise ImportError(f"swehr_params size mismatch: C {L.swehr_params_size()} vs ctypes {C.sizeof(SwehrParams)}")
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Simulation:
    """One SWEHR run on the GPU through the C ABI."""

    def __init__(self, case, precision: int = FP64, budget: bool = False):
        self.L = load()
        self.case = case
        self.params = case.make_params()
        if budget:
            self.params.budget = 1
        self._topo = np.ascontiguousarray(case.topo, dtype=np.float64)
        self._rain = np.ascontiguousarray(case.rain, dtype=np.float64)
        self._ds = np.ascontiguousarray(case.ds, dtype=np.float64)
        self._pf = np.ascontiguousarray(case.pfrac, dtype=np.float64)
        self._ks = None if case.ks is None else np.ascontiguousarray(case.ks, dtype=np.float64)
        inp = SwehrInputs(_dptr(self._topo), _dptr(self._rain), _dptr(self._ds), _dptr(self._pf),
                          _dptr(self._ks) if self._ks is not None else None)
        self.ctx = C.c_void_p()
        st = self.L.swehr_create(C.byref(self.params), C.byref(inp), precision, C.byref(self.ctx))
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())

    def advance(self, t_stop: float = float("inf"), max_steps: int = -1) -> SwehrProgress:
        pr = SwehrProgress()
        st = self.L.swehr_advance(self.ctx, t_stop, max_steps, C.byref(pr))
        self.status = st
        if st not in (0, 1, 2):
            raise SwehrError(st, self.L.swehr_last_error().decode())
        return pr

    def set_timing(self, on: bool):
        self.L.swehr_set_timing(self.ctx, 1 if on else 0)

    def field(self, name: str, k: int = 0) -> np.ndarray:
        out = np.empty((self.case.nx, self.case.ny))
        st = self.L.swehr_read_field(self.ctx, FIELD_NAMES[name], k, out.ctypes.data)
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        return out

    def fields(self) -> dict:
        names = ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth", "vel")
        d = {n: self.field(n) for n in names}
        for g in ("U", "M", "sed"):
            d[g] = np.stack([self.field(g, k) for k in range(1, self.case.sclass + 1)])
        return d

    def write_field(self, name: str, arr: np.ndarray, k: int = 0):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        st = self.L.swehr_write_field(self.ctx, FIELD_NAMES[name], k, a.ctypes.data)
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())

    def series(self, max_rows: int = 200000):
        st = np.empty((max_rows, 24))
        sf = np.empty((max_rows, 18))
        rows = C.c_int64()
        r = self.L.swehr_read_series(self.ctx, st.ctypes.data, sf.ctypes.data, max_rows, C.byref(rows))
        if r != 0:
            raise SwehrError(r, self.L.swehr_last_error().decode())
        return st[: rows.value].copy(), sf[: rows.value].copy()

    def budget(self) -> SwehrBudget:
        b = SwehrBudget()
        st = self.L.swehr_get_budget(self.ctx, C.byref(b))
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        return b

    def close(self):
        if getattr(self, "ctx", None):
            self.L.swehr_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
