"""ctypes binding of libswehr.so (the C ABI in include/swehr.h).

The library is loaded from this package directory only; if it is missing
the import fails loudly -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .params import (SwehrParams, SwehrInputs, SwehrProgress, SwehrBudget, SwehrPoolStats, FIELD_NAMES,
                     PER_CLASS_FIELDS, STATUS, STATUS_BUSY, FP64)

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
    L.swehr_pool_create.restype = i32
    L.swehr_pool_create.argtypes = [i32, i32, i32, C.c_size_t, i32, C.POINTER(vp)]
    L.swehr_pool_submit.restype = i32
    L.swehr_pool_submit.argtypes = [vp, vp, vp, i64, C.POINTER(i32)]
    L.swehr_pool_run.restype = i32
    L.swehr_pool_run.argtypes = [vp, i64, vp]
    L.swehr_pool_tune.restype = i32
    L.swehr_pool_tune.argtypes = [vp, i64, vp]
    L.swehr_pool_poll.restype = i32
    L.swehr_pool_poll.argtypes = [vp, i32, vp]
    L.swehr_pool_scenario.restype = i32
    L.swehr_pool_scenario.argtypes = [vp, i32, C.POINTER(vp)]
    L.swehr_pool_release.restype = i32
    L.swehr_pool_release.argtypes = [vp, i32]
    L.swehr_pool_stats_get.restype = i32
    L.swehr_pool_stats_get.argtypes = [vp, vp]
    L.swehr_pool_destroy.argtypes = [vp]
    L.swehr_slab_create.restype = i32
    L.swehr_slab_create.argtypes = [vp, vp, i32, i32, i32, C.POINTER(vp)]
    L.swehr_slab_rows.restype = i32
    L.swehr_slab_rows.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    for n in ("swehr_slab_wave", "swehr_slab_update", "swehr_slab_pack", "swehr_slab_unpack"):
        getattr(L, n).restype = i32
        getattr(L, n).argtypes = [vp]
    L.swehr_slab_smax_ptr.restype = i32
    L.swehr_slab_smax_ptr.argtypes = [vp, C.POINTER(vp)]
    L.swehr_slab_buffers.restype = i32
    L.swehr_slab_buffers.argtypes = [vp, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_size_t)]
    L.swehr_slab_stream.restype = i32
    L.swehr_slab_stream.argtypes = [vp, C.POINTER(vp)]
    L.swehr_slab_progress.restype = i32
    L.swehr_slab_progress.argtypes = [vp, vp]
    L.swehr_slab_reduce_local.restype = i32
    L.swehr_slab_reduce_local.argtypes = [C.POINTER(vp), i32]
    L.swehr_slab_copy_halo.restype = i32
    L.swehr_slab_copy_halo.argtypes = [vp, i32, vp]
    if L.swehr_params_size() != C.sizeof(SwehrParams):
        raise ImportError(f"swehr_params size mismatch: C {L.swehr_params_size()} vs ctypes {C.sizeof(SwehrParams)}")
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class CaseInputs:
    """A case's parameters and input arrays held in C layout (kept alive as
    long as the C side may read them)."""

    def __init__(self, case, budget: bool = False):
        self.params = case.make_params()
        if budget:
            self.params.budget = 1
        self._topo = np.ascontiguousarray(case.topo, dtype=np.float64)
        self._rain = np.ascontiguousarray(case.rain, dtype=np.float64)
        self._ds = np.ascontiguousarray(case.ds, dtype=np.float64)
        self._pf = np.ascontiguousarray(case.pfrac, dtype=np.float64)
        self._ks = None if case.ks is None else np.ascontiguousarray(case.ks, dtype=np.float64)
        solid = getattr(case, "solid", None)
        self._solid = None if solid is None else np.ascontiguousarray(solid, dtype=np.int32)
        self.inputs = SwehrInputs(_dptr(self._topo), _dptr(self._rain), _dptr(self._ds), _dptr(self._pf),
                                  _dptr(self._ks) if self._ks is not None else None,
                                  self._solid.ctypes.data_as(C.POINTER(C.c_int32)) if self._solid is not None
                                  else None)

    @property
    def host_bytes(self) -> int:
        n = self._topo.nbytes + self._rain.nbytes + self._ds.nbytes + self._pf.nbytes
        n += self._solid.nbytes if self._solid is not None else 0
        return n + (self._ks.nbytes if self._ks is not None else 0)


class _Reader:
    """Field, series and budget reads of one context handle."""

    def _check(self, st):
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())

    def field(self, name: str, k: int = 0) -> np.ndarray:
        out = np.empty((self.case.nx, self.case.ny))
        self._check(self.L.swehr_read_field(self.ctx, FIELD_NAMES[name], k, out.ctypes.data))
        return out

    def fields(self, names=None) -> dict:
        if names is None:
            names = ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth", "vel",
                     "U", "M", "sed")
        d = {}
        for n in names:
            if FIELD_NAMES[n] in PER_CLASS_FIELDS:
                # each class read straight into its slice: no stacking copy
                out = np.empty((self.case.sclass, self.case.nx, self.case.ny))
                for k in range(1, self.case.sclass + 1):
                    self._check(self.L.swehr_read_field(self.ctx, FIELD_NAMES[n], k, out[k - 1].ctypes.data))
                d[n] = out
            else:
                d[n] = self.field(n)
        return d

    def series(self, max_rows: int = 200000):
        st = np.empty((max_rows, 24))
        sf = np.empty((max_rows, 18))
        rows = C.c_int64()
        self._check(self.L.swehr_read_series(self.ctx, st.ctypes.data, sf.ctypes.data, max_rows, C.byref(rows)))
        return st[: rows.value].copy(), sf[: rows.value].copy()

    def budget(self) -> SwehrBudget:
        b = SwehrBudget()
        self._check(self.L.swehr_get_budget(self.ctx, C.byref(b)))
        return b


class Simulation(_Reader):
    """One SWEHR run on the GPU through the C ABI."""

    def __init__(self, case, precision: int = FP64, budget: bool = False):
        self.L = load()
        self.case = case
        self._in = CaseInputs(case, budget)
        self.params = self._in.params
        self.ctx = C.c_void_p()
        st = self.L.swehr_create(C.byref(self.params), C.byref(self._in.inputs), precision, C.byref(self.ctx))
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

    def write_field(self, name: str, arr: np.ndarray, k: int = 0):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        st = self.L.swehr_write_field(self.ctx, FIELD_NAMES[name], k, a.ctypes.data)
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())

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


class PoolScenario(_Reader):
    """A scenario resident in a Pool (reads only; the pool steps it)."""

    def __init__(self, pool, sid: int, case, inputs: CaseInputs):
        self.L = pool.L
        self.pool = pool
        self.id = sid
        self.case = case
        self._in = inputs
        self.ctx = C.c_void_p()
        self._check(self.L.swehr_pool_scenario(pool.handle, sid, C.byref(self.ctx)))

    def progress(self) -> SwehrProgress:
        pr = SwehrProgress()
        self._check(self.L.swehr_pool_poll(self.pool.handle, self.id, C.byref(pr)))
        return pr


class Pool:
    """Many scenarios stepped by shared persistent launches (swehr_pool_*)."""

    def __init__(self, precision: int = FP64, max_classes: int = 16, budget: bool = False, hbm_limit: int = 0,
                 max_scenarios: int = 4096):
        self.L = load()
        self.budget_on = budget
        self.handle = C.c_void_p()
        st = self.L.swehr_pool_create(precision, max_classes, 1 if budget else 0, hbm_limit, max_scenarios,
                                      C.byref(self.handle))
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        self.scenarios = {}

    def submit(self, case, max_steps: int = -1, budget: bool = False):
        """The new PoolScenario, or None when the pool is full right now."""
        inp = CaseInputs(case, budget)
        sid = C.c_int()
        st = self.L.swehr_pool_submit(self.handle, C.byref(inp.params), C.byref(inp.inputs), max_steps,
                                      C.byref(sid))
        if st == STATUS_BUSY:
            return None
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        sc = PoolScenario(self, sid.value, case, inp)
        self.scenarios[sid.value] = sc
        return sc

    def run(self, steps: int = -1) -> SwehrPoolStats:
        s = SwehrPoolStats()
        st = self.L.swehr_pool_run(self.handle, steps, C.byref(s))
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        return s

    def tune(self, steps_per_trial: int = 8) -> SwehrPoolStats:
        s = SwehrPoolStats()
        st = self.L.swehr_pool_tune(self.handle, steps_per_trial, C.byref(s))
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        return s

    def stats(self) -> SwehrPoolStats:
        s = SwehrPoolStats()
        self.L.swehr_pool_stats_get(self.handle, C.byref(s))
        return s

    def release(self, sc):
        st = self.L.swehr_pool_release(self.handle, sc.id)
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())
        self.scenarios.pop(sc.id, None)

    def close(self):
        if getattr(self, "handle", None):
            self.L.swehr_pool_destroy(self.handle)
            self.handle = None
            self.scenarios = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SlabDomain:
    """One domain split into slabs of whole rows (swehr_slab_*), every slab
    driven by this process: a step is the wave pass of every slab, the
    largest wave speed over all of them, every slab's update, and the halo
    rows moved between neighbours by device copies (peer copies when the
    slabs sit on different devices).  devices: the device of each slab
    (default: the current one for all)."""

    def __init__(self, case, slabs: int, precision: int = FP64, devices=None):
        from .slabs import plan
        self.L = load()
        self.case = case
        self._in = CaseInputs(case, False)
        self.plan = plan(case.nx, slabs)
        self.ctx = []
        self.rows = []
        torch = None
        if devices is not None:
            import torch                     # device selection only
            cur = torch.cuda.current_device()
        try:
            for k, s in enumerate(self.plan):
                if torch is not None:
                    torch.cuda.set_device(devices[k])
                c = C.c_void_p()
                self._check(self.L.swehr_slab_create(C.byref(self._in.params), C.byref(self._in.inputs), precision,
                                                     s.own[0], s.own[1], C.byref(c)))
                self.ctx.append(c)
                lo, own, hi = C.c_int(), C.c_int(), C.c_int()
                self._check(self.L.swehr_slab_rows(c, C.byref(lo), C.byref(own), C.byref(hi)))
                self.rows.append((lo.value, own.value, hi.value))
        finally:
            if torch is not None:
                torch.cuda.set_device(cur)
        self._arr = (C.c_void_p * len(self.ctx))(*[c.value for c in self.ctx])

    def _check(self, st):
        if st != 0:
            raise SwehrError(st, self.L.swehr_last_error().decode())

    def step(self, n: int = 1):
        L, ctx = self.L, self.ctx
        for _ in range(n):
            for c in ctx:
                self._check(L.swehr_slab_wave(c))
            self._check(L.swehr_slab_reduce_local(self._arr, len(ctx)))
            for c in ctx:
                self._check(L.swehr_slab_update(c))
                self._check(L.swehr_slab_pack(c))
            for a, b in zip(ctx, ctx[1:]):
                self._check(L.swehr_slab_copy_halo(a, 1, b))     # a's last own rows -> b's upper halo
                self._check(L.swehr_slab_copy_halo(b, 0, a))     # b's first own rows -> a's lower halo
            for c in ctx:
                self._check(L.swehr_slab_unpack(c))

    def progress(self) -> SwehrProgress:
        pr = SwehrProgress()
        for c in self.ctx:
            self._check(self.L.swehr_slab_progress(c, C.byref(pr)))
        return pr

    def field(self, name: str, k: int = 0) -> np.ndarray:
        """the whole domain's field, each slab's own rows"""
        parts = []
        for c, (lo, own, hi) in zip(self.ctx, self.rows):
            out = np.empty((lo + own + hi, self.case.ny))
            self._check(self.L.swehr_read_field(c, FIELD_NAMES[name], k, out.ctypes.data))
            parts.append(out[lo:lo + own])
        return np.concatenate(parts, axis=0)

    def fields(self, names) -> dict:
        d = {}
        for n in names:
            if FIELD_NAMES[n] in PER_CLASS_FIELDS:
                d[n] = np.stack([self.field(n, k) for k in range(1, self.case.sclass + 1)])
            else:
                d[n] = self.field(n)
        return d

    def close(self):
        for c in self.ctx:
            if c:
                self.L.swehr_destroy(c)
        self.ctx = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
