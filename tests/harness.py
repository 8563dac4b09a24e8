"""Test-side drivers: the CPU oracle (oracle/_build/*.so), the reference
program built from SWEHR.c (oracle/_ref/), and the product library, all fed
from the same swehr_b200.workloads.Case.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

from swehr_b200 import io as swio
from swehr_b200.params import (SwehrInputs, SwehrProgress, SwehrBudget, FIELD_NAMES, PER_CLASS_FIELDS)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_BUILD = os.path.join(ORACLE_DIR, "_build")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

STATE_FIELDS = ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth")
CLASS_FIELDS = ("U", "M", "sed")


def build_oracle() -> None:
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _Inputs:
    """Keeps the numpy arrays alive while C holds pointers to them."""

    def __init__(self, case):
        self.topo = np.ascontiguousarray(case.topo, dtype=np.float64)
        self.rain = np.ascontiguousarray(case.rain, dtype=np.float64)
        self.ds = np.ascontiguousarray(case.ds, dtype=np.float64)
        self.pf = np.ascontiguousarray(case.pfrac, dtype=np.float64)
        self.ks = None if case.ks is None else np.ascontiguousarray(case.ks, dtype=np.float64)
        solid = getattr(case, "solid", None)
        self.solid = None if solid is None else np.ascontiguousarray(solid, dtype=np.int32)
        self.s = SwehrInputs(_dptr(self.topo), _dptr(self.rain), _dptr(self.ds), _dptr(self.pf),
                             _dptr(self.ks) if self.ks is not None else None,
                             self.solid.ctypes.data_as(C.POINTER(C.c_int32)) if self.solid is not None else None)


class OracleRun:
    """One simulation on the CPU restatement.  variant: 'shim' (project math,
    the GPU's bit-exact twin) or 'glibc' (libm, the reference's twin)."""

    _libs = {}

    @classmethod
    def lib(cls, variant: str):
        if variant not in cls._libs:
            path = os.path.join(ORACLE_BUILD, f"liborc_{variant}.so")
            if not os.path.exists(path):
                build_oracle()
            L = C.CDLL(path)
            L.orc_create.restype = C.c_void_p
            L.orc_create.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_advance.restype = C.c_int
            L.orc_advance.argtypes = [C.c_void_p, C.c_double, C.c_int64, C.c_void_p]
            L.orc_read_field.restype = C.c_int
            L.orc_read_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            L.orc_read_series.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
            L.orc_get_budget.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_destroy.argtypes = [C.c_void_p]
            L.orc_time.restype = C.c_double
            L.orc_time.argtypes = [C.c_void_p]
            L.orc_steps.restype = C.c_int64
            L.orc_steps.argtypes = [C.c_void_p]
            L.orc_threads.restype = C.c_int
            L.orc_counter.restype = C.c_int64
            L.orc_counter.argtypes = [C.c_void_p, C.c_int]
            for fn in ("orc_m_pow",):
                getattr(L, fn).restype = C.c_double
                getattr(L, fn).argtypes = [C.c_double, C.c_double]
            for fn in ("orc_m_powh", "orc_m_exp", "orc_m_cosatan", "orc_m_sinatan"):
                getattr(L, fn).restype = C.c_double
                getattr(L, fn).argtypes = [C.c_double]
            cls._libs[variant] = L
        return cls._libs[variant]

    def __init__(self, case, variant: str = "shim"):
        self.case = case
        self.L = self.lib(variant)
        self.params = case.make_params()
        self.inp = _Inputs(case)
        self.ctx = self.L.orc_create(C.byref(self.params), C.byref(self.inp.s))
        if not self.ctx:
            raise ValueError("orc_create rejected the case")

    def advance(self, t_stop: float = float("inf"), max_steps: int = -1) -> SwehrProgress:
        pr = SwehrProgress()
        self.status = self.L.orc_advance(self.ctx, t_stop, max_steps, C.byref(pr))
        return pr

    @property
    def t(self):
        return self.L.orc_time(self.ctx)

    @property
    def steps(self):
        return self.L.orc_steps(self.ctx)

    def counters(self) -> dict:
        """Cell-steps so far that took a rare branch: slope failure, debris
        forcing (DFMASK > 0), the debris-flow override of every source."""
        return {n: int(self.L.orc_counter(self.ctx, k)) for k, n in enumerate(("fail", "dfmask", "debris"))}

    def field(self, name: str, k: int = 0) -> np.ndarray:
        out = np.empty((self.case.nx, self.case.ny))
        st = self.L.orc_read_field(self.ctx, FIELD_NAMES[name], k, out.ctypes.data)
        assert st == 0
        return out

    def fields(self) -> dict:
        d = {n: self.field(n) for n in STATE_FIELDS}
        d["vel"] = self.field("vel")
        for g in CLASS_FIELDS:
            d[g] = np.stack([self.field(g, k) for k in range(1, self.case.sclass + 1)])
        return d

    def series(self, max_rows: int = 200000):
        st = np.empty((max_rows, 24))
        sf = np.empty((max_rows, 18))
        rows = C.c_int64()
        self.L.orc_read_series(self.ctx, st.ctypes.data, sf.ctypes.data, max_rows, C.byref(rows))
        return st[: rows.value].copy(), sf[: rows.value].copy()

    def budget(self) -> SwehrBudget:
        b = SwehrBudget()
        self.L.orc_get_budget(self.ctx, C.byref(b))
        return b

    def close(self):
        if self.ctx:
            self.L.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_binary(omp: bool = False) -> str:
    return os.path.join(REF_DIR, "swehr_ref_omp" if omp else "swehr_ref")


def have_reference_binary() -> bool:
    return os.path.exists(ref_binary(False))


def run_reference(case, max_steps: int = -1, omp: bool = False, threads: int = 1, workdir: str = None,
                  dump: bool = True, timeout: float = 3600.0):
    """Run the reference program (built from SWEHR.c) on a Case; returns
    (parsed swehr_dump.txt or None, stdout)."""
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="swehr_ref_")
    swio.write_inputs(case, wd)
    swio.write_ref_cfg(case, wd, max_steps=max_steps, movies=0)
    if not dump:
        with open(os.path.join(wd, "swehr_ref.cfg"), "a") as f:
            f.write("dump 0\n")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([ref_binary(omp)], cwd=wd, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr[-2000:]}")
    out = swio.read_ref_dump(os.path.join(wd, "swehr_dump.txt")) if dump else None
    if own:
        import shutil
        shutil.rmtree(wd, ignore_errors=True)
    return out, r.stdout


def compare(a: dict, b: dict, names=STATE_FIELDS + CLASS_FIELDS) -> dict:
    """Per-field relative L-infinity difference, NaN-position aware:
    returns {name: (rel_linf, nan_positions_equal, bit_equal)}."""
    out = {}
    for n in names:
        x, y = np.asarray(a[n]), np.asarray(b[n])
        nx_, ny_ = np.isnan(x), np.isnan(y)
        same_nan = bool(np.array_equal(nx_, ny_))
        m = ~(nx_ | ny_)
        scale = np.max(np.abs(y[m])) if m.any() else 0.0
        diff = np.max(np.abs(x[m] - y[m])) if m.any() else 0.0
        rel = diff / scale if scale > 0 else diff
        bit = same_nan and bool(np.array_equal(x[m], y[m]))
        out[n] = (float(rel), same_nan, bit)
    return out


GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def load_golden(name: str):
    """(Case, {tag: {field: array}}) from tests/golden/<name>.npz."""
    import json
    from swehr_b200.workloads import Case
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"), allow_pickle=False)
    params = json.loads(str(z["params_json"]))
    if "bndry" in params:
        params["bndry"] = tuple(params["bndry"])
    case = Case(str(z["name"]), params, z["topo"], z["rain"], z["ds"], z["pfrac"],
                ks=z["ks"] if "ks" in z.files else None, solid=z["solid"] if "solid" in z.files else None)
    dumps = {}
    for key in z.files:
        if "__" in key:
            tag, f = key.split("__", 1)
            dumps.setdefault(tag, {})[f] = z[key]
    for d in dumps.values():
        d["steps"] = int(d["steps"])
        d["t"] = float(d["t"])
    return case, dumps
