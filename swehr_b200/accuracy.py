"""Error measures of the mixed form against the plain FP64 form.

rel_linf: relative L-infinity difference of two fields, NaN-position aware.
quantized_case: the case with every real input the mixed form holds in FP32
rounded to FP32 (z, Green-Ampt and time stepping stay FP64, as in the mixed
form).  Running the plain FP64 form on it measures how far an FP32
representation of the inputs alone moves the result -- the envelope against
which the mixed form's own error is read, since SWEHR's wet/dry, shallow-flow
and deposition thresholds amplify last-bit differences over many steps.
"""
from __future__ import annotations

import numpy as np

from . import workloads as W
from .params import REFERENCE_DEFAULTS

# parameters the mixed form keeps in FP64 (time stepping, Green-Ampt, storm track)
KEEP64 = {"dx", "tend", "rint", "stageint", "thetas", "theta0", "hf", "ks", "vinf0", "cstable", "maxstep",
          "storm_peak", "storm_radius", "storm_x0", "storm_y0", "storm_vx", "storm_vy"}


class EmptyField(ValueError):
    """The reference field of an error measure is identically zero (or all
    NaN): a relative error of it says nothing."""


def rel_linf(a, b, require_nonzero: bool = False) -> float:
    """max |a - b| / max |b| over positions finite in both (inf if the NaN
    positions differ).  When b is zero everywhere the absolute difference is
    returned -- unless require_nonzero, which raises EmptyField instead, so
    a comparison of two empty fields cannot pass for an accuracy result."""
    a, b = np.asarray(a), np.asarray(b)
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return float("inf")
    m = ~na
    if not m.any():
        if require_nonzero:
            raise EmptyField("no finite values to compare")
        return 0.0
    scale = float(np.max(np.abs(b[m])))
    diff = float(np.max(np.abs(a[m] - b[m])))
    if scale == 0 and require_nonzero:
        raise EmptyField("reference field is zero everywhere")
    return diff / scale if scale > 0 else diff


def _f32(x):
    return float(np.float32(x))


def quantized_case(case: W.Case) -> W.Case:
    p = dict(REFERENCE_DEFAULTS)
    p.update(case.params)
    for k, v in list(p.items()):
        if isinstance(v, float) and k not in KEEP64:
            p[k] = _f32(v)
    q = lambda a: None if a is None else np.asarray(a).astype(np.float32).astype(np.float64)  # noqa: E731
    return W.Case(case.name + "_q32", p, case.topo, q(case.rain), q(case.ds), q(case.pfrac), ks=q(case.ks),
                  max_steps=case.max_steps)
