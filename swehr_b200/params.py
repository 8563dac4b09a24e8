"""ctypes mirror of include/swehr.h (parameters, inputs, progress, budget).

The field order is the C struct order; `swehr_params_size()` in the shared
library is checked against ctypes.sizeof(SwehrParams) at load time.
"""
import ctypes as C

MAX_CLASSES = 16

FIELD_H, FIELD_HU, FIELD_HV, FIELD_Z, FIELD_VINF, FIELD_U, FIELD_M, FIELD_TOTM, \
    FIELD_TOTSED, FIELD_VEL, FIELD_MAXVEL, FIELD_MAXDEPTH, FIELD_DEP, FIELD_SED = range(14)

PER_CLASS_FIELDS = (FIELD_U, FIELD_M, FIELD_SED)

FIELD_NAMES = {
    "h": FIELD_H, "hu": FIELD_HU, "hv": FIELD_HV, "z": FIELD_Z, "vinf": FIELD_VINF,
    "U": FIELD_U, "M": FIELD_M, "totm": FIELD_TOTM, "totsed": FIELD_TOTSED, "vel": FIELD_VEL,
    "maxvel": FIELD_MAXVEL, "maxdepth": FIELD_MAXDEPTH, "dep": FIELD_DEP, "sed": FIELD_SED,
}

STATUS = {0: "ok", 1: "cfl_error", 2: "nan", 3: "timeout", 4: "cuda_error", 5: "invalid",
          6: "oom", 7: "no_device", 8: "busy"}

FP64, MIXED = 0, 1


class SwehrParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("dx", C.c_double), ("F", C.c_double), ("manning0", C.c_double), ("tend", C.c_double),
        ("a", C.c_double), ("ad", C.c_double), ("h0", C.c_double), ("mtstar0", C.c_double),
        ("rnum", C.c_int32), ("sclass", C.c_int32),
        ("rint", C.c_double), ("J", C.c_double),
        ("hcfriction", C.c_double), ("depthdependentexponent", C.c_double), ("b", C.c_double),
        ("af", C.c_double), ("afr", C.c_double),
        ("cstable", C.c_double), ("maxstep", C.c_double),
        ("g", C.c_double), ("hfilm", C.c_double), ("phi", C.c_double), ("rhos", C.c_double),
        ("rhow", C.c_double), ("nu", C.c_double), ("frictionangle", C.c_double),
        ("cohesion", C.c_double), ("lambda_", C.c_double), ("cthreshold", C.c_double),
        ("betabedload", C.c_double),
        ("roughness", C.c_double), ("ks", C.c_double), ("theta0", C.c_double), ("thetas", C.c_double),
        ("hf", C.c_double), ("vinf0", C.c_double), ("uc", C.c_double), ("uc2", C.c_double),
        ("bndry", C.c_int32 * 4), ("inflow", C.c_int32), ("stop_on_nan", C.c_int32),
        ("stageint", C.c_double), ("outlet_row", C.c_int32), ("npoints", C.c_int32),
        ("xpoint", C.c_int32 * 6), ("ypoint", C.c_int32 * 6),
        ("storm_peak", C.c_double), ("storm_radius", C.c_double), ("storm_x0", C.c_double),
        ("storm_y0", C.c_double), ("storm_vx", C.c_double), ("storm_vy", C.c_double),
        ("budget", C.c_int32), ("reserved_i", C.c_int32 * 7), ("reserved_d", C.c_double * 8),
    ]


class SwehrInputs(C.Structure):
    _fields_ = [
        ("topo", C.POINTER(C.c_double)), ("rain", C.POINTER(C.c_double)),
        ("ds", C.POINTER(C.c_double)), ("pfrac", C.POINTER(C.c_double)),
        ("ks", C.POINTER(C.c_double)), ("solid", C.POINTER(C.c_int32)),
    ]


class SwehrProgress(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("courant", C.c_double), ("rain", C.c_double),
        ("steps", C.c_int64), ("steps_this_call", C.c_int64),
        ("device_ms", C.c_double), ("kernel_ms", C.c_double), ("kernel_launches", C.c_int64),
        ("status", C.c_int32), ("done", C.c_int32), ("t_step", C.c_double),
    ]


class SwehrBudget(C.Structure):
    _fields_ = [
        ("water_now", C.c_double), ("water_init", C.c_double),
        ("rain_in", C.c_double), ("outflow", C.c_double), ("clamp_gain", C.c_double),
        ("bulking", C.c_double), ("infiltration", C.c_double), ("water_residual", C.c_double),
        ("sed_now", C.c_double * MAX_CLASSES), ("sed_init", C.c_double * MAX_CLASSES),
        ("detach", C.c_double * MAX_CLASSES), ("sed_outflow", C.c_double * MAX_CLASSES),
        ("sed_residual", C.c_double * MAX_CLASSES),
        ("sclass", C.c_int32), ("valid", C.c_int32),
        ("rounding", C.c_double), ("sed_rounding", C.c_double * MAX_CLASSES),
    ]


class SwehrPoolStats(C.Structure):
    _fields_ = [
        ("resident", C.c_int32), ("running", C.c_int32), ("finished_now", C.c_int32), ("tuned", C.c_int32),
        ("pool_steps", C.c_int64), ("cell_steps", C.c_int64), ("device_ms", C.c_double),
        ("hbm_used", C.c_size_t), ("hbm_limit", C.c_size_t),
        ("grid_wave", C.c_int32), ("grid_update", C.c_int32),
        ("tile_i", C.c_int32), ("tile_j", C.c_int32),
    ]


STATUS_BUSY = 8

# Reference defaults: SWEHR.c:490-494 (friction/splash exponents), 617-650
# (boundaries, stepping, physical constants), 236-246 (soil), 709-715 (points).
REFERENCE_DEFAULTS = dict(
    hcfriction=0.003, depthdependentexponent=-0.33, b=1.0, af=1.0, afr=1.0,
    cstable=0.05, maxstep=0.25,
    g=9.81, hfilm=1e-5, phi=0.4, rhos=2600.0, rhow=1000.0, nu=1.2e-6, frictionangle=0.8693,
    cohesion=400.0, lambda_=0.65, cthreshold=0.4, betabedload=0.5,
    roughness=0.1, ks=0.0, theta0=0.05, thetas=0.4, hf=0.001, vinf0=1e-4, uc=0.0, uc2=0.0,
    bndry=(1, 0, 1, 1), inflow=1, stop_on_nan=0, stageint=1.0, outlet_row=1, npoints=6,
    xpoint=(2, 2, 2, 2, 2, 2), ypoint=(1, 10, 20, 30, 40, 50),
    storm_peak=0.0, storm_radius=1.0, storm_x0=0.0, storm_y0=0.0, storm_vx=0.0, storm_vy=0.0,
    budget=0,
)

INPUT_TXT_ORDER = ("nx", "ny", "dx", "F", "manning0", "tend", "a", "ad", "h0", "mtstar0",
                   "rnum", "rint", "sclass", "J")


def make_params(**kw) -> SwehrParams:
    """A SwehrParams with the reference defaults, updated by keyword."""
    p = SwehrParams()
    vals = dict(REFERENCE_DEFAULTS)
    vals.update(kw)
    for k, v in vals.items():
        if k == "lambda":
            k = "lambda_"
        cur = getattr(p, k)
        if isinstance(cur, C.Array):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(p, k, v)
    return p


def params_dict(p: SwehrParams) -> dict:
    out = {}
    for name, _ in SwehrParams._fields_:
        v = getattr(p, name)
        out[name] = list(v) if isinstance(v, C.Array) else v
    return out
