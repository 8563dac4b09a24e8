"""What SWEHR.c's main() writes, reproduced from any engine with the C-ABI
shape (advance / field / series): the oracle or the GPU library.

The stepping mirrors SWEHR.c: a movie frame and a console line each time t
reaches the next print time (printint = max(1, tend/1000), SWEHR.c:626-627,
1679-1698; a print time that falls behind gets one step per frame), the ten
result grids and the stage / point series at the end (SWEHR.c:1705-1761).
Grids come back as the reference prints them: rows j, columns i.  Values go
through the reference's text formats (%10.10lf for grids, %lf for series and
console lines), so two engines that agree on every printed digit give equal
arrays here.
"""
import numpy as np

MOVIES = (("topomovie", "z"), ("depthmovie", "h"), ("velocitymovie", "vel"), ("cmovie", "totsed"),
          ("Mmovie", "totm"))
RESULTS = (("topoout", "z", 0), ("depth", "h", 0), ("uh", "hu", 0), ("vh", "hv", 0), ("ch", "U", 1),
           ("m", "totm", 0), ("c", "totsed", 0), ("vel", "vel", 0), ("maxvel", "maxvel", 0),
           ("maxdepth", "maxdepth", 0))


def printed(a, fmt="%10.10f"):
    """Round-trip through the reference's text format."""
    f = np.vectorize(lambda v: float(fmt % v), otypes=[float])
    return f(np.asarray(a, dtype=np.float64))


def grid(a):
    """A nx*ny field (i-major) as printed: rows j, columns i."""
    return printed(np.asarray(a).T)


def run_like_reference(eng, tend: float, movies: bool = True) -> dict:
    printint = max(1.0, tend / 1000.0)
    printinterval = printint
    t, steps = 0.0, 0
    out = {name: [] for name, _ in MOVIES}
    lines = []
    while t < tend:
        if not movies:
            pr = eng.advance()
        elif t >= printinterval:
            pr = eng.advance(max_steps=1)
        else:
            pr = eng.advance(t_stop=printinterval)
        if pr.steps == steps and pr.status == 0:
            break
        t, steps = pr.t, pr.steps
        if movies and t >= printinterval:
            lines.append([float("%f" % v) for v in (t, pr.courant, pr.dt, pr.rain)])
            printinterval += printint
            for name, field in MOVIES:
                out[name].append(grid(eng.field(field)))
        if pr.status != 0:
            break
    res = {name: np.array(v) for name, v in out.items()}
    res["frame_lines"] = np.array(lines)
    for name, field, k in RESULTS:
        res[name] = grid(eng.field(field, k))
    st, sf = eng.series()
    res["stage"] = printed(st, "%f")
    res["saveflow"] = printed(sf, "%f")
    res["steps"] = steps
    return res


def read_table(path):
    with open(path) as f:
        return np.array([[float(v) for v in line.split()] for line in f if line.strip()])


def read_run_dir(wd, ny: int, stdout: str) -> dict:
    """Parse what a run (of swehr_gpu or the reference) left in wd."""
    import os
    res = {}
    for name, _ in MOVIES:
        m = read_table(os.path.join(wd, name + ".txt"))
        res[name] = m.reshape(-1, ny, m.shape[1]) if m.size else np.zeros((0, ny, 0))
    for name, _, _ in RESULTS:
        res[name] = read_table(os.path.join(wd, name + ".txt"))
    res["stage"] = read_table(os.path.join(wd, "stage.txt"))
    res["saveflow"] = read_table(os.path.join(wd, "saveflow.txt"))
    lines = [ln for ln in stdout.splitlines() if ln.count("\t") == 3 and not ln.startswith("Point")]
    res["frame_lines"] = np.array([[float(v) for v in ln.split()] for ln in lines])
    return res


def same(a, b) -> bool:
    """Equal arrays, NaN positions included (the sign of a printed NaN is
    not compared)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and bool(np.array_equal(a, b, equal_nan=True))


def max_diff(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    if a.shape != b.shape or not np.array_equal(np.isnan(a), np.isnan(b)):
        return float("inf")
    m = ~np.isnan(a)
    return float(np.max(np.abs(a[m] - b[m]))) if m.any() else 0.0
