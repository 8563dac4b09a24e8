"""swehr_cfl_noalloc: the CFL time step for callers that cannot allocate
device memory (a framework that owns all allocations through its own pool,
or code running where the allocator is locked).

The entry point allocates nothing; this test plays the caller, which owns
the device buffers (allocated here through the CUDA runtime), and checks the
result against the dt the regular stepping path computes for the same state,
bit for bit (the FP64 tolerance of every parity test here), on two calls in
a row -- the second call shows the shared scratch was left ready for reuse.
"""
import ctypes as C
import os

import numpy as np
import pytest

from swehr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cudart():
    for path in ("/usr/local/cuda/lib64/libcudart.so", "libcudart.so", "libcudart.so.12"):
        try:
            L = C.CDLL(path)
            break
        except OSError:
            continue
    else:
        pytest.skip("libcudart not found")
    L.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    L.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    L.cudaFree.argtypes = [C.c_void_p]
    L.cudaDeviceSynchronize.argtypes = []
    return L


class DeviceBuf:
    def __init__(self, rt, arr: np.ndarray):
        self.rt = rt
        self.nbytes = arr.nbytes
        self.ptr = C.c_void_p()
        assert rt.cudaMalloc(C.byref(self.ptr), self.nbytes) == 0
        assert rt.cudaMemcpy(self.ptr, arr.ctypes.data, self.nbytes, 1) == 0  # host to device

    def read(self, shape):
        out = np.empty(shape)
        assert self.rt.cudaMemcpy(out.ctypes.data, self.ptr, out.nbytes, 2) == 0  # device to host
        return out

    def free(self):
        self.rt.cudaFree(self.ptr)


def _noalloc_dt(L, rt, sim, zprev, t):
    """Call swehr_cfl_noalloc on the simulation's current state."""
    h, hu, hv = (np.ascontiguousarray(sim.field(n)) for n in ("h", "hu", "hv"))
    bufs = [DeviceBuf(rt, a) for a in (h, hu, hv, np.ascontiguousarray(zprev), np.zeros(2))]
    try:
        st = L.swehr_cfl_noalloc(C.byref(sim.params), bufs[0].ptr, bufs[1].ptr, bufs[2].ptr, bufs[3].ptr,
                                 sim.case.ny, t, bufs[4].ptr, None)
        assert st == 0, L.swehr_last_error()
        assert rt.cudaDeviceSynchronize() == 0
        return bufs[4].read((2,))
    finally:
        for b in bufs:
            b.free()


@pytest.mark.parametrize("which", ["fractal", "shipped_inflow", "walls_odd"])
def test_noalloc_cfl_matches_stepping_path_two_calls(which):
    from swehr_b200.lib import Simulation, load
    from harness import load_golden
    L = load()
    rt = _cudart()
    if which == "fractal":
        case = W.fractal_domain(nx=300, ny=170, dx=2.0, steps=100)
        warm = 40
    elif which == "walls_odd":
        # every side a wall, sizes that fill no block or tile evenly
        case = W.fractal_domain(nx=131, ny=77, dx=2.0, steps=100)
        case.params["bndry"] = (1, 1, 1, 1)
        warm = 60
    else:
        case, _ = load_golden("shipped")
        warm = 500
    with Simulation(case) as sim:
        sim.advance(max_steps=warm - 1)
        zprev = sim.field("z")                  # topography of step n-1
        pr = sim.advance(max_steps=1)            # state of step n
        for call in range(2):
            t = pr.t
            res = _noalloc_dt(L, rt, sim, zprev, t)
            zprev = sim.field("z")
            pr = sim.advance(max_steps=1)        # the stepping path's dt for the same state
            assert res[1] == pr.dt, (call, res[1], pr.dt)
            assert res[0] * pr.dt * (1 / case.params["dx"]) == pr.courant, (call, res[0], pr.courant)


def test_noalloc_rejects_oversize_and_bad_arguments():
    from swehr_b200.lib import load
    from swehr_b200.params import make_params
    L = load()
    p = make_params(nx=4097, ny=4096, dx=1.0, tend=10.0, rnum=1, rint=1.0, sclass=1)
    fake = C.c_void_p(16)   # never dereferenced: the size check comes first
    st = L.swehr_cfl_noalloc(C.byref(p), fake, fake, fake, fake, 4096, 0.0, fake, None)
    assert st == 5 and b"SWEHR_NOALLOC_MAX_CELLS" in L.swehr_last_error()
    p = make_params(nx=8, ny=8, dx=1.0, tend=10.0, rnum=1, rint=1.0, sclass=1)
    assert L.swehr_cfl_noalloc(C.byref(p), fake, fake, fake, fake, 4, 0.0, fake, None) == 5   # pitch < ny
    assert L.swehr_cfl_noalloc(C.byref(p), None, fake, fake, fake, 8, 0.0, fake, None) == 5
    # a pitch the kernel's 32-bit row stride cannot hold
    assert L.swehr_cfl_noalloc(C.byref(p), fake, fake, fake, fake, 2 ** 31, 0.0, fake, None) == 5
    assert b"INT32_MAX" in L.swehr_last_error()
