"""Build libswehr.so in-tree with nvcc for sm_100a.

  python -m swehr_b200.build            # builds swehr_b200/libswehr.so
  python -m swehr_b200.build --ptxas-v  # also prints registers / spills per kernel

The FP64 step kernels are compiled with --fmad=false: the plain form must be
bit-identical to the CPU restatement, so no multiply-add may be contracted
(the math bodies in swehr_math.h use explicit fma where they want one).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libswehr.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", os.path.join(HERE, "..", "include")]

# (source, extra flags)
SOURCES = [
    ("swehr_step_f64.cu", ["--fmad=false"]),
    ("swehr_step_f32.cu", []),
    ("swehr_capi.cu", []),
    ("swehr_pool.cu", []),
    ("swehr_cfl_noalloc.cu", ["--fmad=false"]),
    ("swehr_batch16_f64.cu", ["--fmad=false"]),
    ("swehr_batch16_f32.cu", []),
    ("swehr_slab.cu", ["--fmad=false"]),
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs, jobs = [], []
    for src, extra in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        srcp = os.path.join(CSRC, src)
        deps = [srcp] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
        deps.append(os.path.join(HERE, "..", "include", "swehr.h"))
        if not os.path.exists(obj) or any(os.path.getmtime(d) > os.path.getmtime(obj) for d in deps) or ptxas_v:
            cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", srcp, "-o", obj]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            jobs.append((src, cmd))
        objs.append(obj)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: (j[0], subprocess.run(j[1], capture_output=True, text=True)), jobs))
    for src, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if ptxas_v:
            sys.stdout.write(r.stderr)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    build_probe(verbose)
    build_driver(verbose)
    return OUT


PROBE = os.path.join(HERE, "libswehr_probe.so")


def build_probe(verbose: bool = False) -> str:
    """The benchmark's device-peak probe (FP64 pipe ceiling), its own library."""
    src = os.path.join(CSRC, "swehr_probe.cu")
    if os.path.exists(PROBE) and os.path.getmtime(PROBE) >= os.path.getmtime(src):
        return PROBE
    cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", src, "-o", PROBE, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return PROBE


DRIVER = os.path.join(HERE, "swehr_gpu")


def build_driver(verbose: bool = False) -> str:
    """The command-line host (plain C, linked against libswehr.so beside it)."""
    src = os.path.join(CSRC, "swehr_gpu.c")
    cmd = ["gcc", "-O2", "-std=c11", "-D_POSIX_C_SOURCE=200809L", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(HERE, "..", "include"), src, "-o", DRIVER, "-L", HERE, "-lswehr",
           "-Wl,-rpath,$ORIGIN", "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return DRIVER


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_v))


if __name__ == "__main__":
    main()
