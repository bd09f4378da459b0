"""Build libofea_gpu.so (sm_100a kernels + C ABI + host I/O) and ofea_cli in-tree.

    python -m openfea_b200.build        # or: python openfea_b200/build.py

nvcc cross-compiles for sm_100a without a GPU.  The CUDA runtime and the C++
runtime are linked statically and their symbols hidden, so the library loads
into any host process (Python, a C++ application) without version clashes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libofea_gpu.so")
CLI = os.path.join(HERE, "ofea_cli")

CU_SOURCES = ["api.cu", "pattern.cu", "integrate.cu", "sell.cu", "precond.cu", "solve.cu", "learned.cu", "batched.cu", "noalloc.cu", "devmem.cu", "ca.cu", "csc.cu", "tc_gemm.cu"]
HOST_SOURCES = ["host/model.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include")]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
    headers += [os.path.join(ROOT, "include", "ofea_gpu.h"), os.path.join(ROOT, "include", "ofea_host.h")]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-fvisibility=hidden", *inc, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    # one nvcc per translation unit, run side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for out in pool.map(_run, jobs):
            if verbose or ptxas_info:
                sys.stdout.write(out)
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", *inc, "-c", s, "-o", o])
    if _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static",
              "-Xcompiler", "-static-libstdc++", "-Xcompiler", "-static-libgcc",
              "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "--no-undefined", "-lrt", "-ldl",
              "-lpthread"])
    cli_src = os.path.join(CSRC, "host", "ofea_cli.cpp")
    if _stale(CLI, [cli_src, LIB]):
        _run(["g++", "-O2", "-std=c++17", *inc, cli_src, "-o", CLI, "-L", HERE, "-lofea_gpu",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
