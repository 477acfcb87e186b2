"""Build the in-tree shared libraries of the B200 TLM step.

``libtlm_b200.so``          the product: C ABI of include/tlm_b200.h
``libtlm_b200_checked.so``  same code with every global index bounds-checked
                            (a violation records a code and skips the access)

Kernels are compiled for sm_100a only, with --fmad=false so that FP32 results
round exactly like the reference's CPU solver. Host math that must match the
reference bit for bit (waveforms, stub tables) is compiled by g++ with
-ffp-contract=off. The CUDA runtime is linked statically, so the libraries
need nothing but the driver at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "-I" + INCLUDE, "-I" + CSRC]
CUDA_SOURCES = ["tlm_solver.cu", "tlm_surface.cu", "fdtd_solver.cu", "tlm_noalloc.cu", "tlm_batch.cu", "tlm_server.cu"]
HOST_SOURCES = ["tlm_host_math.cpp", "emsim_io.cpp"]

LIBS = {
    "libtlm_b200.so": [],
    "libtlm_b200_checked.so": ["-DTLM_CHECKED"],
}


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    return out.stdout + out.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> dict:
    """Compile every library; returns {name: path}. Rebuilds only what changed;
    the compilations run in parallel, one per host core."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    jobs = []                          # (object, command)
    host_objs = []
    for src in HOST_SOURCES:
        obj = os.path.join(BUILD, src.replace(".cpp", ".o"))
        if force or _stale(obj, deps):
            jobs.append((obj, ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-I" + CSRC,
                               "-I" + INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]))
        host_objs.append(obj)
    lib_objs = {}
    for lib, defs in LIBS.items():
        tag = lib.replace(".so", "")
        objs = []
        for src in CUDA_SOURCES:
            obj = os.path.join(BUILD, f"{tag}_{src.replace('.cu', '.o')}")
            if force or _stale(obj, deps):
                flags = list(NVCC_FLAGS) + defs
                if ptxas_info:
                    flags += ["-Xptxas", "-v"]
                jobs.append((obj, [nvcc] + ARCH + flags + ["-c", os.path.join(CSRC, src), "-o", obj]))
            objs.append(obj)
        lib_objs[lib] = objs
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        logs = list(ex.map(lambda j: _run(j[1], verbose), jobs))
    if ptxas_info:
        for log in logs:
            print(log)
    out = {}
    for lib, objs in lib_objs.items():
        target = os.path.join(HERE, lib)
        if force or _stale(target, objs + host_objs):
            _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", target] + objs + host_objs,
                 verbose)
        out[lib] = target
    return out


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
