"""Builds the native libraries of capaz_b200 in-tree (capaz_b200/lib/).

    python -m capaz_b200.build [--force] [--verbose]

- libcapaz_b200.so       the C ABI (include/capaz_b200.h) and every CUDA kernel,
                         compiled for sm_100a only;
- libcapaz_dropin_2ph.so the reference's two-phase arch-backend call surface
                         (include/capaz_refabi.h) over that C ABI.

Kernels whose results must match the reference bit for bit are compiled with
-fmad=false (no FMA contraction), the others with the default contraction.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "lib", "obj")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]

# (source, extra flags).  Order is the link order.
CUDA_SOURCES = [
    ("step2_fp64.cu", ["-fmad=false"]),
    ("step2_fp32c.cu", []),
    ("step2_fp32c_tma.cu", []),
    ("step3_fp64.cu", ["-fmad=false"]),
    ("step3_fp32c.cu", []),
    ("step3_fp32c_tma.cu", []),
    ("step_bl.cu", ["-fmad=false"]),
    ("step3e.cu", ["-fmad=false"]),
    ("fields.cu", []),
    ("capaz_api.cu", []),
    ("capaz_run.cu", []),
    ("batch.cu", []),
    ("adjoint.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("io.cu", []),
    ("media.cu", []),
    ("slab.cu", []),
]
HEADERS = ["capaz_internal.h", "capaz_ctx.h", "phys3.cuh", "phys3f.cuh", "diag_reduce.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> dict:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "capaz_b200.h")]
    objs = []
    for src, extra in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s, __file__] + hdrs):
            flags = list(extra)
            if ptxas_verbose:
                flags += ["-Xptxas", "-v"]
            _run([NVCC] + NVFLAGS + flags + ["-c", s, "-o", o], verbose)
    lib = os.path.join(LIB, "libcapaz_b200.so")
    if force or _newer(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-cudart", "static"], verbose)

    out = {"libcapaz_b200": lib}
    dsrc = os.path.join(CSRC, "dropin.cpp")
    if os.path.exists(dsrc):
        dh = [os.path.join(INCLUDE, "capaz_refabi.h"), os.path.join(INCLUDE, "capaz_b200.h")]
        cuda = os.path.dirname(os.path.dirname(NVCC))
        for tag, defs in (("2ph", []), ("3ph", ["-DCAPAZ_REFABI_THREE_PHASE"])):
            dlib = os.path.join(LIB, f"libcapaz_dropin_{tag}.so")
            if force or _newer(dlib, [dsrc, lib] + dh):
                _run([CXX, "-O2", "-fPIC", "-shared", "-std=c++17"] + defs +
                     ["-I" + INCLUDE, "-I" + os.path.join(cuda, "include"), dsrc, "-o", dlib, "-L" + LIB,
                      "-lcapaz_b200", "-L" + os.path.join(cuda, "lib64"), "-lcudart_static", "-ldl", "-lrt",
                      "-lpthread", "-Wl,-rpath,$ORIGIN"], verbose)
            out[f"libcapaz_dropin_{tag}"] = dlib
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill report")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))


if __name__ == "__main__":
    main()
