"""Build libgxcorr.so in-tree (nvcc, sm_100a).

    python -m difx_b200.build            # builds difx_b200/libgxcorr.so

The host C++ is compiled by the system g++ (``-ccbin``) so the library links
the system libstdc++ dynamically, like every other extension loaded into the
Python process.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgxcorr.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["gx_fstep.cu", "gx_fstep_sb.cu", "gx_xstep.cu", "gx_tcxmac.cu", "gx_noalloc.cu", "gx_vis.cu", "gx_api.cpp", "gx_input.cpp",
           "gx_server.cpp", "gx_batch.cpp", "gx_vdifmux.cu", "gx_ring.cu", "gx_monitor.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "gxcorr.h")]
    newest = max(os.path.getmtime(p) for p in deps)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
              "-I" + os.path.join(HERE, "..", "include")]

    def compile_one(s):
        o = os.path.join(BUILD, s + ".o")
        cmd = [nvcc()] + ARCH + common + ["-c", os.path.join(CSRC, s), "-o", o]
        if s.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        return s, o, cmd, subprocess.run(cmd, capture_output=True, text=True)

    # one nvcc per source, in parallel (the F-step source alone takes most of a minute)
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = []
    for s, o, cmd, r in results:
        if verbose:
            print(" ".join(cmd))
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {s}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        objs.append(o)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-ccbin", host_cxx(), "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
