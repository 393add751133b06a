"""Build recipe of the B200 backend: ``xpulse_recon_b200/lib/libxpr.so`` and the
``xprecon`` command-line tool (drop-in for the reference's ``XPRecon``).

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
host C++ sources with g++.  Floating-point contraction is disabled everywhere
(``--fmad=false`` / ``-ffp-contract=off``): the projector's arithmetic contracts
are written operation by operation and must not be re-associated or fused.
The CUDA runtime is linked statically so the library does not depend on the
runtime version a host process (e.g. PyTorch) brings.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "lib")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(OUT, "libxpr.so")
CLI = os.path.join(OUT, "xprecon")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-Wall",
             "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I/usr/local/cuda/include"]


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("build step failed: %s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return p.stdout + p.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    hdr = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                 glob.glob(os.path.join(CSRC, "host", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h")))
    return cu, cpp, hdr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp, hdr = sources()
    objs = []
    log = []
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src, __file__] + hdr):
            log.append(_run([NVCC, *ARCH, *NVCC_FLAGS, "-Xptxas", "-v", "-c", src, "-o", obj]))
        objs.append(obj)
    host_objs = []
    for src in cpp:
        obj = os.path.join(BUILD, "host_" + os.path.basename(src) + ".o")
        if force or _stale(obj, [src, __file__] + hdr):
            _run(["g++", *CXX_FLAGS, "-c", src, "-o", obj])
        if os.path.basename(src) == "cli_main.cpp":
            continue
        host_objs.append(obj)
    if force or _stale(LIB, objs + host_objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, *host_objs,
              "-Xcompiler", "-fopenmp", "-lgomp"])
    cli_obj = os.path.join(BUILD, "host_cli_main.cpp.o")
    if os.path.exists(cli_obj) and (force or _stale(CLI, [cli_obj, LIB])):
        _run(["g++", "-o", CLI, cli_obj, "-L" + OUT, "-lxpr", "-Wl,-rpath,$ORIGIN", "-fopenmp"])
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
