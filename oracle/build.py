#!/usr/bin/env python3
"""Build recipe for the CPU oracle (test infrastructure only).

Two libraries are produced:

* ``oracle/_build/libxpr_oracle.so`` -- the C restatement in ``xpr_oracle.c``.
* ``oracle/_ref/libxpr_ref.so`` -- the reference's own OpenCL kernel sources
  (``src/reconstruction/gpu/kernels/Kernel*.cl`` of ebarjou/xpulse_recon),
  compiled for the CPU through ``ref_shim.hpp``.
* ``oracle/_ref/libxpr_ref_relaxed.so`` -- the same generated sources compiled with
  relaxed floating point (``-ffast-math -mfma``: contraction into fma, reassociation,
  reciprocal division, no signed zeros), a CPU stand-in for the reference's own build
  flags (src/reconstruction/gpu/kernel.hpp:26-30 builds every program with
  ``-cl-fast-relaxed-math -cl-mad-enable -cl-no-signed-zeros
  -cl-unsafe-math-optimizations -cl-finite-math-only``).  It measures how far a legitimate relaxed compilation of the
  reference lands from its IEEE interpretation.  The sources are read where
  they lie in the reference checkout; only generated, git-ignored files are
  written under ``oracle/_ref/``.  The pre-pass is textual and mechanical:

  1. inline ``#include "utils.cl"`` / ``#include "constants.cl"`` exactly as the
     reference's CMakeLists.txt:3-15 does before handing the text to OpenCL;
  2. take the OpenCL branch of constants.cl:8-14 (its ``__cplusplus`` branch
     redefines float4 for host code);
  3. rewrite OpenCL vector literals ``(float2)(a, b)`` -> ``float2(a, b)`` (in C++
     the former is a cast of a comma expression) and swizzles ``.even`` ->
     ``.even()``;
  4. make FLOAT_TO_FIXED saturating (constants.cl:22's C cast is undefined for
     NaN / out-of-range values; GPUs saturate and map NaN to 0).

The reference checkout is only needed to (re)generate ``oracle/_ref``; where it
is absent the prebuilt libraries are used as they are.  Its location is the
``XPR_REFERENCE`` environment variable, else a ``reference`` directory beside the
repository checkout.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD_DIR, "libxpr_oracle.so")
REF_SO = os.path.join(REF_DIR, "libxpr_ref.so")
REF_RELAXED_SO = os.path.join(REF_DIR, "libxpr_ref_relaxed.so")
DEFAULT_REFERENCE = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
KERNEL_DIR = os.path.join("src", "reconstruction", "gpu", "kernels")

CFLAGS = ["-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC"]
RELAXED_CFLAGS = ["-O2", "-fopenmp", "-ffast-math", "-mfma", "-mavx2", "-fPIC"]

# kernel name -> launcher (the reference's argument lists, constants.cl:30-88)
LAUNCHERS = {
    "KernelForward": r'''
extern "C" void refk_forward(const float *vol, uint32_t *sum, const void *pd, const uint32_t size4[4],
                             const float origin4[4], uint32_t angles, uint32_t modules,
                             const int32_t vmin[3], const int32_t vmax[3], const int32_t line_offset[2],
                             const float voxel4[4], uint64_t global)
{
    using namespace oclshim;
    const uint4 s(size4[0], size4[1], size4[2], size4[3]);
    const float4 o(origin4[0], origin4[1], origin4[2], origin4[3]);
    const float4 v(voxel4[0], voxel4[1], voxel4[2], voxel4[3]);
    const uint3 mn((uint)vmin[0], (uint)vmin[1], (uint)vmin[2]);
    const uint3 mx((uint)vmax[0], (uint)vmax[1], (uint)vmax[2]);
    const uint2 lo((uint)line_offset[0], (uint)line_offset[1]);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t g = 0; g < (int64_t)global; ++g) {
        g_gid = (size_t)g;
        NS::Forward(vol, sum, (const NS::ProjData *)pd, s, o, angles, modules, mn, mx, lo, v);
    }
}
''',
    "KernelBackward": r'''
extern "C" void refk_backward(float *vol, const float *ratio, const void *pd, const uint32_t size4[4],
                              const float origin4[4], uint32_t angles, uint32_t modules,
                              const int32_t vmin[3], const int32_t vmax[3], const int32_t line_offset[2],
                              const float voxel4[4], uint64_t global)
{
    using namespace oclshim;
    const uint4 s(size4[0], size4[1], size4[2], size4[3]);
    const float4 o(origin4[0], origin4[1], origin4[2], origin4[3]);
    const float4 v(voxel4[0], voxel4[1], voxel4[2], voxel4[3]);
    const uint3 mn((uint)vmin[0], (uint)vmin[1], (uint)vmin[2]);
    const uint3 mx((uint)vmax[0], (uint)vmax[1], (uint)vmax[2]);
    const uint2 lo((uint)line_offset[0], (uint)line_offset[1]);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t g = 0; g < (int64_t)global; ++g) {
        g_gid = (size_t)g;
        NS::Backward(vol, ratio, (const NS::ProjData *)pd, s, o, angles, modules, mn, mx, lo, v);
    }
}
''',
    "KernelError": r'''
extern "C" void refk_error(const float *images, uint32_t *sum, const uint32_t size4[4], uint32_t elements,
                           float weight, uint64_t global)
{
    using namespace oclshim;
    const uint4 s(size4[0], size4[1], size4[2], size4[3]);
#pragma omp parallel for schedule(static, 65536)
    for (int64_t g = 0; g < (int64_t)global; ++g) {
        g_gid = (size_t)g;
        NS::Error(images, sum, s, elements, weight);
    }
}
''',
    "KernelForwardH": r'''
extern "C" void refk_forwardh(const float *vol, uint32_t *sum, const void *pd, const uint16_t *idx,
                              const uint16_t *img, uint32_t angles, uint32_t y_offset, const float origin4[4],
                              float voxel, uint32_t det_w, uint32_t det_h, uint32_t vol_w, uint64_t global)
{
    using namespace oclshim;
    const float4 o(origin4[0], origin4[1], origin4[2], origin4[3]);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t g = 0; g < (int64_t)global; ++g) {
        g_gid = (size_t)g;
        NS::ForwardH(vol, sum, (const NS::ProjData *)pd, idx, img, angles, y_offset, o, voxel, det_w, det_h, vol_w);
    }
}
''',
    "KernelBackwardH": r'''
extern "C" void refk_backwardh(float *vol, const float *ratio, const void *pd, const uint16_t *idx,
                               const uint16_t *img, uint32_t angles, uint32_t y_offset, const float origin4[4],
                               float voxel, uint32_t det_w, uint32_t det_h, uint32_t vol_w, uint64_t global)
{
    using namespace oclshim;
    const float4 o(origin4[0], origin4[1], origin4[2], origin4[3]);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t g = 0; g < (int64_t)global; ++g) {
        g_gid = (size_t)g;
        NS::BackwardH(vol, ratio, (const NS::ProjData *)pd, idx, img, angles, y_offset, o, voxel, det_w, det_h, vol_w);
    }
}
''',
}


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), proc.stdout, proc.stderr))


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "xpr_oracle.c")
    hdr = os.path.join(HERE, "xpr_oracle.h")
    os.makedirs(BUILD_DIR, exist_ok=True)
    if force or not _newer(ORACLE_SO, [src, hdr, __file__]):
        _run(["gcc", "-std=c11", "-shared", *CFLAGS, "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


def preprocess_kernel(reference_root: str, name: str) -> str:
    """Return the C++-compilable text of reference kernel `name` (see module doc)."""
    kdir = os.path.join(reference_root, KERNEL_DIR)
    with open(os.path.join(kdir, name + ".cl")) as f:
        text = f.read()
    with open(os.path.join(kdir, "utils.cl")) as f:
        utils = f.read()
    with open(os.path.join(kdir, "constants.cl")) as f:
        constants = f.read()
    text = text.replace('#include "utils.cl"', utils)
    text = text.replace('#include "constants.cl"', constants)
    text = text.replace("#ifdef __cplusplus", "#if 0")
    text = re.sub(r"(#define FLOAT_TO_FIXED\(x\)[^\n]*\n)",
                  r"\1#undef FLOAT_TO_FIXED\n#define FLOAT_TO_FIXED(x) oclshim::float_to_fixed_sat(x)\n",
                  text, count=1)
    text = re.sub(r"\((float|int|uint|ushort)([234])\)\s*\(", r"\1\2(", text)
    text = re.sub(r"\.(even|odd|lo|hi)\b(?!\s*\()", r".\1()", text)
    return text


def build_ref(reference_root: str | None = None, force: bool = False) -> str | None:
    """Generate and compile oracle/_ref/libxpr_ref.so.  Returns its path, or None
    when neither the reference checkout nor a prebuilt library is available."""
    root = reference_root or os.environ.get("XPR_REFERENCE", DEFAULT_REFERENCE)
    kdir = os.path.join(root, KERNEL_DIR)
    if not os.path.isdir(kdir):
        return REF_SO if os.path.exists(REF_SO) else None
    os.makedirs(REF_DIR, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.hpp")
    cl_files = [os.path.join(kdir, n + ".cl") for n in LAUNCHERS] + [
        os.path.join(kdir, "utils.cl"), os.path.join(kdir, "constants.cl")]
    deps = cl_files + [shim, __file__, os.path.join(HERE, "xpr_oracle.c")]
    if not force and _newer(REF_SO, deps) and _newer(REF_RELAXED_SO, deps):
        return REF_SO
    objs = []
    for name, launcher in LAUNCHERS.items():
        body = preprocess_kernel(root, name)
        ns = "ref_" + name
        cpp = os.path.join(REF_DIR, name + ".cpp")
        with open(cpp, "w") as f:
            f.write("// generated by oracle/build.py from %s -- do not edit\n" % os.path.join(KERNEL_DIR, name + ".cl"))
            f.write('#include "../ref_shim.hpp"\n')
            f.write("namespace %s {\nusing namespace oclshim;\n" % ns)
            f.write("#define kernel\n#define global\n#define constant\n#define restrict __restrict\n")
            f.write(body)
            f.write("\n#undef kernel\n#undef global\n#undef constant\n#undef restrict\n}\n")
            f.write("#define NS %s\n" % ns)
            f.write(launcher)
        obj = cpp[:-4] + ".o"
        _run(["g++", "-std=c++17", "-c", *CFLAGS, "-w", "-o", obj, cpp])
        objs.append(obj)
    common = os.path.join(REF_DIR, "ref_common.cpp")
    with open(common, "w") as f:
        f.write('#include "../ref_shim.hpp"\nthread_local size_t oclshim::g_gid = 0;\n')
    _run(["g++", "-std=c++17", "-c", *CFLAGS, "-o", common[:-4] + ".o", common])
    objs.append(common[:-4] + ".o")
    orc_obj = os.path.join(REF_DIR, "orc_math.o")
    _run(["gcc", "-std=c11", "-c", *CFLAGS, "-o", orc_obj, os.path.join(HERE, "xpr_oracle.c")])
    objs.append(orc_obj)
    _run(["g++", "-shared", "-fopenmp", "-o", REF_SO, *objs, "-lm"])
    # the relaxed-math build of the same kernel sources (exp / log stay the oracle's)
    robjs = []
    for name in LAUNCHERS:
        cpp = os.path.join(REF_DIR, name + ".cpp")
        obj = os.path.join(REF_DIR, name + ".relaxed.o")
        _run(["g++", "-std=c++17", "-c", *RELAXED_CFLAGS, "-w", "-o", obj, cpp])
        robjs.append(obj)
    _run(["g++", "-shared", "-fopenmp", "-o", REF_RELAXED_SO, *robjs, common[:-4] + ".o", orc_obj, "-lm"])
    return REF_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    ref = sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv else None
    print(build_ref(ref, force="--force" in sys.argv))
