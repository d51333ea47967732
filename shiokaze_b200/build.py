"""Build the sm_100a CUDA library ``libshkz_b200.so`` in-tree with nvcc.

    python -m shiokaze_b200.build          # or build() from Python

Every translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); the assembly unit is compiled
with ``-fmad=false`` so its FP64 face arithmetic rounds like the reference's
CPU code. The CUDA runtime is linked statically so the library does not
depend on which libcudart the host process already loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libshkz_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
UNITS = {
    "assemble.cu": ["-fmad=false"],
    "solver.cu": [],
    "learned.cu": [],
    "api.cu": [],
    "noalloc.cu": [],
    "warmstart.cu": [],
    "extend.cu": ["-fmad=false"],
    "splat.cu": ["-fmad=false"],
    "csr_mic0.cu": [],
}
HEADERS = ["common.cuh", "kernels.h", "solver.h", "learned.h", "tc_conv.cuh", "csr_mic0.h"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, extra=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "shkz_b200.h")]
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + flags + (extra or []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


PLUGINS = {"libshiokaze_macpressuresolver3_b200.so": "macpressuresolver3_b200.cpp",
           "libshiokaze_pcg_b200.so": "pcg_b200.cpp",
           "libshiokaze_macnbflip3_b200.so": "macnbflip3_b200.cpp"}

# modules that subclass a reference module compile its source from the
# reference tree (include path of that source file, and the file itself as
# a dependency)
PLUGIN_REFERENCE_SOURCES = {"macnbflip3_b200.cpp": "src/flip/macnbflip3.cpp"}


def build_plugins(reference_root: str, verbose: bool = False) -> list:
    """Build the Shiokaze module(s) that wrap the C ABI. They compile against
    the reference's public headers (``<reference_root>/include`` and
    ``local/include``) with the reference's build defines, and link
    ``libshkz_b200.so`` from this directory."""
    inc = os.path.join(reference_root, "include")
    if not os.path.isdir(inc):
        return []
    lib = build(verbose=verbose)
    out = []
    for so, src in PLUGINS.items():
        target = os.path.join(HERE, so)
        source = os.path.join(HERE, "plugin", src)
        deps = [source, lib, os.path.join(HERE, "..", "include", "shkz_b200.h")]
        extra_inc = []
        if src in PLUGIN_REFERENCE_SOURCES:
            ref_src = os.path.join(reference_root, PLUGIN_REFERENCE_SOURCES[src])
            deps.append(ref_src)
            extra_inc = ["-I" + os.path.dirname(ref_src)]
        if _stale(target, deps):
            cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-w",
                   '-DSHKZ_SUFFIX=""', "-DSHKZ_RELEASE=1", f"-DNUM_THREAD={os.cpu_count() or 4}",
                   "-I" + inc, "-I" + os.path.join(reference_root, "local", "include"),
                   "-I" + os.path.join(HERE, "..", "include")] + extra_inc + [source, "-o", target,
                   "-L" + HERE, "-lshkz_b200", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        out.append(target)
    return out


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
