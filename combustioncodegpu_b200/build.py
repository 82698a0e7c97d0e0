"""Builds the in-tree CUDA library libcc_b200.so for sm_100a.

Every translation unit is compiled in parallel with nvcc
(-gencode arch=compute_100a,code=sm_100a -lineinfo) and linked with the
static CUDA runtime into combustioncodegpu_b200/libcc_b200.so.

build(bounds=True) builds libcc_b200_bounds.so from the same sources with
-DCC_BOUNDS_CHECK: the kernels check the arena, scratch and plane indices
they compute and report an index out of range in the status word instead of
accessing it (a stand-in for compute-sanitizer's memory check).
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcc_b200.so")
BUILD_BOUNDS = os.path.join(HERE, "_build_bounds")
LIB_BOUNDS = os.path.join(HERE, "libcc_b200_bounds.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = [
    "api.cu", "misc.cu", "halo_plan.cpp", "noalloc.cu", "closure_train.cu",
    "inst_d0.cu", "inst_d9.cu", "inst_dn.cu", "inst_f0.cu", "inst_f9.cu", "inst_fn.cu",
]


def _nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return exe


def _flags():
    return ["-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC,
            "-I", os.path.join(os.path.dirname(HERE), "include")]


def _stale(src, obj):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "cc_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, jobs=None, bounds=False):
    build_dir, lib = (BUILD_BOUNDS, LIB_BOUNDS) if bounds else (BUILD, LIB)
    extra = ["-DCC_BOUNDS_CHECK"] if bounds else []
    os.makedirs(build_dir, exist_ok=True)
    nvcc = _nvcc()
    cmds = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(build_dir, s + ".o")
        objs.append(obj)
        if _stale(src, obj):
            lang = ["-x", "cu"] if s.endswith(".cu") else []
            cmds.append([nvcc, *_flags(), *extra, *lang, "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        return cmd

    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd in ex.map(run, cmds):
            if verbose:
                print("compiled", cmd[-1], flush=True)
    if cmds or not os.path.exists(lib):
        link = [nvcc, *ARCH, "-shared", "-o", lib, *objs]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, bounds="--bounds" in sys.argv))
