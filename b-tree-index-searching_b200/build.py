"""Build recipe for the engine's shared library (sm_100a only).

    python b-tree-index-searching_b200/build.py        # -> lib/libbtree_b200.so

nvcc cross-compiles for sm_100a without a GPU.  The library is built in-tree
so it travels with the working tree; nothing is installed.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libbtree_b200.so")
COMPAT_DRIVER = os.path.join(LIBDIR, "compat_driver")

SOURCES = [
    "bt_runtime.cu",
    "bt_build.cu",
    "bt_search.cu",
    "bt_group.cu",
    "bt_capi.cu",
    "bt_compat.cu",
    "bt_noalloc.cu",
    "bt_learned.cu",
    "bt_server.cu",
    "bt_forest.cu",
    "bt_rect.cu",
    "bt_probe.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"),
]


def _nvcc():
    for cand in ("nvcc", "/usr/local/cuda/bin/nvcc"):
        try:
            subprocess.run([cand, "--version"], check=True, capture_output=True)
            return cand
        except (OSError, subprocess.CalledProcessError):
            continue
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_info=False):
    """Compile every .cu of csrc/ and link lib/libbtree_b200.so."""
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + \
                ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    drv_src = os.path.join(ROOT, "tests", "compat_driver.cpp")
    if os.path.exists(drv_src) and (force or _stale(COMPAT_DRIVER, [drv_src, LIB] + headers)):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), drv_src,
               "-o", COMPAT_DRIVER, "-L", LIBDIR, "-lbtree_b200",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
