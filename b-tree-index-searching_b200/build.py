"""Build recipe for the engine's shared library (sm_100a only).

    python b-tree-index-searching_b200/build.py        # -> lib/libbtree_b200.so
                                                       #    lib/btree (the reference's CLI)
                                                       #    lib/libbt_probe.so (bench probes)

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
CLI_SRC = os.path.join(PKG, "cli", "btree_main.cpp")
CLI = os.path.join(LIBDIR, "btree")
PROBE_SRC = os.path.join(PKG, "probe", "bt_probe.cu")
PROBE_LIB = os.path.join(LIBDIR, "libbt_probe.so")

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
    # the benchmark's probes: a separate library the engine does not link
    if force or _stale(PROBE_LIB, [PROBE_SRC]):
        cmd = [nvcc] + NVCC_FLAGS + ["-shared", PROBE_SRC, "-o", PROBE_LIB]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    # the reference program's command line over the compat API (lib/btree)
    if force or _stale(CLI, [CLI_SRC, LIB] + headers):
        cmd = [nvcc] + ARCH + ["-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), CLI_SRC,
                               "-o", CLI, "-L", LIBDIR, "-lbtree_b200", "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
