"""Build recipe for the in-tree CUDA library ``bmmpy_b200/libbmm_b200.so``.

    python -m bmmpy_b200.build [--verbose]

Compiles every ``csrc/*.cu`` for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``), one nvcc process per file in parallel
(objects in ``bmmpy_b200/_build/``), and links one shared library with the CUDA
runtime linked statically, so the library has no Python or torch dependency
and travels as a single file.  Rebuilds only when a source is newer than the
library.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbmm_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler",
                 "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
LINK_FLAGS = ["-shared", "-cudart", "static"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + _headers()


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "bmm_b200.h")]


def _compile(src: str, ptxas_info: bool, force: bool) -> tuple[str, int, str]:
    obj = os.path.join(HERE, "_build", os.path.basename(src) + ".o")
    if not force and not ptxas_info and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if all(os.path.getmtime(p) <= t for p in [src, *_headers()]):
            return obj, 0, ""
    cmd = [nvcc(), *ARCH, *COMPILE_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src,
           "-o", obj]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    return obj, proc.returncode, proc.stdout + proc.stderr


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compile each csrc/*.cu in parallel (one nvcc per file), then link."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as pool:
        results = list(pool.map(lambda s: _compile(s, ptxas_info, force), srcs))
    failed = [out for _, rc, out in results if rc != 0]
    if verbose or ptxas_info or failed:
        for _, _, out in results:
            sys.stderr.write(out)
    if failed:
        raise RuntimeError("nvcc failed building libbmm_b200.so")
    cmd = [nvcc(), *ARCH, *LINK_FLAGS, "-o", LIB + ".tmp", *[o for o, _, _ in results]]
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed linking libbmm_b200.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


BINDING_SRC = os.path.join(HERE, "bindings", "_bmmpy.cpp")


def binding_path() -> str:
    import sysconfig

    return os.path.join(HERE, "_bmmpy" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def build_binding(verbose: bool = False, force: bool = False) -> str:
    """The pybind11 module bmmpy_b200/_bmmpy*.so (the reference's native module
    name) over include/bmmpy/, linked to libbmm_b200.so next to it."""
    import sysconfig

    import pybind11

    out = binding_path()
    deps = [BINDING_SRC, LIB] + sorted(glob.glob(os.path.join(ROOT, "include", "bmmpy", "**",
                                                              "*.hpp"), recursive=True))
    if not force and os.path.exists(out) and all(os.path.getmtime(p) <= os.path.getmtime(out)
                                                  for p in deps):
        return out
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           "-I", os.path.join(ROOT, "include"), BINDING_SRC, "-o", out + ".tmp",
           "-L", HERE, "-lbmm_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("g++ failed building the _bmmpy module")
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv,
          ptxas_info="--ptxas" in sys.argv)
    build_binding(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
