"""Build the sm_100a shared library in-tree.

    python -m opendynamo_b200.build [--force]

Compiles every ``csrc/*.cu`` / ``csrc/*.cpp`` translation unit with nvcc /
g++ in parallel into ``opendynamo_b200/_build/`` and links
``opendynamo_b200/lib/libopendynamo.so`` (plus the ``odrun`` host executable).
Kernels are built for sm_100a only.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libopendynamo.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
            "-I/usr/local/cuda/include"]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    return cu, cpp


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _obj(src):
    return os.path.join(BUILD, os.path.basename(src) + ".o")


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or hdr_mtime > t


def _compile(src):
    obj = _obj(src)
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, *NVFLAGS, "-c", src, "-o", obj]
    else:
        cmd = ["g++", *CXXFLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    cu, cpp = _sources()
    hdr = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    todo = [s for s in cu + cpp if force or _stale(_obj(s), s, hdr)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(_compile, todo))
    objs = [_obj(s) for s in cu + cpp]
    lib_objs = [o for o in objs if not os.path.basename(o).startswith("odrun_main")]
    if force or todo or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *lib_objs, "-o", tmp, "-lz", "-ldl", "-lpthread"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    main_objs = [o for o in objs if os.path.basename(o).startswith("odrun_main")]
    if main_objs:
        exe = os.path.join(LIBDIR, "odrun")
        if force or todo or not os.path.exists(exe):
            cmd = ["g++", *main_objs, "-o", exe, "-L" + LIBDIR, "-lopendynamo", "-Wl,-rpath,$ORIGIN",
                   "-L/usr/local/cuda/lib64", "-lcudart", "-lpthread"]
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
