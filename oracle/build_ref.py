"""Build recipe for the reference's own kernels (test infrastructure).

The reference JIT-compiles its four CUDA sources with NVRTC at start-up
(src/solver.rs:380-447): constants.cuh, device_functions.cuh, rhs.cu and rk.cu
concatenated with newlines, options --use_fast_math (when fast_math),
--gpu-architecture=compute_XY of the running device, -DU_REAL/-DQ_REAL/
-DRHS_REAL/-DCOMPUTE_REAL, -DFR_ORDER=3, -DBC_Y_WALL, the unused viscosity
macros and -DFLUX_SCHEME_*. This recipe does the same, from the sources where
they lie under the reference tree, for compute_100 (B200), and writes one
PTX module per variant into oracle/_ref/. The driver JIT-compiles the PTX at
load time, as cudarc's load_module does for the reference. The PTX is loaded,
never inspected.

It also builds oracle/_ref/libodref.so, the driver-API runner that replays the
reference's launch shapes and sequence (oracle/ref_harness.cpp).

Outputs go to oracle/_ref/ only (git-ignored; it travels to the GPU box).
"""

from __future__ import annotations

import ctypes
import itertools
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
CUDA_FILES = ("constants.cuh", "device_functions.cuh", "rhs.cu", "rk.cu")  # solver.rs:437-443 order
HARNESS_SRC = os.path.join(HERE, "ref_harness.cpp")
HARNESS_SO = os.path.join(OUT, "libodref.so")

FLUX_MACRO = {"slau2": "FLUX_SCHEME_SLAU2", "ausm+": "FLUX_SCHEME_AUSMPLUS", "rusanov": "FLUX_SCHEME_RUSANOV"}
CTYPE = {"f32": "float", "f64": "double"}


def variant_name(u, q, r, c, flux, wall, fast_math=True) -> str:
    f = {"slau2": "slau2", "ausm+": "ausm", "rusanov": "rusanov"}[flux]
    return f"ref_{u}{q}{r}{c}_{f}_{'wall' if wall else 'per'}_{'fm' if fast_math else 'ieee'}"


def ptx_path(u, q, r, c, flux, wall, fast_math=True) -> str:
    return os.path.join(OUT, variant_name(u, q, r, c, flux, wall, fast_math) + ".ptx")


def variants():
    """Every variant the tests and the bench load."""
    out = []
    for prec, flux, wall in itertools.product(("f32", "f64"), FLUX_MACRO, (True, False)):
        out.append((prec, prec, prec, prec, flux, wall, True))
    out.append(("f64", "f32", "f32", "f32", "slau2", True, True))    # constants.cuh defaults
    out.append(("f64", "f32", "f32", "f64", "slau2", True, True))    # f64 compute, f32 Q / RHS
    for flux in FLUX_MACRO:                                            # strict IEEE f32, every flux
        out.append(("f32", "f32", "f32", "f32", flux, True, False))
    return out


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    raise OSError("libnvrtc not found")


def _options(u, q, r, c, flux, wall, fast_math):
    # solver.rs:380-430 (mu_ref / t_ref / s_suth printed as Rust prints the f32 defaults)
    opts = []
    if fast_math:
        opts.append("--use_fast_math")
    opts.append("--gpu-architecture=compute_100")
    opts += [f"-DU_REAL={CTYPE[u]}", f"-DQ_REAL={CTYPE[q]}", f"-DRHS_REAL={CTYPE[r]}", f"-DCOMPUTE_REAL={CTYPE[c]}",
             "-DFR_ORDER=3", f"-DBC_Y_WALL={1 if wall else 0}", "-DMU_REF=0.00016", "-DT_REF=273.15",
             "-DS_SUTH=110.4", f"-D{FLUX_MACRO[flux]}"]
    return opts


def compile_variant(source: str, v, dest: str) -> None:
    nv = _nvrtc()
    prog = ctypes.c_void_p()
    rc = nv.nvrtcCreateProgram(ctypes.byref(prog), source.encode(), b"opendynamo.cu", 0, None, None)
    if rc != 0:
        raise RuntimeError(f"nvrtcCreateProgram failed: {rc}")
    opts = [o.encode() for o in _options(*v)]
    arr = (ctypes.c_char_p * len(opts))(*opts)
    rc = nv.nvrtcCompileProgram(prog, len(opts), arr)
    if rc != 0:
        size = ctypes.c_size_t()
        nv.nvrtcGetProgramLogSize(prog, ctypes.byref(size))
        log = ctypes.create_string_buffer(size.value)
        nv.nvrtcGetProgramLog(prog, log)
        raise RuntimeError(f"NVRTC compile error ({v}): {log.value.decode(errors='replace')}")
    size = ctypes.c_size_t()
    nv.nvrtcGetPTXSize(prog, ctypes.byref(size))
    buf = ctypes.create_string_buffer(size.value)
    nv.nvrtcGetPTX(prog, buf)
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    tmp = dest + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(buf.raw[: size.value])
    os.replace(tmp, dest)


def reference_tree(tree: str | None = None) -> str:
    """The reference source tree: the argument, else $OD_REFERENCE_TREE."""
    tree = tree or os.environ.get("OD_REFERENCE_TREE")
    if not tree:
        raise FileNotFoundError("no reference tree given (argument or OD_REFERENCE_TREE); "
                                f"using the prebuilt modules in {OUT}")
    return tree


def reference_source(tree: str) -> str:
    parts = []
    for f in CUDA_FILES:
        with open(os.path.join(tree, "src", "cuda", f)) as fh:
            parts.append(fh.read())
    return "\n".join(parts)  # format!("{}\n{}\n{}\n{}", ...)


def build_harness(force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    if force or not os.path.exists(HARNESS_SO) or os.path.getmtime(HARNESS_SRC) > os.path.getmtime(HARNESS_SO):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", HARNESS_SRC, "-o", HARNESS_SO + ".tmp",
               "-I/usr/local/cuda/include", "-ldl"]
        subprocess.run(cmd, check=True)
        os.replace(HARNESS_SO + ".tmp", HARNESS_SO)
    return HARNESS_SO


def build(force: bool = False, tree: str | None = None) -> None:
    os.makedirs(OUT, exist_ok=True)
    build_harness(force)
    tree = reference_tree(tree)
    if not os.path.isdir(os.path.join(tree, "src", "cuda")):
        raise FileNotFoundError(f"reference tree not found at {tree}; using the prebuilt modules in {OUT}")
    src = reference_source(tree)
    src_mtime = max(os.path.getmtime(os.path.join(tree, "src", "cuda", f)) for f in CUDA_FILES)
    for v in variants():
        dest = ptx_path(*v)
        if force or not os.path.exists(dest) or os.path.getmtime(dest) < src_mtime:
            compile_variant(src, v, dest)


if __name__ == "__main__":
    import sys
    args = [a for a in sys.argv[1:] if a != "--force"]
    build(force="--force" in sys.argv, tree=args[0] if args else None)
