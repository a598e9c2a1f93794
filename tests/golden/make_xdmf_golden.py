"""Golden ParaView conversions from the reference's own script.

Imports scripts/h5_to_xdmf.py from the reference tree (read-only) and runs
its ``process`` on small synthetic states. h5py is absent here, so a stand-in
module serves the script's reads (attributes and the five planes of a state
held in memory) and records its writes (each create_dataset call with its
data and options); the .xmf text is the file the script writes, and the
printed line is captured. No arithmetic of the script is replaced.

    python tests/golden/make_xdmf_golden.py [/path/to/reference]

writes tests/golden/xdmf_reference.npz.
"""

from __future__ import annotations

import contextlib
import io
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
VARS = ["rho", "rhou", "rhov", "rhow", "E"]

CASES = [
    dict(name="flow_f32_000500.h5", nx=3, ny=2, nz=5, step=500, t=0.05, lx=float(np.float32(2 * np.pi)), ly=2.0,
         lz=float(np.float32(np.pi)), dtype="f4", seed=1),
    dict(name="checkpoint_f64_000012.h5", nx=2, ny=3, nz=9, step=12, t=1.2345678901e-3,
         lx=float(np.float32(2 * np.pi)), ly=float(np.float32(2 * np.pi)), lz=float(np.float32(2 * np.pi)),
         dtype="f8", seed=2),
]


def state(c):
    rng = np.random.default_rng(c["seed"])
    n = c["nx"] * c["ny"] * c["nz"] * 64
    a = np.empty((5, n), dtype=c["dtype"])
    a[0] = 1 + 0.1 * rng.standard_normal(n)
    a[1:4] = 0.3 * rng.standard_normal((3, n))
    a[4] = 2.5 + 0.2 * rng.standard_normal(n)
    # the script's guards: non-positive density, pressure below its floor, NaN
    a[0, 3], a[0, 10], a[0, 17] = 0.0, -0.5, 1e-35
    a[4, 5] = 0.0
    a[2, 40] = np.nan
    a[1, 41] = np.inf
    return a


class _Dataset:
    compression = None

    def __init__(self, arr):
        self.arr = arr

    def __array__(self, dtype=None, copy=None):
        return self.arr if dtype is None else self.arr.astype(dtype)


class _ReadFile:
    def __init__(self, c, planes):
        self.attrs = {"nx": np.uint64(c["nx"]), "ny": np.uint64(c["ny"]), "nz": np.uint64(c["nz"]),
                      "step": np.uint64(c["step"]), "t": np.float64(c["t"]), "lx": np.float64(c["lx"]),
                      "ly": np.float64(c["ly"]), "lz": np.float64(c["lz"])}
        self.groups = {"data": {v: _Dataset(planes[i]) for i, v in enumerate(VARS)}}

    def __getitem__(self, k):
        return self.groups[k]


class _WriteFile:
    def __init__(self, log):
        self.log = log

    def create_group(self, name):
        log = self.log

        class G:
            def create_dataset(self, n, data, **kw):
                log.append((name, n, np.array(data), kw))

        return G()


def main(ref_root: str) -> None:
    sys.path.insert(0, os.path.join(ref_root, "scripts"))
    fake = types.ModuleType("h5py")
    current = {}

    @contextlib.contextmanager
    def File(path, mode="r"):
        if mode == "r":
            yield current["read"]
        else:
            yield _WriteFile(current["log"])

    fake.File = File
    sys.modules["h5py"] = fake
    import h5_to_xdmf as ref  # noqa: E402

    out = {}
    with tempfile.TemporaryDirectory() as td:
        for n, c in enumerate(CASES):
            planes = state(c)
            current["read"] = _ReadFile(c, planes)
            current["log"] = []
            src = Path(td) / c["name"]
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                ref.process(src)
            out[f"case{n}_planes"] = planes
            out[f"case{n}_xmf"] = np.array(src.with_suffix(".xmf").read_text())
            out[f"case{n}_line"] = np.array(buf.getvalue())
            names = []
            for grp, name, data, kw in current["log"]:
                names.append(f"{grp}/{name}")
                out[f"case{n}_{name}"] = data
                out[f"case{n}_{name}_opts"] = np.array(repr(sorted(kw.items())))
            out[f"case{n}_names"] = np.array(names)
    out["cases"] = np.array([repr(c) for c in CASES])
    np.savez_compressed(os.path.join(HERE, "xdmf_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "xdmf_reference.npz"))


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OD_REFERENCE_TREE")
    if not tree:
        raise SystemExit("usage: python tests/golden/make_xdmf_golden.py REFERENCE_TREE (or set OD_REFERENCE_TREE)")
    main(tree)
