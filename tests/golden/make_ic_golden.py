"""Golden initial states from the reference's own IC generator.

Imports scripts/make_initial_state.py from the reference tree (read-only)
and evaluates its ``initial_condition`` for a few small configurations.
Two stand-ins make it importable in this environment, neither touching its
arithmetic: ``h5py`` is stubbed (only its writer uses it), and
``math.fma`` — absent before Python 3.13 — is provided as an exact rational
fused multiply-add (Fraction product + sum, one correctly rounded
conversion), which is what math.fma computes.

    python tests/golden/make_ic_golden.py [/path/to/reference]

writes tests/golden/ic_reference.npz.
"""

from __future__ import annotations

import math
import os
import sys
import types
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    dict(nx=3, ny=4, nz=5, lx=2 * math.pi, ly=2.0, lz=math.pi, mach_bulk=0.2, initial_condition="channel",
         perturbation_amplitude=0.01, perturbation_modes=16, perturbation_seed=42),
    dict(nx=2, ny=3, nz=2, lx=4 * math.pi, ly=2.0, lz=(4.0 / 3.0) * math.pi, mach_bulk=0.3,
         initial_condition="channel", perturbation_amplitude=0.0, perturbation_modes=16, perturbation_seed=7),
    dict(nx=2, ny=2, nz=3, lx=2 * math.pi, ly=2.0, lz=math.pi, mach_bulk=0.25, initial_condition="uniform",
         perturbation_amplitude=0.2, perturbation_modes=5, perturbation_seed=3),
    dict(nx=4, ny=3, nz=2, lx=3.0, ly=1.5, lz=2.0, mach_bulk=0.1, initial_condition="channel",
         perturbation_amplitude=0.05, perturbation_modes=24, perturbation_seed=0),
]


def main(ref_root: str) -> None:
    if not hasattr(math, "fma"):
        math.fma = lambda a, b, c: float(Fraction(a) * Fraction(b) + Fraction(c))
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path.insert(0, os.path.join(ref_root, "scripts"))
    import make_initial_state as mis  # noqa: E402

    out = {}
    for n, c in enumerate(CASES):
        planes = mis.initial_condition(dict(c))
        for v, p in enumerate(planes):
            out[f"case{n}_v{v}"] = np.asarray(p, dtype=np.float32)
    out["cases"] = np.array([repr(c) for c in CASES])
    out["gl_points"] = np.array(mis.gauss_legendre_points())
    np.savez_compressed(os.path.join(HERE, "ic_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "ic_reference.npz"))


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OD_REFERENCE_TREE")
    if not tree:
        raise SystemExit("usage: python tests/golden/make_ic_golden.py REFERENCE_TREE (or set OD_REFERENCE_TREE)")
    main(tree)
