"""Build recipe for the test-only CPU oracle (and, when the reference tree is
present, the reference kernels compiled from their own sources).

    python -m oracle.build            # oracle/liboracle.so (+ oracle/_ref/ when possible)

The oracle is a checker: tests, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg load it; the product never does.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SRC = os.path.join(HERE, "od_oracle.cpp")
ORACLE_SO = os.path.join(HERE, "liboracle.so")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle(force: bool = False) -> str:
    if force or _stale(ORACLE_SO, [ORACLE_SRC]):
        tmp = ORACLE_SO + ".tmp"
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread",
               "-ffp-contract=off", ORACLE_SRC, "-o", tmp]
        subprocess.run(cmd, check=True)
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def build_all(force: bool = False) -> None:
    build_oracle(force)
    from . import build_ref  # noqa: WPS433 (local import keeps the oracle build standalone)
    build_ref.build(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
