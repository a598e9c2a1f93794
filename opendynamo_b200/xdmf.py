"""ParaView conversion of state files (the reference's scripts/h5_to_xdmf.py).

``python -m opendynamo_b200.xdmf FILE|DIR ...`` converts each solver-native
state file into ``<stem>.pv.h5`` (group /data with the 3-D point fields rho,
rhou, rhov, rhow, E, vel, p; chunks of 48, shuffle + gzip 4) and
``<stem>.xmf`` (3DRectMesh, cell-centred attributes). The reorder and the
derived fields run on the GPU (od_point_fields); files are read and written
by the library's own HDF5 code, so blosc-compressed dumps need no plugin.

As in the script (h5_to_xdmf.py:137-159): a directory expands to its
``*.h5`` files in sorted order, and when more than one file is given,
checkpoint files (``checkpoint_*``) are skipped.

Differences: the script fails on meshes with fewer than 48 points along an
axis (h5py rejects a (48, 48, 48) chunk larger than the dataset); here the
chunk is clamped to the dataset. Files this conversion writes (``*.pv.h5``)
are not state files and are skipped when a directory is expanded.
"""

from __future__ import annotations

import ctypes
import sys
from pathlib import Path

from . import _native

FIELDS = ["rho", "rhou", "rhov", "rhow", "E", "vel", "p"]


def convert(src) -> tuple[Path, Path]:
    """Convert one state file; returns (point-field file, xmf file)."""
    L = _native.lib()
    h5 = ctypes.create_string_buffer(4096)
    xmf = ctypes.create_string_buffer(4096)
    err = ctypes.create_string_buffer(1024)
    rc = L.od_xdmf_convert(str(src).encode(), h5, len(h5), xmf, len(xmf), err, len(err))
    if rc != 0:
        raise RuntimeError(err.value.decode() or _native.ERRORS.get(rc, str(rc)))
    return Path(h5.value.decode()), Path(xmf.value.decode())


def process(src: Path) -> None:
    """Convert and report like h5_to_xdmf.py:134."""
    from .state_io import state_info
    info = state_info(str(src))
    h5, xmf = convert(src)
    print(f"{src.name} (step {info['step']}, t={info['t']:.5g}): fields {sorted(FIELDS)} -> {h5.name} + {xmf.name}")


def select(args: list[str]) -> list[tuple[Path, bool]]:
    """(file, convert?) for the command-line arguments (h5_to_xdmf.py:140-155)."""
    files: list[Path] = []
    for a in args:
        p = Path(a)
        if p.is_dir():
            files.extend(f for f in sorted(p.glob("*.h5")) if not f.name.endswith(".pv.h5"))
        elif p.exists():
            files.append(p)
        else:
            raise SystemExit(f"no such path: {a}")
    skip = len(files) > 1
    return [(f, not (skip and f.name.startswith("checkpoint_"))) for f in files]


def main(argv: list[str] | None = None) -> None:
    args = sys.argv[1:] if argv is None else argv
    if not args:
        raise SystemExit(__doc__)
    for f, do in select(args):
        if not do:
            print(f"skip checkpoint {f.name} (resume file; pass it explicitly to view)")
            continue
        try:
            process(f)
        except (RuntimeError, _native.OdError) as e:
            raise SystemExit(str(e))


if __name__ == "__main__":
    main()
