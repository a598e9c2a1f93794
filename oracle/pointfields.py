"""TEST INFRASTRUCTURE — CPU oracle of the ParaView conversion.

A numpy restatement of the reference's scripts/h5_to_xdmf.py for one state:
the reorder of the element-major planes into the global solution-point
tensor (h5_to_xdmf.py:35-44), the derived fields (h5_to_xdmf.py:74-82) in
float32 with numpy's operation order, and the .xmf text
(h5_to_xdmf.py:84-120). Used only by the tests to check od_point_fields,
od_xdmf_text and od_xdmf_convert.
"""

from __future__ import annotations

import numpy as np

VAR_NAMES = ["rho", "rhou", "rhov", "rhow", "E"]
FIELD_NAMES = VAR_NAMES + ["vel", "p"]
GAMMA = 1.4


def to_tensor(flat: np.ndarray, nx: int, ny: int, nz: int, p1: int = 4) -> np.ndarray:
    """Element-major plane (index elem * p1^3 + k p1^2 + j p1 + i, elem = ex +
    nx ey + nx ny ez) -> array [nx p1, ny p1, nz p1] indexed (ex p1 + i,
    ey p1 + j, ez p1 + k) (h5_to_xdmf.py:35-44)."""
    blocks = flat.reshape(nz, ny, nx, p1, p1, p1)          # [ez, ey, ex, k, j, i]
    return np.ascontiguousarray(np.moveaxis(blocks, (2, 5, 1, 4, 0, 3), (0, 1, 2, 3, 4, 5))).reshape(
        nx * p1, ny * p1, nz * p1)


def to_tensor_loops(flat: np.ndarray, nx: int, ny: int, nz: int, p1: int = 4) -> np.ndarray:
    """The same reorder written point by point (small meshes; pins to_tensor)."""
    out = np.empty((nx * p1, ny * p1, nz * p1), flat.dtype)
    for ez in range(nz):
        for ey in range(ny):
            for ex in range(nx):
                e = ex + nx * (ey + ny * ez)
                for k in range(p1):
                    for j in range(p1):
                        for i in range(p1):
                            out[ex * p1 + i, ey * p1 + j, ez * p1 + k] = flat[e * p1 ** 3 + k * p1 * p1 + j * p1 + i]
    return out


def point_fields(planes: np.ndarray, nx: int, ny: int, nz: int) -> dict:
    """The seven point fields of a state (5 planes of any float type, read as
    float32 like h5_to_xdmf.py:69)."""
    raw = [np.asarray(planes[v], dtype=np.float32).reshape(-1) for v in range(5)]
    f = {n: to_tensor(p, nx, ny, nz) for n, p in zip(VAR_NAMES, raw)}
    rho, u, v, w, e = (f[n] for n in VAR_NAMES)
    with np.errstate(all="ignore"):
        r = np.maximum(rho, 1e-30)
        f["vel"] = np.sqrt(u * u + v * v + w * w) / r
        f["p"] = np.maximum(1e-7, (GAMMA - 1.0) * (e - 0.5 * (u * u + v * v + w * w) / r))
    return f


def xdmf_text(h5_name: str, npx: int, npy: int, npz: int, lx: float, ly: float, lz: float, step: int,
              t: float) -> str:
    """The .xmf document of one converted file (h5_to_xdmf.py:84-120)."""
    axes = [np.linspace(0.0, L, n + 1) for L, n in zip((lx, ly, lz), (npx, npy, npz))]
    attrs = []
    for n in FIELD_NAMES:
        attrs.append(
            f'      <Attribute Name="{n}" AttributeType="Scalar" Center="Cell">\n'
            f'        <DataItem Dimensions="{npz} {npy} {npx}" NumberType="Float" Precision="4" Format="HDF">\n'
            f'          {h5_name}:/data/{n}\n'
            f'        </DataItem>\n'
            f'      </Attribute>')
    geo = "".join(
        f'        <DataItem Dimensions="{len(a)}" NumberType="Float" Precision="8" Format="XML">\n'
        f'          {" ".join(f"{x:.10g}" for x in a)}\n'
        f'        </DataItem>\n' for a in axes)
    return ('<?xml version="1.0" ?>\n'
            '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n'
            '<Xdmf Version="2.0">\n'
            '  <Domain>\n'
            f'    <Grid Name="FR_Grid" GridType="Uniform" t_step="{step}" t_time="{t:.6g}">\n'
            f'      <Topology TopologyType="3DRectMesh" Dimensions="{npz + 1} {npy + 1} {npx + 1}"/>\n'
            '      <Geometry GeometryType="VXVYVZ">\n'
            f'{geo}'
            '      </Geometry>\n'
            + "\n".join(attrs) + "\n"
            '    </Grid>\n'
            '  </Domain>\n'
            '</Xdmf>\n')
