"""ParaView conversion on the GPU (scripts/h5_to_xdmf.py): od_point_fields
against the reference script's own outputs (tests/golden/xdmf_reference.npz)
and the oracle, bit for bit, and the whole conversion of state files in
every compression and precision — point-field file, .xmf text and the
printed line."""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from opendynamo_b200 import _native as N
from opendynamo_b200 import state_io as S
from opendynamo_b200 import xdmf as X
from oracle import pointfields as PF

from h5walk import Walker

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "xdmf_reference.npz"))
CASES = [eval(c) for c in GOLDEN["cases"]]


def device_fields(planes, nx, ny, nz):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(planes)).cuda()
    npts = nx * ny * nz * 64
    out = torch.full((7 * npts,), -7.0, dtype=torch.float32, device="cuda")
    rc = N.lib().od_point_fields(ctypes.c_void_p(d.data_ptr()), int(planes.dtype == np.float64), nx, ny, nz,
                                 ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(7, 4 * nx, 4 * ny, 4 * nz)


@pytest.mark.gpu
@pytest.mark.parametrize("n", range(len(CASES)))
def test_point_fields_match_the_reference_script(n):
    c = CASES[n]
    got = device_fields(GOLDEN[f"case{n}_planes"], c["nx"], c["ny"], c["nz"])
    for i, k in enumerate(PF.FIELD_NAMES):
        assert np.array_equal(got[i], GOLDEN[f"case{n}_{k}"], equal_nan=True), k


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", [(1, 1, 1), (5, 4, 17), (16, 3, 8), (2, 9, 24)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_point_fields_match_the_oracle(mesh, dtype):
    nx, ny, nz = mesh
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz)
    npts = nx * ny * nz * 64
    a = np.empty((5, npts), dtype)
    a[0] = rng.uniform(-0.1, 2.0, npts)
    a[1:4] = rng.standard_normal((3, npts))
    a[4] = rng.uniform(-1.0, 5.0, npts)
    a.reshape(-1)[rng.integers(0, a.size, 8)] = np.nan
    got = device_fields(a, nx, ny, nz)
    ref = PF.point_fields(a, nx, ny, nz)
    for i, k in enumerate(PF.FIELD_NAMES):
        assert np.array_equal(got[i], ref[k], equal_nan=True), k


def convert_case(tmp_path, capsys, n, comp):
    c = CASES[n]
    planes = GOLDEN[f"case{n}_planes"]
    src = tmp_path / c["name"]
    S.save_state(str(src), planes, c["nx"], c["ny"], c["nz"], step=c["step"], t=c["t"], lx=c["lx"], ly=c["ly"],
                 lz=c["lz"], compression=comp)
    X.main([str(src)])
    return c, src, capsys.readouterr().out


@pytest.mark.gpu
@pytest.mark.parametrize("comp", ["none", "gzip1", "blosc-lz4", "blosc-zstd"])
@pytest.mark.parametrize("n", range(len(CASES)))
def test_convert_state_file(tmp_path, capsys, n, comp):
    c, src, line = convert_case(tmp_path, capsys, n, comp)
    assert line == str(GOLDEN[f"case{n}_line"])
    stem = src.with_suffix("")
    assert (tmp_path / (stem.name + ".xmf")).read_text() == str(GOLDEN[f"case{n}_xmf"])
    w = Walker((tmp_path / (stem.name + ".pv.h5")).read_bytes())
    members = w.group_members(w.group_members(w.root_ohdr)["data"])
    assert sorted(members) == sorted(PF.FIELD_NAMES)
    for k in PF.FIELD_NAMES:
        info = w.dataset(members[k])
        assert info["dims"] == (4 * c["nx"], 4 * c["ny"], 4 * c["nz"])
        assert info["cdims"] == tuple(min(48, d) for d in info["dims"])
        assert [f for f, _ in info["filters"]] == [2, 1] and info["filters"][1][1] == [4]
        assert np.array_equal(w.read_array(members[k]), GOLDEN[f"case{n}_{k}"], equal_nan=True), k


@pytest.mark.gpu
def test_convert_directory_skips_checkpoints(tmp_path, capsys):
    rng = np.random.default_rng(5)
    nx = ny = nz = 2
    npts = nx * ny * nz * 64
    a = np.stack([1 + 0.1 * rng.standard_normal(npts), *(0.1 * rng.standard_normal((3, npts))),
                  2.5 + 0.1 * rng.standard_normal(npts)]).astype(np.float32)
    for name in ("flow_f32_000001.h5", "flow_f32_000002.h5", "checkpoint_f32_000002.h5"):
        S.save_state(str(tmp_path / name), a, nx, ny, nz, step=int(name[-9:-3]), t=0.1)
    X.main([str(tmp_path)])
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "skip checkpoint checkpoint_f32_000002.h5 (resume file; pass it explicitly to view)"
    assert out[1].startswith("flow_f32_000001.h5 (step 1, t=0.1): fields")
    assert out[2].startswith("flow_f32_000002.h5 (step 2, t=0.1): fields")
    assert sorted(p.name for p in tmp_path.glob("*.xmf")) == ["flow_f32_000001.xmf", "flow_f32_000002.xmf"]
    # a second pass ignores the point-field files it wrote
    X.main([str(tmp_path)])
    assert len(capsys.readouterr().out.splitlines()) == 3


@pytest.mark.gpu
def test_convert_missing_file_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="not found"):
        X.convert(tmp_path / "nothing.h5")
