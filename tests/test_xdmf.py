"""ParaView conversion, host side (scripts/h5_to_xdmf.py): the oracle's reorder
against a point-by-point restatement, the 3-D point-field file writer read
back by the independent walker, the .xmf text against the oracle, and the
command line's file selection. CPU only (no device work)."""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from opendynamo_b200 import _native as N
from opendynamo_b200 import xdmf as X
from oracle import pointfields as PF

from h5walk import Walker


def test_oracle_reorder_matches_point_loops():
    rng = np.random.default_rng(3)
    nx, ny, nz = 3, 2, 5
    flat = rng.standard_normal(nx * ny * nz * 64).astype(np.float32)
    assert np.array_equal(PF.to_tensor(flat, nx, ny, nz), PF.to_tensor_loops(flat, nx, ny, nz))


def save_fields(path, arrs, chunk, comp):
    n0, n1, n2 = arrs[0].shape
    data = np.ascontiguousarray(np.stack(arrs), dtype=np.float32)
    names = (ctypes.c_char_p * len(arrs))(*[f"f{i}".encode() for i in range(len(arrs))])
    rc = N.lib().od_fields_save(str(path).encode(), data.ctypes.data_as(ctypes.c_void_p), len(arrs), names, n0, n1,
                                n2, chunk, comp.encode())
    assert rc == 0, N.lib().od_state_error()


@pytest.mark.parametrize("shape,chunk", [((20, 36, 52), 16), ((8, 12, 60), 48), ((1, 1, 5), 48), ((49, 3, 2), 48)])
@pytest.mark.parametrize("comp", ["none", "gzip4", "blosc-lz4"])
def test_fields_file_round_trip(tmp_path, shape, chunk, comp):
    rng = np.random.default_rng(sum(shape))
    arrs = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    arrs[1].flat[3] = np.nan
    p = tmp_path / "f.pv.h5"
    save_fields(p, arrs, chunk, comp)
    w = Walker(p.read_bytes())
    assert w.attributes(w.root_ohdr) == {}
    top = w.group_members(w.root_ohdr)
    assert list(top) == ["data"]
    members = w.group_members(top["data"])
    assert sorted(members) == ["f0", "f1", "f2"]
    for i, a in enumerate(arrs):
        info = w.dataset(members[f"f{i}"])
        assert info["dims"] == shape and info["size"] == 4
        if comp == "none":
            assert info["layout"] == 1
        else:
            assert info["cdims"] == tuple(min(chunk, d) for d in shape)
            fids = [f for f, _ in info["filters"]]
            assert fids == ([2, 1] if comp == "gzip4" else [32001])
            if comp == "gzip4":
                assert info["filters"][0][1] == [4] and info["filters"][1][1] == [4]
        b = w.read_array(members[f"f{i}"])
        assert np.array_equal(b, a, equal_nan=True)


def test_fields_file_many_chunks_multilevel_index(tmp_path):
    # 130 chunks of 4^3: more than one leaf of the chunk index (64 per node)
    shape = (8, 4, 260)
    a = np.arange(np.prod(shape), dtype=np.float32).reshape(shape)
    p = tmp_path / "m.pv.h5"
    save_fields(p, [a], 4, "gzip1")
    w = Walker(p.read_bytes())
    m = w.group_members(w.group_members(w.root_ohdr)["data"])
    info = w.dataset(m["f0"])
    assert len(w.chunks(info["btree"], 3)) == 2 * 1 * 65
    assert np.array_equal(w.read_array(m["f0"]), a)


def test_fields_file_rejects_bad_arguments(tmp_path):
    a = np.zeros((2, 2, 2), np.float32)
    names = (ctypes.c_char_p * 1)(b"x")
    L = N.lib()
    assert L.od_fields_save(str(tmp_path / "a.h5").encode(), a.ctypes.data_as(ctypes.c_void_p), 1, names, 2, 2, 2, 0,
                            b"gzip4") != 0
    assert L.od_fields_save(str(tmp_path / "b.h5").encode(), a.ctypes.data_as(ctypes.c_void_p), 1, names, 2, 2, 2, 4,
                            b"gzip0") != 0
    assert "invalid compression" in L.od_state_error().decode()


def xdmf_text(*args):
    L = N.lib()
    n = L.od_xdmf_text(None, 0, *args)
    assert n > 0
    buf = ctypes.create_string_buffer(n + 1)
    assert L.od_xdmf_text(buf, n + 1, *args) == n
    return buf.value.decode()


@pytest.mark.parametrize("case", [
    ("flow_f32_000500.pv.h5", 192, 8, 128, float(np.float32(2 * np.pi)), 2.0, float(np.float32(np.pi)), 500, 0.05),
    ("checkpoint_f64_000003.pv.h5", 32, 32, 32, float(np.float32(2 * np.pi)), float(np.float32(2 * np.pi)),
     float(np.float32(2 * np.pi)), 3, 1.2345678901e-3),
    ("a.pv.h5", 4, 12, 20, 4 * np.pi, 2.0, 4 * np.pi / 3, 0, 0.0),
    ("b.pv.h5", 7, 3, 5, 1e-3, 12345.678, 0.1, 18446744073709551615, 98765.4321),
])
def test_xdmf_text_matches_oracle(case):
    name, npx, npy, npz, lx, ly, lz, step, t = case
    got = xdmf_text(name.encode(), npx, npy, npz, lx, ly, lz, step, t)
    assert got == PF.xdmf_text(name, npx, npy, npz, lx, ly, lz, step, t)


def test_command_line_selection(tmp_path):
    for n in ("flow_f32_000002.h5", "checkpoint_f32_000002.h5", "flow_f32_000001.h5", "flow_f32_000001.pv.h5",
              "notes.txt"):
        (tmp_path / n).write_bytes(b"")
    sel = X.select([str(tmp_path)])
    assert [(f.name, do) for f, do in sel] == [("checkpoint_f32_000002.h5", False), ("flow_f32_000001.h5", True),
                                                ("flow_f32_000002.h5", True)]
    one = X.select([str(tmp_path / "checkpoint_f32_000002.h5")])
    assert [(f.name, do) for f, do in one] == [("checkpoint_f32_000002.h5", True)]
    with pytest.raises(SystemExit):
        X.select([str(tmp_path / "missing.h5")])
    with pytest.raises(SystemExit):
        X.main([])


GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "xdmf_reference.npz"))
GOLDEN_CASES = [eval(c) for c in GOLDEN["cases"]]


@pytest.mark.parametrize("n", range(len(GOLDEN_CASES)))
def test_oracle_pinned_to_the_reference_script(n):
    c = GOLDEN_CASES[n]
    planes = GOLDEN[f"case{n}_planes"]
    f = PF.point_fields(planes, c["nx"], c["ny"], c["nz"])
    assert list(GOLDEN[f"case{n}_names"]) == [f"data/{k}" for k in PF.FIELD_NAMES]
    for k in PF.FIELD_NAMES:
        g = GOLDEN[f"case{n}_{k}"]
        assert g.dtype == np.float32 and f[k].dtype == np.float32
        assert np.array_equal(f[k], g, equal_nan=True), k
        assert str(GOLDEN[f"case{n}_{k}_opts"]) == "[('chunks', (48, 48, 48)), ('compression', 'gzip'), " \
                                                   "('compression_opts', 4), ('shuffle', True)]"
    npx, npy, npz = 4 * c["nx"], 4 * c["ny"], 4 * c["nz"]
    stem = c["name"][:-3]
    assert PF.xdmf_text(stem + ".pv.h5", npx, npy, npz, c["lx"], c["ly"], c["lz"], c["step"], c["t"]) == \
        str(GOLDEN[f"case{n}_xmf"])
    assert str(GOLDEN[f"case{n}_line"]) == (
        f"{c['name']} (step {c['step']}, t={c['t']:.5g}): fields {sorted(PF.FIELD_NAMES)} -> {stem}.pv.h5 + "
        f"{stem}.xmf\n")


@pytest.mark.parametrize("n", range(len(GOLDEN_CASES)))
def test_xdmf_text_matches_the_reference_script(n):
    c = GOLDEN_CASES[n]
    stem = c["name"][:-3]
    got = xdmf_text((stem + ".pv.h5").encode(), 4 * c["nx"], 4 * c["ny"], 4 * c["nz"], c["lx"], c["ly"], c["lz"],
                    c["step"], c["t"])
    assert got == str(GOLDEN[f"case{n}_xmf"])
