"""State files (src/io.rs): lossless round trips for every compression,
attribute layout, validation errors with the reference's messages, files
cross-checked by an independent reader, and Blosc frames in the split-stream
layout c-blosc writes by default. CPU only (the library is loaded, no
device work)."""

import os
import struct

import numpy as np
import pytest

from opendynamo_b200 import _native as N
from opendynamo_b200 import state_io as S

from h5walk import Walker, blosc_encode_split

COMPRESSIONS = ["none", "gzip1", "gzip4", "gzip9", "blosc-lz4", "blosc-zstd"]


def planes(nx, ny, nz, dtype, seed=0):
    rng = np.random.default_rng(seed)
    npts = nx * ny * nz * 64
    a = np.empty((5, npts), dtype=dtype)
    a[0] = 1 + 0.05 * rng.standard_normal(npts)
    a[1:4] = 0.2 * rng.standard_normal((3, npts))
    a[4] = 2.5 + 0.1 * rng.standard_normal(npts)
    return a


@pytest.mark.parametrize("comp", COMPRESSIONS)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_round_trip_bitwise(tmp_path, comp, dtype):
    # 17x16x16 elements: 278 528 points per plane, two chunks, the last partial
    nx, ny, nz = 17, 16, 16
    a = planes(nx, ny, nz, dtype)
    a[2, 5] = np.nan
    a[3, 7] = -0.0
    a[4, 9] = np.inf
    kind = "f64" if dtype == np.float64 else "f32"
    p = str(tmp_path / f"s_{kind}_{comp}.h5")
    S.save_state(p, a, nx, ny, nz, step=123456, t=0.0123, lx=2 * np.pi, ly=2.0, lz=np.pi, compression=comp)
    b, step, t = S.load_state(p, nx, ny, nz, kind)
    assert (step, t) == (123456, 0.0123)
    assert b.dtype == dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("comp", COMPRESSIONS)
def test_independent_reader(tmp_path, comp):
    nx, ny, nz = 17, 16, 16
    a = planes(nx, ny, nz, np.float32, seed=3)
    p = str(tmp_path / "w.h5")
    S.save_state(p, a, nx, ny, nz, step=7, t=0.5, lx=2 * np.pi, ly=2.0, lz=np.pi, compression=comp)
    data = open(p, "rb").read()
    w = Walker(data)
    assert w.eof == len(data)
    assert (w.leaf_k, w.internal_k) == (4, 16)
    attrs = w.attributes(w.root_ohdr)
    assert {k: v[2] for k, v in attrs.items()} == {
        "nx": 17, "ny": 16, "nz": 16, "fr_order": 3, "step": 7, "t": 0.5,
        "lx": float(np.float32(2 * np.pi)), "ly": 2.0, "lz": float(np.float32(np.pi)), "u_real": "f32"}
    assert attrs["u_real"][:2] == (3, 3)  # fixed 3-byte string
    top = w.group_members(w.root_ohdr)
    assert list(top) == ["data"]
    members = w.group_members(top["data"])
    assert sorted(members) == sorted(S.VAR_NAMES)
    for v, name in enumerate(S.VAR_NAMES):
        info = w.dataset(members[name])
        assert info["n"] == nx * ny * nz * 64 and info["size"] == 4
        if comp == "none":
            assert info["layout"] == 1 and not info["filters"]
        else:
            assert info["layout"] == 2 and info["chunk"] == 1 << 18 and info["esize"] == 4
            ids = [f[0] for f in info["filters"]]
            assert ids == ([2, 1] if comp.startswith("gzip") else [32001])
            if comp.startswith("gzip"):
                assert info["filters"][1][1] == [int(comp[4:])]
            else:
                cv = info["filters"][0][1]
                assert cv[2:] == [4, 4 << 18, 9 if comp == "blosc-lz4" else 5, 1, 1 if comp == "blosc-lz4" else 5]
        raw = w.read_plane(members[name])
        assert raw == a[v].tobytes()


def test_attributes_and_info(tmp_path):
    a = planes(2, 3, 4, np.float64)
    p = str(tmp_path / "i.h5")
    S.save_state(p, a, 2, 3, 4, step=2**40 + 5, t=-1.5, compression="none")
    info = S.state_info(p)
    assert info == {"nx": 2, "ny": 3, "nz": 4, "fr_order": 3, "step": 2**40 + 5, "t": -1.5,
                    "lx": float(np.float32(4 * np.pi)), "ly": 2.0, "lz": float(np.float32(4 * np.pi / 3)),
                    "u_real": "f64"}


def test_file_name():
    assert S.file_name("out", "flow", "f32", 42) == os.path.join("out", "flow_f32_000042.h5")
    assert S.file_name("o", "checkpoint", "f64", 1234567) == os.path.join("o", "checkpoint_f64_1234567.h5")


def test_validation_messages(tmp_path):
    a = planes(3, 2, 2, np.float32)
    p = str(tmp_path / "v.h5")
    S.save_state(p, a, 3, 2, 2, compression="gzip1")
    with pytest.raises(N.OdError, match=r"initial_state mesh 3x2x2 does not match config 3x2x3; refusing to load"):
        S.load_state(p, 3, 2, 3, "f32")
    with pytest.raises(N.OdError, match=r"initial_state u_real 'f32' does not match the configured pipeline "
                                        r"\('f64'\); refusing to load"):
        S.load_state(p, 3, 2, 2, "f64")
    with pytest.raises(N.OdError, match="initial_state file not found"):
        S.load_state(str(tmp_path / "missing.h5"), 3, 2, 2, "f32")
    # fr_order attribute rewritten to 4 (name padded to 16, datatype 16, dataspace 8)
    data = bytearray(open(p, "rb").read())
    at = data.index(b"fr_order\0")
    assert struct.unpack_from("<Q", data, at + 40)[0] == 3
    struct.pack_into("<Q", data, at + 40, 4)
    q = str(tmp_path / "fr.h5")
    open(q, "wb").write(bytes(data))
    with pytest.raises(N.OdError, match="initial_state fr_order 4 != configured FR_ORDER 3"):
        S.load_state(q, 3, 2, 2, "f32")


def test_invalid_compression(tmp_path):
    a = planes(1, 1, 1, np.float32)
    with pytest.raises(N.OdError, match=r"invalid compression 'gzip0': expected \"none\", \"gzip1\"..\"gzip9\", "
                                        r"\"blosc-lz4\" or \"blosc-zstd\""):
        S.save_state(str(tmp_path / "c.h5"), a, 1, 1, 1, compression="gzip0")
    assert not os.path.exists(tmp_path / "c.h5")


@pytest.mark.parametrize("cut", [0, 10, 95, 200, 1000, -100])
def test_truncated_or_corrupt_file_fails_cleanly(tmp_path, cut):
    a = planes(2, 2, 2, np.float32)
    p = str(tmp_path / "t.h5")
    S.save_state(p, a, 2, 2, 2, compression="gzip1")
    data = open(p, "rb").read()
    q = str(tmp_path / "cut.h5")
    open(q, "wb").write(data[:cut] if cut >= 0 else data[:cut])
    with pytest.raises(N.OdError):
        S.load_state(q, 2, 2, 2, "f32")
    # flipped bytes inside the compressed chunks: an error or different values, never a crash
    bad = bytearray(data)
    for k in range(len(bad) // 2, len(bad) // 2 + 64):
        bad[k] ^= 0x5A
    open(q, "wb").write(bytes(bad))
    try:
        S.load_state(q, 2, 2, 2, "f32")
    except N.OdError:
        pass


@pytest.mark.parametrize("codec", ["lz4", "zstd"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_blosc_split_stream_frames(tmp_path, codec, dtype):
    """Chunks rewritten as c-blosc's default split-stream frames (one stream
    per byte of the type, as c-blosc 1.x writes for typesize <= 16) load to
    the same values."""
    nx, ny, nz = 17, 16, 16
    a = planes(nx, ny, nz, dtype, seed=5)
    p = str(tmp_path / "b.h5")
    S.save_state(p, a, nx, ny, nz, compression=f"blosc-{codec}")
    data = bytearray(open(p, "rb").read())
    w = Walker(bytes(data))
    members = w.group_members(w.group_members(w.root_ohdr)["data"])
    es = np.dtype(dtype).itemsize
    for name in S.VAR_NAMES:
        info = w.dataset(members[name])
        for off, addr, size, mask, keypos in w.chunks(info["btree"]):
            chunk = np.zeros(1 << 18, dtype=dtype)
            v = S.VAR_NAMES.index(name)
            cnt = min(1 << 18, a.shape[1] - off)
            chunk[:cnt] = a[v, off:off + cnt]
            frame = blosc_encode_split(chunk.tobytes(), es, codec)
            assert frame[2] & 0x10 == 0
            new_addr = len(data)
            data += frame
            while len(data) % 8:
                data.append(0)
            struct.pack_into("<I", data, keypos, len(frame))
            struct.pack_into("<Q", data, keypos + 24, new_addr)
    struct.pack_into("<Q", data, 40, len(data))  # end-of-file address
    q = str(tmp_path / "split.h5")
    open(q, "wb").write(bytes(data))
    b, _, _ = S.load_state(q, nx, ny, nz, "f64" if dtype == np.float64 else "f32")
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
