"""Snapshot interop: the esdat HDF5 files of save_esdat / inipcl
(src/io/snap.F90:203-356, src/pcl/inipcl.F90:362-425) written and read by
ctca_b200.snapshot, bit for bit, and the file's HDF5 structures checked
against the format specification's layout (superblock version 0, symbol
table root group, version 1 object headers, contiguous data)."""
import struct

import numpy as np
import pytest

from ctca_b200 import inputs, snapshot
from ctca_b200.emses import PARTICLE_DTYPE


def records(n, seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    for f in ("x", "y", "z"):
        p[f] = rng.random(n) * 32
    for f in ("vx", "vy", "vz"):
        p[f] = rng.normal(0, 0.01, n)
    p["preside"] = rng.integers(-2, 2, n)
    p["spec"] = np.where(np.arange(n) < n // 2, 1, 2)
    return p


def test_h5_round_trip_of_every_kind(tmp_path):
    d = {f"d{i:02d}": np.arange(i + 1, dtype=np.float64) * np.pi for i in range(11)}
    d["ints"] = np.array([[1, -2, 3], [4, 5, -6]], dtype=np.int32)
    d["cube"] = np.random.default_rng(1).random((3, 4, 5))
    d["empty"] = np.zeros(0, np.float64)
    path = tmp_path / "t.h5"
    snapshot.write_h5(path, d)
    back = snapshot.read_h5(path)
    assert sorted(back) == sorted(d)
    for k, v in d.items():
        assert back[k].dtype == v.dtype and back[k].shape == v.shape
        assert np.array_equal(back[k].view(np.uint8), v.view(np.uint8)), k


def test_h5_structures(tmp_path):
    path = tmp_path / "s.h5"
    snapshot.write_h5(path, {"a": np.ones(3), "b": np.zeros(2, np.int32)})
    raw = path.read_bytes()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n"
    ver, fsver, rootver, _, shver, so, sl, _ = raw[8:16]
    assert (ver, so, sl) == (0, 8, 8)
    leaf_k, int_k, flags = struct.unpack_from("<HHI", raw, 16)
    assert (leaf_k, int_k) == (4, 16)
    base, free, eof, drv = struct.unpack_from("<QQQQ", raw, 24)
    assert base == 0 and eof == len(raw) and free == drv == 0xFFFFFFFFFFFFFFFF
    _, root, cache, _, btree, heap = struct.unpack_from("<QQIIQQ", raw, 56)
    assert cache == 1 and raw[btree:btree + 4] == b"TREE" and raw[heap:heap + 4] == b"HEAP"
    hver, _, nmsg, refs, size = struct.unpack_from("<BBHII", raw, root)
    assert (hver, nmsg, refs) == (1, 1, 1)
    mtype, msize = struct.unpack_from("<HH", raw, root + 16)
    assert (mtype, msize) == (0x0011, 16)
    assert struct.unpack_from("<QQ", raw, root + 24) == (btree, heap)


def test_h5_rejects_what_it_cannot_read(tmp_path):
    path = tmp_path / "x.h5"
    path.write_bytes(b"not hdf5" * 20)
    with pytest.raises(snapshot.SnapshotError):
        snapshot.read_h5(path)
    with pytest.raises(snapshot.SnapshotError):
        snapshot.write_h5(tmp_path / "y.h5", {"f32": np.ones(2, np.float32)})


def test_esdat_round_trip(tmp_path):
    p = records(1000)
    tp = np.array([500, 500])
    u = inputs.units()
    rens = (1.0, u["renv"], u["renrho"], u["renq"])
    rhobk = np.random.default_rng(2).random((9, 8, 7))
    path = tmp_path / snapshot.esdat_name(0)
    snapshot.write_esdat(path, p, tp, rens, sdoms=[[0, 6], [0, 7], [0, 8]], rhobk=rhobk, chgacm=[0.5, -0.25])
    d = snapshot.read_esdat(path)
    assert np.array_equal(d["totalp"], tp)
    for f in ("x", "y", "z", "vx", "vy", "vz", "preside", "spec"):
        assert np.array_equal(d["pbuf"][f], p[f]), f
    assert np.array_equal(d["rens"], np.array(rens))
    assert np.array_equal(d["rhobk"], rhobk)
    assert np.array_equal(d["chgacm"], [0.5, -0.25])
    assert d["sdoms"].tolist() == [[0, 6], [0, 7], [0, 8]]
    assert int(d["nspec"][0]) == 2 and int(d["npc"][0]) == 2 and int(d["nnode"][0]) == 1
    assert sorted(d) == sorted(["nnode", "nspec", "np", "npc", "sdoms", "rens", "px", "py", "pz", "pvx", "pvy",
                                "pvz", "pres", "pis", "rhobk", "chgacm", "pbuf", "totalp"])
