"""Particle snapshots in the reference's esdat format (HDF5), for restarts
from and to a run of the reference.

The reference writes one file per rank, ./SNAPSHOT1/esdat%04d.h5, in
save_esdat (src/io/snap.F90:203-356), and reads it back at a restart in
inipcl (src/pcl/inipcl.F90:362-425).  Its datasets:

    nnode  int32 [1]      (rank 0 only)   number of ranks
    nspec  int32 [1]                      species
    np     int32 [nspec]                  particles per species
    npc    int32 [1]                      bodies
    sdoms  int32 [3][2]                   the rank's subdomain bounds (lower, upper per axis)
    rens   float64 [4]                    renr, renv, renrho, renq (unit factors of rescal)
    px py pz pvx pvy pvz  float64 [n]     particle positions and velocities (internal units)
    pres   int32 [n]                      preside
    pis    int32 [n]                      species (1-based)
    rhobk  float64 [nz+1][ny+1][nx+1]     rhobk(1,0:nx,0:ny,0:nz,3), the accumulated background charge
    chgacm float64 [npc]                  accumulated body charge

(shapes in HDF5's C order: the Fortran API reverses the dimensions).  The
particles are those of pbuf(1:pbase(3)) in buffer order, species after
species.

No HDF5 library or binding exists in this environment, so this module
writes and reads the subset of the HDF5 file format (version 0 superblock)
that the HDF5 library produces for these files with its default
properties: a root group stored as a symbol table (a version 1 B-tree of
group nodes over symbol table nodes, names in a local heap), version 1
object headers, and datasets with contiguous storage of little-endian
32-bit integers or IEEE 754 doubles.  The reader also follows object header
continuation messages and compact storage, and reads B-trees of any depth;
chunked or filtered datasets are refused with a clear error.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

from .emses import PARTICLE_DTYPE

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4        # group leaf node K: a symbol table node holds 2K entries
INTERNAL_K = 16   # group internal node K: a B-tree node holds 2K children

# header message types
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL_OLD, MSG_FILL = 0x0000, 0x0001, 0x0003, 0x0004, 0x0005
MSG_LAYOUT, MSG_CONTINUATION, MSG_SYMBOL_TABLE = 0x0008, 0x0010, 0x0011


class SnapshotError(ValueError):
    pass


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ---------------------------------------------------------------- writing
def _datatype_msg(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    if dt == np.dtype("<i4"):
        # class 0 (fixed point), version 1; little endian, signed; offset 0, precision 32
        return struct.pack("<B3BI", 0x10, 0x08, 0, 0, 4) + struct.pack("<HH", 0, 32)
    if dt == np.dtype("<f8"):
        # class 1 (floating point), version 1; little endian, mantissa normalised
        # (msb implied), sign at bit 63; exponent 52..62 (bias 1023), mantissa 0..51
        return (struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) +
                struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023))
    raise SnapshotError(f"no esdat datatype for {dt}")


def _dataspace_msg(shape) -> bytes:
    # version 1: rank, no maximum dimensions
    out = struct.pack("<BBBB4x", 1, len(shape), 0, 0)
    for d in shape:
        out += struct.pack("<Q", int(d))
    return out


def _fill_msg() -> bytes:
    # version 2: allocation late, fill value written when set, no fill value defined
    return struct.pack("<BBBB", 2, 2, 2, 0)


def _layout_msg(addr: int, size: int) -> bytes:
    # version 3, contiguous
    return struct.pack("<BBQQ", 3, 1, addr, size)


def _object_header(messages: list[tuple[int, bytes]]) -> bytes:
    """Version 1 object header: 16-byte prefix, then the messages, each padded
    to a multiple of 8 bytes."""
    body = b""
    for mtype, data in messages:
        n = _pad8(len(data))
        body += struct.pack("<HHB3x", mtype, n, 0) + data + b"\x00" * (n - len(data))
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body


class _Writer:
    def __init__(self):
        self.buf = bytearray()

    def alloc(self, data: bytes, align: int = 8) -> int:
        while len(self.buf) % align:
            self.buf.append(0)
        addr = len(self.buf)
        self.buf += data
        return addr


def write_h5(path, datasets: dict) -> None:
    """Writes `datasets` (name -> numpy array of int32 or float64, C order)
    as an HDF5 file whose root group holds them."""
    names = sorted(datasets)  # the symbol tables keep names in strcmp order
    for nm in names:
        if not nm or "/" in nm or not nm.isascii():
            raise SnapshotError(f"bad dataset name {nm!r}")
    w = _Writer()
    w.alloc(b"\x00" * 96)  # the superblock, filled in at the end
    # local heap of the root group: "" at offset 0, then the names
    heap = bytearray(b"\x00" * 8)
    name_off = {}
    for nm in names:
        name_off[nm] = len(heap)
        raw = nm.encode() + b"\x00"
        heap += raw + b"\x00" * (_pad8(len(raw)) - len(raw))
    heap_data = w.alloc(bytes(heap))
    heap_hdr = w.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), UNDEF, heap_data))
    # datasets: data, then object header
    headers = {}
    for nm in names:
        a = np.ascontiguousarray(datasets[nm])
        if a.dtype == np.int32 or a.dtype == np.float64:
            a = a.astype(a.dtype.newbyteorder("<"), copy=False)
        else:
            raise SnapshotError(f"{nm}: dtype {a.dtype} (int32 or float64 only)")
        shape = a.shape if a.ndim else (1,)
        data_addr = w.alloc(a.tobytes(), 16) if a.size else UNDEF
        hdr = _object_header([(MSG_DATASPACE, _dataspace_msg(shape)), (MSG_DATATYPE, _datatype_msg(a.dtype)),
                              (MSG_FILL, _fill_msg()), (MSG_LAYOUT, _layout_msg(data_addr, a.nbytes))])
        headers[nm] = w.alloc(hdr)
    # symbol table nodes of 2K entries, and the B-tree (one level) over them
    per = 2 * LEAF_K
    groups = [names[i:i + per] for i in range(0, len(names), per)] or [[]]
    if len(groups) > 2 * INTERNAL_K:
        raise SnapshotError("too many datasets for a one-level group B-tree")
    snods = []
    for grp in groups:
        ent = b""
        for nm in grp:
            ent += struct.pack("<QQII16x", name_off[nm], headers[nm], 0, 0)
        ent += b"\x00" * (40 * per - len(ent))
        snods.append(w.alloc(b"SNOD" + struct.pack("<BBH", 1, 0, len(grp)) + ent))
    # keys: key 0 the empty name, key i+1 the last name of child i
    keys = [0] + [name_off[g[-1]] if g else 0 for g in groups]
    tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(groups), UNDEF, UNDEF)
    for i, child in enumerate(snods):
        tree += struct.pack("<QQ", keys[i], child)
    tree += struct.pack("<Q", keys[len(snods)])
    tree += b"\x00" * ((2 * INTERNAL_K - len(snods)) * 16)  # the node's full size
    btree = w.alloc(tree)
    root = w.alloc(_object_header([(MSG_SYMBOL_TABLE, struct.pack("<QQ", btree, heap_hdr))]))
    eof = len(w.buf)
    sb = (SIGNATURE + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0) + struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
          + struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
          + struct.pack("<QQII", 0, root, 1, 0) + struct.pack("<QQ", btree, heap_hdr))
    assert len(sb) == 96
    w.buf[0:96] = sb
    Path(path).write_bytes(bytes(w.buf))


# ---------------------------------------------------------------- reading
class _File:
    def __init__(self, data: bytes):
        self.d = data

    def u(self, fmt: str, off: int):
        return struct.unpack_from("<" + fmt, self.d, off)

    def cstr(self, off: int) -> str:
        end = self.d.index(b"\x00", off)
        return self.d[off:end].decode()


def _messages(f: _File, addr: int):
    """(type, data offset, size) of every message of a version 1 object
    header, following continuation messages."""
    ver, _, nmsg, _refs, size = f.u("BBHII", addr)
    if ver != 1:
        raise SnapshotError(f"object header version {ver} at {addr} (version 1 only)")
    blocks = [(addr + 16, size)]
    out = []
    while blocks and len(out) < nmsg:
        start, size = blocks.pop(0)
        pos = start
        while pos + 8 <= start + size and len(out) < nmsg:
            mtype, msize, _flags = f.u("HHB", pos)
            out.append((mtype, pos + 8, msize))
            if mtype == MSG_CONTINUATION:
                caddr, clen = f.u("QQ", pos + 8)
                blocks.append((caddr, clen))
            pos += 8 + msize
    return out


def _dtype(f: _File, off: int) -> np.dtype:
    cv, b0, b1, b2, size = f.u("B3BI", off)
    cls, ver = cv & 0x0F, cv >> 4
    big = bool(b0 & 1)
    if cls == 0:
        signed = bool(b0 & 0x08)
        return np.dtype(("i" if signed else "u") + str(size)).newbyteorder(">" if big else "<")
    if cls == 1 and size in (4, 8):
        return np.dtype("f" + str(size)).newbyteorder(">" if big else "<")
    raise SnapshotError(f"datatype class {cls} version {ver} size {size} not supported")


def _dataspace(f: _File, off: int) -> tuple:
    ver, rank, flags = f.u("BBB", off)
    if ver == 1:
        dims = f.u("Q" * rank, off + 8)
    elif ver == 2:
        dims = f.u("Q" * rank, off + 4)
    else:
        raise SnapshotError(f"dataspace version {ver}")
    return tuple(int(x) for x in dims)


def _read_dataset(f: _File, addr: int) -> np.ndarray:
    shape, dt, layout = None, None, None
    for mtype, off, size in _messages(f, addr):
        if mtype == MSG_DATASPACE:
            shape = _dataspace(f, off)
        elif mtype == MSG_DATATYPE:
            dt = _dtype(f, off)
        elif mtype == MSG_LAYOUT:
            ver = f.u("B", off)[0]
            if ver == 3:
                cls = f.u("B", off + 1)[0]
                if cls == 1:
                    layout = ("contiguous",) + f.u("QQ", off + 2)
                elif cls == 0:
                    n = f.u("H", off + 2)[0]
                    layout = ("compact", off + 4, n)
                else:
                    raise SnapshotError("chunked datasets are not supported")
            elif ver in (1, 2):
                rank, cls = f.u("BB", off + 1)
                if cls != 1:
                    raise SnapshotError(f"layout class {cls} (contiguous only)")
                layout = ("contiguous", f.u("Q", off + 8)[0], None)
            else:
                raise SnapshotError(f"layout message version {ver}")
    if shape is None or dt is None or layout is None:
        raise SnapshotError(f"object at {addr} is not a dataset")
    n = int(np.prod(shape)) if shape else 1
    if layout[0] == "compact":
        raw = f.d[layout[1]:layout[1] + layout[2]]
    else:
        daddr = layout[1]
        if daddr == UNDEF:
            raw = b"\x00" * (n * dt.itemsize)
        else:
            raw = f.d[daddr:daddr + n * dt.itemsize]
    a = np.frombuffer(raw, dtype=dt, count=n).reshape(shape)
    return a.astype(dt.newbyteorder("="))


def _group_entries(f: _File, btree: int, heap: int) -> dict:
    sig, ver, _r, dsize, _free, data = f.u("4sB3sQQQ", heap)
    if sig != b"HEAP":
        raise SnapshotError("bad local heap")
    out = {}

    def node(addr):
        sig, ntype, level, used = f.u("4sBBH", addr)
        if sig != b"TREE" or ntype != 0:
            raise SnapshotError("bad group B-tree node")
        pos = addr + 8 + 16
        for i in range(used):
            child = f.u("Q", pos + 8)[0]
            if level > 0:
                node(child)
            else:
                s, _v, _r, nsym = f.u("4sBBH", child)
                if s != b"SNOD":
                    raise SnapshotError("bad symbol table node")
                for e in range(nsym):
                    name_off, ohdr = f.u("QQ", child + 8 + 40 * e)
                    out[f.cstr(data + name_off)] = ohdr
            pos += 16

    node(btree)
    return out


def read_h5(path) -> dict:
    """The datasets of the root group of an HDF5 file (superblock version 0
    or 1, symbol-table groups), as numpy arrays."""
    f = _File(Path(path).read_bytes())
    if f.d[:8] != SIGNATURE:
        raise SnapshotError("not an HDF5 file")
    ver = f.d[8]
    if ver not in (0, 1):
        raise SnapshotError(f"superblock version {ver} (0 or 1 only)")
    so, sl = f.d[13], f.d[14]
    if so != 8 or sl != 8:
        raise SnapshotError("8-byte offsets and lengths only")
    pos = 24 + (4 if ver == 1 else 0) + 32  # flags, (indexed storage K), addresses
    _name, root, cache, _r = f.u("QQII", pos)
    btree, heap = f.u("QQ", pos + 24)
    if cache != 1:
        for mtype, off, size in _messages(f, root):
            if mtype == MSG_SYMBOL_TABLE:
                btree, heap = f.u("QQ", off)
                break
        else:
            raise SnapshotError("root group is not a symbol table")
    return {name: _read_dataset(f, addr) for name, addr in _group_entries(f, btree, heap).items()}


# ---------------------------------------------------------------- esdat
def esdat_name(rank: int = 0) -> str:
    return f"esdat{rank:04d}.h5"


def write_esdat(path, pbuf: np.ndarray, totalp, rens, sdoms=None, rhobk=None, chgacm=None, nnode: int | None = 1,
                nspec: int | None = None) -> None:
    """save_esdat (snap.F90:203-356) for one rank: pbuf the particle records
    (species segments of totalp, buffer order), rens = (renr, renv, renrho,
    renq), sdoms[3][2] the subdomain bounds (lower, upper) per axis, rhobk the
    background charge on the nodes 0..n as numpy (z, y, x), chgacm per
    body.  nnode is written by rank 0 only (None leaves it out)."""
    totalp = np.asarray(totalp, dtype=np.int64)
    ns = int(nspec if nspec is not None else totalp.size)
    n = int(totalp[:ns].sum())
    p = np.ascontiguousarray(pbuf[:n])
    if p.dtype != PARTICLE_DTYPE:
        raise SnapshotError("pbuf must hold emsesg particle records")
    d = {"nspec": np.array([ns], np.int32), "np": totalp[:ns].astype(np.int32),
         "npc": np.array([0 if chgacm is None else len(chgacm)], np.int32),
         "sdoms": np.zeros((3, 2), np.int32) if sdoms is None else np.asarray(sdoms, np.int32).reshape(3, 2),
         "rens": np.asarray(rens, np.float64).reshape(4),
         "px": p["x"].astype(np.float64), "py": p["y"].astype(np.float64), "pz": p["z"].astype(np.float64),
         "pvx": p["vx"].astype(np.float64), "pvy": p["vy"].astype(np.float64), "pvz": p["vz"].astype(np.float64),
         "pres": p["preside"].astype(np.int32), "pis": p["spec"].astype(np.int32),
         "chgacm": np.zeros(0, np.float64) if chgacm is None else np.asarray(chgacm, np.float64)}
    if nnode is not None:
        d["nnode"] = np.array([nnode], np.int32)
    if rhobk is not None:
        d["rhobk"] = np.ascontiguousarray(rhobk, dtype=np.float64)
    write_h5(path, d)


def read_esdat(path) -> dict:
    """The restart read of inipcl (inipcl.F90:362-425): returns
    {"pbuf": records (pid 0, nid 0), "totalp": per species, "rens": ...} plus
    every other dataset of the file as it is."""
    d = read_h5(path)
    for key in ("np", "px", "py", "pz", "pvx", "pvy", "pvz", "pres", "pis"):
        if key not in d:
            raise SnapshotError(f"esdat file without {key}")
    totalp = d["np"].astype(np.int64)
    n = int(totalp.sum())
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    for f, k in (("x", "px"), ("y", "py"), ("z", "pz"), ("vx", "pvx"), ("vy", "pvy"), ("vz", "pvz")):
        if d[k].size != n:
            raise SnapshotError(f"{k}: {d[k].size} values for {n} particles")
        p[f] = d[k]
    p["preside"] = d["pres"][:n]
    p["spec"] = d["pis"][:n]
    out = dict(d)
    out["pbuf"] = p
    out["totalp"] = totalp
    return out


def save(g, path, rens, fx: bool = True, rank: int = 0, nnode: int | None = 1) -> None:
    """Writes the particles of the context g (with fx, the FP32 form's state
    as FP64 records) with its background charge rhobk on the nodes 0..n and
    the bodies' chgacm as esdat; rens = (renr, renv, renrho, renq) of the
    run's units."""
    cfg = g.cfg
    if fx:
        g.fx_store()
    p, tp = g.download_particles()
    rb = g.download_field("rhobk")[1:cfg.nz + 2, 1:cfg.ny + 2, 1:cfg.nx + 2, 0]
    chg = g.get_counters().as_dict()["chgacm"][:cfg.npc, 0]
    sd = [[0, cfg.nx], [0, cfg.ny], [0, cfg.nz]]
    write_esdat(path, p, tp[:cfg.nspec], rens, sdoms=sd, rhobk=rb, chgacm=chg, nnode=nnode if rank == 0 else None)


def load(g, path, fx: bool = True) -> dict:
    """Starts the context g from an esdat file (inipcl's restart read): its
    particles become g's, converted into the FP32 form when fx; returns the
    file's datasets."""
    d = read_esdat(path)
    p = d["pbuf"].copy()
    p["nid"] = 0
    p["pid"] = 0
    g.upload_particles(p, d["totalp"])
    if fx:
        g.fx_load()
    return d
