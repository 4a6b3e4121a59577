"""Mesh and state IO: XDMF (XML light data) with HDF5 or raw binary heavy data.

The reference reads its example meshes with DOLFINx / adios4dolfinx (``io_utils/mesh.py``,
``examples/*/Relax.py``) and writes states as XDMF (``io.XDMFFile``) and ADIOS2 ``.bp``
checkpoints (``gpu/solvers/llg_module_GPU.py:1948-1956``).  Neither DOLFINx nor h5py is
available here, so this module reads the files itself:

* ``read_hdf5(path)``: the datasets of an HDF5 file written with the library defaults of
  the format's first version (superblock version 0, symbol-table groups: a version-1 B-tree
  with SNOD nodes and a local heap; version-1 object headers with continuation blocks;
  contiguous, compact or chunked datasets (version-1 B-tree chunk index) of little- or
  big-endian integers and floats, with the deflate, shuffle and fletcher32 filters).  This
  is what meshio writes for the examples' ``*.h5`` files (gzip-compressed chunks).  Later
  superblock versions and other filters raise ``NotImplementedError``.
* ``read_xdmf_mesh(path)``: points, tetrahedra and cell attributes of an XDMF 2/3 file whose
  DataItems are ``Format="HDF"`` (file.h5:/path), ``"XML"`` (inline) or ``"Binary"`` (raw).
* ``XDMFWriter``: a mesh plus a time series of nodal vector fields as XDMF with raw binary
  heavy data (one little-endian file per array), readable by ParaView and by
  ``read_xdmf_mesh`` / ``read_xdmf_series``.
* ``write_mesh`` / ``write_function`` / ``read_mesh`` / ``read_function``: checkpoints for a
  restart, with adios4dolfinx's call names, in this module's own directory format (ADIOS2 BP
  itself is not part of this build).
"""
from __future__ import annotations

import struct
import xml.etree.ElementTree as ET
import zlib
from pathlib import Path

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class _H5:
    def __init__(self, path):
        self.path = str(path)
        self.b = Path(path).read_bytes()
        b = self.b
        if b[:8] != b"\x89HDF\r\n\x1a\n":
            raise ValueError(f"{path}: not an HDF5 file")
        ver = b[8]
        if ver not in (0, 1):
            raise NotImplementedError(f"{path}: HDF5 superblock version {ver} is not supported")
        self.so, self.sl = b[13], b[14]
        if self.so != 8 or self.sl != 8:
            raise NotImplementedError("only 8-byte offsets and lengths are supported")
        p = 24 + (4 if ver == 1 else 0)
        self.base = self.u64(p)
        root = p + 32  # base, free space, end of file, driver info
        self.root_header = self.u64(root + 8)

    def u8(self, p):
        return self.b[p]

    def u16(self, p):
        return struct.unpack_from("<H", self.b, p)[0]

    def u32(self, p):
        return struct.unpack_from("<I", self.b, p)[0]

    def u64(self, p):
        return struct.unpack_from("<Q", self.b, p)[0]

    # ---------------------------------------------------------------- object headers
    def messages(self, addr):
        """(type, data offset, size) of every message of a version-1 object header."""
        a = self.base + addr
        if self.u8(a) != 1:
            raise NotImplementedError("only version-1 object headers are supported")
        nmsg = self.u16(a + 2)
        size = self.u32(a + 8)
        blocks = [(a + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(out) < nmsg:
                mtype, msize = self.u16(p), self.u16(p + 2)
                out.append((mtype, p + 8, msize))
                if mtype == 0x10:  # continuation
                    blocks.append((self.base + self.u64(p + 8), self.u64(p + 16)))
                p += 8 + msize
        return out

    # ---------------------------------------------------------------- groups
    def group_links(self, header_addr):
        btree = heap = None
        for t, p, _ in self.messages(header_addr):
            if t == 0x11:  # symbol table message
                btree, heap = self.u64(p), self.u64(p + 8)
        if btree is None:
            raise NotImplementedError("only symbol-table groups are supported")
        return self._btree_links(btree, heap)

    def _heap_name(self, heap, off):
        h = self.base + heap
        if self.b[h:h + 4] != b"HEAP":
            raise ValueError("bad local heap")
        data = self.base + self.u64(h + 24)
        end = self.b.index(b"\0", data + off)
        return self.b[data + off:end].decode()

    def _btree_links(self, node, heap):
        a = self.base + node
        if self.b[a:a + 4] != b"TREE":
            raise ValueError("bad B-tree node")
        level, used = self.u8(a + 5), self.u16(a + 6)
        p = a + 24 + 8  # first key
        links = {}
        for _ in range(used):
            child = self.u64(p)
            if level > 0:
                links.update(self._btree_links(child, heap))
            else:
                s = self.base + child
                if self.b[s:s + 4] != b"SNOD":
                    raise ValueError("bad symbol-table node")
                for k in range(self.u16(s + 6)):
                    e = s + 8 + 40 * k
                    links[self._heap_name(heap, self.u64(e))] = self.u64(e + 8)
            p += 16
        return links

    # ---------------------------------------------------------------- datasets
    def _filters(self, p):
        v, nf = self.u8(p), self.u8(p + 1)
        q = p + (8 if v == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self.u16(q)
            if v == 1 or fid >= 256:
                nlen = self.u16(q + 2)
                flags, nval = self.u16(q + 4), self.u16(q + 6)
                q += 8 + ((nlen + 7) // 8 * 8 if v == 1 else nlen)
            else:
                flags, nval = self.u16(q + 2), self.u16(q + 4)
                q += 6
            vals = [self.u32(q + 4 * i) for i in range(nval)]
            q += 4 * nval + (4 if v == 1 and nval % 2 else 0)
            out.append((fid, flags, vals))
        return out

    def _chunks(self, node, ndl, out):
        a = self.base + node
        if self.b[a:a + 4] != b"TREE" or self.u8(a + 4) != 1:
            raise ValueError("bad chunk B-tree node")
        level, used = self.u8(a + 5), self.u16(a + 6)
        p = a + 24
        ks = 8 + 8 * ndl
        for _ in range(used):
            size, mask = self.u32(p), self.u32(p + 4)
            offs = [self.u64(p + 8 + 8 * i) for i in range(ndl)]
            child = self.u64(p + ks)
            if level > 0:
                self._chunks(child, ndl, out)
            else:
                out.append((offs, size, mask, child))
            p += ks + 8
        return out

    def _unfilter(self, raw, filters, mask, esize):
        for k in range(len(filters) - 1, -1, -1):
            fid = filters[k][0]
            if mask & (1 << k):
                continue
            if fid == 1:
                raw = zlib.decompress(raw)
            elif fid == 2:
                n = len(raw) // esize
                raw = np.frombuffer(raw, dtype=np.uint8, count=n * esize).reshape(esize, n).T.tobytes() + \
                    raw[n * esize:]
            elif fid == 3:
                raw = raw[:-4]
            else:
                raise NotImplementedError(f"HDF5 filter {fid} is not supported")
        return raw

    def dataset(self, header_addr):
        dims = dtype = None
        layout = None
        filters = []
        for t, p, size in self.messages(header_addr):
            if t == 0x01:  # dataspace
                v, nd = self.u8(p), self.u8(p + 1)
                q = p + (8 if v == 1 else 4)
                dims = [self.u64(q + 8 * i) for i in range(nd)]
            elif t == 0x03:  # datatype
                cls, ver = self.u8(p) & 0x0F, self.u8(p) >> 4
                bits = self.u8(p + 1)
                esize = self.u32(p + 4)
                order = ">" if bits & 1 else "<"
                if cls == 0:
                    dtype = np.dtype(f"{order}{'i' if bits & 0x08 else 'u'}{esize}")
                elif cls == 1:
                    dtype = np.dtype(f"{order}f{esize}")
                else:
                    raise NotImplementedError(f"datatype class {cls} is not supported")
                _ = ver
            elif t == 0x0B:
                filters = self._filters(p)
            elif t == 0x08:  # layout
                v = self.u8(p)
                if v == 3:
                    cls = self.u8(p + 1)
                    if cls == 1:
                        layout = ("contiguous", self.u64(p + 2), self.u64(p + 10))
                    elif cls == 0:
                        n = self.u16(p + 2)
                        layout = ("compact", p + 4, n)
                    elif cls == 2:
                        ndl = self.u8(p + 2)
                        cdims = [self.u32(p + 11 + 4 * i) for i in range(ndl)]
                        layout = ("chunked", self.u64(p + 3), ndl, cdims)
                    else:
                        raise NotImplementedError(f"layout class {cls} is not supported")
                elif v in (1, 2):
                    nd, cls = self.u8(p + 1), self.u8(p + 2)
                    if cls != 1:
                        raise NotImplementedError("only contiguous version-1/2 layouts are supported")
                    layout = ("contiguous", self.u64(p + 8), None)
                else:
                    raise NotImplementedError(f"layout message version {v}")
        if dims is None or dtype is None or layout is None:
            raise ValueError("incomplete dataset header")
        count = int(np.prod(dims)) if dims else 1
        if layout[0] == "chunked":
            _, bt, ndl, cdims = layout
            cd = cdims[:-1]
            nat = dtype.newbyteorder("=")
            out = np.zeros(dims, dtype=nat)
            if bt == UNDEF:
                return out
            for offs, size, mask, addr in self._chunks(bt, ndl, []):
                raw = self._unfilter(self.b[self.base + addr:self.base + addr + size], filters, mask, dtype.itemsize)
                blk = np.frombuffer(raw, dtype=dtype, count=int(np.prod(cd))).astype(nat).reshape(cd)
                sl = tuple(slice(o, min(o + c, d)) for o, c, d in zip(offs[:-1], cd, dims))
                out[sl] = blk[tuple(slice(0, q.stop - q.start) for q in sl)]
            return out
        if filters:
            raise NotImplementedError("filtered contiguous datasets do not exist in HDF5")
        if layout[0] == "contiguous":
            if layout[1] == UNDEF:
                return np.zeros(dims, dtype=dtype.newbyteorder("="))
            start = self.base + layout[1]
        else:
            start = layout[1]
        arr = np.frombuffer(self.b, dtype=dtype, count=count, offset=start)
        return arr.astype(dtype.newbyteorder("="), copy=True).reshape(dims)

    def get(self, path):
        parts = [q for q in str(path).split("/") if q]
        addr = self.root_header
        for i, name in enumerate(parts):
            links = self.group_links(addr)
            if name not in links:
                raise KeyError(f"{self.path}: no object {path!r}")
            addr = links[name]
        return self.dataset(addr)

    def walk(self, addr=None, prefix=""):
        addr = self.root_header if addr is None else addr
        out = {}
        for name, child in self.group_links(addr).items():
            kinds = {t for t, _, _ in self.messages(child)}
            if 0x11 in kinds:
                out.update(self.walk(child, prefix + "/" + name))
            else:
                out[prefix + "/" + name] = self.dataset(child)
        return out


def read_hdf5(path, name=None):
    """One dataset (``name`` like "/data0") or a dict of every dataset of an HDF5 file."""
    f = _H5(path)
    return f.get(name) if name is not None else f.walk()


# -------------------------------------------------------------------- XDMF
def _dataitem(item, base: Path):
    fmt = item.get("Format", "XML")
    dims = [int(v) for v in item.get("Dimensions").split()]
    dt = item.get("DataType", item.get("NumberType", "Float"))
    prec = int(item.get("Precision", "4"))
    np_t = {("Float", 4): np.float32, ("Float", 8): np.float64, ("Int", 4): np.int32, ("Int", 8): np.int64,
            ("UInt", 4): np.uint32, ("UInt", 8): np.uint64}.get((dt, prec), np.float64)
    text = (item.text or "").strip()
    if fmt == "HDF":
        fname, _, dpath = text.partition(":")
        return np.asarray(read_hdf5(base / fname, dpath)).reshape(dims)
    if fmt == "Binary":
        endian = "<" if item.get("Endian", "Little") != "Big" else ">"
        a = np.fromfile(base / text, dtype=np.dtype(np_t).newbyteorder(endian))
        return a.astype(np_t).reshape(dims)
    return np.array(text.split(), dtype=np_t).reshape(dims)


def _grids(root):
    for g in root.iter("Grid"):
        if g.get("GridType", "Uniform") == "Uniform":
            yield g


def read_xdmf_mesh(path):
    """(X [N, 3] float64, tets [E, 4] int32, cell attributes) of the first uniform grid."""
    path = Path(path)
    root = ET.parse(path).getroot()
    grid = next(_grids(root))
    geo = grid.find("Geometry")
    X = _dataitem(geo.find("DataItem"), path.parent).astype(np.float64).reshape(-1, 3)
    top = grid.find("Topology")
    if top.get("TopologyType", top.get("Type", "")).lower() != "tetrahedron":
        raise NotImplementedError("only tetrahedral meshes are supported")
    T = _dataitem(top.find("DataItem"), path.parent).astype(np.int64).reshape(-1, 4)
    attrs = {}
    for a in grid.findall("Attribute"):
        if a.get("Center") == "Cell":
            attrs[a.get("Name")] = _dataitem(a.find("DataItem"), path.parent)
    if T.min() < 0 or T.max() >= X.shape[0]:
        raise ValueError("tetrahedron vertex index out of range")
    return X, np.ascontiguousarray(T, dtype=np.int32), attrs


def read_xdmf_series(path, name):
    """[(time, nodal field [N, k])] of attribute ``name`` over the grids of a temporal collection."""
    path = Path(path)
    root = ET.parse(path).getroot()
    out = []
    for g in _grids(root):
        t = g.find("Time")
        for a in g.findall("Attribute"):
            if a.get("Name") == name:
                out.append((float(t.get("Value")) if t is not None else 0.0, _dataitem(a.find("DataItem"),
                                                                                       path.parent)))
    return out


class XDMFWriter:
    """Mesh + time series of nodal fields as XDMF 3 with raw binary heavy data."""

    def __init__(self, path, X, tets):
        self.path = Path(path)
        self.stem = self.path.with_suffix("")
        self.X = np.ascontiguousarray(X, dtype="<f8").reshape(-1, 3)
        self.T = np.ascontiguousarray(tets, dtype="<i4").reshape(-1, 4)
        self.steps = []
        self._write_array("geometry", self.X)
        self._write_array("topology", self.T)

    def _write_array(self, tag, a):
        fname = f"{self.stem.name}_{tag}.bin"
        np.ascontiguousarray(a).tofile(self.path.parent / fname)
        return fname

    def write_function(self, values, time=0.0, name="m"):
        """Append one state (nodal vectors, length 3N, numpy or torch) at ``time``."""
        if hasattr(values, "detach"):
            values = values.detach().cpu().numpy()
        v = np.ascontiguousarray(np.asarray(values, dtype="<f8")[: 3 * self.X.shape[0]]).reshape(-1, 3)
        fname = self._write_array(f"{name}_{len(self.steps):05d}", v)
        self.steps.append((float(time), name, fname, v.shape[0]))
        self.flush()

    def flush(self):
        N, E = self.X.shape[0], self.T.shape[0]
        geo = (f'<Geometry GeometryType="XYZ"><DataItem DataType="Float" Precision="8" Format="Binary" '
               f'Endian="Little" Dimensions="{N} 3">{self.stem.name}_geometry.bin</DataItem></Geometry>')
        top = (f'<Topology TopologyType="Tetrahedron" NumberOfElements="{E}" NodesPerElement="4"><DataItem '
               f'DataType="Int" Precision="4" Format="Binary" Endian="Little" Dimensions="{E} 4">'
               f'{self.stem.name}_topology.bin</DataItem></Topology>')
        grids = []
        for t, name, fname, n in self.steps or [(0.0, None, None, 0)]:
            attr = "" if name is None else (
                f'<Attribute Name="{name}" AttributeType="Vector" Center="Node"><DataItem DataType="Float" '
                f'Precision="8" Format="Binary" Endian="Little" Dimensions="{n} 3">{fname}</DataItem></Attribute>')
            grids.append(f'<Grid Name="mesh" GridType="Uniform"><Time Value="{t!r}"/>{geo}{top}{attr}</Grid>')
        xml = ('<?xml version="1.0"?>\n<Xdmf Version="3.0"><Domain><Grid Name="TimeSeries" '
               'GridType="Collection" CollectionType="Temporal">' + "".join(grids) + "</Grid></Domain></Xdmf>\n")
        self.path.write_text(xml)


# ------------------------------------------------------------------ checkpoints
# The reference saves a relaxed state with adios4dolfinx (write_mesh + write_function into
# "Relax.bp", llg_module_GPU.py:2035-2042, 2373-2376) and restarts from it with read_mesh +
# read_function (examples/gpu/Current_driven_skyrmion_Torus/Dynamics.py:33-43).  The same four
# calls are offered here.  ADIOS2 is not in this image, so the checkpoint is this module's own
# format, not ADIOS2 BP: a directory (as a BP file is) with index.json and raw little-endian
# FP64 / int32 arrays; values round-trip exactly.

def _ckpt_index(d: Path):
    import json
    f = d / "index.json"
    return json.loads(f.read_text()) if f.exists() else {"format": "spinfemx_b200 checkpoint", "version": 1,
                                                          "mesh": None, "functions": {}}


def _ckpt_save(d: Path, idx):
    import json
    (d / "index.json").write_text(json.dumps(idx, indent=1))


def write_mesh(filename, X, tets):
    """Start a checkpoint at ``filename`` (a directory) with the mesh (X [N][3] nm, tets [E][4])."""
    d = Path(filename)
    d.mkdir(parents=True, exist_ok=True)
    X = np.ascontiguousarray(X, dtype="<f8").reshape(-1, 3)
    T = np.ascontiguousarray(tets, dtype="<i4").reshape(-1, 4)
    X.tofile(d / "mesh_X.f64")
    T.tofile(d / "mesh_tets.i32")
    idx = {"format": "spinfemx_b200 checkpoint", "version": 1, "functions": {},
           "mesh": {"nodes": int(X.shape[0]), "cells": int(T.shape[0])}}
    _ckpt_save(d, idx)


def write_function(filename, values, time=0.0, name="m"):
    """Add nodal vectors (3N values, numpy or torch) named ``name`` at ``time`` (replacing an
    entry of the same name and time)."""
    d = Path(filename)
    idx = _ckpt_index(d)
    if idx.get("mesh") is None:
        raise ValueError(f"{d}: write_mesh first")
    if hasattr(values, "detach"):
        values = values.detach().cpu().numpy()
    v = np.ascontiguousarray(np.asarray(values, dtype="<f8").reshape(-1))
    if v.size != 3 * idx["mesh"]["nodes"]:
        raise ValueError(f"expected {3 * idx['mesh']['nodes']} values, got {v.size}")
    entries = [e for e in idx["functions"].get(name, []) if e["time"] != float(time)]
    serial = int(idx.get("arrays_written", 0))
    fname = f"{name}_{serial:05d}.f64"
    idx["arrays_written"] = serial + 1
    v.tofile(d / fname)
    entries.append({"time": float(time), "file": fname})
    idx["functions"][name] = entries
    _ckpt_save(d, idx)


def read_mesh(filename):
    """(X [N][3], tets [E][4]) of a checkpoint."""
    d = Path(filename)
    idx = _ckpt_index(d)
    if idx.get("mesh") is None:
        raise FileNotFoundError(f"{d}: no checkpoint mesh")
    X = np.fromfile(d / "mesh_X.f64", dtype="<f8").reshape(-1, 3)
    T = np.fromfile(d / "mesh_tets.i32", dtype="<i4").reshape(-1, 4)
    return X, T


def read_function(filename, time=0.0, name="m"):
    """The 3N values of ``name`` stored at exactly ``time`` (KeyError otherwise)."""
    d = Path(filename)
    for e in _ckpt_index(d)["functions"].get(name, []):
        if e["time"] == float(time):
            return np.fromfile(d / e["file"], dtype="<f8")
    raise KeyError(f"{d}: no function {name!r} at time {time!r}")


__all__ = ["read_hdf5", "read_xdmf_mesh", "read_xdmf_series", "XDMFWriter", "write_mesh", "write_function",
           "read_mesh", "read_function"]
