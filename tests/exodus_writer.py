"""A small netCDF classic writer (CDF-1, CDF-2, CDF-5) for Exodus II test
meshes: the library's Exodus reader is checked against files written here,
and this writer against scipy's netCDF reader (CDF-1/2)."""
import struct

import numpy as np

NC = {"i1": 1, "S1": 2, "i2": 3, "i4": 4, "f4": 5, "f8": 6, "i8": 10}


def _pad(b):
    return b + b"\0" * ((4 - len(b) % 4) % 4)


class Writer:
    def __init__(self, version=1):
        assert version in (1, 2, 5)
        self.version = version
        self.dims = []   # (name, length)
        self.vars = []   # (name, dim names, array, {attr: str})

    def dim(self, name, length):
        self.dims.append((name, int(length)))

    def var(self, name, dims, data, attrs=None):
        self.vars.append((name, list(dims), data, attrs or {}))

    def _count(self, n):
        return struct.pack(">Q" if self.version == 5 else ">I", n)

    def _name(self, s):
        b = s.encode()
        return self._count(len(b)) + _pad(b)

    def _attrs(self, attrs):
        if not attrs:
            return struct.pack(">I", 0) + self._count(0)
        out = struct.pack(">I", 0x0C) + self._count(len(attrs))
        for k, v in attrs.items():
            b = v.encode()
            out += self._name(k) + struct.pack(">I", 2) + self._count(len(b)) + _pad(b)
        return out

    def _header(self, begins):
        h = b"CDF" + bytes([self.version]) + self._count(0)
        h += struct.pack(">I", 0x0A) + self._count(len(self.dims))
        for n, l in self.dims:
            h += self._name(n) + self._count(l)
        h += struct.pack(">I", 0) + self._count(0)  # no global attributes
        h += struct.pack(">I", 0x0B) + self._count(len(self.vars))
        names = [d[0] for d in self.dims]
        for (n, dims, data, attrs), b in zip(self.vars, begins):
            h += self._name(n) + self._count(len(dims))
            for d in dims:
                h += self._count(names.index(d))
            h += self._attrs(attrs)
            code = NC[data.dtype.str[1:]]
            h += struct.pack(">I", code) + self._count(len(_pad(self._raw(data))))
            h += struct.pack(">I" if self.version == 1 else ">Q", b)
        return h

    @staticmethod
    def _raw(data):
        return np.ascontiguousarray(data).astype(data.dtype.newbyteorder(">")).tobytes()

    def bytes(self):
        size = len(self._header([0] * len(self.vars)))
        begins, off = [], size
        for _, _, data, _ in self.vars:
            begins.append(off)
            off += len(_pad(self._raw(data)))
        out = self._header(begins)
        for _, _, data, _ in self.vars:
            out += _pad(self._raw(data))
        return out

    def write(self, path):
        with open(path, "wb") as f:
            f.write(self.bytes())


def exodus_box(path, cells, coords, node_sets, version=1, blocks=2, combined_coord=False, coord_dtype=np.float64,
               int_dtype=np.int32, names=True, elem_type="TETRA"):
    """An Exodus II file of a tet mesh: cells split into `blocks` element
    blocks, node sets {name: 0-based ids} (ids 10, 20, ...)."""
    w = Writer(version)
    N, C = coords.shape[0], cells.shape[0]
    w.dim("len_string", 33)
    w.dim("len_name", 33)
    w.dim("num_dim", 3)
    w.dim("num_nodes", N)
    w.dim("num_elem", C)
    w.dim("num_el_blk", blocks)
    parts = np.array_split(np.arange(C), blocks)
    for b, part in enumerate(parts, 1):
        w.dim(f"num_el_in_blk{b}", part.size)
        w.dim(f"num_nod_per_el{b}", 4)
    w.dim("num_node_sets", len(node_sets))
    for s, (name, ids) in enumerate(node_sets.items(), 1):
        w.dim(f"num_nod_ns{s}", len(ids))
    if combined_coord:
        w.var("coord", ["num_dim", "num_nodes"], coords.T.astype(coord_dtype))
    else:
        for d, nm in enumerate(("coordx", "coordy", "coordz")):
            w.var(nm, ["num_nodes"], coords[:, d].astype(coord_dtype))
    w.var("eb_prop1", ["num_el_blk"], np.arange(1, blocks + 1, dtype=np.int32))
    for b, part in enumerate(parts, 1):
        w.var(f"connect{b}", [f"num_el_in_blk{b}", f"num_nod_per_el{b}"], (cells[part] + 1).astype(int_dtype),
              {"elem_type": elem_type})
    w.var("ns_prop1", ["num_node_sets"], 10 * np.arange(1, len(node_sets) + 1, dtype=np.int32))
    if names:
        arr = np.zeros((len(node_sets), 33), "S1")
        for s, name in enumerate(node_sets):
            for k, ch in enumerate(name.encode()):
                arr[s, k] = bytes([ch])
        w.var("ns_names", ["num_node_sets", "len_name"], arr)
    for s, (name, ids) in enumerate(node_sets.items(), 1):
        w.var(f"node_ns{s}", [f"num_nod_ns{s}"], (np.asarray(ids) + 1).astype(int_dtype))
    w.write(path)
