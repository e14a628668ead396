"""The packed ``.ntiga`` Bezier-extraction database, in numpy.

Binary layout (little endian), as read by the reference's ``iga::Database``
(solvers/cpu/include/IgaDatabase.hpp:28-161) and written by ``iga_pack``
(solvers/cpu/src/iga_pack.cpp:337-403):

  header   magic "NTIGADB2", u32 version (3/4/5), u32 ranks, u64 elements,
           u64 nodes, u32 bezier_points (=64), u32 reserved, u64 rank_index_offset,
           v5: f64 source_origin[3], f64 units_per_normalized_unit, f64 length_scale_to_m
  index    u64 element_offsets[elements+1] (the last one ends the records),
           i32 owners[elements]
  element  u64 id, i32 type, i32 owner, u32 nen, v>=4: i32 face_labels[6],
           i32 connectivity[nen], per basis row: u8 nnz, nnz x (u8 column, f64 value),
           f64 bezier_points[64][3]
  ranks    at rank_index_offset: u64 rank_offsets[ranks+1], u64 rank_elements[...]

``FlatMesh`` is the flattened in-memory form the device path consumes
(the layout of solvers/cuda/include/DeviceMesh.hpp:16-57).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

MAGIC = b"NTIGADB2"
VERSION = 5


@dataclass
class FlatMesh:
    nodes: int
    element_offsets: np.ndarray          # int32 [E+1]
    connectivity: np.ndarray             # int32 [sum nen]
    extraction_offsets: np.ndarray       # int32 [sum nen + 1]
    extraction_columns: np.ndarray       # uint8 [nnz]
    extraction_values: np.ndarray        # float64 [nnz]
    bezier_points: np.ndarray            # float64 [E*64*3]
    boundary_labels: np.ndarray          # int32 [E*6]
    geometry_transform: tuple = (0.0, 0.0, 0.0, 1.0, 1.0)
    version: int = VERSION
    ranks: int = 1
    owners: np.ndarray | None = None
    ids: np.ndarray | None = None
    types: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def elements(self) -> int:
        return len(self.element_offsets) - 1

    @property
    def max_basis(self) -> int:
        return int(np.diff(self.element_offsets).max())

    def element(self, e: int):
        """Dense (connectivity, extraction[nen,64], bezier[64,3], labels[6]) of one element."""
        b, t = int(self.element_offsets[e]), int(self.element_offsets[e + 1])
        conn = self.connectivity[b:t]
        C = np.zeros((t - b, 64))
        for a in range(t - b):
            lo, hi = int(self.extraction_offsets[b + a]), int(self.extraction_offsets[b + a + 1])
            C[a, self.extraction_columns[lo:hi]] = self.extraction_values[lo:hi]
        X = self.bezier_points[e * 192:(e + 1) * 192].reshape(64, 3)
        return conn, C, X, self.boundary_labels[6 * e:6 * e + 6]

    def contiguous(self) -> "FlatMesh":
        self.element_offsets = np.ascontiguousarray(self.element_offsets, np.int32)
        self.connectivity = np.ascontiguousarray(self.connectivity, np.int32)
        self.extraction_offsets = np.ascontiguousarray(self.extraction_offsets, np.int32)
        self.extraction_columns = np.ascontiguousarray(self.extraction_columns, np.uint8)
        self.extraction_values = np.ascontiguousarray(self.extraction_values, np.float64)
        self.bezier_points = np.ascontiguousarray(self.bezier_points, np.float64)
        self.boundary_labels = np.ascontiguousarray(self.boundary_labels, np.int32)
        return self


def read(path) -> FlatMesh:
    """Read a v3/v4/v5 database into a FlatMesh (all elements, rank 0 view)."""
    data = Path(path).read_bytes()
    if data[:8] != MAGIC:
        raise ValueError("not a supported .ntiga database")
    version, ranks, elements, nodes, bez, _reserved, rio = struct.unpack_from("<IIQQIIQ", data, 8)
    off = 8 + struct.calcsize("<IIQQIIQ")
    if version not in (3, 4, 5):
        raise ValueError("unsupported database version")
    transform = (0.0, 0.0, 0.0, 1.0, 1.0)
    if version >= 5:
        transform = struct.unpack_from("<5d", data, off)
        off += 40
    if bez != 64:
        raise ValueError("unsupported Bezier point count")
    if nodes == 0 or rio == 0:
        raise ValueError("invalid database ownership index")
    offsets = np.frombuffer(data, "<u8", elements + 1, off)
    off += 8 * (elements + 1)
    owners = np.frombuffer(data, "<i4", elements, off).copy()
    eo = [0]
    conn, xo, xc, xv, bz, labels, ids, types = [], [0], [], [], [], [], [], []
    for e in range(elements):
        o = int(offsets[e])
        eid, typ, _own, nen = struct.unpack_from("<QiiI", data, o)
        o += 20
        lab = (-1,) * 6
        if version >= 4:
            lab = struct.unpack_from("<6i", data, o)
            o += 24
        if nen == 0 or nen > 4096:
            raise ValueError("invalid element basis count")
        conn.append(np.frombuffer(data, "<i4", nen, o))
        o += 4 * nen
        for _a in range(nen):
            nz = data[o]
            o += 1
            rec = np.frombuffer(data, dtype=np.dtype([("c", "u1"), ("v", "<f8")]), count=nz, offset=o)
            o += 9 * nz
            if nz and rec["c"].max() >= 64:
                raise ValueError("invalid extraction column")
            xc.append(rec["c"]); xv.append(rec["v"])
            xo.append(xo[-1] + nz)
        bz.append(np.frombuffer(data, "<f8", 192, o))
        labels.append(lab); ids.append(eid); types.append(typ)
        eo.append(eo[-1] + nen)
    return FlatMesh(
        nodes=int(nodes),
        element_offsets=np.array(eo, np.int32),
        connectivity=np.concatenate(conn).astype(np.int32),
        extraction_offsets=np.array(xo, np.int32),
        extraction_columns=np.concatenate(xc).astype(np.uint8),
        extraction_values=np.concatenate(xv).astype(np.float64),
        bezier_points=np.concatenate(bz).astype(np.float64),
        boundary_labels=np.array(labels, np.int32).ravel(),
        geometry_transform=tuple(transform), version=int(version), ranks=int(ranks),
        owners=owners, ids=np.array(ids, np.uint64), types=np.array(types, np.int32))


def write(path, mesh: FlatMesh) -> None:
    """Write a single-rank v5 database (all elements owned by rank 0); element ids and types are
    kept when the mesh carries them (a database read by `read`)."""
    E = mesh.elements
    rec_dtype = np.dtype([("c", "u1"), ("v", "<f8")])
    head = bytearray()
    head += MAGIC
    head += struct.pack("<IIQQII", VERSION, 1, E, mesh.nodes, 64, 0)
    rio_pos = len(head)
    head += struct.pack("<Q", 0)
    head += struct.pack("<5d", *mesh.geometry_transform)
    index_pos = len(head)
    body_start = index_pos + 8 * (E + 1) + 4 * E
    chunks = []
    offsets = np.zeros(E + 1, np.uint64)
    pos = body_start
    for e in range(E):
        offsets[e] = pos
        b, t = int(mesh.element_offsets[e]), int(mesh.element_offsets[e + 1])
        nen = t - b
        eid = int(mesh.ids[e]) if mesh.ids is not None else e
        typ = int(mesh.types[e]) if mesh.types is not None else 0
        parts = [struct.pack("<QiiI", eid, typ, 0, nen),
                 np.asarray(mesh.boundary_labels[6 * e:6 * e + 6], "<i4").tobytes(),
                 np.asarray(mesh.connectivity[b:t], "<i4").tobytes()]
        for a in range(nen):
            lo, hi = int(mesh.extraction_offsets[b + a]), int(mesh.extraction_offsets[b + a + 1])
            rec = np.empty(hi - lo, rec_dtype)
            rec["c"] = mesh.extraction_columns[lo:hi]
            rec["v"] = mesh.extraction_values[lo:hi]
            parts.append(bytes([hi - lo]))
            parts.append(rec.tobytes())
        parts.append(np.asarray(mesh.bezier_points[192 * e:192 * (e + 1)], "<f8").tobytes())
        blob = b"".join(parts)
        chunks.append(blob)
        pos += len(blob)
    offsets[E] = pos
    rank_index = np.concatenate([np.array([0, E], np.uint64), np.arange(E, dtype=np.uint64)]).tobytes()
    struct.pack_into("<Q", head, rio_pos, pos)
    with open(path, "wb") as f:
        f.write(head)
        f.write(offsets.astype("<u8").tobytes())
        f.write(np.zeros(E, "<i4").tobytes())
        for blob in chunks:
            f.write(blob)
        f.write(rank_index)
