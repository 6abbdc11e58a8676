"""Synthetic PLY files for the PLY ingest tests (seeded; no public models).

Each case is the bytes of one file.  Together they cover what the
reference's reader (src/dort/ply_mesh.cpp over rply) distinguishes: the three
formats, scalar types of coordinates, list count and index types, extra
vertex and face properties before and after the ones read, other elements,
polygons of mixed size (fans), faces with fewer than three indices, a vertex
element whose z is not its last coordinate (the point is emitted when z is
read), a face list not named "vertex_indices" (not read), and no faces.
"""
from __future__ import annotations

import numpy as np

_END = {"binary_little_endian": "<", "binary_big_endian": ">"}
_NP = {"char": "i1", "uchar": "u1", "short": "i2", "ushort": "u2", "int": "i4",
       "uint": "u4", "float": "f4", "double": "f8", "uint8": "u1", "int32": "i4",
       "float32": "f4"}


def _ply(fmt: str, elements) -> bytes:
    """elements: [(name, [(prop, type) | (prop, 'list', count_type, type)],
    rows)], rows a list of tuples (a list value is a sequence)."""
    head = ["ply", f"format {fmt} 1.0", "comment synthetic test mesh"]
    for name, props, rows in elements:
        head.append(f"element {name} {len(rows)}")
        for p in props:
            if len(p) == 4:
                head.append(f"property list {p[2]} {p[3]} {p[0]}")
            else:
                head.append(f"property {p[1]} {p[0]}")
    head.append("end_header")
    out = ("\n".join(head) + "\n").encode()
    if fmt == "ascii":
        lines = []
        for _, props, rows in elements:
            for r in rows:
                w = []
                for p, v in zip(props, r):
                    if len(p) == 4:
                        w.append(str(len(v)))
                        w += [str(int(x)) for x in v]
                    elif p[1] in ("float", "double", "float32"):
                        w.append(repr(float(v)))
                    else:
                        w.append(str(int(v)))
                lines.append(" ".join(w))
        return out + ("\n".join(lines) + "\n").encode()
    e = _END[fmt]
    body = bytearray()
    for _, props, rows in elements:
        for r in rows:
            for p, v in zip(props, r):
                if len(p) == 4:
                    body += np.array([len(v)], e + _NP[p[2]]).tobytes()
                    body += np.asarray(v, e + _NP[p[3]]).tobytes()
                else:
                    body += np.array([v], e + _NP[p[1]]).tobytes()
    return out + bytes(body)


def _grid(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32)


def cases() -> dict[str, bytes]:
    rng = np.random.default_rng(1234)
    c = {}
    xyz = [("x", "float"), ("y", "float"), ("z", "float")]

    p = _grid(6, 1)
    c["ascii_triangles"] = _ply("ascii", [
        ("vertex", xyz, [tuple(v) for v in p]),
        ("face", [("vertex_indices", "list", "uchar", "int")],
         [([0, 1, 2],), ([2, 3, 4],), ([4, 5, 0],), ([1, 3, 5],)])])

    p = _grid(12, 2)
    nrm = rng.normal(size=(12, 3))
    faces = [[0, 1, 2], [2, 3, 4, 5], [5, 6, 7, 8, 9], [9, 10, 11], [11, 0, 3, 6]]
    c["ascii_mixed_polygons"] = _ply("ascii", [
        ("vertex", xyz + [("nx", "float"), ("ny", "float"), ("nz", "float")],
         [tuple(v) + tuple(n) for v, n in zip(p, nrm)]),
        ("edge", [("vertex1", "int"), ("vertex2", "int")], [(0, 1), (1, 2)]),
        ("face", [("vertex_indices", "list", "uchar", "int")], [(f,) for f in faces])])

    p = _grid(200, 3)
    quads = rng.integers(0, 200, (150, 4))
    c["ble_uniform_quads"] = _ply("binary_little_endian", [
        ("vertex", [("confidence", "float")] + xyz + [("red", "uchar")],
         [(0.5,) + tuple(v) + (7,) for v in p]),
        ("face", [("flags", "uchar"), ("vertex_indices", "list", "uchar", "int"),
                  ("material", "ushort")], [(1, list(q), 3) for q in quads])])

    p = rng.uniform(-1e3, 1e3, (40, 3))
    faces = [list(rng.integers(0, 40, rng.integers(3, 8))) for _ in range(60)]
    c["bbe_double_mixed"] = _ply("binary_big_endian", [
        ("vertex", [("x", "double"), ("y", "double"), ("z", "double")],
         [tuple(v) for v in p]),
        ("face", [("vertex_indices", "list", "uint8", "uint")], [(f,) for f in faces])])

    p = _grid(30, 5)
    tris = rng.integers(0, 30, (40, 3))
    c["ble_z_not_last"] = _ply("binary_little_endian", [
        ("vertex", [("y", "float"), ("z", "float"), ("x", "float")],
         [(v[1], v[2], v[0]) for v in p]),
        ("face", [("vertex_indices", "list", "uchar", "int")], [(list(t),) for t in tris])])

    p = _grid(25, 6)
    faces = [[0, 1, 2], [3], [], [4, 5], [6, 7, 8, 9], [10, 11, 12]]
    c["ble_short_faces"] = _ply("binary_little_endian", [
        ("vertex", xyz, [tuple(v) for v in p]),
        ("face", [("vertex_indices", "list", "int", "int")], [(f,) for f in faces])])

    p = _grid(9, 7)
    c["ascii_vertex_index_name"] = _ply("ascii", [
        ("vertex", xyz, [tuple(v) for v in p]),
        ("face", [("vertex_index", "list", "uchar", "int")], [([0, 1, 2],), ([3, 4, 5],)])])

    p = _grid(17, 8)
    c["ble_points_only"] = _ply("binary_little_endian", [
        ("vertex", xyz, [tuple(v) for v in p])])

    p = _grid(2000, 9)
    tris = rng.integers(0, 2000, (4000, 3))
    c["ble_large_triangles"] = _ply("binary_little_endian", [
        ("vertex", xyz, [tuple(v) for v in p]),
        ("face", [("vertex_indices", "list", "uchar", "uint")], [(list(t),) for t in tris])])
    return c
