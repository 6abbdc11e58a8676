"""PLY mesh ingest: the reference's reader restated over numpy.

Follows read_ply_callbacks (src/dort/ply_mesh.cpp:9-78), which reads through
the rply library the reference vendors (extern/rply, version 1.1.x):

  - formats ascii, binary_little_endian and binary_big_endian;
  - points come from the "vertex" element's x, y and z properties, rounded to
    float; a point is emitted when its z is read (ply_mesh.cpp:33-42), so a
    vertex element without z gives no points;
  - triangles come from the "face" element's "vertex_indices" list, a polygon
    (i0, i1, ..., ik) fanned into (i0, i1, i2), (i0, i2, i3), ...
    (ply_mesh.cpp:44-62); other elements and properties are skipped.

Unlike the reference, an index that does not name a point is an error here
(the reference would read out of bounds when it builds the triangles).

Binary elements whose properties are all scalars, and face lists whose
polygons all have the same size, are decoded in one numpy pass; anything else
falls back to a per-record loop.
"""
from __future__ import annotations

import numpy as np

_TYPES = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1",
    "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
    "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
    "float": "f4", "float32": "f4", "double": "f8", "float64": "f8",
}


class PlyError(ValueError):
    pass


class _Prop:
    __slots__ = ("name", "type", "count_type")

    def __init__(self, name, type_, count_type=None):
        self.name, self.type, self.count_type = name, type_, count_type


class _Elem:
    __slots__ = ("name", "count", "props")

    def __init__(self, name, count):
        self.name, self.count, self.props = name, count, []


def _header(data: bytes):
    end = data.find(b"end_header")
    if not data.startswith(b"ply") or end < 0:
        raise PlyError("not a PLY file")
    nl = data.find(b"\n", end)
    body = nl + 1 if nl >= 0 else len(data)
    fmt, elems = None, []
    for raw in data[:end].decode("ascii", "replace").splitlines()[1:]:
        w = raw.split()
        if not w:
            continue
        if w[0] == "format":
            fmt = w[1] if len(w) > 1 else ""
        elif w[0] == "element":
            elems.append(_Elem(w[1], int(w[2])))
        elif w[0] == "property":
            if not elems:
                raise PlyError("PLY property before element")
            if w[1] == "list":
                if w[2] not in _TYPES or w[3] not in _TYPES:
                    raise PlyError(f"unknown PLY type in: {raw.strip()}")
                elems[-1].props.append(_Prop(w[4], w[3], w[2]))
            else:
                if w[1] not in _TYPES:
                    raise PlyError(f"unknown PLY type in: {raw.strip()}")
                elems[-1].props.append(_Prop(w[2], w[1]))
    if fmt not in ("ascii", "binary_little_endian", "binary_big_endian"):
        raise PlyError(f"unknown PLY format: {fmt}")
    return fmt, elems, body


class _Points:
    """The reference's point callback: x / y / z update one persistent point,
    which is emitted when z is read."""

    def __init__(self):
        self.cur = np.zeros(3, np.float32)
        self.out = []

    def record(self, names, values):
        for name, v in zip(names, values):
            if name in ("x", "y", "z"):
                self.cur["xyz".index(name)] = np.float32(v)
                if name == "z":
                    self.out.append(self.cur.copy())

    def block(self, names, cols):
        """All records of a vertex element at once (columns by property)."""
        axes = [n for n in names if n in ("x", "y", "z")]
        if "z" not in axes or len(cols["z"]) == 0:
            # no point is emitted; only the persistent point changes
            for n in axes:
                if len(cols[n]):
                    self.cur["xyz".index(n)] = np.float32(cols[n][-1])
            return
        count = len(cols["z"])
        pts = np.empty((count, 3), np.float32)
        zi = names.index("z")
        for a, n in enumerate("xyz"):
            if n not in axes:
                pts[:, a] = self.cur[a]
                continue
            v = np.asarray(cols[n]).astype(np.float32)
            if names.index(n) <= zi:
                pts[:, a] = v                      # read before (or as) z of the record
            else:
                pts[0, a] = self.cur[a]            # read after z: the previous record's
                pts[1:, a] = v[:-1]
        self.out.append(pts)
        self.cur = np.array([np.float32(cols[n][-1]) if n in axes else self.cur[a]
                             for a, n in enumerate("xyz")], np.float32)

    def array(self):
        if not self.out:
            return np.zeros((0, 3), np.float32)
        return np.concatenate([np.asarray(o, np.float32).reshape(-1, 3) for o in self.out])


def _fan_uniform(idx: np.ndarray) -> np.ndarray:
    """Fans of polygons of equal size k (rows of idx), polygon-major."""
    k = idx.shape[1]
    if k < 3:
        return np.zeros((0, 3), np.int64)
    j = np.arange(2, k)
    tri = np.empty((idx.shape[0], k - 2, 3), np.int64)
    tri[:, :, 0] = idx[:, :1]
    tri[:, :, 1] = idx[:, j - 1]
    tri[:, :, 2] = idx[:, j]
    return tri.reshape(-1, 3)


def _fan_one(face) -> np.ndarray:
    k = len(face)
    if k < 3:
        return np.zeros((0, 3), np.int64)
    return np.array([[face[0], face[j - 1], face[j]] for j in range(2, k)], np.int64)


def _read_ascii(text: bytes, elems):
    tok = text.split()
    pos = 0
    points = _Points()
    tris = []

    def take(n):
        nonlocal pos
        if pos + n > len(tok):
            raise PlyError("truncated PLY file")
        v = tok[pos:pos + n]
        pos += n
        return v

    for e in elems:
        if all(p.count_type is None for p in e.props):
            n = len(e.props)
            vals = np.array(take(n * e.count), np.float64).reshape(e.count, n) if n else \
                np.zeros((e.count, 0))
            if e.name == "vertex":
                points.block([p.name for p in e.props],
                             {p.name: vals[:, i] for i, p in enumerate(e.props)})
            continue
        for _ in range(e.count):
            names, values, face = [], [], None
            for p in e.props:
                if p.count_type is not None:
                    cnt = int(float(take(1)[0]))
                    lst = [float(t) for t in take(cnt)]
                    if e.name == "face" and p.name == "vertex_indices":
                        face = lst
                else:
                    names.append(p.name)
                    values.append(float(take(1)[0]))
            if e.name == "vertex":
                points.record(names, values)
            if face is not None:
                tris.append(_fan_one(np.array(face, np.float64).astype(np.int64)))
    return points.array(), tris


def _read_binary(body: memoryview, elems, big: bool):
    end = ">" if big else "<"
    pos = 0
    points = _Points()
    tris = []
    for e in elems:
        if all(p.count_type is None for p in e.props):
            dt = np.dtype([(f"p{i}", end + _TYPES[p.type]) for i, p in enumerate(e.props)])
            need = dt.itemsize * e.count
            if pos + need > len(body):
                raise PlyError("truncated PLY file")
            rec = np.frombuffer(body, dt, e.count, pos)
            pos += need
            if e.name == "vertex":
                points.block([p.name for p in e.props],
                             {p.name: rec[f"p{i}"].astype(np.float64)
                              for i, p in enumerate(e.props)})
            continue
        # one list property and scalar properties: try the uniform layout
        done = False
        lists = [i for i, p in enumerate(e.props) if p.count_type is not None]
        if len(lists) == 1 and e.count > 0:
            li = lists[0]
            lp = e.props[li]
            pre = np.dtype([(f"p{i}", end + _TYPES[p.type]) for i, p in enumerate(e.props[:li])])
            cdt = np.dtype(end + _TYPES[lp.count_type])
            first = pos + pre.itemsize
            if first + cdt.itemsize <= len(body):
                k = int(np.frombuffer(body, cdt, 1, first)[0])
                fields = [(f"p{i}", end + _TYPES[p.type]) for i, p in enumerate(e.props[:li])]
                fields.append(("n", cdt.str))
                if k > 0:
                    fields.append(("v", end + _TYPES[lp.type], (k,)))
                fields += [(f"q{i}", end + _TYPES[p.type]) for i, p in enumerate(e.props[li + 1:])]
                dt = np.dtype(fields)
                need = dt.itemsize * e.count
                if pos + need <= len(body):
                    rec = np.frombuffer(body, dt, e.count, pos)
                    if np.all(rec["n"] == k):
                        pos += need
                        if e.name == "face" and lp.name == "vertex_indices" and k > 0:
                            tris.append(_fan_uniform(
                                rec["v"].reshape(e.count, k).astype(np.float64).astype(np.int64)))
                        done = True
        if done:
            continue
        for _ in range(e.count):
            names, values, face = [], [], None
            for p in e.props:
                if p.count_type is not None:
                    cdt = np.dtype(end + _TYPES[p.count_type])
                    if pos + cdt.itemsize > len(body):
                        raise PlyError("truncated PLY file")
                    cnt = int(np.frombuffer(body, cdt, 1, pos)[0])
                    pos += cdt.itemsize
                    vdt = np.dtype(end + _TYPES[p.type])
                    if pos + vdt.itemsize * cnt > len(body):
                        raise PlyError("truncated PLY file")
                    lst = np.frombuffer(body, vdt, cnt, pos)
                    pos += vdt.itemsize * cnt
                    if e.name == "face" and p.name == "vertex_indices":
                        face = lst.astype(np.float64).astype(np.int64)
                else:
                    vdt = np.dtype(end + _TYPES[p.type])
                    if pos + vdt.itemsize > len(body):
                        raise PlyError("truncated PLY file")
                    names.append(p.name)
                    values.append(float(np.frombuffer(body, vdt, 1, pos)[0]))
                    pos += vdt.itemsize
            if e.name == "vertex":
                points.record(names, values)
            if face is not None:
                tris.append(_fan_one(face))
    return points.array(), tris


def read_ply(path: str) -> tuple[np.ndarray, np.ndarray]:
    """Reads a PLY file: (points float32 (n, 3), vertex indices int64 (3m,)),
    the triangle fan of every face in file order."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise OSError(f"Could not open ply mesh file for reading: {path}") from e
    try:
        fmt, elems, body = _header(data)
        if fmt == "ascii":
            pts, tris = _read_ascii(data[body:], elems)
        else:
            pts, tris = _read_binary(memoryview(data)[body:], elems, fmt == "binary_big_endian")
    except PlyError as e:
        raise PlyError(f"Could not read ply file: {path} ({e})") from None
    verts = (np.concatenate([t.reshape(-1, 3) for t in tris]).reshape(-1) if tris
             else np.zeros(0, np.int64))
    if verts.size and (verts.min() < 0 or verts.max() >= len(pts)):
        raise PlyError(f"Could not read ply file: {path} (face index out of range)")
    return pts, verts.astype(np.int64)
