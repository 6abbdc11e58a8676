"""Writes tests/golden/ply_golden.npz: every file of ply_cases.py (its bytes)
with the points and triangle indices the reference's own PLY reader
(read_ply_to_mesh, src/dort/ply_mesh.cpp, compiled from the reference tree
into oracle/_ref/ by oracle/Makefile) makes of it.

    make -C oracle ref REF=<reference tree>
    python tests/golden/gen_ply_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ply_cases  # noqa: E402
import pyoracle  # noqa: E402


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, data in ply_cases.cases().items():
            path = os.path.join(tmp, name + ".ply")
            with open(path, "wb") as f:
                f.write(data)
            pts, verts = pyoracle.ref_read_ply(path)
            out[name + "/file"] = np.frombuffer(data, np.uint8)
            out[name + "/points"] = pts
            out[name + "/vertices"] = verts
            print(f"{name}: {len(data)} bytes, {len(pts)} points, {len(verts) // 3} triangles")
    np.savez_compressed(os.path.join(HERE, "ply_golden.npz"), **out)


if __name__ == "__main__":
    main()
