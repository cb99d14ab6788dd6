"""Comparison helpers shared by the tests."""
from __future__ import annotations

import struct

import numpy as np


def face_keys(starts: np.ndarray, nodes: np.ndarray):
    return [tuple(sorted(nodes[starts[i]:starts[i + 1]].tolist())) for i in range(len(starts) - 1)]


def face_map(starts_a, nodes_a, starts_b, nodes_b) -> np.ndarray:
    """perm with face b[perm[i]] == face a[i] (faces matched by node set)."""
    kb = {k: i for i, k in enumerate(face_keys(starts_b, nodes_b))}
    return np.array([kb[k] for k in face_keys(starts_a, nodes_a)], dtype=np.int64)


def rel_max(a, b) -> float:
    """max |a - b| / max |b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def read_fvm(path: str):
    """Parse a .fvm file (layout of src/meshio.cu:1150-1216)."""
    d = open(path, "rb").read()
    pos = 0

    def u():
        nonlocal pos
        v = struct.unpack_from("<I", d, pos)[0]
        pos += 4
        return v

    nn = u()
    nodes = np.frombuffer(d, np.float32, nn * 3, pos).reshape(nn, 3)
    pos += nn * 12
    nf, _ = u(), u()
    faces = []
    for _ in range(nf):
        s = u()
        faces.append(struct.unpack_from("<%dI" % s, d, pos))
        pos += 4 * s
    ncg, _ = u(), u()
    cells = []
    for _ in range(ncg):
        s = u()
        f = struct.unpack_from("<%dI" % s, d, pos)
        pos += 4 * s
        c = struct.unpack_from("<%dI" % s, d, pos)
        pos += 4 * s
        cells.append((f, c))
    nr, _ = u(), u()
    regions = []
    for _ in range(nr):
        name = d[pos:pos + 128].split(b"\0")[0].decode()
        pos += 128
        s = u()
        regions.append((name, struct.unpack_from("<%dI" % s, d, pos)))
        pos += 4 * s
    assert pos == len(d)
    return nodes, faces, cells, regions
