"""Procedural unstructured meshes for the finite-volume Euler path.

The reference ships no meshes (its cases are built with gmsh from ``.geo``
scripts), so every workload here is generated: a structured block of hexes is
laid out in index space, mapped to physical space, and each hex is split into
tets (Kuhn/Freudenthal split, 6 tets around the main diagonal) or into two
prisms (wall layers).  The split patterns are chosen so that neighbouring
cells always share identical faces, including across the O-grid seam and the
collapsed slit beyond a wing tip, so the result is a conforming unstructured
mesh.  Boundary faces are recovered by face de-duplication and classified by
node tags.

Element kinds and local node orders follow the SU2 native format that the
reference reads (src/meshio.cu:297-475): 5 triangle, 9 quad, 10 tetra,
12 hexahedron, 13 wedge (prism), 14 pyramid.

Node coordinates are rounded to float32 before they are stored, so a float32
reader (the reference's ``fscanf("%f")``, src/meshio.cu:863) and a float64
reader see exactly the same geometry.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

TRI, QUAD, TET, HEX, PRISM, PYRAMID = 5, 9, 10, 12, 13, 14
NODES_PER_KIND = {TRI: 3, QUAD: 4, TET: 4, HEX: 8, PRISM: 6, PYRAMID: 5}

# Local faces per element kind, in the order the reference's converter lists
# them (src/meshio.cu:315-475).  The per-cell face order decides the order in
# which a cell sums its face contributions.
LOCAL_FACES = {
    TET: [(0, 2, 1), (0, 1, 3), (1, 2, 3), (0, 3, 2)],
    HEX: [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7), (3, 2, 1, 0), (4, 5, 6, 7)],
    PRISM: [(0, 1, 2), (3, 5, 4), (0, 2, 5, 3), (1, 4, 5, 2), (1, 0, 3, 4)],
    PYRAMID: [(0, 1, 2, 3), (0, 4, 3), (0, 1, 4), (1, 2, 4), (2, 3, 4)],
}


@dataclasses.dataclass
class ElementMesh:
    """Nodes, volume elements and boundary markers of an unstructured mesh.

    ``blocks`` holds the volume elements as ``(kind, int64[n, k])`` in SU2
    order; ``markers`` maps a boundary region name to its boundary faces as a
    list of ``(kind, int64[m, k])`` (triangles and quads).
    """

    nodes: np.ndarray
    blocks: List[Tuple[int, np.ndarray]]
    markers: Dict[str, List[Tuple[int, np.ndarray]]]
    name: str = "mesh"

    @property
    def n_cells(self) -> int:
        return int(sum(b.shape[0] for _, b in self.blocks))

    @property
    def n_ghosts(self) -> int:
        return int(sum(a.shape[0] for faces in self.markers.values() for _, a in faces))

    def counts(self) -> Dict[str, int]:
        s = sum(len(LOCAL_FACES[k]) * b.shape[0] for k, b in self.blocks)
        g = self.n_ghosts
        return {"cells": self.n_cells, "ghosts": g, "faces": (s + g) // 2,
                "cell_faces": s, "nodes": int(self.nodes.shape[0])}

    def write_su2(self, path: str) -> None:
        """Write the mesh in SU2 native text format (3-D)."""
        with open(path, "w") as f:
            f.write("NDIME= 3\n")
            f.write(f"NELEM= {self.n_cells}\n")
            eid = 0
            for kind, conn in self.blocks:
                n = conn.shape[0]
                arr = np.empty((n, conn.shape[1] + 2), dtype=np.int64)
                arr[:, 0] = kind
                arr[:, 1:-1] = conn
                arr[:, -1] = np.arange(eid, eid + n)
                eid += n
                _write_int_rows(f, arr)
            f.write(f"NPOIN= {self.nodes.shape[0]}\n")
            pts = self.nodes
            ids = np.arange(pts.shape[0])
            lines = [f"{x:.17g} {y:.17g} {z:.17g} {i}\n" for (x, y, z), i in zip(pts.tolist(), ids.tolist())]
            f.write("".join(lines))
            f.write(f"NMARK= {len(self.markers)}\n")
            for name, faces in self.markers.items():
                m = sum(a.shape[0] for _, a in faces)
                f.write(f"MARKER_TAG= {name}\n")
                f.write(f"MARKER_ELEMS= {m}\n")
                for kind, conn in faces:
                    arr = np.empty((conn.shape[0], conn.shape[1] + 1), dtype=np.int64)
                    arr[:, 0] = kind
                    arr[:, 1:] = conn
                    _write_int_rows(f, arr)


def _write_int_rows(f, arr: np.ndarray) -> None:
    if arr.shape[0] == 0:
        return
    fmt = " ".join(["%d"] * arr.shape[1])
    chunk = 1 << 16
    for s in range(0, arr.shape[0], chunk):
        block = arr[s:s + chunk]
        f.write("\n".join(fmt % tuple(r) for r in block.tolist()))
        f.write("\n")


def _f32(x: np.ndarray) -> np.ndarray:
    return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


# ---------------------------------------------------------------------------
# Hex splitting in index space.  A hex cell is addressed by its lower corner;
# corner (a, b, c) in {0,1}^3 is offset a along axis 0, b along axis 1, c
# along axis 2.  ``corner_ids`` has shape (n_cells, 2, 2, 2).
# ---------------------------------------------------------------------------
_KUHN_PATHS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def _kuhn_tets(corner_ids: np.ndarray, mirror0: np.ndarray | None = None) -> np.ndarray:
    """6 tets per hex around the diagonal (0,0,0)-(1,1,1).

    Where ``mirror0`` is set, axis 0 is reflected (diagonal (1,0,0)-(0,1,1)).
    All faces of a cell are cut along the diagonal through the face's lowest
    corner (reflected in axis 0 for mirrored cells), so equally oriented
    neighbours agree on every shared face.
    """
    n = corner_ids.shape[0]
    out = np.empty((n, 6, 4), dtype=np.int64)
    if mirror0 is None:
        mirror0 = np.zeros(n, dtype=bool)
    for t, path in enumerate(_KUHN_PATHS):
        p = np.zeros(3, dtype=np.int64)
        verts = [p.copy()]
        for ax in path:
            p[ax] = 1
            verts.append(p.copy())
        for v, (a, b, c) in enumerate(verts):
            plain = corner_ids[:, a, b, c]
            mirr = corner_ids[:, 1 - a, b, c]
            out[:, t, v] = np.where(mirror0, mirr, plain)
    return out.reshape(n * 6, 4)


def _prisms(corner_ids: np.ndarray, mirror0: np.ndarray | None = None) -> np.ndarray:
    """2 prisms per hex, extruded along axis 2, triangles in the (0,1) plane.

    The triangle diagonal is (0,0)-(1,1), or (1,0)-(0,1) where ``mirror0`` is
    set, matching the Kuhn split's cut of the axis-2 faces.
    """
    n = corner_ids.shape[0]
    if mirror0 is None:
        mirror0 = np.zeros(n, dtype=bool)
    tris_plain = [((0, 0), (1, 0), (1, 1)), ((0, 0), (1, 1), (0, 1))]
    tris_mirr = [((1, 0), (1, 1), (0, 1)), ((1, 0), (0, 1), (0, 0))]
    out = np.empty((n, 2, 6), dtype=np.int64)
    for t in range(2):
        for v in range(3):
            for c in range(2):
                (a0, b0), (a1, b1) = tris_plain[t][v], tris_mirr[t][v]
                out[:, t, 3 * c + v] = np.where(mirror0, corner_ids[:, a1, b1, c], corner_ids[:, a0, b0, c])
    return out.reshape(n * 2, 6)


def _hex_corner_ids(node_index: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Corner node ids for hex cells given by lower-corner index triples."""
    i, j, k = cells[:, 0], cells[:, 1], cells[:, 2]
    out = np.empty((cells.shape[0], 2, 2, 2), dtype=np.int64)
    n0 = node_index.shape[0]
    for a in range(2):
        for b in range(2):
            for c in range(2):
                out[:, a, b, c] = node_index[(i + a) % n0, j + b, k + c]
    return out


def _element_faces(blocks: Sequence[Tuple[int, np.ndarray]]):
    tri_list, quad_list = [], []
    for kind, conn in blocks:
        for lf in LOCAL_FACES[kind]:
            (tri_list if len(lf) == 3 else quad_list).append(conn[:, list(lf)])
    tris = np.concatenate(tri_list) if tri_list else np.zeros((0, 3), np.int64)
    quads = np.concatenate(quad_list) if quad_list else np.zeros((0, 4), np.int64)
    return tris, quads


def _boundary_faces(blocks):
    """Faces that belong to exactly one volume element."""
    out = []
    for faces, kind in zip(_element_faces(blocks), (TRI, QUAD)):
        if faces.shape[0] == 0:
            continue
        key = np.sort(faces, axis=1)
        _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
        inv = inv.reshape(-1)
        if cnt.max() > 2:
            raise ValueError("non-manifold mesh: a face is shared by more than two elements")
        out.append((kind, faces[cnt[inv] == 1]))
    return out


def _classify(bfaces, tags: Dict[str, np.ndarray]):
    """Assign each boundary face to the first region whose node tag holds all its nodes."""
    markers: Dict[str, List[Tuple[int, np.ndarray]]] = {name: [] for name in tags}
    for kind, faces in bfaces:
        left = np.ones(faces.shape[0], dtype=bool)
        for name, tag in tags.items():
            sel = left & np.all(tag[faces], axis=1)
            if sel.any():
                markers[name].append((kind, faces[sel]))
            left &= ~sel
        if left.any():
            raise ValueError(f"{int(left.sum())} boundary faces match no region")
    return {k: v for k, v in markers.items() if v}


# ---------------------------------------------------------------------------
# Channel with a circular-arc bump (all tets).
# ---------------------------------------------------------------------------
def channel_bump(nx: int = 60, ny: int = 20, nz: int = 4, length: float = 3.0, height: float = 1.0,
                 width: float = 0.2, bump_height: float = 0.1, cells: str = "tet") -> ElementMesh:
    """Channel [0,L]x[0,H]x[0,W] with a circular-arc bump of chord 1 on x in [1,2].

    ``cells`` = "tet" (6 tets per hex), "hex", "prism" (2 per hex),
    "pyramid" (6 pyramids per hex around a centre node), "mixed" (hexes,
    prisms and pyramids in thirds of the columns along x: every face between
    them is a whole quad on both sides) or "layered" (prisms in the lower
    half of the z layers, tets above: the prisms' triangles are cut along the
    tets' diagonal).  Regions: inlet, outlet, lower (bump wall), upper, sides.
    """
    xs = np.linspace(0.0, length, nx + 1)
    r = (0.25 + bump_height ** 2) / (2 * bump_height) if bump_height > 0 else 0.0
    yw = np.zeros_like(xs)
    if bump_height > 0:
        inb = (xs >= 1.0) & (xs <= 2.0)
        yw[inb] = np.sqrt(np.maximum(r * r - (xs[inb] - 1.5) ** 2, 0.0)) - (r - bump_height)
    eta = np.linspace(0.0, 1.0, ny + 1)
    zs = np.linspace(0.0, width, nz + 1)
    X = np.broadcast_to(xs[:, None, None], (nx + 1, ny + 1, nz + 1))
    Y = yw[:, None, None] + (height - yw[:, None, None]) * eta[None, :, None]
    Y = np.broadcast_to(Y, (nx + 1, ny + 1, nz + 1))
    Z = np.broadcast_to(zs[None, None, :], (nx + 1, ny + 1, nz + 1))
    nodes = _f32(np.stack([X, Y, Z], axis=-1).reshape(-1, 3))
    node_index = np.arange(nodes.shape[0]).reshape(nx + 1, ny + 1, nz + 1)
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cells_ijk = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)
    # node_index's first axis must not wrap: pad so (i + 1) % n0 is i + 1.
    pad = np.concatenate([node_index, node_index[:1]], axis=0)
    corners = _hex_corner_ids(pad, cells_ijk)
    def hexes(cs):
        order = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
        return np.stack([cs[:, a, b, c] for a, b, c in order], axis=1)

    def pyramids(nodes, cs):
        centres = nodes[cs.reshape(-1, 8)].mean(axis=1)
        cid = nodes.shape[0] + np.arange(cs.shape[0])
        quads = [[(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)], [(0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)],
                 [(0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)], [(0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)],
                 [(0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)], [(1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)]]
        pyr = np.empty((cs.shape[0], 6, 5), dtype=np.int64)
        for q, quad in enumerate(quads):
            for v, (a, b, c) in enumerate(quad):
                pyr[:, q, v] = cs[:, a, b, c]
            pyr[:, q, 4] = cid
        return np.concatenate([nodes, _f32(centres)]), pyr.reshape(-1, 5)

    if cells == "tet":
        blocks = [(TET, _kuhn_tets(corners))]
    elif cells == "hex":
        blocks = [(HEX, hexes(corners))]
    elif cells == "prism":
        blocks = [(PRISM, _prisms(corners))]
    elif cells == "pyramid":
        nodes, pyr = pyramids(nodes, corners)
        blocks = [(PYRAMID, pyr)]
    elif cells == "mixed":
        col = cells_ijk[:, 0]
        zone = np.where(col < nx // 3, 0, np.where(col < 2 * nx // 3, 1, 2))
        nodes, pyr = pyramids(nodes, corners[zone == 2])
        blocks = [(HEX, hexes(corners[zone == 0])), (PRISM, _prisms(corners[zone == 1])), (PYRAMID, pyr)]
    elif cells == "layered":
        low = cells_ijk[:, 2] < max(nz // 2, 1)
        blocks = [(PRISM, _prisms(corners[low])), (TET, _kuhn_tets(corners[~low]))]
    else:
        raise ValueError(cells)
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    n_struct = (nx + 1) * (ny + 1) * (nz + 1)

    def tag(mask):
        t = np.zeros(nodes.shape[0], dtype=bool)
        t[:n_struct] = mask.ravel()
        return t

    tags = {"inlet": tag(ii == 0), "outlet": tag(ii == nx), "lower": tag(jj == 0),
            "upper": tag(jj == ny), "sides": tag((kk == 0) | (kk == nz))}
    markers = _classify(_boundary_faces(blocks), tags)
    return ElementMesh(nodes, blocks, markers, name=f"channel_bump_{nx}x{ny}x{nz}_{cells}")


# ---------------------------------------------------------------------------
# NACA 0012 sections.
# ---------------------------------------------------------------------------
def naca0012_contour(n: int, closed_te: bool = True, cluster: float = 1.0) -> Tuple[np.ndarray, np.ndarray]:
    """O-grid contour with ``n`` points (n even), index 0 at the trailing edge,
    running over the upper surface to the leading edge (n/2) and back along
    the lower surface; unit chord.  Points are a blend of cosine clustering at
    both edges (weight ``cluster``) and even spacing in x."""
    assert n % 2 == 0
    half = n // 2
    beta = np.linspace(0.0, math.pi, half + 1)
    x = cluster * 0.5 * (1.0 + np.cos(beta)) + (1.0 - cluster) * (1.0 - beta / math.pi)   # TE -> LE
    a4 = -0.1036 if closed_te else -0.1015
    t = 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 + a4 * x ** 4)
    xu, zu = x, t
    xl, zl = x[::-1][1:-1], -t[::-1][1:-1]
    return np.concatenate([xu, xl]), np.concatenate([zu, zl])


def _radial(n: int, first: float, total: float) -> np.ndarray:
    """n+1 increasing distances 0..total, first step ~``first``, geometric."""
    if n == 1:
        return np.array([0.0, total])
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        q = 0.5 * (lo + hi)
        s = first * (q ** n - 1) / (q - 1)
        if s > total:
            hi = q
        else:
            lo = q
    q = 0.5 * (lo + hi)
    d = first * (q ** np.arange(n + 1) - 1) / (q - 1)
    return d * (total / d[-1])



def _contour_normals(xc: np.ndarray, zc: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Outward unit normals of a closed contour (either orientation),
    averaged over the two edges at each point."""
    px, pz = np.roll(xc, 1), np.roll(zc, 1)
    nx_, nz_ = np.roll(xc, -1), np.roll(zc, -1)
    e1 = np.stack([xc - px, zc - pz], 1)
    e2 = np.stack([nx_ - xc, nz_ - zc], 1)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
    t = e1 + e2
    n = np.stack([t[:, 1], -t[:, 0]], 1)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    # orient outward: away from the contour's centroid
    c = np.array([xc.mean(), zc.mean()])
    if np.sum((np.stack([xc, zc], 1) - c) * n) < 0:
        n = -n
    return n[:, 0], n[:, 1]


def _ogrid_lines(cx, cz, fx, fz, d, delta):
    """Grid lines from contour points (cx, cz) to far points (fx, fz) at the
    distance fractions d: they leave the surface along its normal and turn
    towards the straight line to the far point over a length ~delta, so the
    first cells are orthogonal to the wall even at sharp corners."""
    nx_, nz_ = _contour_normals(cx, cz)
    L = np.hypot(fx - cx, fz - cz)
    sx, sz = (fx - cx) / L, (fz - cz) / L
    dist = d[None, :] * L[:, None]
    w = np.exp(-dist / delta)
    dx = w * nx_[:, None] + (1 - w) * sx[:, None]
    dz = w * nz_[:, None] + (1 - w) * sz[:, None]
    nrm = np.hypot(dx, dz)
    X = cx[:, None] + dx / nrm * dist
    Z = cz[:, None] + dz / nrm * dist
    return X, Z


def airfoil_2d_prisms(n_around: int, n_radial: int, span: float = 0.1, r_far: float = 20.0,
                      first: float = 2e-3, cluster: float = 0.5) -> ElementMesh:
    """2-D NACA 0012 O-grid, quads cut into 2 triangles, extruded one layer in y.

    Triangles = 2 * n_around * n_radial = cells (prisms).  Regions: wing,
    farfield, sides (the two span planes).
    """
    xc, zc = naca0012_contour(n_around, cluster=cluster)
    centre = np.array([0.5, 0.0])
    theta = 2.0 * math.pi * np.arange(n_around) / n_around     # even far-field angles
    d = _radial(n_radial, first / r_far, 1.0)
    # blend from contour to far circle along each grid line
    far_x = centre[0] + r_far * np.cos(theta)
    far_z = centre[1] + r_far * np.sin(theta)
    X2, Z2 = _ogrid_lines(xc, zc, far_x, far_z, d, 0.1)
    ys = np.array([0.0, span])
    X = np.broadcast_to(X2[:, :, None], (n_around, n_radial + 1, 2))
    Z = np.broadcast_to(Z2[:, :, None], (n_around, n_radial + 1, 2))
    Y = np.broadcast_to(ys[None, None, :], (n_around, n_radial + 1, 2))
    nodes = _f32(np.stack([X, Y, Z], axis=-1).reshape(-1, 3))
    node_index = np.arange(nodes.shape[0]).reshape(n_around, n_radial + 1, 2)
    ci, ck = np.meshgrid(np.arange(n_around), np.arange(n_radial), indexing="ij")
    # axes: 0 = around (periodic), 1 = radial, 2 = span.  Prisms extrude along
    # axis 2 here, so build corners with (around, radial, span).
    cells = np.stack([ci.ravel(), ck.ravel(), np.zeros(ci.size, dtype=np.int64)], axis=1)
    corners = _hex_corner_ids(node_index, cells)
    blocks = [(PRISM, _prisms(corners))]
    ii, kk, jj = np.meshgrid(np.arange(n_around), np.arange(n_radial + 1), np.arange(2), indexing="ij")
    tags = {"wing": (kk == 0).ravel(), "farfield": (kk == n_radial).ravel(), "sides": np.ones(nodes.shape[0], bool)}
    markers = _classify(_boundary_faces(blocks), tags)
    return ElementMesh(nodes, blocks, markers, name=f"airfoil2d_{2 * n_around * n_radial}")


AIRFOIL_SIZES = {50_000: (250, 100), 120_000: (400, 150), 300_000: (600, 250)}


def airfoil_extruded(n_triangles: int) -> ElementMesh:
    """The 50k / 120k / 300k triangle airfoil meshes (one prism layer)."""
    if n_triangles in AIRFOIL_SIZES:
        na, nr = AIRFOIL_SIZES[n_triangles]
    else:
        nr = max(4, int(round(math.sqrt(n_triangles / 2 / 1.6))))
        na = max(8, int(round(n_triangles / 2 / nr / 2)) * 2)
    return airfoil_2d_prisms(na, nr)


# ---------------------------------------------------------------------------
# Swept, tapered NACA 0012 semispan wing with a flat tip cap: prism layers +
# tets out to a far-field sphere (truncated by a flat cap).  Beyond the tip
# the tip section continues spanwise and its interior is filled with a core
# block of tets, so no cell is degenerate.
# ---------------------------------------------------------------------------
def naca0012_blunt_contour(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """O-grid contour of n points (n even) with a blunt trailing edge (the
    open-TE NACA 0012, base 0.25 % chord): index 0 is the middle of the base,
    1 the upper TE corner, n/2 the leading edge, n-1 the lower TE corner."""
    assert n % 2 == 0 and n >= 8
    half = n // 2
    beta = np.linspace(0.0, math.pi, half)            # upper corner .. LE: half points
    x = 0.5 * (1.0 + np.cos(beta))
    t = 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1015 * x ** 4)
    xu, zu = x, t                                      # indices 1 .. half
    xl, zl = x[::-1][1:-1], -t[::-1][1:-1]             # indices half+1 .. n-1 (LE excluded, corner kept below)
    xl = np.concatenate([xl, [x[0]]])
    zl = np.concatenate([zl, [-t[0]]])
    return np.concatenate([[1.0], xu, xl]), np.concatenate([[0.0], zu, zl])


def _prism_to_tets(b, t, third_from_p: bool) -> np.ndarray:
    """Split prisms with bottom (s, p, q) = b[:, 0..2], top t[:, 0..2] into 3
    tets.  The quad faces s-p and s-q are cut from s (bottom) to the top
    vertex; face p-q from p (bottom) to q' (top) if third_from_p, else from q
    to p' (the diagonal orientation that avoids a cycle)."""
    s, p, q = b[:, 0], b[:, 1], b[:, 2]
    s1, p1, q1 = t[:, 0], t[:, 1], t[:, 2]
    if third_from_p:
        tets = [(s, p, q, q1), (s, p, q1, p1), (s, p1, q1, s1)]
    else:
        tets = [(s, p, q, p1), (s, q, q1, p1), (s, p1, q1, s1)]
    return np.stack([np.stack(tt, axis=1) for tt in tets], axis=1).reshape(-1, 4)


def _min_angle(p0, p1, p2):
    """Smallest interior angle of triangles (arrays of 2-D points)."""
    def ang(a, b, c):
        u, v = b - a, c - a
        cosv = np.sum(u * v, -1) / (np.linalg.norm(u, axis=-1) * np.linalg.norm(v, axis=-1))
        return np.arccos(np.clip(cosv, -1.0, 1.0))
    return np.minimum(np.minimum(ang(p0, p1, p2), ang(p1, p2, p0)), ang(p2, p0, p1))


def _anti_diagonal(X: np.ndarray, Z: np.ndarray) -> np.ndarray:
    """For the quads of a periodic-in-i structured section grid (X, Z of
    shape [i, k]), True where the cut (1,0)-(0,1) keeps a larger minimum angle
    than the cut (0,0)-(1,1)."""
    P = np.stack([X, Z], axis=-1)
    p00, p10 = P[:, :-1], np.roll(P, -1, axis=0)[:, :-1]
    p01, p11 = P[:, 1:], np.roll(P, -1, axis=0)[:, 1:]
    main = np.minimum(_min_angle(p00, p10, p11), _min_angle(p00, p11, p01))
    anti = np.minimum(_min_angle(p10, p11, p01), _min_angle(p10, p01, p00))
    return anti > main


def swept_wing(n_around: int = 160, n_radial: int = 48, n_span_wing: int = 40, n_span_out: int = 32,
               semispan: float = 1.5, sweep_deg: float = 30.0, taper: float = 0.56, r_far: float = 20.0,
               first: float = 2e-3, tip_cluster: float = 0.5, phi_max_deg: float = 75.0) -> ElementMesh:
    """Semispan wing on the symmetry plane y = 0 (about 1.1 M cells by default).

    Stations are planes y = const: ``n_span_wing`` layers from the root to the
    tip (mildly clustered towards the tip) and ``n_span_out`` layers beyond it
    out to y = 3 semispans, where a flat far-field cap closes the domain.
    Each station is an O-grid from the section out to the circle where the
    far-field sphere of radius ``r_far`` cuts the station plane; radial grid
    lines leave the section along its normal.  Cells are prisms extruded
    along the span with triangles in the section plane (well shaped from the
    wall to the far field; wall-parallel triangles or tets cut from the
    strongly anisotropic hexes give nearly singular least-squares systems).
    Beyond the flat tip cap the tip section continues as an interior surface
    that grows with the distance from the tip; inside it is a core of prisms.
    Regions: wing (surface and tip cap), symmetry, farfield (sphere and cap).
    """
    ni = n_around
    half = ni // 2
    xc, zc = naca0012_contour(ni, cluster=0.5)
    tan_sw = math.tan(math.radians(sweep_deg))
    u = np.linspace(0.0, 1.0, n_span_wing + 1)
    yw = semispan * ((1 - tip_cluster) * u + tip_cluster * np.sin(0.5 * math.pi * u))   # clustered to the tip
    g = _radial(n_span_out, (yw[-1] - yw[-2]) * 1.2, 2.0 * semispan)[1:]
    ys = np.concatenate([yw, semispan + g])
    nj = ys.size - 1
    jt = n_span_wing                                   # tip station
    chord = np.where(ys <= semispan, 1.0 - (1.0 - taper) * ys / semispan, taper)
    x_le = np.minimum(ys, semispan) * tan_sw
    theta = 2.0 * math.pi * np.arange(ni) / ni
    phi = math.radians(phi_max_deg) * np.arange(nj + 1) / nj
    x0 = 0.5 * semispan * tan_sw + 0.5
    nk = n_radial
    X = np.empty((ni, nk + 1, nj + 1))
    Y = np.empty_like(X)
    Z = np.empty_like(X)
    for j in range(nj + 1):
        ctr_x = x_le[j] + 0.5 * chord[j]
        cx = x_le[j] + chord[j] * xc
        cz = chord[j] * zc
        cy = np.full(ni, ys[j])
        # far points evenly spaced in longitude theta and latitude phi on the
        # sphere, so that cells grow in all three directions with the distance
        fx = x0 + r_far * math.cos(phi[j]) * np.cos(theta)
        fy = np.full(ni, r_far * math.sin(phi[j]))
        fz = r_far * math.cos(phi[j]) * np.sin(theta)
        nx_, nz_ = _contour_normals(cx, cz)
        L = np.sqrt((fx - cx) ** 2 + (fy - cy) ** 2 + (fz - cz) ** 2)
        d = _radial(n_radial, first / L.mean(), 1.0)
        dist = d[None, :] * L[:, None]
        w = np.exp(-dist / (1.0 * chord[j]))
        dx = w * nx_[:, None] + (1 - w) * ((fx - cx) / L)[:, None]
        dy = (1 - w) * ((fy - cy) / L)[:, None]
        dz = w * nz_[:, None] + (1 - w) * ((fz - cz) / L)[:, None]
        nrm = np.sqrt(dx * dx + dy * dy + dz * dz)
        X[:, :, j] = cx[:, None] + dx / nrm * dist
        Y[:, :, j] = cy[:, None] + dy / nrm * dist
        Z[:, :, j] = cz[:, None] + dz / nrm * dist
    n_og = ni * (nk + 1) * (nj + 1)
    node_index = np.arange(n_og).reshape(nj + 1, nk + 1, ni).transpose(2, 1, 0)   # [i, k, j]
    pts = np.stack([X, Y, Z], axis=-1).transpose(2, 1, 0, 3).reshape(-1, 3)      # id order (j, k, i)
    # core mid-thickness nodes for a = 1 .. half-1 at stations j >= jt
    mid_index = np.full((half, nj + 1), -1, dtype=np.int64)
    mid_pts = []
    nxt = n_og
    for j in range(jt, nj + 1):
        for a in range(1, half):
            mid_index[a, j] = nxt
            nxt += 1
            mid_pts.append(0.5 * (np.array([X[a, 0, j], Y[a, 0, j], Z[a, 0, j]]) +
                                  np.array([X[ni - a, 0, j], Y[ni - a, 0, j], Z[ni - a, 0, j]])))
    nodes = _f32(np.concatenate([pts, np.array(mid_pts).reshape(-1, 3)]))
    # O-grid cells: hexes (i around, k radial, j span) cut into 2 prisms
    # extruded along the span, triangles in the section plane.  Each section
    # quad is cut along the diagonal that keeps the larger minimum angle (at
    # the root station; the same cut at every station keeps faces shared).
    ci, ck, cj = np.meshgrid(np.arange(ni), np.arange(nk), np.arange(nj), indexing="ij")
    order = np.lexsort((ck.ravel(), ci.ravel(), cj.ravel()))            # SU2 order (j, i, k)
    cells = np.stack([ci.ravel(), ck.ravel(), cj.ravel()], axis=1)[order]
    corners = _hex_corner_ids(node_index, cells)
    anti = _anti_diagonal(X[:, :, 0], Z[:, :, 0])                        # [i, k]
    mirror = anti[cells[:, 0], cells[:, 1]]
    prisms = [_prisms(corners, mirror)]
    # core beyond the tip: hexes (a, row, j) for a = 1 .. half-2, rows 0 (upper
    # to mid) and 1 (mid to lower), cut into 2 span-extruded prisms; the
    # leading- and trailing-edge fans are one prism per row
    up = lambda a, j: node_index[a % ni, 0, j]
    lo = lambda a, j: node_index[(ni - a) % ni, 0, j]
    col = lambda a, j: (up(a, j), mid_index[a, j], lo(a, j))
    for j in range(jt, nj):
        cs = []
        for a in range(1, half - 1):
            for row in range(2):
                c = np.empty((2, 2, 2), dtype=np.int64)     # [a, c, j]
                for da in range(2):
                    for dj in range(2):
                        cc = col(a + da, j + dj)
                        c[da, 0, dj], c[da, 1, dj] = cc[row], cc[row + 1]
                cs.append(c)
        prisms.append(_prisms(np.array(cs)))
        le, le1 = node_index[half, 0, j], node_index[half, 0, j + 1]
        te, te1 = node_index[0, 0, j], node_index[0, 0, j + 1]
        n, n1 = col(half - 1, j), col(half - 1, j + 1)
        m, m1 = col(1, j), col(1, j + 1)
        fans = []
        for r in range(2):
            fans.append([le, n[r], n[r + 1], le1, n1[r], n1[r + 1]])
            fans.append([te, m[r], m[r + 1], te1, m1[r], m1[r + 1]])
        prisms.append(np.array(fans, dtype=np.int64))
    blocks = [(PRISM, np.concatenate(prisms))]
    # node tags
    kk = np.broadcast_to(np.arange(nk + 1)[None, :, None], node_index.shape)
    jj = np.broadcast_to(np.arange(nj + 1)[None, None, :], node_index.shape)

    def tag(mask, extra=None):
        t = np.zeros(nodes.shape[0], dtype=bool)
        t[node_index[mask]] = True
        if extra is not None:
            t[extra] = True
        return t

    tags = {"wing": tag((kk == 0) & (jj <= jt), mid_index[1:, jt]), "symmetry": tag(jj == 0),
            "farfield": tag((kk == nk) | (jj == nj), mid_index[1:, nj])}
    markers = _classify(_boundary_faces(blocks), tags)
    n_cells = sum(b.shape[0] for _, b in blocks)
    return ElementMesh(nodes, blocks, markers, name=f"swept_wing_{n_cells}")


def cylinder_ogrid(n_around: int = 400, n_radial: int = 250, ratio: float = 1.03, r_far: float = 30.0,
                   span: float = 0.1) -> ElementMesh:
    """O-grid of hexes around a unit-diameter cylinder, one cell in span.

    Radial spacing grows geometrically by ``ratio`` out to ``r_far``.
    Regions: cylinder, farfield, sides.
    """
    q = ratio
    first = (r_far - 0.5) * (q - 1) / (q ** n_radial - 1)
    r = 0.5 + first * (q ** np.arange(n_radial + 1) - 1) / (q - 1)
    th = np.linspace(0, 2 * math.pi, n_around, endpoint=False)
    X = np.cos(th)[:, None, None] * r[None, :, None] * np.ones((1, 1, 2))
    Z = np.sin(th)[:, None, None] * r[None, :, None] * np.ones((1, 1, 2))
    Y = np.broadcast_to(np.array([0.0, span])[None, None, :], X.shape)
    nodes = _f32(np.stack([X, Y, Z], axis=-1).reshape(-1, 3))
    node_index = np.arange(nodes.shape[0]).reshape(n_around, n_radial + 1, 2)
    ci, ck = np.meshgrid(np.arange(n_around), np.arange(n_radial), indexing="ij")
    cells = np.stack([ci.ravel(), ck.ravel(), np.zeros(ci.size, dtype=np.int64)], axis=1)
    corners = _hex_corner_ids(node_index, cells)
    order = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    blocks = [(HEX, np.stack([corners[:, a, b, c] for a, b, c in order], axis=1))]
    ii, kk, jj = np.meshgrid(np.arange(n_around), np.arange(n_radial + 1), np.arange(2), indexing="ij")
    tags = {"cylinder": (kk == 0).ravel(), "farfield": (kk == n_radial).ravel(), "sides": np.ones(nodes.shape[0], bool)}
    markers = _classify(_boundary_faces(blocks), tags)
    return ElementMesh(nodes, blocks, markers, name=f"cylinder_{n_around}x{n_radial}")


def signed_tet_volumes(mesh: ElementMesh) -> np.ndarray:
    """Absolute volumes of all tets in the mesh (mesh validity checks)."""
    vols = []
    for kind, conn in mesh.blocks:
        if kind != TET:
            continue
        p = mesh.nodes[conn]
        v = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6.0
        vols.append(np.abs(v))
    return np.concatenate(vols) if vols else np.zeros(0)
