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

    ``cells`` = "tet" (6 tets per hex), "hex", "prism" (2 per hex) or
    "pyramid" (6 pyramids per hex around a centre node).  Regions: inlet,
    outlet, lower (bump wall), upper, sides.
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
    if cells == "tet":
        blocks = [(TET, _kuhn_tets(corners))]
    elif cells == "hex":
        order = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
        blocks = [(HEX, np.stack([corners[:, a, b, c] for a, b, c in order], axis=1))]
    elif cells == "prism":
        blocks = [(PRISM, _prisms(corners))]
    elif cells == "pyramid":
        centres = nodes[corners.reshape(-1, 8)].mean(axis=1)
        cid = nodes.shape[0] + np.arange(corners.shape[0])
        nodes = np.concatenate([nodes, _f32(centres)])
        quads = [[(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)], [(0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)],
                 [(0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)], [(0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)],
                 [(0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)], [(1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)]]
        pyr = np.empty((corners.shape[0], 6, 5), dtype=np.int64)
        for q, quad in enumerate(quads):
            for v, (a, b, c) in enumerate(quad):
                pyr[:, q, v] = corners[:, a, b, c]
            pyr[:, q, 4] = cid
        blocks = [(PYRAMID, pyr.reshape(-1, 5))]
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
def naca0012_contour(n: int, closed_te: bool = True) -> Tuple[np.ndarray, np.ndarray]:
    """O-grid contour with ``n`` points (n even), index 0 at the trailing edge,
    running over the upper surface to the leading edge (n/2) and back along
    the lower surface.  Cosine clustering at both edges; unit chord."""
    assert n % 2 == 0
    half = n // 2
    beta = np.linspace(0.0, math.pi, half + 1)
    x = 0.5 * (1.0 + np.cos(beta))          # 1 -> 0 (TE to LE)
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


def airfoil_2d_prisms(n_around: int, n_radial: int, span: float = 0.1, r_far: float = 20.0,
                      first: float = 2e-3) -> ElementMesh:
    """2-D NACA 0012 O-grid, quads cut into 2 triangles, extruded one layer in y.

    Triangles = 2 * n_around * n_radial = cells (prisms).  Regions: wing,
    farfield, sides (the two span planes).
    """
    xc, zc = naca0012_contour(n_around)
    centre = np.array([0.5, 0.0])
    theta = np.arctan2(zc - centre[1], xc - centre[0])
    d = _radial(n_radial, first / r_far, 1.0)
    # blend from contour to far circle along each grid line
    far_x = centre[0] + r_far * np.cos(theta)
    far_z = centre[1] + r_far * np.sin(theta)
    w = d[None, :]
    # blend with a radius-stretching so near-wall spacing is ~first
    X2 = xc[:, None] + (far_x - xc)[:, None] * w
    Z2 = zc[:, None] + (far_z - zc)[:, None] * w
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
# Swept, tapered NACA 0012 semispan wing: prism layers + tets to a far-field
# hemisphere (truncated by a flat cap), with a rounded tip that closes onto a
# slit beyond which upper and lower O-grid nodes coincide.
# ---------------------------------------------------------------------------
def swept_wing(n_around: int = 144, n_radial: int = 37, n_prism: int = 8, n_span_wing: int = 24,
               n_span_tip: int = 4, n_span_out: int = 12, semispan: float = 1.5, sweep_deg: float = 30.0,
               taper: float = 0.56, r_far: float = 20.0, first: float = 2e-3) -> ElementMesh:
    """Semispan wing on the symmetry plane y = 0.

    Stations are planes y = const: ``n_span_wing`` layers over the wing,
    ``n_span_tip`` layers over a rounded tip cap of span equal to the tip
    thickness, and ``n_span_out`` layers beyond, where the section has
    collapsed onto its chord line (a slit whose upper and lower nodes are
    shared, so the faces on it are interior).  Each station is an O-grid from
    the section (or slit) out to the circle where the far-field sphere of
    radius ``r_far`` cuts the station plane; the last station is a flat cap.
    Cells: prisms in the first ``n_prism`` radial layers, 6 tets per hex
    beyond.  Regions: wing, symmetry, farfield.
    """
    ni = n_around
    half = ni // 2
    xc, zc = naca0012_contour(ni)
    tan_sw = math.tan(math.radians(sweep_deg))
    c_tip = taper
    t_tip = 0.12 * c_tip
    tip_len = t_tip * 0.5
    y_end = semispan + tip_len
    y_last = 0.85 * r_far
    # spanwise stations
    yw = semispan * (1 - np.cos(np.linspace(0, math.pi / 2, n_span_wing + 1)))      # clustered to tip
    yt = semispan + tip_len * np.sin(np.linspace(0, math.pi / 2, n_span_tip + 1))[1:]
    g = _radial(n_span_out, (yw[-1] - yw[-2]) * 1.5, y_last - y_end)[1:]
    yo = y_end + g
    ys = np.concatenate([yw, yt, yo])
    nj = ys.size - 1
    j_end = n_span_wing + n_span_tip            # first station that is a slit
    # section scale per station
    chord = np.where(ys <= semispan, 1.0 - (1.0 - taper) * ys / semispan, c_tip)
    x_le = np.minimum(ys, semispan) * tan_sw
    thick = np.ones_like(ys)
    tip_sel = ys > semispan
    thick[tip_sel] = np.sqrt(np.clip(1.0 - ((ys[tip_sel] - semispan) / tip_len) ** 2, 0.0, 1.0))
    thick[j_end:] = 0.0
    # radial distribution (fraction of the way from contour to far circle)
    d = _radial(n_radial, first / r_far, 1.0)
    nk = n_radial
    X = np.empty((ni, nk + 1, nj + 1))
    Y = np.empty_like(X)
    Z = np.empty_like(X)
    for j in range(nj + 1):
        cx = x_le[j] + chord[j] * xc
        cz = chord[j] * zc * thick[j]
        ctr_x = x_le[j] + 0.5 * chord[j]
        r_st = math.sqrt(max(r_far ** 2 - ys[j] ** 2, 1e-12))
        theta = np.arctan2(chord[j] * zc, cx - ctr_x)
        fx = ctr_x + r_st * np.cos(theta)
        fz = r_st * np.sin(theta)
        X[:, :, j] = cx[:, None] + (fx - cx)[:, None] * d[None, :]
        Z[:, :, j] = cz[:, None] + (fz - cz)[:, None] * d[None, :]
        Y[:, :, j] = ys[j]
    pts = np.stack([X, Y, Z], axis=-1)
    # node numbering with the slit merge: for j >= j_end, k = 0, node (i) and
    # (ni - i) are one node.
    node_index = -np.ones((ni, nk + 1, nj + 1), dtype=np.int64)
    count = 0
    flat_pts = []
    for j in range(nj + 1):
        for k in range(nk + 1):
            for_i = np.arange(ni)
            if j >= j_end and k == 0:
                own = for_i <= half
                ids = np.empty(ni, dtype=np.int64)
                ids[own] = count + np.arange(own.sum())
                ids[~own] = ids[ni - for_i[~own]]
                node_index[:, k, j] = ids
                flat_pts.append(pts[own, k, j])
                count += int(own.sum())
            else:
                node_index[:, k, j] = count + for_i
                flat_pts.append(pts[:, k, j])
                count += ni
    nodes = _f32(np.concatenate(flat_pts))
    # cells: axes (i around, j span, k radial) so that prisms extrude along k
    # and lie in the (i, j) wall plane.
    node_ijk = np.transpose(node_index, (0, 2, 1))            # [i, j, k]
    ci, cj, ck = np.meshgrid(np.arange(ni), np.arange(nj), np.arange(nk), indexing="ij")
    cells = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)
    corners = _hex_corner_ids(node_ijk, cells)
    mirror = cells[:, 0] >= half
    is_prism = cells[:, 2] < n_prism
    # SU2 order: prisms first (wall layers), then tets, each in (j, i, k) order
    order_p = np.lexsort((cells[is_prism, 2], cells[is_prism, 0], cells[is_prism, 1]))
    order_t = np.lexsort((cells[~is_prism, 2], cells[~is_prism, 0], cells[~is_prism, 1]))
    prisms = _prisms(corners[is_prism][order_p], mirror[is_prism][order_p])
    tets = _kuhn_tets(corners[~is_prism][order_t], mirror[~is_prism][order_t])
    blocks = [(PRISM, prisms), (TET, tets)]
    # node tags
    kk = np.broadcast_to(np.arange(nk + 1)[None, :, None], node_index.shape)
    jj = np.broadcast_to(np.arange(nj + 1)[None, None, :], node_index.shape)

    def tag(mask):
        t = np.zeros(nodes.shape[0], dtype=bool)
        t[node_index[mask]] = True
        return t

    tags = {"wing": tag((kk == 0) & (jj <= j_end)), "symmetry": tag(jj == 0),
            "farfield": tag((kk == nk) | (jj == nj))}
    markers = _classify(_boundary_faces(blocks), tags)
    return ElementMesh(nodes, blocks, markers, name=f"swept_wing_{prisms.shape[0] + tets.shape[0]}")


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
