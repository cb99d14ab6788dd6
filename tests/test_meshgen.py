"""Procedural meshes: sizes, validity and conformity."""
import numpy as np
import pytest

from graphite_b200 import meshgen
from oracle import OracleMesh


def test_channel_bump_sizes():
    """60 x 20 x 4 hexes x 6 tets: 28,800 cells, 6,080 boundary faces,
    60,640 faces."""
    m = meshgen.channel_bump()
    c = m.counts()
    assert (c["cells"], c["ghosts"], c["faces"]) == (28800, 6080, 60640)
    assert meshgen.signed_tet_volumes(m).min() > 0


@pytest.mark.parametrize("cells", ["tet", "hex", "prism", "pyramid"])
def test_element_kinds_conform(cells):
    """Every face is shared by exactly two cells (ghosts included): the
    oracle's converter would reject the mesh otherwise."""
    m = meshgen.channel_bump(5, 3, 2, cells=cells)
    om = OracleMesh(m)
    assert om.N == m.n_cells and om.G == m.n_ghosts
    vol = om.get("cell_volumes")[: om.N]
    assert vol.min() > 0
    # the volumes of any split of the hex grid add up to the channel volume
    ref = OracleMesh(meshgen.channel_bump(5, 3, 2, cells="hex")).get("cell_volumes")[:30].sum()
    assert abs(vol.sum() - ref) < 1e-9 * ref


def test_airfoil_sizes():
    m = meshgen.airfoil_2d_prisms(40, 12)
    assert m.n_cells == 2 * 40 * 12
    om = OracleMesh(m)
    assert om.get("cell_volumes")[: om.N].min() > 0
    assert set(m.markers) == {"wing", "farfield", "sides"}


def test_swept_wing_small_is_valid():
    """Span-extruded prisms around the wing and the core beyond the tip: a
    conforming mesh (the oracle's converter checks that every face has two
    cells) with positive volumes, three boundary regions and well-conditioned
    least-squares systems."""
    m = meshgen.swept_wing(n_around=24, n_radial=8, n_span_wing=4, n_span_out=3)
    om = OracleMesh(m)
    assert set(m.markers) == {"wing", "symmetry", "farfield"}
    vol = om.get("cell_volumes")[: om.N]
    assert vol.min() > 0
    N = om.N
    cfs, cc = om.get("cell_faces_starts"), om.get("cell_connects")
    c = om.get("cell_centers").reshape(-1, 3)
    owner = np.repeat(np.arange(N), np.diff(cfs[: N + 1]))
    d = c[cc[: cfs[N]]] - c[owner]
    u = d / np.linalg.norm(d, axis=1, keepdims=True)
    a = np.zeros((N, 3, 3))
    np.add.at(a, owner, u[:, :, None] * u[:, None, :])
    assert np.linalg.eigvalsh(a)[:, 0].min() > 1e-3
    # the symmetry plane is flat at y = 0
    sym = np.concatenate([c.reshape(-1) for _, c in m.markers["symmetry"]])
    assert np.allclose(m.nodes[sym, 1], 0.0)


def test_su2_round_trip(tmp_path):
    m = meshgen.channel_bump(3, 2, 2)
    p = tmp_path / "c.su2"
    m.write_su2(str(p))
    text = p.read_text().splitlines()
    assert text[0] == "NDIME= 3"
    assert text[1] == f"NELEM= {m.n_cells}"
    # node coordinates are float32 values written exactly
    npo = text.index(f"NPOIN= {m.nodes.shape[0]}")
    xyz = np.array([[float(v) for v in line.split()[:3]] for line in text[npo + 1: npo + 1 + m.nodes.shape[0]]])
    assert np.array_equal(xyz, m.nodes)
    assert np.array_equal(xyz.astype(np.float32).astype(np.float64), xyz)
