"""The C ABI without a GPU: exported symbols, the SU2 -> .fvm converter
against the reference converter's own output, and error reporting."""
import os

import numpy as np
import pytest

import cases
from graphite_b200 import capi
from helpers import read_fvm

GOLDEN = os.path.dirname(cases.__file__)


def test_library_exports_every_declared_function():
    lib = capi.load()
    names = capi.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_header():
    # cuMeshBase: 2 ints, 5 size_t, 14 pointers; FvmField: 4 pointers + impl
    import ctypes as C
    assert C.sizeof(capi.gb_vector) == 12
    assert C.sizeof(capi.gb_tensor) == 36
    assert C.sizeof(capi.cuMeshBase) == 8 + 5 * 8 + 14 * 8
    assert C.sizeof(capi.FvmField) == 5 * 8
    assert C.sizeof(capi.gbBc) == 4 + 4 + 12 + 4 + 4


@pytest.mark.parametrize("name", ["tet_6x3x2", "hex_6x3x2", "prism_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2", "tet_12x6x2"])
def test_converter_matches_reference_converter(name, su2_paths, workdir):
    """cuMeshFromSu2 writes the file the reference's converter writes: same
    float32 nodes, same faces with the same node order, same cells (face
    lists in element-local order, neighbours), same regions; faces are
    numbered in first-appearance order instead of hash-bucket order."""
    out = str(workdir / f"{name}_mine.fvm")
    assert capi.load().cuMeshFromSu2(su2_paths(name).encode(), out.encode()) == 0, capi.last_error()
    rn, rf, rc, rr = read_fvm(os.path.join(GOLDEN, f"{name}_ref.fvm"))
    mn, mf, mc, mr = read_fvm(out)
    assert np.array_equal(rn, mn)
    key = {tuple(sorted(f)): i for i, f in enumerate(rf)}
    perm = [key[tuple(sorted(f))] for f in mf]          # my face -> reference face
    assert sorted(perm) == list(range(len(rf)))
    for i, f in enumerate(mf):
        assert rf[perm[i]] == f
    assert len(rc) == len(mc)
    for (rfaces, rconn), (mfaces, mconn) in zip(rc, mc):
        assert tuple(perm[f] for f in mfaces) == rfaces
        assert mconn == rconn
    assert rr == mr


@pytest.mark.parametrize("cells,shape", [("tet", (60, 30, 20)), ("hex", (60, 40, 60)), ("prism", (60, 30, 40)),
                                         ("pyramid", (60, 30, 13)), ("mixed", (60, 30, 30)),
                                         ("layered", (60, 30, 20))])
def test_parallel_converter_matches_oracle_topology(workdir, cells, shape):
    """With 130k-216k elements the converter builds the face records, sorts
    them and numbers the faces on several host threads; its file equals the
    oracle's serial topology (both number faces in first-appearance order)
    exactly, for triangle faces, quad faces and both mixed."""
    from graphite_b200 import meshgen
    from oracle import OracleMesh
    nx, ny, nz = shape
    mesh = meshgen.channel_bump(nx=nx, ny=ny, nz=nz, cells=cells)
    su2, out = str(workdir / f"par_{cells}.su2"), str(workdir / f"par_{cells}.fvm")
    mesh.write_su2(su2)
    assert capi.load().cuMeshFromSu2(su2.encode(), out.encode()) == 0, capi.last_error()
    nodes, faces, cells, regions = read_fvm(out)
    om = OracleMesh(mesh, metric_bits=64)
    assert (len(cells), len(faces)) == (om.N + om.G, om.F)
    fs, fn = om.get("face_nodes_starts"), om.get("face_nodes")
    assert np.array_equal(np.cumsum([0] + [len(f) for f in faces]), fs)
    assert np.array_equal(np.concatenate([np.array(f) for f in faces]), fn)
    cs = om.get("cell_faces_starts")
    assert np.array_equal(np.cumsum([0] + [len(c[0]) for c in cells]), cs)
    assert np.array_equal(np.concatenate([np.array(c[0]) for c in cells]), om.get("cell_faces"))
    assert np.array_equal(np.concatenate([np.array(c[1]) for c in cells]), om.get("cell_connects"))
    assert [r[0] for r in regions] == list(mesh.markers)


@pytest.mark.parametrize("first,second,message", [
    ("few", "kind", "element 100: too few nodes"),
    ("kind", "few", "element 100: unsupported volume element kind 7")])
def test_parallel_parse_reports_the_first_bad_element(workdir, first, second, message):
    """A 140k-element file parses on several host threads; with two bad
    elements in different threads' ranges the error still names the first
    one, with the check that fails first on its line."""
    from graphite_b200 import meshgen
    path = str(workdir / "two_errors.su2")
    meshgen.channel_bump(nx=60, ny=30, nz=13, cells="tet").write_su2(path)
    lines = open(path).read().split("\n")
    start = next(i for i, l in enumerate(lines) if l.startswith("NELEM=")) + 1
    def spoil(line, how):
        parts = line.split()
        return " ".join(parts[:3]) if how == "few" else " ".join(["7"] + parts[1:])
    lines[start + 100] = spoil(lines[start + 100], first)
    lines[start + 120000] = spoil(lines[start + 120000], second)
    with open(path, "w") as f:
        f.write("\n".join(lines))
    out = str(workdir / "two_errors.fvm").encode()
    assert capi.load().cuMeshFromSu2(path.encode(), out) != 0
    assert message in capi.last_error(), capi.last_error()


def test_parallel_builder_rejects_a_face_of_three_elements(workdir):
    """A 140k-element mesh with one element listed twice: its faces are shared
    by three elements, which the parallel grouping reports as non-manifold."""
    from graphite_b200 import meshgen
    path = str(workdir / "dup.su2")
    meshgen.channel_bump(nx=60, ny=30, nz=13, cells="tet").write_su2(path)
    lines = open(path).read().split("\n")
    at = next(i for i, l in enumerate(lines) if l.startswith("NELEM="))
    n = int(lines[at].split("=")[1])
    lines[at] = f"NELEM= {n + 1}"
    lines.insert(at + 1 + 70000, lines[at + 1 + 70000])
    with open(path, "w") as f:
        f.write("\n".join(lines))
    out = str(workdir / "dup.fvm").encode()
    assert capi.load().cuMeshFromSu2(path.encode(), out) != 0
    assert "non-manifold" in capi.last_error(), capi.last_error()


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)
    return path


def test_converter_errors(workdir):
    lib = capi.load()
    out = str(workdir / "bad.fvm").encode()
    assert lib.cuMeshFromSu2(b"/nonexistent/mesh.su2", out) != 0
    assert "cannot open" in capi.last_error()
    p = _write(str(workdir / "dim2.su2"), "NDIME= 2\n")
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "3D" in capi.last_error()
    # no elements at all
    p = _write(str(workdir / "empty.su2"), "NDIME= 3\nNELEM= 0\nNPOIN= 0\nNMARK= 0\n")
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "no elements" in capi.last_error()
    # a single tet with no boundary markers: open mesh
    tet = "NDIME= 3\nNELEM= 1\n10 0 1 2 3 0\nNPOIN= 4\n0 0 0 0\n1 0 0 1\n0 1 0 2\n0 0 1 3\n"
    p = _write(str(workdir / "open.su2"), tet)
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "open mesh" in capi.last_error()
    # node index out of range
    p = _write(str(workdir / "range.su2"), tet.replace("10 0 1 2 3 0", "10 0 1 2 9 0"))
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "out of range" in capi.last_error()
    # unknown element kind
    p = _write(str(workdir / "kind.su2"), tet.replace("10 0 1 2 3 0", "11 0 1 2 3 0"))
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "kind" in capi.last_error()
    # a marker face that matches no element face
    closed = tet + "NMARK= 1\nMARKER_TAG= wall\nMARKER_ELEMS= 1\n9 0 1 2 3\n"
    p = _write(str(workdir / "nomatch.su2"), closed)
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "matches no element face" in capi.last_error()
    # the same boundary face listed twice
    twice = tet + "NMARK= 1\nMARKER_TAG= wall\nMARKER_ELEMS= 2\n5 0 2 1\n5 1 0 2\n"
    p = _write(str(workdir / "twice.su2"), twice)
    assert lib.cuMeshFromSu2(p.encode(), out) != 0 and "already has two cells" in capi.last_error()
    # the closed single tet converts
    ok = tet + "NMARK= 1\nMARKER_TAG= wall\nMARKER_ELEMS= 4\n5 0 2 1\n5 0 1 3\n5 1 2 3\n5 0 3 2\n"
    p = _write(str(workdir / "ok.su2"), ok)
    assert lib.cuMeshFromSu2(p.encode(), out) == 0, capi.last_error()
    nodes, faces, cells, regions = read_fvm(out.decode())
    assert len(faces) == 4 and len(cells) == 5 and regions[0][0] == "wall"
    assert cells[0][1] == (1, 2, 3, 4)       # each face of the tet leads to its ghost


def test_fvm_reader_rejects_corrupt_files(workdir):
    lib = capi.load()
    p = str(workdir / "trunc.fvm")
    data = open(os.path.join(GOLDEN, "tet_6x3x2_ref.fvm"), "rb").read()
    with open(p, "wb") as f:
        f.write(data[: len(data) // 2])
    assert not lib.cuMeshFromFile(p.encode())
    assert "truncated" in capi.last_error() or "bad" in capi.last_error()
    assert not lib.cuMeshFromFile(b"/nonexistent/x.fvm")
    assert "cannot open" in capi.last_error()


def test_field_api_without_gpu_reports_errors():
    """FvmFieldNew needs device memory; without a GPU it fails loudly (NULL
    with a CUDA message), never silently."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = capi.load()
    assert not lib.FvmFieldNew(4, 10, b"rho", 1)
    assert capi.last_error()
    assert not lib.FvmFieldNew(7, 10, b"bad", 1)
    assert "elem_size" in capi.last_error()
