"""VTU output (FieldsWriteVtu, gbFieldsWriteVtuBinary): the written file
parses, its cells are the mesh's polyhedra and its cell data are the fields."""
import ctypes as C
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import cases
from graphite_b200 import capi
from graphite_b200.euler import EulerCase

pytestmark = pytest.mark.gpu


def _ascii_arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {}
    for da in root.iter("DataArray"):
        dt = np.float64 if da.get("type") == "Float32" else np.int64
        out[da.get("Name")] = np.array(da.text.split(), dtype=np.float64).astype(dt)
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), out


def _binary_arrays(path):
    raw = open(path, "rb").read()
    head, data = raw.split(b"<AppendedData encoding=\"raw\">", 1)
    data = data[data.index(b"_") + 1:]
    piece = re.search(rb'NumberOfPoints="(\d+)" NumberOfCells="(\d+)"', head)
    out = {}
    for m in re.finditer(rb'<DataArray type="(\w+)" Name="(\w+)"[^>]*offset="(\d+)"', head):
        typ, name, off = m.group(1).decode(), m.group(2).decode(), int(m.group(3))
        nbytes = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        dt = np.float32 if typ == "Float32" else np.int64
        out[name] = np.frombuffer(data[off + 8: off + 8 + nbytes], dt)
    return int(piece.group(1)), int(piece.group(2)), out


@pytest.mark.parametrize("name", ["prism_6x3x2", "tet_6x3x2"])
def test_vtu_ascii_and_binary(su2_paths, workdir, name):
    c = EulerCase(su2_paths(name))
    bcs = cases.channel_bcs()
    c.init(cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)
    c.run(bcs, 0.8, 20)
    rho, rhou, _ = c.fields()              # VarGpuToCpu: host values current
    lib = capi.load()
    vars_ = (capi.FieldP * 2)(c.rho, c.rhou)
    base = c.mesh.contents._cpu.contents
    N, n_nodes = c.n_cells, int(base.n_nodes)
    pa, pb = str(workdir / f"{name}.vtu"), str(workdir / f"{name}_bin.vtu")
    assert lib.FieldsWriteVtu(pa.encode(), c.mesh, vars_, 2) == 0
    assert lib.gbFieldsWriteVtuBinary(pb.encode(), c.mesh, vars_, 2) == 0
    for npts, ncells, arr in (_ascii_arrays(pa), _binary_arrays(pb)):
        assert npts == n_nodes and ncells == N
        np.testing.assert_allclose(arr["rho"], rho[:N], rtol=1e-7)
        np.testing.assert_allclose(np.asarray(arr["rhou"]).reshape(-1, 3), rhou[:N], rtol=1e-7, atol=1e-30)
        assert len(arr["offsets"]) == N and arr["offsets"][-1] == len(arr["connectivity"])
        assert np.all(arr["types"] == 42)
        assert arr["connectivity"].min() >= 0 and arr["connectivity"].max() < n_nodes
        per_cell = np.diff(np.concatenate([[0], arr["offsets"]]))
        expected = 6 if name.startswith("prism") else 4
        assert np.all(per_cell == expected)
        # every cell's face list names exactly its nodes
        faces, fo = arr["faces"], arr["faceoffsets"]
        start = 0
        for e in range(N):
            f = faces[start:fo[e]]
            nf, k, seen = int(f[0]), 1, set()
            for _ in range(nf):
                m = int(f[k]); seen.update(int(x) for x in f[k + 1:k + 1 + m]); k += 1 + m
            assert k == len(f)
            assert seen == set(int(x) for x in arr["connectivity"][(arr["offsets"][e - 1] if e else 0):arr["offsets"][e]])
            start = fo[e]
    assert lib.FieldsWriteVtu(b"/nonexistent_dir/x.vtu", c.mesh, vars_, 2) != 0
    c.close()
