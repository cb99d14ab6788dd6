"""A C program compiled against include/graphite_b200.h (tests/abi/
physics_euler.c) and linked with libgraphite_b200.so.

CPU: the header's structs have the reference's fields in the reference's
order (include/mesh.cuh:18-63, include/fvmfields.cuh:16-30) with the C
layout the ctypes binding assumes, and the program links.  GPU: the
program's PhysicsEuler loop (the reference's call sequence, written in C)
gives bit for bit the residuals and density of the same loop driven from
Python, and agrees with the float64 oracle."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import cases
from graphite_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "abi", "physics_euler.c")
LIBDIR = os.path.join(ROOT, "graphite_b200")

# Field order of the reference's structs (include/mesh.cuh:18-63,
# include/fvmfields.cuh:16-30, include/datatypes.cuh:36-54); the gb structs
# are this library's own (gbBc, gbBatchInstance, gbFvmTerm).
ORDER = {
    "gb_vector": ["x", "y", "z"],
    "gb_tensor": ["u", "v", "w"],
    "cuMeshBase": ["type", "allocated", "n_cells", "n_faces", "n_nodes", "n_ghosts", "n_regions", "cell_faces",
                   "cell_connects", "cell_faces_starts", "cell_volumes", "cell_centers", "cell_matrices",
                   "face_nodes", "face_nodes_starts", "face_areas", "face_centers", "face_normals", "nodes",
                   "ghost_cell_ids", "ghost_cell_starts"],
    "cuMesh": ["_cpu", "_hgpu", "_gpu", "region_names", "region_names_alloc", "region_names_size", "impl"],
    "FvmFieldBase": ["elem_size", "size", "value", "gradient", "limiter"],
    "FvmField": ["_cpu", "_hgpu", "_gpu", "name", "impl"],
    "gbBc": ["type", "region_id", "mach", "pressure", "temperature"],
    "gbBatchInstance": ["mesh", "n_bc", "bcs"],
    "gbFvmTerm": ["op", "coef", "u", "phi", "phi_const"],
}
CTYPES = {"gb_vector": capi.gb_vector, "gb_tensor": capi.gb_tensor, "cuMeshBase": capi.cuMeshBase,
          "cuMesh": capi.cuMesh, "FvmFieldBase": capi.FvmFieldBase, "FvmField": capi.FvmField, "gbBc": capi.gbBc,
          "gbBatchInstance": capi.gbBatchInstance, "gbFvmTerm": capi.gbFvmTerm}


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    capi.load()          # the library must be built
    out = str(tmp_path_factory.mktemp("abi") / "physics_euler")
    r = subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-pedantic",
                        "-I", os.path.join(ROOT, "include"), SRC, "-o", out, "-L", LIBDIR, "-lgraphite_b200",
                        f"-Wl,-rpath,{LIBDIR}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_header_structs_have_the_reference_layout(exe):
    r = subprocess.run([exe, "layout"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    offs, sizes = {}, {}
    for line in r.stdout.splitlines():
        a, b, *c = line.split()
        if b == "sizeof":
            sizes[a] = int(c[0])
        else:
            s, f = a.split(".")
            offs.setdefault(s, []).append((f, int(b), int(c[0])))
    assert set(offs) == set(ORDER)
    for s, fields in ORDER.items():
        got = offs[s]
        assert [f for f, _, _ in got] == fields
        o = [x for _, x, _ in got]
        assert o == sorted(o) and len(set(o)) == len(o), (s, got)     # declaration order in memory
        ct = CTYPES[s]
        for f, off, size in got:
            assert getattr(ct, f).offset == off and getattr(ct, f).size == size, (s, f, off, size)
        assert sizes[s] == C.sizeof(ct), (s, sizes[s], C.sizeof(ct))


@pytest.mark.gpu
def test_c_caller_runs_the_physics_euler_loop(exe, su2_paths, tmp_path):
    from graphite_b200.euler import EulerCase
    from oracle import OracleMesh, OracleSolver

    iters = 10
    path = su2_paths("tet_6x3x2")
    r = subprocess.run([exe, "run", path, str(tmp_path / "m.fvm"), str(iters)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    res = np.array([float(l.split()[2]) for l in lines if l.startswith("residual")], np.float32)
    rho = np.array([float(l.split()[2]) for l in r.stdout.splitlines() if l.startswith("rho")], np.float32)
    assert len(res) == iters
    bcs = cases.channel_bcs()
    with EulerCase(path) as c:
        # the header's inline CSR helpers read the host mirror as the arrays say
        fs, fn = capi.mesh_array(c.mesh, "face_nodes_starts"), capi.mesh_array(c.mesh, "face_nodes")
        faces = [l.split()[2:] for l in lines if l.startswith("face ")]
        assert len(faces) == len(fs) - 1
        for i, f in enumerate(faces):
            assert int(f[0]) == fs[i + 1] - fs[i] and [int(x) for x in f[1:]] == list(fn[fs[i]:fs[i + 1]])
        cs, cf = capi.mesh_array(c.mesh, "cell_faces_starts"), capi.mesh_array(c.mesh, "cell_faces")
        cc = capi.mesh_array(c.mesh, "cell_connects")
        cells = [l.split()[2:] for l in lines if l.startswith("cell ")]
        assert len(cells) == len(cs) - 1
        for i, x in enumerate(cells):
            pairs = [tuple(int(y) for y in p.split(":")) for p in x[1:1 + int(x[0])]]
            assert pairs == list(zip(cf[cs[i]:cs[i + 1]], cc[cs[i]:cs[i + 1]]))
            if "ghostface" in x:
                assert int(x[-1]) == cf[cs[i]]
        gs = capi.mesh_array(c.mesh, "ghost_cell_starts")
        regions = [int(l.split()[2]) for l in lines if l.startswith("region ")]
        assert regions == list(np.diff(gs))
        c.init(cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)
        py = np.array([c.iterate(bcs, 0.8) for _ in range(iters)], np.float32)
        py_rho = c.fields()[0][: c.n_cells]
        n = c.n_cells
    assert len(rho) == n
    assert np.array_equal(res, py), (res, py)              # the same calls from C and from Python
    assert np.array_equal(rho, py_rho)
    mesh = cases.MESHES["tet_6x3x2"]()
    s = OracleSolver(OracleMesh(mesh, metric_bits=64), bits=64)
    s.init(cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)
    h = s.run(bcs, iters, 0.8)
    assert np.max(np.abs(res - h) / h) < 1e-4, (res, h)
    ref = s.get("rho")[:n]
    assert np.max(np.abs(rho - ref)) / np.max(np.abs(ref)) < 1e-4
