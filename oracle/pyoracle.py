"""ctypes bindings for oracle/_build/liboracle.so (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, List, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    lib.orc_last_error.restype = C.c_char_p
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_max_threads.restype = C.c_int
    lib.orc_mesh_new.restype = _P
    lib.orc_mesh_new.argtypes = [_I64, _P, _I64, _P, _P, _P, _I64, C.c_char_p, _P, _P, _P, _P, C.c_int]
    lib.orc_mesh_free.argtypes = [_P]
    lib.orc_mesh_sizes.argtypes = [_P, _P]
    lib.orc_mesh_get.restype = _I64
    lib.orc_mesh_get.argtypes = [_P, C.c_char_p, _P]
    lib.orc_region_id.restype = _I64
    lib.orc_region_id.argtypes = [_P, C.c_char_p]
    lib.orc_solver_new.restype = _P
    lib.orc_solver_new.argtypes = [_P, C.c_int, C.c_int]
    lib.orc_solver_free.argtypes = [_P]
    lib.orc_init.argtypes = [_P, _D, _D, _D, _D, _D]
    lib.orc_set_state.argtypes = [_P, _P, _P, _P]
    lib.orc_get.restype = _I64
    lib.orc_get.argtypes = [_P, C.c_char_p, _P]
    lib.orc_bc_slip.argtypes = [_P, _I64]
    lib.orc_bc_farfield.argtypes = [_P, _I64, _D, _D, _D, _D, _D]
    lib.orc_prepare.argtypes = [_P]
    lib.orc_step.argtypes = [_P, _D]
    lib.orc_reduce_error.restype = _D
    lib.orc_reduce_error.argtypes = [_P]
    lib.orc_run.argtypes = [_P, _I64, _D, _I64, _P, _P, _P, _P]
    lib.orc_sample_step.argtypes = [_P, _D, _I64, _I64]
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def mesh_arrays(mesh) -> Dict[str, object]:
    """Flatten a meshgen.ElementMesh into the arrays the C entry points take."""
    kinds, offs, nodes = [], [0], []
    for kind, conn in mesh.blocks:
        kinds.append(np.full(conn.shape[0], kind, dtype=np.int32))
        nodes.append(conn.reshape(-1))
        offs.append(np.full(conn.shape[0], conn.shape[1], dtype=np.int64))
    ek = np.concatenate(kinds)
    eo = np.concatenate([np.zeros(1, np.int64), np.cumsum(np.concatenate(offs[1:]))])
    en = np.concatenate(nodes).astype(np.int64)
    names, roff, bk, bo, bn = [], [0], [], [], []
    for name, faces in mesh.markers.items():
        names.append(name)
        cnt = 0
        for kind, conn in faces:
            bk.append(np.full(conn.shape[0], kind, dtype=np.int32))
            bo.append(np.full(conn.shape[0], conn.shape[1], dtype=np.int64))
            bn.append(conn.reshape(-1))
            cnt += conn.shape[0]
        roff.append(roff[-1] + cnt)
    return {
        "nodes": np.ascontiguousarray(mesh.nodes, dtype=np.float64),
        "kinds": ek, "eoff": eo, "enodes": en,
        "names": names, "roff": np.array(roff, dtype=np.int64),
        "bkinds": np.concatenate(bk).astype(np.int32),
        "boff": np.concatenate([np.zeros(1, np.int64), np.cumsum(np.concatenate(bo))]),
        "bnodes": np.concatenate(bn).astype(np.int64),
    }


class OracleMesh:
    """Reference-semantics mesh (cells in SU2 order, ghosts per marker) with
    metrics computed in ``metric_bits`` precision."""

    INT_ARRAYS = ("cell_faces_starts", "cell_faces", "cell_connects", "face_nodes_starts", "face_nodes",
                  "ghost_cell_ids", "ghost_cell_starts")
    FLOAT_ARRAYS = ("face_areas", "face_normals", "face_centers", "cell_volumes", "cell_centers", "cell_matrices")

    def __init__(self, mesh, metric_bits: int = 64):
        lib = load()
        a = mesh_arrays(mesh)
        self._keep = a
        names = b"".join(n.encode() + b"\0" for n in a["names"])
        h = lib.orc_mesh_new(a["nodes"].shape[0], _ptr(a["nodes"]), a["kinds"].shape[0], _ptr(a["kinds"]),
                             _ptr(a["eoff"]), _ptr(a["enodes"]), len(a["names"]), names, _ptr(a["roff"]),
                             _ptr(a["bkinds"]), _ptr(a["boff"]), _ptr(a["bnodes"]), metric_bits)
        if not h:
            raise ValueError(lib.orc_last_error().decode())
        self.h = h
        self.region_names: List[str] = list(a["names"])
        s = np.zeros(7, dtype=np.int64)
        lib.orc_mesh_sizes(h, _ptr(s))
        self.N, self.G, self.F, self.S, self.n_nodes, self.n_regions, self.n_face_nodes = (int(x) for x in s)

    def get(self, name: str) -> np.ndarray:
        lib = load()
        n = lib.orc_mesh_get(self.h, name.encode(), None)
        dt = np.int64 if name in self.INT_ARRAYS else np.float64
        out = np.empty(n, dtype=dt)
        lib.orc_mesh_get(self.h, name.encode(), _ptr(out))
        return out

    def region_id(self, name: str) -> int:
        r = load().orc_region_id(self.h, name.encode())
        if r < 0:
            raise KeyError(name)
        return int(r)

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_mesh_free(self.h)
            self.h = None


class OracleSolver:
    """Euler state and operators on an OracleMesh, in float32 or float64."""

    def __init__(self, mesh: OracleMesh, bits: int = 64, transposed_momentum: bool = True):
        self.mesh = mesh
        self.h = load().orc_solver_new(mesh.h, bits, 1 if transposed_momentum else 0)
        self.n = mesh.N + mesh.G

    def init(self, mach: Sequence[float], p: float, t: float):
        load().orc_init(self.h, mach[0], mach[1], mach[2], p, t)

    def set_state(self, rho, rhou, rhoe):
        r = np.ascontiguousarray(rho, dtype=np.float64)
        u = np.ascontiguousarray(np.asarray(rhou).reshape(-1), dtype=np.float64)
        e = np.ascontiguousarray(rhoe, dtype=np.float64)
        assert r.size == self.n and u.size == 3 * self.n and e.size == self.n
        load().orc_set_state(self.h, _ptr(r), _ptr(u), _ptr(e))

    _COMPS = {"rho": 1, "rhoe": 1, "err": 1, "err_rho": 1, "lim_rho": 1, "lim_rhoe": 1, "rhou": 3, "lim_rhou": 3,
              "grad_rho": 3, "grad_rhoe": 3, "grad_rhou": 9}

    def get(self, name: str) -> np.ndarray:
        k = self._COMPS[name]
        out = np.empty(self.n * k, dtype=np.float64)
        load().orc_get(self.h, name.encode(), _ptr(out))
        return out.reshape(self.n, k) if k > 1 else out

    def apply_bcs(self, bcs):
        lib = load()
        for b in bcs:
            rid = self.mesh.region_id(b[1])
            if b[0] == "slip":
                lib.orc_bc_slip(self.h, rid)
            else:
                lib.orc_bc_farfield(self.h, rid, *[float(x) for x in b[2:7]])

    def prepare(self):
        load().orc_prepare(self.h)

    def step(self, cfl: float):
        load().orc_step(self.h, cfl)

    def reduce_error(self) -> float:
        return float(load().orc_reduce_error(self.h))

    def sample_step(self, cfl: float, c0: int, c1: int) -> None:
        """Gradients, limiters and flux/update of interior cells [c0, c1)."""
        load().orc_sample_step(self.h, cfl, c0, c1)

    def run(self, bcs, n_iter: int, cfl: float) -> np.ndarray:
        types = np.array([0 if b[0] == "slip" else 1 for b in bcs], dtype=np.int32)
        regions = np.array([self.mesh.region_id(b[1]) for b in bcs], dtype=np.int64)
        params = np.zeros((len(bcs), 5), dtype=np.float64)
        for i, b in enumerate(bcs):
            if b[0] != "slip":
                params[i] = [float(x) for x in b[2:7]]
        hist = np.zeros(n_iter, dtype=np.float64)
        load().orc_run(self.h, n_iter, cfl, len(bcs), _ptr(types), _ptr(regions), _ptr(params), _ptr(hist))
        return hist

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_solver_free(self.h)
            self.h = None


def set_threads(n: int) -> None:
    load().orc_set_threads(n)


def max_threads() -> int:
    return int(load().orc_max_threads())


def wall_force(mesh: "OracleMesh", rho, rhou, rhoe, region) -> np.ndarray:
    """Pressure force on a boundary region from a state in reference order,
    in float64: the sum over the region's ghosts of p A n, with p the pressure
    of the ghost's interior cell and n its face normal oriented away from that
    cell (the orientation of src/models/euler.cu:422-434)."""
    r = mesh.region_id(region) if isinstance(region, str) else int(region)
    gs, gid = mesh.get("ghost_cell_starts"), mesh.get("ghost_cell_ids")
    cfs, cf, cc = mesh.get("cell_faces_starts"), mesh.get("cell_faces"), mesh.get("cell_connects")
    area = mesh.get("face_areas")
    nrm = mesh.get("face_normals").reshape(-1, 3)
    fctr = mesh.get("face_centers").reshape(-1, 3)
    cctr = mesh.get("cell_centers").reshape(-1, 3)
    g = gid[gs[r]:gs[r + 1]]
    c1 = cc[cfs[g]]
    face = cf[cfs[g]]
    n = nrm[face]
    sign = np.where(np.einsum("ij,ij->i", n, fctr[face] - cctr[c1]) >= 0, 1.0, -1.0)
    rho = np.asarray(rho, np.float64)
    rhou = np.asarray(rhou, np.float64).reshape(-1, 3)
    rhoe = np.asarray(rhoe, np.float64)
    p = 0.4 * (rhoe[c1] - 0.5 * np.einsum("ij,ij->i", rhou[c1], rhou[c1]) / rho[c1])
    return np.sum((p * area[face] * sign)[:, None] * n, axis=0)


def lift_drag(force, mach) -> tuple:
    """(lift, drag): components of the force normal and parallel to the free
    stream, the normal taken in the x-z plane (mach = M (cos a, 0, sin a))."""
    m = np.asarray(mach, np.float64)
    d = m / np.linalg.norm(m)
    l = np.array([-d[2], 0.0, d[0]])
    f = np.asarray(force, np.float64)
    return float(f @ l), float(f @ d)
