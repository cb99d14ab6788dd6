"""The reference's PhysicsEuler driver loop, over the C ABI.

``EulerCase`` does what PhysicsEuler (src/models/euler.cu:12-175) does with
the reference's entry points -- load the mesh, create rho/rhou/rhoe/error,
initialise from a free stream, and per iteration apply the boundary
conditions, prepare gradients and limiters, step, and reduce the residual --
but calls libgraphite_b200.so.  ``run`` uses the graph-replayed loop
(gbEulerRun) instead of one C call per stage.

Boundary conditions are tuples ``("slip", region)`` or
``("farfield", region, mach_x, mach_y, mach_z, pressure, temperature)``.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import Sequence, Tuple

import numpy as np

from . import capi


def lift_drag(force, mach) -> Tuple[float, float]:
    """(lift, drag) of a force: its components normal and parallel to the free
    stream, the normal taken in the x-z plane (mach = M (cos a, 0, sin a))."""
    m = np.asarray(mach, np.float64)
    d = m / np.linalg.norm(m)
    n = np.array([-d[2], 0.0, d[0]])
    f = np.asarray(force, np.float64)
    return float(f @ n), float(f @ d)


class EulerCase:
    def __init__(self, mesh_path: str, via_fvm: bool = True):
        """Load an SU2 mesh, either through cuMeshFromSu2 + cuMeshFromFile
        (the reference's path, float32 node coordinates) or directly."""
        lib = capi.load()
        self.lib = lib
        self._tmp = None
        if mesh_path.endswith(".su2") and via_fvm:
            self._tmp = tempfile.mkdtemp(prefix="gb_mesh_")
            fvm = os.path.join(self._tmp, os.path.basename(mesh_path)[:-3] + "fvm")
            capi.check(lib.cuMeshFromSu2(mesh_path.encode(), fvm.encode()), "cuMeshFromSu2")
            mesh = lib.cuMeshFromFile(fvm.encode())
        elif mesh_path.endswith(".su2"):
            mesh = lib.gbMeshFromSu2(mesh_path.encode())
        else:
            mesh = lib.cuMeshFromFile(mesh_path.encode())
        if not mesh:
            raise capi.GraphiteError(f"mesh load failed: {capi.last_error()}")
        self.mesh = mesh
        base = mesh.contents._cpu.contents
        self.n_cells = int(base.n_cells)
        self.n_ghosts = int(base.n_ghosts)
        self.n_faces = int(base.n_faces)
        n = int(lib.cuMeshGetVarSize(mesh))
        self.rho = lib.FvmFieldNew(4, n, b"rho", 1)
        self.rhou = lib.FvmFieldNew(12, n, b"rhou", 1)
        self.rhoe = lib.FvmFieldNew(4, n, b"rhoe", 1)
        self.error = lib.FvmFieldNew(4, n, b"error", 1)
        if not (self.rho and self.rhou and self.rhoe and self.error):
            raise capi.GraphiteError(f"FvmFieldNew failed: {capi.last_error()}")
        self.err0 = None

    @property
    def regions(self):
        m = self.mesh.contents
        return [m.region_names[i].decode() for i in range(m.region_names_size)]

    def init(self, mach: Sequence[float], pressure: float, temperature: float) -> None:
        capi.check(self.lib.FvmEulerInit(self.mesh, self.rho, self.rhou, self.rhoe, capi.vec(mach), pressure,
                                         temperature), "FvmEulerInit")

    def set_state(self, rho: np.ndarray, rhou: np.ndarray, rhoe: np.ndarray) -> None:
        """Upload a state given in reference order (cells then ghosts)."""
        for f, v in ((self.rho, rho), (self.rhou, rhou), (self.rhoe, rhoe)):
            capi.set_field_values(f, v)
            capi.check(self.lib.gbVarCpuToGpu(self.mesh, f), "gbVarCpuToGpu")

    def upload_mirrors(self) -> None:
        """gbVarCpuToGpu of rho, rhou and rhoe: the device state becomes what
        their pinned host mirrors (FvmField _cpu->value) hold."""
        for f in (self.rho, self.rhou, self.rhoe):
            capi.check(self.lib.gbVarCpuToGpu(self.mesh, f), "gbVarCpuToGpu")

    def download_mirrors(self) -> None:
        """VarGpuToCpu of rho, rhou and rhoe into their pinned host mirrors."""
        for f in (self.rho, self.rhou, self.rhoe):
            self.lib.VarGpuToCpu(f)
            if capi.last_error():
                raise capi.GraphiteError(capi.last_error())

    def state_bytes(self) -> int:
        """Bytes of the host mirrors of rho, rhou and rhoe (cells and ghosts)."""
        n = self.n_cells + self.n_ghosts
        return n * (4 + 12 + 4)

    def apply_bcs(self, bcs) -> None:
        # the calls' arguments are built once per list of conditions
        key = tuple(tuple(b) for b in bcs)
        if getattr(self, "_bc_key", None) != key:
            calls = []
            for b in bcs:
                if b[0] == "slip":
                    calls.append((self.lib.FvmEulerSlipBc, (self.mesh, self.rho, self.rhou, self.rhoe,
                                                            b[1].encode()), b))
                else:
                    calls.append((self.lib.FvmEulerInletOutletBc,
                                  (self.mesh, self.rho, self.rhou, self.rhoe, capi.vec(b[2:5]), float(b[5]),
                                   float(b[6]), b[1].encode()), b))
            self._bc_key, self._bc_calls = key, calls
        for fn, args, b in self._bc_calls:
            rc = fn(*args)
            if rc != 0:
                capi.check(rc, f"boundary condition {b[0]} on {b[1]}")

    def prepare(self) -> None:
        capi.check(self.lib.FvmEulerStepPrepare(self.mesh, self.rho, self.rhou, self.rhoe), "FvmEulerStepPrepare")

    def step(self, cfl: float) -> None:
        capi.check(self.lib.FvmEulerStep(self.mesh, self.rho, self.rhou, self.rhoe, cfl, b"steady", None,
                                         self.error), "FvmEulerStep")

    def residual(self) -> float:
        r = float(self.lib.FvmFieldReduceSum(self.mesh, self.error))
        if r != r:
            raise capi.GraphiteError(f"FvmFieldReduceSum failed: {capi.last_error()}")
        return r

    def iterate(self, bcs, cfl: float) -> float:
        """One PhysicsEuler::step (src/models/euler.cu:99-175); returns the
        residual sum of this iteration."""
        self.apply_bcs(bcs)
        self.prepare()
        self.step(cfl)
        return self.residual()

    def bc_structs(self, bcs):
        arr = (capi.gbBc * max(len(bcs), 1))()
        for i, b in enumerate(bcs):
            rid = self.lib.cuMeshGetRegionId(self.mesh, b[1].encode())
            if rid == 0xFFFFFFFF:
                raise capi.GraphiteError(capi.last_error())
            if b[0] == "slip":
                arr[i] = capi.gbBc(0, rid, capi.vec(0, 0, 0), 0.0, 0.0)
            else:
                arr[i] = capi.gbBc(1, rid, capi.vec(b[2:5]), float(b[5]), float(b[6]))
        return arr

    def run(self, bcs, cfl: float, n_iter: int, tolerance: float = 0.0, check_every: int = 100) -> np.ndarray:
        """n_iter iterations as replayed CUDA graphs; returns the residual
        history (stops early below ``tolerance`` relative to the first)."""
        arr = self.bc_structs(bcs)
        hist = np.zeros(max(n_iter, 1), dtype=np.float64)
        done = self.lib.gbEulerRun(self.mesh, self.rho, self.rhou, self.rhoe, self.error, cfl, n_iter, arr, len(bcs),
                                   tolerance, check_every, hist.ctypes.data_as(C.POINTER(C.c_double)))
        if done < 0:
            raise capi.GraphiteError(f"gbEulerRun failed: {capi.last_error()}")
        return hist[:done]

    def run_density(self, bcs, cfl: float, n_iter: int, tolerance: float = 0.0, check_every: int = 100):
        """run() that also returns the density part of the residual per
        iteration (sum of F_rho^2 V): (residual history, density history)."""
        arr = self.bc_structs(bcs)
        hist = np.zeros(max(n_iter, 1), dtype=np.float64)
        dens = np.zeros(max(n_iter, 1), dtype=np.float64)
        done = self.lib.gbEulerRunDensityResidual(self.mesh, self.rho, self.rhou, self.rhoe, self.error, cfl, n_iter,
                                                  arr, len(bcs), tolerance, check_every,
                                                  hist.ctypes.data_as(C.POINTER(C.c_double)),
                                                  dens.ctypes.data_as(C.POINTER(C.c_double)))
        if done < 0:
            raise capi.GraphiteError(f"gbEulerRunDensityResidual failed: {capi.last_error()}")
        return hist[:done], dens[:done]

    def fields(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(rho, rhou, rhoe) in reference order, cells then ghosts."""
        out = []
        for f in (self.rho, self.rhou, self.rhoe):
            self.lib.VarGpuToCpu(f)
            if capi.last_error():
                raise capi.GraphiteError(capi.last_error())
            out.append(capi.field_values(f))
        return tuple(out)

    def gradients(self):
        """{name: (gradient, limiter)} after VarAllGpuToCpu, reference layout."""
        out = {}
        for name, f in (("rho", self.rho), ("rhou", self.rhou), ("rhoe", self.rhoe)):
            self.lib.VarAllGpuToCpu(f)
            out[name] = capi.field_gradients(f)
        return out

    def error_values(self) -> np.ndarray:
        self.lib.VarGpuToCpu(self.error)
        return capi.field_values(self.error)

    def wall_force(self, region: str) -> np.ndarray:
        """Pressure force on a boundary region (gbWallForce), float64 [3]."""
        rid = self.lib.cuMeshGetRegionId(self.mesh, region.encode())
        f = np.zeros(3, np.float64)
        capi.check(self.lib.gbWallForce(self.mesh, self.rho, self.rhou, self.rhoe, rid, f.ctypes.data), "gbWallForce")
        return f

    def close(self) -> None:
        if getattr(self, "mesh", None):
            for f in (self.rho, self.rhou, self.rhoe, self.error):
                if f:
                    self.lib.FvmFieldFree(f)
            self.lib.cuMeshFree(self.mesh)
            self.mesh = None
        if self._tmp:
            import shutil
            shutil.rmtree(self._tmp, ignore_errors=True)
            self._tmp = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
