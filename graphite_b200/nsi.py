"""The incompressible Navier-Stokes driver over the C ABI (FvmNSI*, gbNSI*).

``NSICase`` holds a mesh with "velocity" and "pressure" fields and runs the
loop the reference's PhysicsNSI (src/models/nsi.cu) lays out -- boundary
conditions, FvmNSIStepPrepare, FvmNSIStep, residual -- or the graph-replayed
gbNSIRun.  Boundary conditions are tuples ``("slip", region)``,
``("wall", region)`` (no-slip) or ``("inletoutlet", region, ux, uy, uz, p)``.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import tempfile
from typing import Sequence

import numpy as np

from . import capi


class NSICase:
    def __init__(self, mesh_path: str):
        lib = capi.load()
        self.lib = lib
        self._tmp = tempfile.mkdtemp(prefix="gb_nsi_")
        if mesh_path.endswith(".su2"):
            fvm = os.path.join(self._tmp, os.path.basename(mesh_path)[:-3] + "fvm")
            capi.check(lib.cuMeshFromSu2(mesh_path.encode(), fvm.encode()), "cuMeshFromSu2")
            mesh_path = fvm
        mesh = lib.cuMeshFromFile(mesh_path.encode())
        if not mesh:
            raise capi.GraphiteError(f"mesh load failed: {capi.last_error()}")
        self.mesh = mesh
        base = mesh.contents._cpu.contents
        self.n_cells = int(base.n_cells)
        self.n_ghosts = int(base.n_ghosts)
        n = int(lib.cuMeshGetVarSize(mesh))
        self.velocity = lib.FvmFieldNew(12, n, b"velocity", 1)
        self.pressure = lib.FvmFieldNew(4, n, b"pressure", 1)
        self.error = lib.FvmFieldNew(4, n, b"error", 1)
        if not (self.velocity and self.pressure and self.error):
            raise capi.GraphiteError(f"FvmFieldNew failed: {capi.last_error()}")

    @staticmethod
    def set_constants(density: float = 1.0, viscosity: float = 0.025, beta: float = 2.0, corrected: bool = True,
                      limited: bool = False):
        capi.check(capi.load().gbNSISetConstants(density, viscosity, beta, 1 if corrected else 0, 1 if limited else 0),
                   "gbNSISetConstants")

    def init(self, velocity: Sequence[float], pressure: float) -> None:
        capi.check(self.lib.FvmNSIInit(self.mesh, self.velocity, self.pressure, capi.vec(velocity), pressure),
                   "FvmNSIInit")

    def set_state(self, velocity: np.ndarray, pressure: np.ndarray) -> None:
        """Upload a state in reference order (cells then ghosts)."""
        for f, v in ((self.velocity, velocity), (self.pressure, pressure)):
            capi.set_field_values(f, v)
            capi.check(self.lib.gbVarCpuToGpu(self.mesh, f), "gbVarCpuToGpu")

    def apply_bcs(self, bcs) -> None:
        for b in bcs:
            if b[0] == "slip":
                rc = self.lib.FvmNSISlipBc(self.mesh, self.velocity, self.pressure, b[1].encode())
            elif b[0] == "wall":
                rc = self.lib.FvmNSIWallBc(self.mesh, self.velocity, self.pressure, b[1].encode())
            else:
                rc = self.lib.FvmNSIInletOutletBc(self.mesh, self.velocity, self.pressure, capi.vec(b[2:5]),
                                                  float(b[5]), b[1].encode())
            capi.check(rc, f"boundary condition {b[0]} on {b[1]}")

    def prepare(self) -> None:
        capi.check(self.lib.FvmNSIStepPrepare(self.mesh, self.velocity, self.pressure), "FvmNSIStepPrepare")

    def step(self, cfl: float) -> None:
        capi.check(self.lib.FvmNSIStep(self.mesh, self.velocity, self.pressure, cfl, b"steady", None, self.error),
                   "FvmNSIStep")

    def residual(self) -> float:
        r = float(self.lib.FvmFieldReduceSum(self.mesh, self.error))
        if r != r:
            raise capi.GraphiteError(f"FvmFieldReduceSum failed: {capi.last_error()}")
        return r

    def iterate(self, bcs, cfl: float) -> float:
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
            elif b[0] == "wall":
                arr[i] = capi.gbBc(2, rid, capi.vec(0, 0, 0), 0.0, 0.0)
            else:
                arr[i] = capi.gbBc(1, rid, capi.vec(b[2:5]), float(b[5]), 0.0)
        return arr

    def run(self, bcs, cfl: float, n_iter: int, tolerance: float = 0.0, check_every: int = 100) -> np.ndarray:
        """gbNSIRun; returns the residual sum of every iteration that ran."""
        arr = self.bc_structs(bcs)
        hist = np.zeros(max(n_iter, 1), np.float64)
        done = self.lib.gbNSIRun(self.mesh, self.velocity, self.pressure, self.error, cfl, n_iter, arr, len(bcs),
                                 tolerance, check_every, hist.ctypes.data_as(C.c_void_p))
        if done < 0:
            raise capi.GraphiteError(f"gbNSIRun failed: {capi.last_error()}")
        return hist[:done]

    def fields(self):
        """(velocity [n][3], pressure [n]) in reference order, cells then ghosts."""
        out = []
        for f in (self.velocity, self.pressure):
            self.lib.VarGpuToCpu(f)
            if capi.last_error():
                raise capi.GraphiteError(capi.last_error())
            out.append(capi.field_values(f))
        return tuple(out)

    def wall_force(self, region: str) -> np.ndarray:
        rid = self.lib.cuMeshGetRegionId(self.mesh, region.encode())
        f = np.zeros(3, np.float64)
        capi.check(self.lib.gbNSIWallForce(self.mesh, self.velocity, self.pressure, rid, f.ctypes.data), "gbNSIWallForce")
        return f

    def close(self) -> None:
        if getattr(self, "mesh", None):
            for f in (self.velocity, self.pressure, self.error):
                if f:
                    self.lib.FvmFieldFree(f)
            self.lib.cuMeshFree(self.mesh)
            self.mesh = None
        if self._tmp:
            shutil.rmtree(self._tmp, ignore_errors=True)
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def recirculation_length(centres: np.ndarray, velocity: np.ndarray, radius: float = 0.5, band: float = None) -> float:
    """Length of the closed wake behind a cylinder centred at the origin with
    the flow along +x in the x-z plane: from the rear of the cylinder to where
    u_x on the wake axis (|z| small) turns positive, linearly interpolated
    between cell centres.  Returns it in diameters."""
    x, z = centres[:, 0], centres[:, 2]
    if band is None:
        sel = (x > radius) & (np.abs(z) < 0.02 + 0.02 * x)
    else:
        sel = (x > radius) & (np.abs(z) < band)
    order = np.argsort(x[sel])
    xs, ux = x[sel][order], velocity[sel][order, 0]
    # cells on the axis come in pairs (either side); average per distinct x
    keys = np.round(xs, 6)
    ux_m = np.array([ux[keys == k].mean() for k in np.unique(keys)])
    xs_m = np.unique(keys)
    neg = ux_m < 0
    if not neg.any():
        return 0.0
    k = int(np.argmax(~neg[np.argmax(neg):]) + np.argmax(neg))
    if k == 0 or neg[k]:
        return float((xs_m[-1] - radius) / (2 * radius))
    x0, x1, u0, u1 = xs_m[k - 1], xs_m[k], ux_m[k - 1], ux_m[k]
    xc = x0 - u0 * (x1 - x0) / (u1 - u0)
    return float((xc - radius) / (2 * radius))
