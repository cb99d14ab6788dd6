"""Batched multi-instance solves over the C ABI (gbBatch*).

``EulerBatch`` advances many instances -- each a mesh with its own boundary
conditions (e.g. Mach and angle of attack) -- together, each to its own
residual drop, with the mesh data of instances that share a mesh reused
from L2.  The meshes are EulerCase objects (which own the device mesh).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import capi


class EulerBatch:
    def __init__(self, cases: Sequence, instances: Sequence[tuple]):
        """cases: EulerCase objects providing the meshes.
        instances: (case index, boundary conditions) per instance, with the
        boundary conditions as for EulerCase.run."""
        lib = capi.load()
        self.lib = lib
        self.cases = list(cases)
        meshes = (capi.MeshP * len(self.cases))(*[c.mesh for c in self.cases])
        self._bc_arrays = []
        inst = (capi.gbBatchInstance * len(instances))()
        for i, (ci, bcs) in enumerate(instances):
            arr = self.cases[ci].bc_structs(bcs)
            self._bc_arrays.append(arr)
            inst[i] = capi.gbBatchInstance(ci, len(bcs), C.cast(arr, C.POINTER(capi.gbBc)))
        h = lib.gbBatchCreate(len(self.cases), meshes, len(instances), inst)
        if not h:
            raise capi.GraphiteError(f"gbBatchCreate failed: {capi.last_error()}")
        self.h = h
        self.n = len(instances)
        self.instance_case = [ci for ci, _ in instances]

    def init_uniform(self, i: int, mach, pressure: float, temperature: float) -> None:
        capi.check(self.lib.gbBatchInitUniform(self.h, i, capi.vec(mach), pressure, temperature), "gbBatchInitUniform")

    def set_state(self, i: int, rho, rhou, rhoe) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float32)
        u = np.ascontiguousarray(rhou, dtype=np.float32).reshape(-1)
        e = np.ascontiguousarray(rhoe, dtype=np.float32)
        capi.check(self.lib.gbBatchSetState(self.h, i, r.ctypes.data, u.ctypes.data, e.ctypes.data), "gbBatchSetState")

    def get_state(self, i: int):
        c = self.cases[self.instance_case[i]]
        n = c.n_cells + c.n_ghosts
        r = np.empty(n, np.float32)
        u = np.empty(3 * n, np.float32)
        e = np.empty(n, np.float32)
        capi.check(self.lib.gbBatchGetState(self.h, i, r.ctypes.data, u.ctypes.data, e.ctypes.data), "gbBatchGetState")
        return r, u.reshape(n, 3), e

    def set_residual_scale(self, i: int, res0: float) -> None:
        """Divide instance i's residuals by res0 instead of its first residual (0: default)."""
        capi.check(self.lib.gbBatchSetResidualScale(self.h, i, float(res0)), "gbBatchSetResidualScale")

    def wall_force(self, i: int, region: str) -> np.ndarray:
        """Pressure force on a boundary region of instance i (gbBatchWallForce), float64 [3]."""
        c = self.cases[self.instance_case[i]]
        rid = self.lib.cuMeshGetRegionId(c.mesh, region.encode())
        f = np.zeros(3, np.float64)
        capi.check(self.lib.gbBatchWallForce(self.h, i, rid, f.ctypes.data), "gbBatchWallForce")
        return f

    def set_tuning(self, tile: int, schedule: int) -> None:
        capi.check(self.lib.gbBatchSetTuning(self.h, tile, schedule), "gbBatchSetTuning")

    def tuning(self):
        t, s = C.c_int(), C.c_int()
        self.lib.gbBatchGetTuning(self.h, C.byref(t), C.byref(s))
        return t.value, s.value

    def autotune(self, cfl: float, trial_iters: int = 5):
        t, s = C.c_int(), C.c_int()
        capi.check(self.lib.gbBatchAutotune(self.h, cfl, trial_iters, C.byref(t), C.byref(s)), "gbBatchAutotune")
        return t.value, s.value

    def run(self, cfl: float, max_iter: int, tolerance: float = 0.0, check_every: int = 100, history: bool = False):
        """Returns (loop iterations, per-instance iterations, residual ratios,
        statuses[, residual history n x max_iter])."""
        its = np.zeros(self.n, np.int64)
        rat = np.zeros(self.n, np.float64)
        st = np.zeros(self.n, np.int32)
        hist = np.zeros((self.n, max_iter), np.float64) if history else None
        done = self.lib.gbBatchRun(self.h, cfl, max_iter, tolerance, check_every,
                                   its.ctypes.data_as(C.POINTER(C.c_int64)), rat.ctypes.data_as(C.POINTER(C.c_double)),
                                   st.ctypes.data_as(C.POINTER(C.c_int)),
                                   hist.ctypes.data_as(C.POINTER(C.c_double)) if history else None)
        if done < 0:
            raise capi.GraphiteError(f"gbBatchRun failed: {capi.last_error()}")
        out = (int(done), its, rat, st)
        return out + (hist,) if history else out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gbBatchFree(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
