"""Learned warm start over the C ABI (gbWarmStart*).

``WarmStart`` owns a per-cell MLP for one mesh: it collects converged fields
(from a batch instance or an EulerCase), trains on them with the library's
tensor-core kernels, and writes predicted initial states into batch instances
or EulerCase fields.  ``solve_warm`` is the warm-started batched solve: the
residual of every instance is measured against the first residual of its
cold start, and an instance whose predicted state is not better than the free
stream falls back to the free stream.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import capi

N_PARAMS = 36864


class WarmStart:
    def __init__(self, case=None, wall: str = "wing", seed: int = 0):
        """case: an EulerCase providing the mesh (None: only the explicit-sample
        calls gradient / forward and the weight calls work)."""
        lib = capi.load()
        self.lib = lib
        self.case = case
        mesh, region = None, 0
        if case is not None:
            mesh = case.mesh
            region = lib.cuMeshGetRegionId(mesh, wall.encode())
            if region == 0xFFFFFFFF:
                raise capi.GraphiteError(f"no region {wall!r}")
        h = lib.gbWarmStartCreate(mesh, region, seed)
        if not h:
            raise capi.GraphiteError(f"gbWarmStartCreate failed: {capi.last_error()}")
        self.h = h

    # ---- parameters ----
    @property
    def weights(self) -> np.ndarray:
        w = np.empty(N_PARAMS, np.float32)
        capi.check(self.lib.gbWarmStartGetWeights(self.h, w.ctypes.data), "gbWarmStartGetWeights")
        return w

    @weights.setter
    def weights(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == N_PARAMS
        capi.check(self.lib.gbWarmStartSetWeights(self.h, w.ctypes.data), "gbWarmStartSetWeights")

    def scales(self):
        g = np.empty(4, np.float32)
        t = np.empty(5, np.float32)
        capi.check(self.lib.gbWarmStartGetScales(self.h, g.ctypes.data, t.ctypes.data), "gbWarmStartGetScales")
        return g, t

    def set_scales(self, target) -> None:
        t = np.ascontiguousarray(target, dtype=np.float32)
        capi.check(self.lib.gbWarmStartSetScales(self.h, t.ctypes.data), "gbWarmStartSetScales")

    def features(self) -> np.ndarray:
        """Mapped geometry inputs per interior cell, reference order: [n][4]."""
        g = np.empty((self.case.n_cells, 4), np.float32)
        capi.check(self.lib.gbWarmStartGetFeatures(self.h, g.ctypes.data), "gbWarmStartGetFeatures")
        return g

    # ---- data ----
    def add_batch_field(self, batch, i: int, mach, pressure: float, temperature: float) -> None:
        capi.check(self.lib.gbWarmStartAddBatchField(self.h, batch.h, i, capi.vec(mach), pressure, temperature),
                   "gbWarmStartAddBatchField")

    def add_field(self, case, mach, pressure: float, temperature: float) -> None:
        capi.check(self.lib.gbWarmStartAddField(self.h, case.rho, case.rhou, case.rhoe, capi.vec(mach), pressure,
                                                temperature), "gbWarmStartAddField")

    @property
    def n_fields(self) -> int:
        return int(self.lib.gbWarmStartFieldCount(self.h))

    # ---- training ----
    def train(self, epochs: int, tiles_per_cta: int = 8, lr: float = 1e-3, history: int = 0):
        """Returns (steps, per-step losses or None)."""
        hist = np.zeros(history, np.float64) if history else None
        n = self.lib.gbWarmStartTrain(self.h, epochs, tiles_per_cta, lr,
                                      hist.ctypes.data if history else None, history)
        if n < 0:
            raise capi.GraphiteError(f"gbWarmStartTrain failed: {capi.last_error()}")
        if hist is not None:
            hist = hist[: min(int(n), history)]
        return int(n), hist

    # ---- prediction ----
    def predict_batch(self, batch, i: int, mach, pressure: float, temperature: float) -> None:
        capi.check(self.lib.gbWarmStartPredictBatch(self.h, batch.h, i, capi.vec(mach), pressure, temperature),
                   "gbWarmStartPredictBatch")

    def predict(self, case, mach, pressure: float, temperature: float) -> None:
        capi.check(self.lib.gbWarmStartPredict(self.h, case.rho, case.rhou, case.rhoe, capi.vec(mach), pressure,
                                               temperature), "gbWarmStartPredict")

    # ---- explicit samples (kernel checks) ----
    def gradient(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(N_PARAMS, np.float32)
        loss = C.c_double()
        capi.check(self.lib.gbWarmStartGradient(self.h, x.shape[0], x.ctypes.data, t.ctypes.data, g.ctypes.data,
                                                C.byref(loss)), "gbWarmStartGradient")
        return g, loss.value

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], 5), np.float32)
        capi.check(self.lib.gbWarmStartForward(self.h, x.shape[0], x.ctypes.data, y.ctypes.data),
                   "gbWarmStartForward")
        return y

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gbWarmStartFree(self.h)
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


def solve_warm(batch, ws_per_instance: Sequence[Optional[WarmStart]], cases: Sequence[tuple], cfl: float,
               max_iter: int, tolerance: float, check_every: int = 25):
    """Warm-started batched solve.

    cases[i] = (mach vector, pressure, temperature) of instance i;
    ws_per_instance[i] = the WarmStart of its mesh, or None for a cold start.
    Every instance's residual is divided by the first residual of its cold
    start, so warm and cold solves stop at the same absolute residual.
    Returns (iterations per instance incl. the first cold and predicted
    iterations, ratios, statuses, fell_back flags)."""
    n = len(cases)
    # 1. cold first residual of every instance
    for i, (m, p, t) in enumerate(cases):
        batch.init_uniform(i, m, p, t)
        batch.set_residual_scale(i, 0.0)
    _, _, _, _, hist = batch.run(cfl, 1, history=True)
    res0 = hist[:, 0].copy()
    # 2. predicted states, measured against the cold first residual
    for i, (m, p, t) in enumerate(cases):
        batch.set_residual_scale(i, float(res0[i]))
        if ws_per_instance[i] is not None:
            ws_per_instance[i].predict_batch(batch, i, m, p, t)
        else:
            batch.init_uniform(i, m, p, t)
    _, _, rat1, _, hist = batch.run(cfl, 1, history=True)
    fell_back = np.zeros(n, bool)
    for i, (m, p, t) in enumerate(cases):
        r = hist[i, 0]
        if ws_per_instance[i] is not None and not (np.isfinite(r) and r < res0[i]):
            batch.init_uniform(i, m, p, t)
            fell_back[i] = True
    # 3. the solve, to tolerance x cold first residual
    done, its, rat, st = batch.run(cfl, max_iter, tolerance=tolerance, check_every=check_every)
    return its + 2, rat, st, fell_back
