"""Generate the golden fixtures by running the reference solver itself.

Needs a GPU and the headless reference build (``make -f oracle/Makefile.ref``
in a tree where the reference sources are present; the built
``oracle/_ref/ref_driver`` then runs anywhere with the same CUDA runtime).

    python tests/golden/make_golden.py --out tests/golden

For each case in cases.py it writes the SU2 mesh, runs the reference harness
(oracle/ref_driver.cu) in one of its modes and stores the arrays as ``<case>_<mode>.npz``:

* metrics  - the reference converter's .fvm file (``<case>_ref.fvm``) and
             the reference's mesh arrays after cuMeshFromSu2/cuMeshFromFile
             (CSR topology, face areas/normals/centres, cell volumes/centres,
             inverse LSQ matrices), for every element kind;
* prepare  - value/gradient/limiter of rho, rhou, rhoe after the boundary
             conditions and FvmEulerStepPrepare, from a seeded synthetic state;
* solve    - residual history and final fields after a fixed number of
             PhysicsEuler::step iterations from the uniform freestream;
* fvmops   - the reference's generic finite-volume operators
             (include/fvmops.cuh:96-219) at every interior cell, from seeded
             smooth fields, with the reference's gradients and limiters of
             those fields (harness oracle/ref_fvmops.cu).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402
import refio  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
FVMOPS = os.path.join(ROOT, "oracle", "_ref", "ref_fvmops")

MIXED = ["mixed_6x3x2", "layered_6x3x2"]     # several element kinds in one mesh
METRICS = ["tet_6x3x2", "hex_6x3x2", "prism_6x3x2", "pyramid_6x3x2", "tet_12x6x2"] + MIXED
PREPARE = ["tet_6x3x2", "hex_6x3x2", "prism_6x3x2", "pyramid_6x3x2", "tet_12x6x2"] + MIXED
SOLVES = [("tet_12x6x2", 20000), ("channel", 2000), ("channel", 40000)]
FVMOPS_MESHES = ["tet_6x3x2", "prism_6x3x2", "hex_6x3x2", "pyramid_6x3x2"] + MIXED
PHI_CONST = (0.7, -0.2, 0.4)


def operator_fields(mesh, seed=4):
    """Seeded smooth fields for the operator fixtures, in reference cell order
    (cells, then ghosts at their ghost centroids): a scalar s, a vector v and
    a vector phi."""
    from oracle.pyoracle import OracleMesh

    x = OracleMesh(mesh).get("cell_centers").reshape(-1, 3)
    n = x.shape[0]
    rng = np.random.default_rng(seed)
    s = np.sin(2 * x[:, 0]) + x[:, 1] ** 2 + 0.05 * rng.standard_normal(n)
    v = np.column_stack([np.cos(x[:, 1]), x[:, 0] * x[:, 2], 1 + 0.1 * rng.standard_normal(n)])
    ph = np.column_stack([1 + 0.2 * x[:, 1], 0.3 * np.ones(n), -0.2 + 0.1 * x[:, 0]])
    return s.astype(np.float32), v.astype(np.float32), ph.astype(np.float32)

FLOAT_KEYS_METRICS = ["nodes", "face_areas", "face_normals", "face_centers", "cell_volumes",
                      "cell_centers", "cell_matrices"]
INT_KEYS_METRICS = ["cell_faces_starts", "cell_faces", "cell_connects", "face_nodes_starts", "face_nodes",
                    "ghost_cell_ids", "ghost_cell_starts"]


def run(args, log):
    t = time.time()
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    log.write(" ".join(args) + f"\n  -> rc={r.returncode} {time.time() - t:.1f}s\n" + r.stdout[-2000:] + "\n")
    log.flush()
    if r.returncode != 0:
        raise SystemExit(f"driver failed: {' '.join(args)}\n{r.stdout[-2000:]}")
    return r.stdout


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "graphite_b200_golden_work"))
    ap.add_argument("--only", default="", help="comma list of metrics,prepare,solve,fvmops")
    ap.add_argument("--cases", default="", help="comma list of mesh names (default: all of each kind)")
    a = ap.parse_args()
    pick = set(a.cases.split(",")) if a.cases else None
    os.makedirs(a.out, exist_ok=True)
    os.makedirs(a.work, exist_ok=True)
    only = set(a.only.split(",")) if a.only else {"metrics", "prepare", "solve", "fvmops"}
    log = open(os.path.join(a.work, "make_golden.log"), "a")
    meshes = {}

    def su2(name):
        if name not in meshes:
            m = cases.MESHES[name]()
            path = os.path.join(a.work, f"{name}.su2")
            m.write_su2(path)
            meshes[name] = (m, path)
        return meshes[name]

    init = cases.CHANNEL_MACH + (cases.P_INF, cases.T_INF)
    bcs = cases.channel_bcs()
    if "metrics" in only:
        for name in METRICS:
            if pick is not None and name not in pick:
                continue
            m, path = su2(name)
            case = os.path.join(a.work, f"{name}_metrics.txt")
            refio.write_case(case, init, bcs)
            out = os.path.join(a.work, f"{name}_metrics.bin")
            run([DRIVER, case, path, out, "metrics"], log)
            rec = refio.read_records(out)
            # the reference converter's own .fvm output, for the converter tests
            shutil.copyfile(path[:-3] + "fvm", os.path.join(a.out, f"{name}_ref.fvm"))
            np.savez_compressed(os.path.join(a.out, f"{name}_metrics.npz"), sizes=rec["sizes"],
                                **{k: rec[k] for k in FLOAT_KEYS_METRICS + INT_KEYS_METRICS})
    if "prepare" in only:
        for name in PREPARE:
            if pick is not None and name not in pick:
                continue
            m, path = su2(name)
            rho, rhou, rhoe = cases.synthetic_state(m)
            state = os.path.join(a.work, f"{name}_state.bin")
            np.concatenate([rho, rhou.reshape(-1), rhoe]).astype(np.float32).tofile(state)
            case = os.path.join(a.work, f"{name}_prepare.txt")
            refio.write_case(case, init, bcs, state=state)
            out = os.path.join(a.work, f"{name}_prepare.bin")
            run([DRIVER, case, path, out, "prepare"], log)
            rec = refio.read_records(out)
            keep = {k: v for k, v in rec.items() if k.split(".")[0] in ("rho", "rhou", "rhoe")}
            np.savez_compressed(os.path.join(a.out, f"{name}_prepare.npz"), sizes=rec["sizes"],
                                state_rho=rho, state_rhou=rhou, state_rhoe=rhoe, **keep)
    if "solve" in only:
        for name, iters in SOLVES:
            if pick is not None and name not in pick:
                continue
            m, path = su2(name)
            case = os.path.join(a.work, f"{name}_solve{iters}.txt")
            refio.write_case(case, init, bcs, cfl=0.8, iters=iters)
            out = os.path.join(a.work, f"{name}_solve{iters}.bin")
            txt = run([DRIVER, case, path, out, "solve"], log)
            rec = refio.read_records(out)
            keep = {k: rec[k] for k in ("rho.value", "rhou.value", "rhoe.value", "residual_history",
                                        "iterations", "wall_seconds", "event_seconds", "sizes")}
            np.savez_compressed(os.path.join(a.out, f"{name}_solve{iters}.npz"), **keep)
            print(name, iters, txt.strip().splitlines()[-1])
    if "fvmops" in only:
        for name in FVMOPS_MESHES:
            if pick is not None and name not in pick:
                continue
            m, path = su2(name)
            sf, vf, pf = operator_fields(m)
            fields = os.path.join(a.work, f"{name}_fvmops_fields.bin")
            np.concatenate([sf, vf.reshape(-1), pf.reshape(-1)]).astype(np.float32).tofile(fields)
            out = os.path.join(a.work, f"{name}_fvmops.bin")
            run([FVMOPS, path, fields, out] + ["%.9g" % c for c in PHI_CONST], log)
            rec = refio.read_records(out)
            np.savez_compressed(os.path.join(a.out, f"{name}_fvmops.npz"), s=sf, v=vf, phi=pf,
                                phi_const=np.array(PHI_CONST, np.float32), **rec)
            print(name, "fvmops", rec["ops"].size // 35, "cells")
    log.close()


if __name__ == "__main__":
    main()
