"""FP64 oracle solves of the held-out warm-start cases (the learned warm
start's evaluation draws on the 120,000-prism NACA 0012 airfoil).

Each case runs the float64 oracle (oracle/fvm_oracle.cpp, the reference's
scheme restated) from the free stream at CFL 0.5 until the reference's
squared residual drops below 1e-3 of its first value, then 1,000
iterations more, recording the residual every iteration and the wall
force's lift and drag every 10 iterations.  bench.py compares the GPU
solves of the same cases with these.  The draws repeat bench.py's seeded
ones (seed 20261204: 512 training draws, then the held-out draws, Mach ~
U[0.3, 0.8], AoA ~ U[-4, 8] deg); the first N_CASES held-out draws are
solved.  Test infrastructure: takes hours on a few host cores.

    python tests/golden/make_warm_fp64.py [n_cases] [threads]
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from graphite_b200 import meshgen  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

SEED, N_TRAIN, N_HELD = 20261204, 512, 64
CFL, TOL, AFTER, EVERY, CAP = 0.5, 1e-3, 1000, 10, 20000
P_INF, T_INF = 1.0, 1.0 / 1.4
OUT = os.path.join(HERE, "warm_heldout_fp64.npz")


def held_out_draws():
    rng = np.random.default_rng(SEED)
    draws = [(float(rng.uniform(0.3, 0.8)), float(rng.uniform(-4.0, 8.0))) for _ in range(N_TRAIN + N_HELD)]
    return draws[N_TRAIN:]


def solve(om, mach_m, aoa):
    a = math.radians(aoa)
    mach = (mach_m * math.cos(a), 0.0, mach_m * math.sin(a))
    bcs = [("farfield", "farfield") + mach + (P_INF, T_INF), ("slip", "sides"), ("slip", "wing")]
    s = po.OracleSolver(om, bits=64)
    s.init(mach, P_INF, T_INF)
    hist, ld = [], []
    stop = None
    while len(hist) < CAP + AFTER:
        h = s.run(bcs, EVERY, CFL)
        hist.extend(h.tolist())
        f = po.wall_force(om, s.get("rho"), s.get("rhou"), s.get("rhoe"), "wing")
        ld.append(po.lift_drag(f, mach))
        if stop is None:
            r = np.array(hist) / hist[0]
            if np.any(r < TOL):
                stop = int(np.argmax(r < TOL)) + 1
        if stop is not None and len(hist) >= stop + AFTER:
            break
    return np.array(hist), np.array(ld), (stop if stop is not None else -1)


def main():
    n_cases = int(sys.argv[1]) if len(sys.argv) > 1 else 16
    if len(sys.argv) > 2:
        po.set_threads(int(sys.argv[2]))
    om = po.OracleMesh(meshgen.airfoil_extruded(120_000))
    draws = held_out_draws()[:n_cases]
    done = {}
    if os.path.exists(OUT):      # resume: keep the cases already solved
        z = np.load(OUT)
        done = {int(k): (z["hist"][k][~np.isnan(z["hist"][k])], z["ld"][k][~np.isnan(z["ld"][k][:, 0])],
                         int(z["stop"][k])) for k in range(len(z["stop"]))}
    results = []
    for k, (m, a) in enumerate(draws):
        if k in done:
            results.append(done[k])
            continue
        t0 = time.time()
        results.append(solve(om, m, a))
        print(f"case {k}: M {m:.4f} AoA {a:.3f} stop {results[-1][2]} ({time.time() - t0:.0f} s)", flush=True)
        save(draws, results)


def save(draws, results):
    n = len(results)
    L = max(len(r[0]) for r in results)
    M = max(len(r[1]) for r in results)
    hist = np.full((n, L), np.nan, np.float32)
    ld = np.full((n, M, 2), np.nan)
    for k, (h, l, _) in enumerate(results):
        hist[k, : len(h)] = h
        ld[k, : len(l)] = l
    np.savez_compressed(OUT, mach=np.array([d[0] for d in draws[:n]]), aoa=np.array([d[1] for d in draws[:n]]),
                        stop=np.array([r[2] for r in results]), hist=hist, ld=ld, every=EVERY, cfl=CFL, tol=TOL)


if __name__ == "__main__":
    main()
