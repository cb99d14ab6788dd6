"""Converged-field parity with the reference's own solver (its sources built
headless by oracle/Makefile.ref, in float32 as shipped and in float64 with
FLOAT_PREC removed) on identical meshes, against the reference's own
run-to-run spread.

The reference updates each cell's state in place while neighbouring threads
still read it (src/models/euler.cu:250-255,376-378), so two of its runs from
the same free stream end in different fields, in either precision.  On
these cases the limited scheme's residual stalls rather than converging
(channel near 1e-2 after 2,000 iterations; airfoil between 4e-4 and 2e-3
over 30,000), so there is no converged field to match to 1e-5; the
statement that holds is that this library's field lies inside the spread of
the reference's own runs: its nearest reference run is closer than the two
farthest reference runs are to each other, and its farthest is about as far
as those.  It also agrees with
the float64 oracle at least as closely as the reference's float32 runs do.

Measured on the B200 (relative L2, the largest over rho, rho u, rho E):
channel, 2,000 iterations -- twelve reference runs 3.1e-6..5.9e-5 apart,
this library 6.4e-6..6.1e-5 from them and 9.3e-6 from the float64 oracle
(the reference's float32 runs 5.6e-5..5.9e-5 from it); airfoil (4,608
prisms), 30,000 iterations -- six reference runs 9.2e-5..3.8e-4 apart, this
library 1.2e-4..3.4e-4 from them and 2.7e-4 from the float64 oracle (the
reference's float32 runs 3.0e-4..3.9e-4)."""
import math
import os
import subprocess

import numpy as np
import pytest

import cases
import refio
from graphite_b200 import capi, meshgen
from graphite_b200.euler import EulerCase
from oracle import pyoracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF32 = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
REF64 = os.path.join(ROOT, "oracle", "_ref", "ref_driver64")


# (mesh, free stream, boundary conditions, CFL, iterations, reference runs per precision)
def _airfoil():
    a = math.radians(3.0)
    m = (0.6 * math.cos(a), 0.0, 0.6 * math.sin(a))
    return (meshgen.airfoil_2d_prisms(96, 24), m,
            [("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")], 0.5,
            30000, 3)


def _channel():
    # the reference's runs of this case end near one of two fields (the race
    # decides); six runs per precision all but certainly show both
    return cases.MESHES["channel"](), cases.CHANNEL_MACH, cases.channel_bcs(), 0.8, 2000, 6


def _fields(rec_or_tuple, n):
    return {k: np.asarray(v, np.float64).reshape(-1)[: n * c] for (k, c), v in
            zip((("rho", 1), ("rhou", 3), ("rhoe", 1)), rec_or_tuple)}


def _dist(a, b):
    return max(float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])) for k in a)


@pytest.mark.skipif(not (os.path.exists(REF32) and os.path.exists(REF64)),
                    reason="the reference builds (oracle/_ref) are not present")
@pytest.mark.parametrize("make_case", [_channel, _airfoil], ids=["channel_2000", "airfoil_30000"])
def test_fields_lie_within_the_reference_run_to_run_spread(workdir, make_case):
    em, mach, bcs, cfl, iters, n_runs = make_case()
    path = str(workdir / f"spread_{em.name}.su2")
    em.write_su2(path)
    init = tuple(mach) + (cases.P_INF, cases.T_INF)
    case = str(workdir / f"spread_{em.name}.txt")
    refio.write_case(case, init, bcs, cfl=cfl, iters=iters)
    refs = {}
    runs = [(f"f32 {k}", REF32) for k in range(n_runs)] + [(f"f64 {k}", REF64) for k in range(n_runs)]
    for tag, exe in runs:
        out = str(workdir / f"spread_{em.name}_{tag.replace(' ', '_')}.bin")
        subprocess.run([exe, case, path, out, "solve"], check=True, capture_output=True, timeout=600)
        rec = refio.read_records(out)
        n = int(rec["sizes"][0])
        refs[tag] = _fields((rec["rho.value"], rec["rhou.value"], rec["rhoe.value"]), n)
    capi.load().gbSetReferenceMomentumReconstruction(1)
    with EulerCase(path) as c:
        c.init(mach, cases.P_INF, cases.T_INF)
        c.run(bcs, cfl, iters)
        ours = _fields(c.fields(), n)
    s = pyoracle.OracleSolver(pyoracle.OracleMesh(em), bits=64)
    s.init(mach, cases.P_INF, cases.T_INF)
    s.run(bcs, iters, cfl)
    o64 = _fields((s.get("rho"), s.get("rhou"), s.get("rhoe")), n)
    tags = list(refs)
    pairs = [_dist(refs[a], refs[b]) for i, a in enumerate(tags) for b in tags[i + 1:]]
    to_refs = [_dist(ours, refs[t]) for t in tags]
    refs_to_oracle = [_dist(refs[t], o64) for t in tags if t.startswith("f32")]
    ours_to_oracle = _dist(ours, o64)
    print(f"{em.name}, {iters} iterations: reference runs apart {min(pairs):.2e}..{max(pairs):.2e}; "
          f"this library from them {min(to_refs):.2e}..{max(to_refs):.2e}; from the FP64 oracle "
          f"{ours_to_oracle:.2e} (FP32 reference runs {min(refs_to_oracle):.2e}..{max(refs_to_oracle):.2e})")
    assert max(pairs) > 0.0                      # the reference's own runs differ
    # inside the cloud of the reference's runs: its nearest run is closer than
    # the cloud's diameter, its farthest about as far as the cloud's two
    # farthest (measured 0.9..1.07 of it; the diameter itself varies with
    # the races of each set of runs)
    assert min(to_refs) <= max(pairs)
    assert max(to_refs) <= 1.25 * max(pairs)
    assert ours_to_oracle <= 1.05 * max(refs_to_oracle)
