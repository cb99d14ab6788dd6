"""30,000 iterations of the reference's own CUDA build (oracle/_ref, the
reference's sources compiled headless) and of this library on the same
airfoil mesh and free stream: the residual histories stall and rebound the
same way (the stall is the scheme's, not a porting error).

The reference updates the state in place while other threads still read it,
so its own history differs from run to run from the first few dozen
iterations on; in the stall phase (after ~2,000 iterations) two of its runs
differ pointwise by up to ~20 %, while their geometric means over 500
iterations agree within ~3 %.  The comparison is therefore pointwise in the
early, converging phase and over such windows afterwards."""
import math
import os
import subprocess

import numpy as np
import pytest

import cases
import refio
from graphite_b200 import capi, meshgen
from graphite_b200.euler import EulerCase

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference build (oracle/_ref) is not present")
@pytest.mark.parametrize("mach,aoa", [(0.6, 3.0), (0.75, 6.0)])
def test_long_run_matches_reference_build(workdir, mach, aoa):
    em = meshgen.airfoil_2d_prisms(96, 24)
    path = str(workdir / "longrun.su2")
    em.write_su2(path)
    a = math.radians(aoa)
    m = (mach * math.cos(a), 0.0, mach * math.sin(a))
    iters = 30000
    case = str(workdir / "longrun_case.txt")
    with open(case, "w") as f:
        f.write(f"init {m[0]} {m[1]} {m[2]} {cases.P_INF} {cases.T_INF}\n"
                f"farfield farfield {m[0]} {m[1]} {m[2]} {cases.P_INF} {cases.T_INF}\n"
                f"slip sides\nslip wing\ncfl 0.5\niters {iters}\n")
    out = str(workdir / "longrun_ref.bin")
    subprocess.run([REF, case, path, out, "solve"], check=True, capture_output=True)
    rh = refio.read_records(out)["residual_history"]
    capi.load().gbSetReferenceMomentumReconstruction(1)
    c = EulerCase(path)
    c.init(m, cases.P_INF, cases.T_INF)
    h = c.run([("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")],
              0.5, iters)
    c.close()
    r, q = rh / rh[0], h / h[0]
    early = [100, 500, 1000, 1500]
    print("reference", [f"{r[k]:.2e}" for k in early])
    print("ours     ", [f"{q[k]:.2e}" for k in early])
    for k in early:
        assert abs(q[k] - r[k]) <= 0.15 * r[k], (k, q[k], r[k])

    def window(x, c, w=250):
        return float(np.exp(np.mean(np.log(x[c - w:c + w]))))

    centres = [2000, 3000, 5000, 8000, 12000, 20000, iters - 250]
    print("reference windows", [f"{window(r, c):.3e}" for c in centres])
    print("ours windows     ", [f"{window(q, c):.3e}" for c in centres])
    for c in centres:
        assert abs(window(q, c) - window(r, c)) <= 0.10 * window(r, c), (c, window(q, c), window(r, c))
    # both stall: the minimum is far from the end, and the end is above it
    assert np.argmin(q) < iters - 1000 and q[-1] > 2 * q.min()
    assert np.argmin(r) < iters - 1000 and r[-1] > 2 * r.min()
