"""Wall force (lift / drag): the GPU reduction against the float64 oracle on
the same state, and the FP32 solver's lift, drag and density against an
FP64 oracle run of the same iterations."""
import math

import numpy as np
import pytest

import cases
from graphite_b200 import capi, meshgen
from graphite_b200.euler import EulerCase
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def airfoil_bcs(mach, aoa_deg):
    a = math.radians(aoa_deg)
    m = (mach * math.cos(a), 0.0, mach * math.sin(a))
    return m, [("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")]


@pytest.fixture(scope="module")
def airfoil(workdir):
    em = meshgen.airfoil_2d_prisms(96, 24)
    p = str(workdir / "force_airfoil.su2")
    em.write_su2(p)
    return em, p


def test_wall_force_matches_oracle_on_same_state(airfoil):
    em, path = airfoil
    capi.load().gbSetReferenceMomentumReconstruction(1)
    c = EulerCase(path)
    mach, bcs = airfoil_bcs(0.6, 4.0)
    c.init(mach, cases.P_INF, cases.T_INF)
    c.run(bcs, 0.5, 300)
    f = c.wall_force("wing")
    rho, rhou, rhoe = c.fields()
    om = pyoracle.OracleMesh(em)
    ref = pyoracle.wall_force(om, rho, rhou, rhoe, "wing")
    assert np.max(np.abs(f - ref)) <= 2e-6 * np.max(np.abs(ref))
    lift, drag = pyoracle.lift_drag(f, mach)
    assert lift > 0.0                      # positive angle of attack
    c.close()


@pytest.mark.parametrize("mach,aoa", [(0.5, 2.0), (0.75, 5.0)])
def test_fp32_solver_against_fp64_oracle(airfoil, mach, aoa):
    """2000 iterations from free stream: the FP32 solver against the FP64
    oracle (the same scheme, reference momentum reconstruction)."""
    em, path = airfoil
    capi.load().gbSetReferenceMomentumReconstruction(1)
    m, bcs = airfoil_bcs(mach, aoa)
    n_it = 2000
    c = EulerCase(path)
    c.init(m, cases.P_INF, cases.T_INF)
    h = c.run(bcs, 0.5, n_it)
    f32 = c.wall_force("wing")
    rho32 = c.fields()[0]
    om = pyoracle.OracleMesh(em)
    s = pyoracle.OracleSolver(om, bits=64)
    s.init(m, cases.P_INF, cases.T_INF)
    h64 = s.run(bcs, n_it, 0.5)
    rho64 = s.get("rho")
    f64 = pyoracle.wall_force(om, rho64, s.get("rhou"), s.get("rhoe"), "wing")
    l32, d32 = pyoracle.lift_drag(f32, m)
    l64, d64 = pyoracle.lift_drag(f64, m)
    N = c.n_cells
    l2 = np.linalg.norm(rho32[:N] - rho64[:N]) / np.linalg.norm(rho64[:N])
    print(f"M {mach} a {aoa}: lift {l32:.6e} vs {l64:.6e}, drag {d32:.6e} vs {d64:.6e}, rho L2 {l2:.2e}")
    # measured on B200: rho L2 3e-5..5e-5, lift 2e-4..6e-4 relative, drag
    # within 2e-3 of the lift.  Once the limiter starts switching (after a
    # few dozen iterations) the residual itself is sensitive to round-off, so
    # the history is compared pointwise early and by its level late.
    assert l2 < 1e-4
    assert abs(l32 - l64) <= 2e-3 * abs(l64)
    assert abs(d32 - d64) <= 5e-3 * abs(l64)
    np.testing.assert_allclose(h[:40] / h[0], h64[:40] / h64[0], rtol=1e-3)
    late, late64 = np.median(h[-500:] / h[0]), np.median(h64[-500:] / h64[0])
    assert abs(late - late64) <= 0.2 * late64
    c.close()
