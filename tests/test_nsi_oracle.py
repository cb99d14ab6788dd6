"""The FP64 incompressible Navier-Stokes oracle on cases with known answers."""
import numpy as np

from graphite_b200 import meshgen
from oracle.pyoracle import OracleMesh
from oracle.nsi_oracle import NSIOracle


def _cylinder():
    return OracleMesh(meshgen.cylinder_ogrid(32, 12, ratio=1.2, r_far=10.0))


def test_uniform_flow_is_preserved():
    """With free-stream conditions on every boundary (the cylinder's too) a
    uniform state has zero residual: the flux is consistent and the discrete
    divergence and Laplacian of constants vanish."""
    o = NSIOracle(_cylinder(), viscosity=0.05, beta=2.0)
    o.init((0.8, 0.0, 0.3), 0.25)
    bcs = [("inletoutlet", r, 0.8, 0.0, 0.3, 0.25) for r in ("cylinder", "farfield")] + [("slip", "sides")]
    h = o.run(bcs, 5, 0.8)
    assert np.max(h) < 1e-24
    assert np.max(np.abs(o.p[: o.N] - 0.25)) < 1e-14 and np.max(np.abs(o.u[: o.N] - [0.8, 0.0, 0.3])) < 1e-14


def test_cylinder_residual_drops_and_drag_points_downstream():
    o = NSIOracle(_cylinder(), viscosity=0.025, beta=2.0)
    o.init((1.0, 0.0, 0.0), 0.0)
    bcs = [("wall", "cylinder"), ("inletoutlet", "farfield", 1.0, 0.0, 0.0, 0.0), ("slip", "sides")]
    h = o.run(bcs, 1000, 0.5)
    assert h[-1] < 1e-2 * h[0]
    f = o.wall_force("cylinder")
    assert f[0] > 0 and abs(f[2]) < 1e-6 * f[0]            # symmetric flow: no lift


def test_plain_average_laplacian_differs_from_corrected():
    o1 = NSIOracle(_cylinder(), corrected=True)
    o0 = NSIOracle(_cylinder(), corrected=False)
    bcs = [("wall", "cylinder"), ("inletoutlet", "farfield", 1.0, 0.0, 0.0, 0.0), ("slip", "sides")]
    for o in (o0, o1):
        o.init((1.0, 0.0, 0.0), 0.0)
        o.run(bcs, 50, 0.5)
    assert np.max(np.abs(o1.u - o0.u)) > 1e-3
