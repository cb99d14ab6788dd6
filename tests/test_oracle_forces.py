"""The float64 wall-force oracle on states with known answers."""
import numpy as np

from graphite_b200 import meshgen
from oracle import pyoracle


def test_uniform_pressure_gives_no_force():
    em = meshgen.airfoil_2d_prisms(40, 12)
    om = pyoracle.OracleMesh(em)
    n = om.N + om.G
    rho = np.full(n, 1.4)
    rhou = np.tile([0.7, 0.0, 0.05], (n, 1))
    rhoe = np.full(n, 2.5 + 0.5 * (0.49 + 0.0025) / 1.4)
    f = pyoracle.wall_force(om, rho, rhou, rhoe, "wing")
    p = 0.4 * (rhoe[0] - 0.5 * (0.49 + 0.0025) / 1.4)
    area = om.get("face_areas")
    assert np.max(np.abs(f)) < 1e-12 * p * area.sum() * 1e3


def test_pressure_difference_gives_lift():
    em = meshgen.airfoil_2d_prisms(40, 12)
    om = pyoracle.OracleMesh(em)
    n = om.N + om.G
    c = om.get("cell_centers").reshape(-1, 3)
    rho = np.full(n, 1.4)
    rhou = np.zeros((n, 3))
    # pressure 1 above the chord line, 1.1 below: net force +0.1 * chord * span in z
    p = np.where(c[:, 2] < 0.0, 1.1, 1.0)
    rhoe = p / 0.4
    f = pyoracle.wall_force(om, rho, rhou, rhoe, "wing")
    nodes = np.asarray(em.nodes)
    span = nodes[:, 1].max() - nodes[:, 1].min()
    assert abs(f[2] - 0.1 * 1.0 * span) < 0.02 * 0.1 * span
    lift, drag = pyoracle.lift_drag(f, (0.5, 0.0, 0.0))
    assert lift > 0 and abs(drag) < 0.05 * lift
