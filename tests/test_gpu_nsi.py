"""Incompressible Navier-Stokes (FvmNSI*, gbNSIRun) against the FP64 oracle,
and the laminar cylinder at Re = 40."""
import numpy as np
import pytest

from graphite_b200 import meshgen
from graphite_b200.nsi import NSICase, recirculation_length
from oracle.nsi_oracle import NSIOracle
from oracle.pyoracle import OracleMesh

pytestmark = pytest.mark.gpu

BCS = [("wall", "cylinder"), ("inletoutlet", "farfield", 1.0, 0.0, 0.0, 0.0), ("slip", "sides")]


@pytest.fixture(scope="module")
def cyl(workdir):
    em = meshgen.cylinder_ogrid(48, 24, ratio=1.15, r_far=15.0)
    p = str(workdir / "nsi_cyl.su2")
    em.write_su2(p)
    return em, p


@pytest.mark.parametrize("corrected,limited", [(True, False), (False, False), (True, True)])
def test_nsi_matches_fp64_oracle(cyl, corrected, limited):
    """600 pseudo-time iterations from a uniform start, FP32 on the GPU
    against the FP64 oracle of the same scheme."""
    em, path = cyl
    NSICase.set_constants(1.0, 0.025, 2.0, corrected, limited)
    try:
        c = NSICase(path)
        c.init((1.0, 0.0, 0.0), 0.0)
        h = c.run(BCS, 0.5, 600)
        u, p = c.fields()
        f = c.wall_force("cylinder")
        o = NSIOracle(OracleMesh(em), viscosity=0.025, beta=2.0, corrected=corrected, limited=limited)
        o.init((1.0, 0.0, 0.0), 0.0)
        h64 = o.run(BCS, 600, 0.5)
        f64 = o.wall_force("cylinder")
        N = c.n_cells
        eu = np.linalg.norm(u[:N] - o.u[:N]) / np.linalg.norm(o.u[:N])
        ep = np.linalg.norm(p[:N] - o.p[:N]) / np.linalg.norm(o.p[:N])
        print(f"corrected={corrected}: velocity L2 {eu:.2e}, pressure L2 {ep:.2e}, drag {f[0]:.6e} vs {f64[0]:.6e}")
        assert eu < 1e-4 and ep < 1e-3
        assert abs(f[0] - f64[0]) <= 1e-3 * abs(f64[0])
        np.testing.assert_allclose(h / h[0], h64 / h64[0], rtol=2e-3)
        c.close()
    finally:
        NSICase.set_constants()


# every region; the span sides left without a condition (their ghosts keep
# their stored state); the sides given two conditions (the later one holds)
NSI_BC_SETS = {"all": BCS, "no_sides": BCS[:2], "sides_twice": BCS + [("wall", "sides")]}


@pytest.mark.parametrize("bcs,limited", [("all", False), ("all", True), ("no_sides", False), ("sides_twice", False)])
def test_nsi_per_call_loop_equals_graph(cyl, bcs, limited):
    """The per-call loop (BC kernels, FvmNSIStepPrepare, FvmNSIStep, residual)
    and the replayed graphs (on this one-layer mesh the gradient kernel applies
    the boundary conditions) give the same bits, ghost values included."""
    _, path = cyl
    NSICase.set_constants(1.0, 0.025, 2.0, True, limited)
    try:
        a, b = NSICase(path), NSICase(path)
        for c in (a, b):
            c.init((1.0, 0.0, 0.0), 0.0)
        h = a.run(NSI_BC_SETS[bcs], 0.5, 40)
        h2 = np.array([b.iterate(NSI_BC_SETS[bcs], 0.5) for _ in range(40)])
        ua, pa = a.fields()
        ub, pb = b.fields()
        assert np.array_equal(ua, ub) and np.array_equal(pa, pb)
        np.testing.assert_allclose(h, h2, rtol=1e-6)
        a.close()
        b.close()
    finally:
        NSICase.set_constants()


def test_nsi_bad_calls_are_rejected(cyl):
    _, path = cyl
    c = NSICase(path)
    from graphite_b200 import capi
    lib = capi.load()
    assert lib.FvmNSIStep(c.mesh, c.velocity, c.pressure, 0.5, b"steady", None, c.error) != 0   # no prepare yet
    assert b"FvmNSIStepPrepare" in lib.gbGetLastError()
    assert lib.FvmNSISlipBc(c.mesh, c.velocity, c.pressure, b"nowhere") != 0
    assert lib.gbNSISetConstants(1.0, 0.025, 0.0, 1, 0) != 0
    c.close()


def test_cylinder_re40_drag_and_wake(workdir):
    """Steady laminar flow past a cylinder at Re = 40 on a 128 x 64 O-grid,
    converged to round-off: the drag coefficient and the closed wake's
    length fall in the range of published values for this Reynolds number
    (Cd about 1.5-1.6, wake about 2.1-2.35 diameters); measured 1.53 and
    2.04 on this grid (400 x 250: 1.53 and 2.23)."""
    em = meshgen.cylinder_ogrid(128, 64, ratio=1.08, r_far=30.0)
    path = str(workdir / "nsi_cyl128.su2")
    em.write_su2(path)
    c = NSICase(path)
    c.init((1.0, 0.0, 0.0), 0.0)
    h = c.run(BCS, 0.8, 80000, tolerance=1e-10, check_every=2000)
    assert h[-1] < 1e-10 * h[0]
    f = c.wall_force("cylinder")
    span = 0.1
    cd = f[0] / (0.5 * 1.0 * 1.0 * 1.0 * span)
    base = c.mesh.contents._cpu.contents
    cent = np.array([[base.cell_centers[i].x, base.cell_centers[i].y, base.cell_centers[i].z]
                     for i in range(c.n_cells)])
    u, _ = c.fields()
    L = recirculation_length(cent, u[: c.n_cells])
    print(f"Re 40: {len(h)} iterations, Cd {cd:.3f}, wake {L:.2f} D")
    assert 1.45 < cd < 1.65
    assert 1.9 < L < 2.4
    assert abs(f[2]) < 1e-3 * f[0]                    # symmetric: no lift
    c.close()


def test_cylinder_400x250_to_1e3_against_fp64(workdir):
    """The config-2 mesh (400 x 250 O-grid, stretching 1.03, far field at 30
    diameters) run to the 1e-3 drop of the squared residual: the FP32 GPU
    state, drag and wake against the FP64 oracle after the same iterations."""
    em = meshgen.cylinder_ogrid(400, 250, ratio=1.03, r_far=30.0)
    path = str(workdir / "nsi_cyl400.su2")
    em.write_su2(path)
    c = NSICase(path)
    c.init((1.0, 0.0, 0.0), 0.0)
    h = c.run(BCS, 0.8, 2000, tolerance=1e-3, check_every=1)
    n_it = len(h)
    assert h[-1] < 1e-3 * h[0] and n_it < 2000
    f = c.wall_force("cylinder")
    u, p = c.fields()
    o = NSIOracle(OracleMesh(em), viscosity=0.025, beta=2.0)
    o.init((1.0, 0.0, 0.0), 0.0)
    h64 = o.run(BCS, n_it, 0.8)
    f64 = o.wall_force("cylinder")
    N = c.n_cells
    eu = np.linalg.norm(u[:N] - o.u[:N]) / np.linalg.norm(o.u[:N])
    base = c.mesh.contents._cpu.contents
    cent = np.array([[base.cell_centers[i].x, base.cell_centers[i].y, base.cell_centers[i].z] for i in range(N)])
    L32, L64 = recirculation_length(cent, u[:N]), recirculation_length(cent, o.u[:N])
    print(f"400x250 to 1e-3: {n_it} iterations, drag {f[0]:.6e} vs {f64[0]:.6e}, velocity L2 {eu:.2e}, "
          f"wake {L32:.4f} vs {L64:.4f} D")
    assert h64[-1] < 1e-3 * h64[0] * 1.01
    assert eu < 1e-4
    assert abs(f[0] - f64[0]) <= 1e-3 * abs(f64[0])
    assert abs(L32 - L64) <= 0.02
    c.close()


CHANNEL_BCS = [("inletoutlet", "inlet", 0.5, 0.0, 0.0, 0.0), ("inletoutlet", "outlet", 0.5, 0.0, 0.0, 0.0),
               ("wall", "lower"), ("slip", "upper"), ("slip", "sides")]


@pytest.mark.parametrize("name", ["tet_12x6x2", "mixed_6x3x2", "layered_6x3x2"])
def test_nsi_3d_meshes_match_fp64_oracle(name, su2_paths):
    """The incompressible scheme on 3-D channels with a bump wall -- tets,
    hexes / prisms / pyramids side by side, prism layers under tets: the
    ghost kernels apply the conditions (these meshes are not ghost-heavy)
    and cells of 4, 5 and 6 faces share each launch.  300 iterations, FP32 on
    the GPU against the FP64 oracle of the same scheme, and the replayed
    graphs bitwise equal to the per-call loop."""
    import cases
    em = cases.MESHES[name]()
    path = su2_paths(name)
    NSICase.set_constants(1.0, 0.02, 2.0, True, False)
    try:
        c = NSICase(path)
        c.init((0.5, 0.0, 0.0), 0.0)
        h = c.run(CHANNEL_BCS, 0.5, 300)
        u, p = c.fields()
        o = NSIOracle(OracleMesh(em), viscosity=0.02, beta=2.0, corrected=True, limited=False)
        o.init((0.5, 0.0, 0.0), 0.0)
        h64 = o.run(CHANNEL_BCS, 300, 0.5)
        N = c.n_cells
        eu = np.linalg.norm(u[:N] - o.u[:N]) / np.linalg.norm(o.u[:N])
        ep = np.linalg.norm(p[:N] - o.p[:N]) / np.linalg.norm(o.p[:N])
        print(f"{name}: velocity L2 {eu:.2e}, pressure L2 {ep:.2e}")
        assert eu < 1e-6 and ep < 1e-5          # measured 1.4e-7..1.5e-7 and 5e-7..1e-6
        np.testing.assert_allclose(h / h[0], h64 / h64[0], rtol=2e-3)
        b = NSICase(path)
        b.init((0.5, 0.0, 0.0), 0.0)
        h2 = np.array([b.iterate(CHANNEL_BCS, 0.5) for _ in range(300)])
        ub, pb = b.fields()
        assert np.array_equal(u, ub) and np.array_equal(p, pb)
        np.testing.assert_allclose(h, h2, rtol=1e-6)
        c.close()
        b.close()
    finally:
        NSICase.set_constants()
