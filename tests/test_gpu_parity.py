"""The sm_100a path, through the C ABI, against the oracle and the reference.

Every call goes through libgraphite_b200.so (graphite_b200.capi); the oracle
(oracle/, float64 unless stated) and the reference's golden outputs are the
checkers.  The kernels compute in float32 from float64 metrics, so parity is
to float32 rounding: tolerances are relative to each array's largest
magnitude and written next to each comparison.
"""
import os

import numpy as np
import pytest

import cases
from graphite_b200 import capi
from graphite_b200.euler import EulerCase
from helpers import face_map, rel_max
from oracle import OracleMesh, OracleSolver

pytestmark = pytest.mark.gpu

SMALL = ["tet_6x3x2", "hex_6x3x2", "prism_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2", "tet_12x6x2"]
BCS = cases.channel_bcs()
INIT = (cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)


def golden(name):
    return np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}.npz")


@pytest.fixture(autouse=True)
def reference_defaults():
    lib = capi.load()
    lib.gbSetReferenceMomentumReconstruction(1)
    lib.gbSetRenumbering(1)
    yield
    lib.gbSetReferenceMomentumReconstruction(1)
    lib.gbSetRenumbering(1)


def oracle_state(name, bits=64, transposed=True):
    om = OracleMesh(cases.MESHES[name](), metric_bits=64)
    return om, OracleSolver(om, bits=bits, transposed_momentum=transposed)


@pytest.mark.parametrize("name", SMALL)
def test_metrics_match_oracle_and_reference(name, su2_paths):
    """float64 device metrics, rounded to float32 in the host mirror, against
    the float64 oracle (float32 rounding only) and the reference's float32
    fast-math metrics."""
    with EulerCase(su2_paths(name)) as c:
        m = c.mesh
        om = OracleMesh(cases.MESHES[name](), metric_bits=64)
        perm = face_map(om.get("face_nodes_starts"), om.get("face_nodes"), capi.mesh_array(m, "face_nodes_starts"),
                        capi.mesh_array(m, "face_nodes"))
        assert rel_max(capi.mesh_array(m, "face_areas")[perm], om.get("face_areas")) < 2e-7
        assert rel_max(capi.mesh_array(m, "face_normals")[perm], om.get("face_normals").reshape(-1, 3)) < 2e-7
        assert rel_max(capi.mesh_array(m, "face_centers")[perm], om.get("face_centers").reshape(-1, 3)) < 2e-7
        assert rel_max(capi.mesh_array(m, "cell_volumes"), om.get("cell_volumes")) < 2e-7
        assert rel_max(capi.mesh_array(m, "cell_centers"), om.get("cell_centers").reshape(-1, 3)) < 2e-7
        assert rel_max(capi.mesh_array(m, "cell_matrices"), om.get("cell_matrices").reshape(-1, 9)) < 2e-7
        g = golden(f"{name}_metrics")
        rperm = face_map(g["face_nodes_starts"], g["face_nodes"], capi.mesh_array(m, "face_nodes_starts"),
                         capi.mesh_array(m, "face_nodes"))
        assert rel_max(capi.mesh_array(m, "face_areas")[rperm], g["face_areas"]) < 1e-6
        assert rel_max(capi.mesh_array(m, "cell_volumes"), g["cell_volumes"]) < 2e-5
        assert rel_max(capi.mesh_array(m, "cell_matrices").reshape(-1), g["cell_matrices"]) < 2e-5


def _prepare(name, su2_paths, transposed=True):
    g = golden(f"{name}_prepare")
    c = EulerCase(su2_paths(name))
    c.set_state(g["state_rho"], g["state_rhou"], g["state_rhoe"])
    c.apply_bcs(BCS)
    c.prepare()
    om, s = oracle_state(name, transposed=transposed)
    s.set_state(g["state_rho"], g["state_rhou"], g["state_rhoe"])
    s.apply_bcs(BCS)
    s.prepare()
    return g, c, s


@pytest.mark.parametrize("name", SMALL)
def test_bcs_gradients_limiters(name, su2_paths):
    """Ghost states (slip, far field), LSQ gradients and limiters of the fused
    kernel vs the float64 oracle and the reference's FvmEulerStepPrepare.
    Gradients: float32 sums of differences, 2e-5 of the largest entry.
    Limiters: smooth switches of gradient ratios, 2e-4 absolute."""
    g, c, s = _prepare(name, su2_paths)
    with c:
        rho, rhou, rhoe = c.fields()
        assert rel_max(rho, s.get("rho")) < 2e-7
        assert rel_max(rhou, s.get("rhou")) < 2e-7
        assert rel_max(rhoe, s.get("rhoe")) < 2e-7
        grads = c.gradients()
        for var, gk, lk in (("rho", "grad_rho", "lim_rho"), ("rhou", "grad_rhou", "lim_rhou"),
                            ("rhoe", "grad_rhoe", "lim_rhoe")):
            grad, lim = grads[var]
            assert rel_max(grad, s.get(gk)) < 2e-5, var
            assert np.max(np.abs(lim - s.get(lk))) < 2e-4, var
            ref_g = g[f"{var}.gradient"].reshape(grad.shape)
            ref_l = g[f"{var}.limiter"].reshape(lim.shape)
            assert rel_max(grad, ref_g) < 3e-5, var
            assert np.max(np.abs(lim - ref_l)) < 3e-4, var


@pytest.mark.parametrize("name", SMALL)
@pytest.mark.parametrize("transposed", [True, False])
def test_one_iteration_matches_oracle(name, transposed, su2_paths):
    """One full iteration (BCs, prepare, flux + update, residual) from the
    seeded state, both momentum reconstructions: updated fields to 1e-5 of
    their largest value, residual per cell to 1e-4, residual sum to 1e-5."""
    capi.load().gbSetReferenceMomentumReconstruction(1 if transposed else 0)
    g, c, s = _prepare(name, su2_paths, transposed=transposed)
    with c:
        c.step(0.8)
        res = c.residual()
        s.step(0.8)
        N = c.n_cells
        rho, rhou, rhoe = c.fields()
        assert rel_max(rho[:N], s.get("rho")[:N]) < 1e-5
        assert rel_max(rhou[:N], s.get("rhou")[:N]) < 1e-5
        assert rel_max(rhoe[:N], s.get("rhoe")[:N]) < 1e-5
        err = c.error_values()[:N]
        assert rel_max(err, s.get("err")[:N]) < 1e-4
        assert abs(res - s.reduce_error()) < 1e-5 * abs(s.reduce_error())


def test_momentum_modes_differ(su2_paths):
    """The reference's transposed reconstruction is a real difference on a
    non-uniform state (so the switch is exercised)."""
    out = []
    for t in (1, 0):
        capi.load().gbSetReferenceMomentumReconstruction(t)
        g, c, s = _prepare("tet_12x6x2", su2_paths)
        with c:
            c.step(0.8)
            out.append(c.fields()[1])
    assert rel_max(out[0], out[1]) > 1e-4


def test_channel_2000_iterations_match_reference(su2_paths):
    """The bump channel for 2000 iterations through the per-call ABI (the
    PhysicsEuler::step loop) against the reference's own run: residual history
    within 5e-3 relative, fields within 1e-3 max / 5e-5 mean of their
    largest value (the reference's in-place update races; this is a Jacobi
    sweep)."""
    g = golden("channel_solve2000")
    with EulerCase(su2_paths("channel")) as c:
        c.init(*INIT)
        h = np.array([c.iterate(BCS, 0.8) for _ in range(2000)])
        ref = g["residual_history"]
        np.testing.assert_allclose(h / h[0], ref / ref[0], rtol=5e-3)
        N = c.n_cells
        for got, key, comps in zip(c.fields(), ("rho.value", "rhou.value", "rhoe.value"), (1, 3, 1)):
            r = g[key].reshape(-1, comps)[:N] if comps > 1 else g[key][:N]
            d = np.abs(got[:N] - r) / np.max(np.abs(r))
            assert d.max() < 1e-3 and d.mean() < 5e-5, (key, d.max(), d.mean())


# every region; one region left without a condition (its ghosts keep their
# stored state); a region given two conditions (the later one holds)
BC_SETS = {"all": BCS, "no_sides": [b for b in BCS if b[1] != "sides"],
           "upper_twice": BCS + [("farfield", "upper") + tuple(cases.CHANNEL_MACH) + (cases.P_INF, cases.T_INF)]}


@pytest.mark.parametrize("mesh,bcs", [("tet_12x6x2", b) for b in BC_SETS] + [("channel", "all"), ("channel", "upper_twice")])
def test_graph_run_is_bitwise_the_per_call_loop(mesh, bcs, su2_paths):
    """gbEulerRun (replayed CUDA graphs) computes exactly what the per-call
    loop computes, ghost values included, whichever regions have conditions:
    on tet_12x6x2 (432 ghosts for 864 cells) its gradient kernel applies the
    conditions, on the channel (6,080 for 28,800) one table-driven ghost
    kernel does, where the per-call loop runs a ghost kernel per condition."""
    hs, fs = [], []
    for mode in ("calls", "graph"):
        with EulerCase(su2_paths(mesh)) as c:
            c.init(*INIT)
            if mode == "calls":
                h = np.array([c.iterate(BC_SETS[bcs], 0.8) for _ in range(57)])
            else:
                h = c.run(BC_SETS[bcs], 0.8, 57)
            hs.append(h)
            fs.append(c.fields())
    assert np.array_equal(hs[0].astype(np.float32), hs[1].astype(np.float32))
    for a, b in zip(fs[0], fs[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("mach,aoa", [(0.6, 3.0), (1.3, 2.0)])
def test_graph_run_is_bitwise_the_per_call_loop_on_airfoil(workdir, mach, aoa):
    """On a one-layer airfoil (two span ghosts per cell) gbEulerRun applies the
    boundary conditions inside its gradient kernel; it still computes exactly
    what the per-call loop with its ghost kernels computes, subsonic and
    supersonic free stream (every far-field branch)."""
    import math
    from graphite_b200 import meshgen
    path = str(workdir / "bitwise_airfoil.su2")
    if not os.path.exists(path):
        meshgen.airfoil_2d_prisms(96, 24).write_su2(path)
    a = math.radians(aoa)
    m = (mach * math.cos(a), 0.0, mach * math.sin(a))
    bcs = [("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")]
    hs, fs = [], []
    for mode in ("calls", "graph"):
        with EulerCase(path) as c:
            c.init(m, cases.P_INF, cases.T_INF)
            if mode == "calls":
                h = np.array([c.iterate(bcs, 0.5) for _ in range(300)])
            else:
                h = c.run(bcs, 0.5, 300)
            hs.append(h)
            fs.append(c.fields())
    assert np.array_equal(hs[0].astype(np.float32), hs[1].astype(np.float32))
    for x, y in zip(fs[0], fs[1]):
        assert np.array_equal(x, y)


def test_runs_are_deterministic(su2_paths):
    out = []
    for _ in range(2):
        with EulerCase(su2_paths("channel")) as c:
            c.init(*INIT)
            h = c.run(BCS, 0.8, 300)
            out.append((h, c.fields()))
    assert np.array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["channel", "mixed_6x3x2", "layered_6x3x2"])
def test_renumbering_does_not_change_results(su2_paths, name):
    """Each cell sums its faces in the reference's element-local order
    whatever the numbering, so fields are bitwise equal with and without the
    reverse Cuthill-McKee renumbering (on the mixed meshes the renumbering
    also interleaves cells of different face counts)."""
    lib = capi.load()
    out = []
    for r in (0, 1):
        lib.gbSetRenumbering(r)
        with EulerCase(su2_paths(name)) as c:
            c.init(*INIT)
            c.run(BCS, 0.8, 200)
            out.append(c.fields())
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_tolerance_stops_on_the_device_at_the_first_iteration_below(su2_paths):
    """With a tolerance the replayed loop stops after the first iteration
    below it, although the host checks only every 50 iterations: the
    remaining iterations of that chunk do nothing, and the state is bitwise
    that of a run of exactly that many iterations (ghost values included)."""
    with EulerCase(su2_paths("tet_12x6x2")) as c:
        c.init(*INIT)
        h = c.run(BCS, 0.8, 5000, tolerance=1e-2, check_every=50)
        r = h / h[0]
        assert len(h) < 5000 and r[-1] < 1e-2 and np.all(r[:-1] >= 1e-2)
        got = c.fields()
        c.init(*INIT)
        h2 = c.run(BCS, 0.8, len(h), check_every=len(h))
        assert np.array_equal(h2, h)
        ref = c.fields()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        # a second run continues from the stopped state and stops again
        h3 = c.run(BCS, 0.8, 20, tolerance=1e-9, check_every=7)
        assert len(h3) == 20


def test_ghost_readback_matches_reference_convention(su2_paths):
    """Ghost gradients/limiters read back as the interior cell's, as the
    reference's fvmScalGradLimBc leaves them."""
    g, c, s = _prepare("tet_6x3x2", su2_paths)
    with c:
        grad, lim = c.gradients()["rho"]
        cfs = capi.mesh_array(c.mesh, "cell_faces_starts")
        conn = capi.mesh_array(c.mesh, "cell_connects")
        for gh in range(c.n_cells, c.n_cells + c.n_ghosts):
            inner = conn[cfs[gh]]
            assert np.array_equal(grad[gh], grad[inner]) and lim[gh] == lim[inner]


def test_errors_are_reported(su2_paths):
    lib = capi.load()
    with EulerCase(su2_paths("tet_6x3x2")) as c:
        c.init(*INIT)
        assert lib.FvmEulerSlipBc(c.mesh, c.rho, c.rhou, c.rhoe, b"nowhere") != 0
        assert "not found" in capi.last_error()
        assert lib.cuMeshGetRegionId(c.mesh, b"nowhere") == 0xFFFFFFFF
        assert lib.FvmEulerStep(c.mesh, c.rho, c.rhou, c.rhoe, 0.8, b"steady", None, c.error) != 0
        assert "Prepare" in capi.last_error()
        assert lib.FvmEulerStep(c.mesh, c.rho, c.rhou, c.rhoe, 0.8, b"unsteady", None, c.error) != 0
        small = lib.FvmFieldNew(4, 7, b"small", 1)
        assert lib.FvmEulerInit(c.mesh, small, c.rhou, c.rhoe, capi.vec(0.5, 0, 0), 1.0, 0.7) != 0
        assert "elements" in capi.last_error()
        assert lib.FvmEulerInit(c.mesh, c.rhou, c.rhou, c.rhoe, capi.vec(0.5, 0, 0), 1.0, 0.7) != 0
        assert "scalar" in capi.last_error()
        lib.FvmFieldFree(small)


def test_deferred_boundary_conditions(su2_paths):
    """FvmEulerSlipBc / FvmEulerInletOutletBc are recorded and applied by the
    next call that uses the fields: reading the fields back shows the
    conditions applied (as the oracle applies them); a later condition on a
    region replaces an earlier one; gbApplyBoundaryConditions applies them
    at once; and a per-call iteration gives bitwise what the replayed loop
    gives."""
    name = "tet_12x6x2"
    lib = capi.load()
    mesh = cases.MESHES[name]()
    rho, rhou, rhoe = cases.synthetic_state(mesh)
    om, s = oracle_state(name)
    with EulerCase(su2_paths(name)) as c:
        c.set_state(rho, rhou, rhoe)
        c.apply_bcs(BCS)
        got = c.fields()                            # VarGpuToCpu applies them first
        s.set_state(rho, rhou, rhoe)
        s.apply_bcs(BCS)
        for g, key in zip(got, ("rho", "rhou", "rhoe")):
            assert rel_max(g, s.get(key)) < 2e-7, key
        # two far-field conditions on the inlet: the later one holds
        other = ("farfield", "inlet", 0.3, 0.0, 0.05, cases.P_INF, cases.T_INF)
        c.set_state(rho, rhou, rhoe)
        c.apply_bcs([BCS[0], other])
        capi.check(lib.gbApplyBoundaryConditions(c.mesh), "gbApplyBoundaryConditions")
        got = c.fields()
        s.set_state(rho, rhou, rhoe)
        s.apply_bcs([other])
        for g, key in zip(got, ("rho", "rhou", "rhoe")):
            assert rel_max(g, s.get(key)) < 2e-7, key
        # per-call iterations against the replayed loop
        c.set_state(rho, rhou, rhoe)
        hp = [c.iterate(BCS, 0.8) for _ in range(5)]
        per_call = c.fields()
        c.set_state(rho, rhou, rhoe)
        hg = c.run(BCS, 0.8, 5, check_every=5)
        graph = c.fields()
        assert np.array_equal(np.float32(hg), np.float32(hp))
        for a, b in zip(per_call, graph):
            assert np.array_equal(a, b)


def test_density_residual_history(su2_paths):
    """gbEulerRunDensityResidual: the same iterates and residual history as
    gbEulerRun (bitwise), and per iteration the density part of the residual,
    sum of F_rho^2 V, against the float64 oracle's."""
    iters = 60
    with EulerCase(su2_paths("tet_12x6x2")) as a, EulerCase(su2_paths("tet_12x6x2")) as b:
        for c in (a, b):
            c.init(*INIT)
        h = a.run(BCS, 0.8, iters)
        h2, d = b.run_density(BCS, 0.8, iters)
        assert np.array_equal(h, h2)
        for x, y in zip(a.fields(), b.fields()):
            assert np.array_equal(x, y)
        assert np.all(d > 0) and np.all(d < h)
    om, s = oracle_state("tet_12x6x2")
    s.init(*INIT)
    d64 = []
    for _ in range(iters):
        s.apply_bcs(BCS)
        s.prepare()
        s.step(0.8)
        d64.append(float(np.sum(s.get("err_rho")[: om.N])))
    d64 = np.array(d64)
    assert np.max(np.abs(d - d64) / d64) < 1e-3, np.max(np.abs(d - d64) / d64)


def test_single_cell_mesh(workdir):
    """The smallest mesh: one tet and its four ghosts (one block of every
    kernel, most of it idle).  Ten iterations through the per-call loop and
    the replayed graphs agree bitwise, and with the float64 oracle."""
    from graphite_b200 import meshgen
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    em = meshgen.ElementMesh(nodes, [(meshgen.TET, np.array([[0, 1, 2, 3]]))],
                             {"wall": [(meshgen.TRI, np.array([[0, 2, 1], [0, 1, 3]]))],
                              "farfield": [(meshgen.TRI, np.array([[1, 2, 3], [0, 3, 2]]))]}, name="one_tet")
    path = str(workdir / "one_tet.su2")
    em.write_su2(path)
    bcs = [("slip", "wall"), ("farfield", "farfield", 0.5, 0.0, 0.1, cases.P_INF, cases.T_INF)]
    with EulerCase(path) as a, EulerCase(path) as b:
        assert a.n_cells == 1 and a.n_ghosts == 4
        for c in (a, b):
            c.init((0.4, 0.0, 0.05), cases.P_INF, cases.T_INF)
        h = np.array([a.iterate(bcs, 0.5) for _ in range(10)])
        h2 = b.run(bcs, 0.5, 10)
        np.testing.assert_array_equal(h, h2)
        for x, y in zip(a.fields(), b.fields()):
            np.testing.assert_array_equal(x, y)
        s = OracleSolver(OracleMesh(em, metric_bits=64), bits=64)
        s.init((0.4, 0.0, 0.05), cases.P_INF, cases.T_INF)
        h64 = s.run(bcs, 10, 0.5)
        np.testing.assert_allclose(h, h64, rtol=1e-4)
        assert rel_max(a.fields()[0][:1], s.get("rho")[:1]) < 1e-5
