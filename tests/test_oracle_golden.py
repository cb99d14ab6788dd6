"""The CPU oracle against outputs of the reference solver itself.

The fixtures in tests/golden were produced by running the reference's own
sources (built headless, oracle/Makefile.ref) on a GPU: make_golden.py.
The reference computes in float32 with --use_fast_math, so agreement is to
float32 rounding of those operations, not bitwise.
"""
import numpy as np
import pytest

import cases
from helpers import face_map, rel_max
from oracle import OracleMesh, OracleSolver

METRIC_MESHES = ["tet_6x3x2", "hex_6x3x2", "prism_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2", "tet_12x6x2"]

# float32 fast-math reference vs float64 restatement: relative to the
# array's max magnitude.  Volumes and LSQ inverses lose a few more bits to
# cancellation in float32.
TOL = {"face_areas": 1e-6, "face_normals": 1e-6, "face_centers": 1e-6, "cell_centers": 1e-6,
       "cell_volumes": 2e-5, "cell_matrices": 2e-5}


@pytest.fixture(scope="module", params=METRIC_MESHES)
def metric_case(request):
    name = request.param
    g = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}_metrics.npz")
    return name, g, OracleMesh(cases.MESHES[name](), metric_bits=64)


def test_topology_matches_reference_converter(metric_case):
    """Same cells, same per-cell face order, same neighbours, same face node
    order (the node order fixes the face orientation); only face numbering
    differs (reference: hash-bucket order, oracle: first appearance)."""
    name, g, om = metric_case
    N, G, F = (int(x) for x in g["sizes"][:3])
    assert (om.N, om.G, om.F) == (N, G, F)
    perm = face_map(g["face_nodes_starts"], g["face_nodes"], om.get("face_nodes_starts"), om.get("face_nodes"))
    assert np.array_equal(om.get("cell_faces_starts"), g["cell_faces_starts"].astype(np.int64))
    assert np.array_equal(perm[g["cell_faces"].astype(np.int64)], om.get("cell_faces"))
    assert np.array_equal(om.get("cell_connects"), g["cell_connects"].astype(np.int64))
    fs, fn = om.get("face_nodes_starts"), om.get("face_nodes")
    gs, gn = g["face_nodes_starts"], g["face_nodes"]
    for i in range(F):
        assert tuple(fn[fs[perm[i]]:fs[perm[i] + 1]]) == tuple(gn[gs[i]:gs[i + 1]])
    assert np.array_equal(om.get("ghost_cell_ids"), g["ghost_cell_ids"].astype(np.int64))
    assert np.array_equal(om.get("ghost_cell_starts"), g["ghost_cell_starts"].astype(np.int64))


@pytest.mark.parametrize("bits", [32, 64])
def test_metrics_match_reference(metric_case, bits):
    name, g, _ = metric_case
    om = OracleMesh(cases.MESHES[name](), metric_bits=bits)
    perm = face_map(g["face_nodes_starts"], g["face_nodes"], om.get("face_nodes_starts"), om.get("face_nodes"))
    for key in ("face_areas", "face_normals", "face_centers"):
        comps = 1 if key == "face_areas" else 3
        mine = om.get(key).reshape(-1, comps)[perm]
        assert rel_max(mine, g[key].reshape(-1, comps)) < TOL[key], key
    for key in ("cell_volumes", "cell_centers", "cell_matrices"):
        assert rel_max(om.get(key), g[key]) < TOL[key], key


PREP_KEYS = [("rho.value", "rho", 1, 2e-7), ("rhou.value", "rhou", 3, 2e-7), ("rhoe.value", "rhoe", 1, 2e-7),
             ("rho.gradient", "grad_rho", 3, 2e-5), ("rhoe.gradient", "grad_rhoe", 3, 2e-5),
             ("rhou.gradient", "grad_rhou", 9, 2e-5), ("rho.limiter", "lim_rho", 1, 1e-4),
             ("rhoe.limiter", "lim_rhoe", 1, 1e-4), ("rhou.limiter", "lim_rhou", 3, 1e-4)]


@pytest.mark.parametrize("name", METRIC_MESHES)
@pytest.mark.parametrize("bits", [32, 64])
def test_bcs_gradients_limiters_match_reference(name, bits):
    """Boundary ghosts (slip and far field), LSQ gradients and limiters after
    the reference's FvmEulerStepPrepare, from a seeded non-uniform state."""
    g = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}_prepare.npz")
    om = OracleMesh(cases.MESHES[name](), metric_bits=bits)
    s = OracleSolver(om, bits=bits)
    s.set_state(g["state_rho"], g["state_rhou"], g["state_rhoe"])
    s.apply_bcs(cases.channel_bcs())
    s.prepare()
    for key, ok, comps, tol in PREP_KEYS:
        ref = g[key].reshape(-1, comps) if comps > 1 else g[key]
        assert rel_max(s.get(ok), ref) < tol, key


def test_channel_2000_iterations_match_reference():
    """2000 iterations of the bump channel (Mach 0.5, CFL 0.8): residual
    history and fields against the reference's own run.  The reference updates
    in place (racy), the oracle as a Jacobi sweep; both stay within float32
    noise of each other over the run."""
    g = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/channel_solve2000.npz")
    om = OracleMesh(cases.MESHES["channel"](), metric_bits=64)
    s = OracleSolver(om, bits=32)
    s.init(cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)
    h = s.run(cases.channel_bcs(), 2000, 0.8)
    ref = g["residual_history"]
    np.testing.assert_allclose(h / h[0], ref / ref[0], rtol=5e-3)
    N = om.N
    for key, ok, comps in (("rho.value", "rho", 1), ("rhou.value", "rhou", 3), ("rhoe.value", "rhoe", 1)):
        r = g[key].reshape(-1, comps)[:N] if comps > 1 else g[key][:N]
        o = s.get(ok)[:N]
        d = np.abs(o - r) / np.max(np.abs(r))
        assert d.max() < 1e-3 and d.mean() < 5e-5, (key, d.max(), d.mean())


# (offset, width) of each operator in the reference harness's 35 outputs per
# cell (oracle/ref_fvmops.cu), by the operator ids of gbFvmApply
FVMOP_SLOTS = {0: (0, 1), 1: (1, 3), 2: (4, 3), 3: (7, 9), 4: (16, 3), 5: (19, 9), 6: (28, 1), 7: (29, 1),
               8: (30, 1), 9: (31, 1), 10: (32, 3)}
VECTOR_OPS = (3, 5, 6, 10)


@pytest.mark.parametrize("name", ["tet_6x3x2", "prism_6x3x2", "hex_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2"])
def test_operator_restatement_matches_reference_operators(name):
    """oracle/fvmops_oracle.py against the reference's own inline fvmOp
    functions (include/fvmops.cuh:96-219) evaluated by oracle/ref_fvmops.cu
    on the B200 (float32, fast math), given the reference's own gradients
    and limiters; and the restated gradient + limiter against the
    reference's ScalarVar/VectorVarComputeGradient and -Limiters."""
    from oracle.fvmops_oracle import OpMesh

    z = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}_fvmops.npz")
    om = OpMesh(OracleMesh(cases.MESHES[name]()))
    N, n = om.N, len(z["s"])
    ops = z["ops"].reshape(N, 35).astype(np.float64)
    s, v = z["s"].astype(np.float64), z["v"].astype(np.float64)
    sg = z["s.gradient"].reshape(n, 3)[:N].astype(np.float64)
    sl = z["s.limiter"][:N].astype(np.float64)
    vg = z["v.gradient"].reshape(n, 3, 3)[:N].astype(np.float64)     # tensor columns = component gradients
    vl = z["v.limiter"].reshape(n, 3)[:N].astype(np.float64)
    g, l = om.gradient(s)
    assert rel_max(g[:, 0], sg) < 2e-5 and np.max(np.abs(l[:, 0] - sl)) < 2e-5
    g, l = om.gradient(v)
    assert rel_max(g, vg) < 2e-5 and np.max(np.abs(l - vl)) < 2e-5
    for op, (o, k) in FVMOP_SLOTS.items():
        u = v if op in VECTOR_OPS else s
        got = om.apply(op, u, grad=sg[:, None, :], lim=sl[:, None], phi=z["phi"].astype(np.float64),
                       phi_c=z["phi_const"].astype(np.float64)).reshape(N, k)
        assert rel_max(got, ops[:, o:o + k]) < 1e-4, op
