"""Batched multi-instance solves (gbBatch*) against plain single solves."""
import math

import numpy as np
import pytest

import cases
from graphite_b200 import capi, meshgen
from graphite_b200.batch import EulerBatch
from graphite_b200.euler import EulerCase

pytestmark = pytest.mark.gpu


def airfoil_bcs(mach, aoa_deg):
    a = math.radians(aoa_deg)
    m = (mach * math.cos(a), 0.0, mach * math.sin(a))
    return m, [("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")]


@pytest.fixture(scope="module")
def meshes(workdir):
    paths = []
    for name, m in (("af_a", meshgen.airfoil_2d_prisms(40, 12)), ("af_b", meshgen.airfoil_2d_prisms(64, 16))):
        p = str(workdir / f"{name}.su2")
        m.write_su2(p)
        paths.append(p)
    return paths


def _instances():
    rng = np.random.default_rng(3)
    return [(k % 2, float(rng.uniform(0.3, 0.8)), float(rng.uniform(-2, 6))) for k in range(5)]


@pytest.mark.parametrize("tuning", [(256, 0), (512, 1), (1024, 3), (2048, 2), (512, 4), (1024, 5), (256, 6),
                                    (512, 7), (1024, 8), (2048, 9)])
def test_batch_equals_plain_solves(meshes, tuning):
    """Every instance of a batch follows, bit for bit, the iterates of a plain
    solve of it, whatever the tile size and schedule (schedules 6-9: the
    persistent kernel)."""
    lib = capi.load()
    lib.gbSetReferenceMomentumReconstruction(1)
    cs = [EulerCase(p) for p in meshes]
    inst = _instances()
    spec = [(k, airfoil_bcs(m, a)[1]) for k, m, a in inst]
    with EulerBatch(cs, spec) as b:
        b.set_tuning(*tuning)
        for i, (k, m, a) in enumerate(inst):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        done, its, rat, st = b.run(0.8, 150)
        assert done == 150 and np.all(its == 150) and np.all(st == 2)
        got = [b.get_state(i) for i in range(len(inst))]
    for i, (k, m, a) in enumerate(inst):
        mach, bcs = airfoil_bcs(m, a)
        c = cs[k]
        c.init(mach, cases.P_INF, cases.T_INF)
        h = c.run(bcs, 0.8, 150)
        ref = c.fields()
        assert np.array_equal(got[i][0], ref[0]), i
        assert np.array_equal(got[i][1], ref[1]), i
        assert np.array_equal(got[i][2], ref[2]), i
        np.testing.assert_allclose(rat[i], h[-1] / h[0], rtol=1e-12)
    for c in cs:
        c.close()


@pytest.mark.parametrize("schedule", [5, 7])
def test_tile_shrinks_as_instances_stop_without_changing_states(meshes, schedule):
    """Once instances stop, the run re-tiles the remaining work into smaller
    items; every instance still ends bit for bit where a plain solve of its
    own iteration count ends, and the tuned tile is back after the run."""
    lib = capi.load()
    lib.gbSetReferenceMomentumReconstruction(1)
    cs = [EulerCase(p) for p in meshes]
    inst = _instances()
    spec = [(k, airfoil_bcs(m, a)[1]) for k, m, a in inst]
    with EulerBatch(cs, spec) as b:
        b.set_tuning(2048, schedule)
        for i, (k, m, a) in enumerate(inst):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        done, its, rat, st = b.run(0.8, 3000, tolerance=3e-2, check_every=10)
        assert np.all(st == 1), st
        assert len(set(its.tolist())) > 1          # they stop at different iterations
        assert b.tuning() == (2048, schedule)
        got = [b.get_state(i) for i in range(len(inst))]
    for i, (k, m, a) in enumerate(inst):
        mach, bcs = airfoil_bcs(m, a)
        c = cs[k]
        c.init(mach, cases.P_INF, cases.T_INF)
        c.run(bcs, 0.8, int(its[i]))
        ref = c.fields()
        for q in range(3):
            assert np.array_equal(got[i][q], ref[q]), (i, q)
    for c in cs:
        c.close()


def test_batch_instances_stop_at_their_own_tolerance(meshes):
    cs = [EulerCase(p) for p in meshes]
    inst = _instances()
    spec = [(k, airfoil_bcs(m, a)[1]) for k, m, a in inst]
    with EulerBatch(cs, spec) as b:
        for i, (k, m, a) in enumerate(inst):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        before = [b.get_state(i) for i in range(len(inst))]
        tile, sched = b.autotune(0.8, trial_iters=3)
        assert tile % 256 == 0 and sched in range(10)
        for i in range(len(inst)):                 # the trials' iterations are undone
            for q in range(3):
                assert np.array_equal(b.get_state(i)[q], before[i][q])
        done, its, rat, st, hist = b.run(0.8, 3000, tolerance=1e-2, check_every=50, history=True)
        assert np.all(st == 1), st
        assert np.all(rat < 1e-2)
        for i in range(len(inst)):
            h = hist[i, : its[i]]
            assert h[-1] / h[0] < 1e-2 and np.all(h[:-1] / h[0] >= 1e-2)
            assert np.all(hist[i, its[i]:] == 0)     # frozen afterwards
    # a plain solve of one instance stops at the same iteration
    k, m, a = inst[0]
    mach, bcs = airfoil_bcs(m, a)
    c = cs[k]
    c.init(mach, cases.P_INF, cases.T_INF)
    h = c.run(bcs, 0.8, 3000, tolerance=1e-2, check_every=1)
    assert len(h) == its[0]
    for c in cs:
        c.close()


def test_batch_warm_start_state_round_trip(meshes):
    cs = [EulerCase(meshes[0])]
    mach, bcs = airfoil_bcs(0.5, 2.0)
    with EulerBatch(cs, [(0, bcs), (0, bcs)]) as b:
        n = cs[0].n_cells + cs[0].n_ghosts
        rng = np.random.default_rng(0)
        rho = (1.4 + 0.01 * rng.standard_normal(n)).astype(np.float32)
        rhou = (np.array(mach) * 1.4 + 0.01 * rng.standard_normal((n, 3))).astype(np.float32)
        rhoe = (2.5 + 0.5 * 1.4 * 0.25 + 0.01 * rng.standard_normal(n)).astype(np.float32)
        b.set_state(1, rho, rhou, rhoe)
        r, u, e = b.get_state(1)
        assert np.array_equal(r, rho) and np.array_equal(u, rhou) and np.array_equal(e, rhoe)
    cs[0].close()


@pytest.mark.parametrize("tuning", [(256, 1), (256, 5), (1024, 9)])
def test_batch_on_3d_mixed_meshes_equals_plain_solves(su2_paths, tuning):
    """A batch over three 3-D channels -- tets, the hex / prism / pyramid mix
    and prism layers under tets (cells of 4, 5 and 6 faces in one launch; not
    ghost-heavy, so the plain solves apply the conditions with the ghost
    kernel while the batch applies them inside its gradient pass) -- follows
    the plain solves bit for bit."""
    lib = capi.load()
    lib.gbSetReferenceMomentumReconstruction(1)
    names = ["tet_12x6x2", "mixed_6x3x2", "layered_6x3x2"]
    cs = [EulerCase(su2_paths(n)) for n in names]
    inst = [(k, mach) for k in range(3) for mach in (0.4, 0.6)]
    spec = [(k, cases.channel_bcs((m, 0.0, 0.0))) for k, m in inst]
    with EulerBatch(cs, spec) as b:
        b.set_tuning(*tuning)
        for i, (k, m) in enumerate(inst):
            b.init_uniform(i, (m, 0.0, 0.0), cases.P_INF, cases.T_INF)
        done, its, rat, st = b.run(0.8, 120)
        assert done == 120 and np.all(its == 120)
        got = [b.get_state(i) for i in range(len(inst))]
    for i, (k, m) in enumerate(inst):
        c = cs[k]
        c.init((m, 0.0, 0.0), cases.P_INF, cases.T_INF)
        h = c.run(cases.channel_bcs((m, 0.0, 0.0)), 0.8, 120)
        ref = c.fields()
        for q in range(3):
            assert np.array_equal(got[i][q], ref[q]), (names[k], m, q)
        np.testing.assert_allclose(rat[i], h[-1] / h[0], rtol=1e-12)
    for c in cs:
        c.close()
