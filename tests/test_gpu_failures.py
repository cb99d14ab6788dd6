"""Failure detection, exercised without a GPU fault: every failure is made on
the host (a non-finite state uploaded through the C ABI) or by a bounded
wait that is made to run out (a tensor-core wait bound of a few cycles, a
grid barrier that no block can complete), and the tests check that the
library reports it and that the next call works normally.  The reference
has no such detection: its only NaN check is commented out
(apps/main_old.cu:133)."""
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
def airfoil(workdir):
    p = str(workdir / "fail_airfoil.su2")
    meshgen.airfoil_2d_prisms(40, 12).write_su2(p)
    return p


DRAWS = [(0.5, 2.0), (0.6, 4.0), (0.7, -1.0)]


def _plain(c, m, a, iters):
    mach, bcs = airfoil_bcs(m, a)
    c.init(mach, cases.P_INF, cases.T_INF)
    c.run(bcs, 0.8, iters)
    return c.fields()


@pytest.mark.parametrize("schedule", [5, 7])
def test_non_finite_instance_stops_alone(airfoil, schedule):
    """A NaN put into one instance's state stops that instance (status 3,
    not finite) at its first residual; the other instances run on and end
    bit for bit where plain solves end."""
    capi.load().gbSetReferenceMomentumReconstruction(1)
    c = EulerCase(airfoil)
    spec = [(0, airfoil_bcs(m, a)[1]) for m, a in DRAWS]
    with EulerBatch([c], spec) as b:
        b.set_tuning(512, schedule)
        for i, (m, a) in enumerate(DRAWS):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        r, u, e = b.get_state(1)
        r = r.copy()
        r[7] = np.nan
        b.set_state(1, r, u, e)
        done, its, rat, st = b.run(0.8, 60, check_every=20)
        assert st.tolist() == [2, 3, 2], st
        assert its[1] == 1 and its[0] == its[2] == 60
        got = [b.get_state(i) for i in (0, 2)]
    for (m, a), g in zip((DRAWS[0], DRAWS[2]), got):
        ref = _plain(c, m, a, 60)
        for q in range(3):
            assert np.array_equal(g[q], ref[q])
    c.close()


def test_non_finite_state_is_reported_by_the_run(airfoil):
    """gbEulerRun reports a non-finite residual (a diverged or corrupted
    state) as an error instead of iterating on; the case runs normally once
    a valid state is back."""
    capi.load().gbSetReferenceMomentumReconstruction(1)
    mach, bcs = airfoil_bcs(0.6, 3.0)
    with EulerCase(airfoil) as c:
        c.init(mach, cases.P_INF, cases.T_INF)
        rho, rhou, rhoe = c.fields()
        bad = rho.copy()
        bad[3] = np.inf
        c.set_state(bad, rhou, rhoe)
        with pytest.raises(capi.GraphiteError, match="not finite"):
            c.run(bcs, 0.8, 50, check_every=10)
        c.set_state(rho, rhou, rhoe)
        h = c.run(bcs, 0.8, 50, check_every=10)
        assert len(h) == 50 and np.all(np.isfinite(h))


def test_mlp_wait_that_gives_up_is_reported_and_recovered():
    """With a wait bound of a few cycles the MLP kernel's first wait for its
    tensor-core work gives up: the call returns an error naming the stage,
    the kernel lets its work finish and frees its tensor memory, and the next
    call with the default bound gives the oracle's gradient."""
    from graphite_b200.warmstart import WarmStart
    from oracle import mlp_oracle as mo

    rng = np.random.default_rng(5)
    x = np.column_stack([rng.uniform(-1, 1, (512, 7)), np.ones(512)]).astype(np.float32)
    t = rng.standard_normal((512, 5)).astype(np.float32)
    w = mo.init_like_kernel(np.random.default_rng(6)).astype(np.float32)
    lib = capi.load()
    with WarmStart(None, seed=1) as ws:
        ws.weights = w
        capi.check(lib.gbWarmStartSetWaitLimit(ws.h, 4), "gbWarmStartSetWaitLimit")
        with pytest.raises(capi.GraphiteError, match="gave up"):
            ws.gradient(x, t)
        capi.check(lib.gbWarmStartSetWaitLimit(ws.h, 0), "gbWarmStartSetWaitLimit")
        g, loss = ws.gradient(x, t)
    lref, gref = mo.loss_and_grad(w.astype(np.float64), x.astype(np.float64), t.astype(np.float64), mode="kernel")
    cos = float(g @ gref / np.linalg.norm(g) / np.linalg.norm(gref))
    assert abs(loss - lref) < 2e-3 * lref and cos > 0.9995, (loss, lref, cos)


def test_persistent_barrier_that_cannot_complete_is_reported(airfoil):
    """The persistent batch kernel's grid barrier, started in a state no
    block can complete, gives up after its bound: the run returns an error
    rather than hanging, and the next run of the same batch is normal."""
    capi.load().gbSetReferenceMomentumReconstruction(1)
    c = EulerCase(airfoil)
    spec = [(0, airfoil_bcs(m, a)[1]) for m, a in DRAWS]
    with EulerBatch([c], spec) as b:
        b.set_tuning(512, 7)
        for i, (m, a) in enumerate(DRAWS):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        capi.check(capi.load().gbBatchInjectBarrierFault(b.h), "gbBatchInjectBarrierFault")
        with pytest.raises(capi.GraphiteError, match="gave up"):
            b.run(0.8, 20, check_every=20)
        for i, (m, a) in enumerate(DRAWS):
            b.init_uniform(i, airfoil_bcs(m, a)[0], cases.P_INF, cases.T_INF)
        done, its, rat, st = b.run(0.8, 40, check_every=20)
        assert done == 40 and np.all(st == 2)
        got = b.get_state(1)
    ref = _plain(c, *DRAWS[1], 40)
    for q in range(3):
        assert np.array_equal(got[q], ref[q])
    c.close()


def test_nsi_non_finite_state_is_reported_by_the_run(workdir):
    """gbNSIRun reports a non-finite residual as an error, like gbEulerRun,
    and runs normally again from a valid state."""
    from graphite_b200.nsi import NSICase
    path = str(workdir / "nsi_fail_cyl.su2")
    meshgen.cylinder_ogrid(32, 16, ratio=1.15, r_far=10.0).write_su2(path)
    bcs = [("wall", "cylinder"), ("inletoutlet", "farfield", 1.0, 0.0, 0.0, 0.0), ("slip", "sides")]
    c = NSICase(path)
    try:
        c.init((1.0, 0.0, 0.0), 0.0)
        u, p = c.fields()
        bad = p.copy()
        bad[5] = np.nan
        c.set_state(u, bad)
        with pytest.raises(capi.GraphiteError, match="not finite"):
            c.run(bcs, 0.5, 40, check_every=10)
        c.set_state(u, p)
        h = c.run(bcs, 0.5, 40, check_every=10)
        assert len(h) == 40 and np.all(np.isfinite(h))
    finally:
        c.close()
