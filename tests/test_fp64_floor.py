"""How far the float64 oracle's own lift and drag move at the stopping rule
the benchmark uses (the reference's squared residual below 1e-3 of its first
value, src/models/euler.cu:158-168,380), when its initial density is
perturbed by one unit in the last place.

On the explicit limited scheme the residual does not converge to round-off:
it stalls near the 1e-3 drop while the limiter switches, so the iteration
at which it crosses 1e-3 and the lift there depend on round-off.  This is
the floor under any lift/drag comparison at that stopping point: an FP32
solve (or a warm-started one) cannot be expected to match the FP64 oracle
more closely than the FP64 oracle matches itself.  Measured here on the
4,608-prism NACA 0012 airfoil (96 x 24 O-grid): the spread is 1e-3 to 5e-3
of the lift, above the 1e-4 a converged solution would allow."""
import math

import numpy as np
import pytest

import cases
from graphite_b200 import meshgen
from oracle import pyoracle as po

CASES = [(0.6, 2.5), (0.4, -2.0)]


def airfoil_bcs(mach_m, aoa_deg):
    a = math.radians(aoa_deg)
    m = (mach_m * math.cos(a), 0.0, mach_m * math.sin(a))
    return m, [("farfield", "farfield") + m + (cases.P_INF, cases.T_INF), ("slip", "sides"), ("slip", "wing")]


def solve_to_drop(om, mach, bcs, bits=64, perturb_seed=0, tol=1e-3, cfl=0.5, cap=20000):
    """(iterations, lift, drag) of the oracle at the first iteration whose
    residual is below tol x the first one; perturb_seed > 0 multiplies the
    initial density by 1 +- 2^-52 (a seeded sign per cell)."""
    s = po.OracleSolver(om, bits=bits)
    s.init(mach, cases.P_INF, cases.T_INF)
    if perturb_seed:
        rng = np.random.default_rng(perturb_seed)
        r = s.get("rho")
        s.set_state(r * (1.0 + 2.0 ** -52 * rng.choice([-1.0, 1.0], r.shape)), s.get("rhou"), s.get("rhoe"))
    h0 = None
    for it in range(cap):
        h = float(s.run(bcs, 1, cfl)[0])
        h0 = h if h0 is None else h0
        if h / h0 < tol:
            break
    f = po.wall_force(om, s.get("rho"), s.get("rhou"), s.get("rhoe"), "wing")
    return (it + 1,) + po.lift_drag(f, mach)


@pytest.fixture(scope="module")
def small_airfoil():
    po.set_threads(min(4, po.max_threads()))
    return po.OracleMesh(meshgen.airfoil_2d_prisms(96, 24))


@pytest.mark.parametrize("mach_m,aoa", CASES)
def test_fp64_oracle_spread_at_the_1e3_drop(small_airfoil, mach_m, aoa):
    mach, bcs = airfoil_bcs(mach_m, aoa)
    base = solve_to_drop(small_airfoil, mach, bcs)
    pert = [solve_to_drop(small_airfoil, mach, bcs, perturb_seed=k) for k in (1, 2)]
    lift = abs(base[1])
    spread_l = max(abs(p[1] - base[1]) for p in pert) / lift
    spread_d = max(abs(p[2] - base[2]) for p in pert) / lift
    iters = [base[0]] + [p[0] for p in pert]
    print(f"M {mach_m} AoA {aoa}: stops at {iters}, lift spread {spread_l:.2e}, drag spread {spread_d:.2e} (of lift)")
    # one ulp of initial density moves the stopping iteration and the lift
    # there by far more than 1e-4
    assert len(set(iters)) > 1
    assert spread_l > 5e-4
