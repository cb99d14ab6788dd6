"""Golden-fixture cases: meshes, freestream, boundary conditions, states.

Shared by make_golden.py (which runs the reference solver on them) and the
tests (which run the oracle and the CUDA path on the same inputs).
"""
from __future__ import annotations

import numpy as np

from graphite_b200 import meshgen

GAMMA = 1.4
# Non-dimensional freestream used by every reference example: p = 1,
# T = 1/1.4, so rho = 1.4 and the speed of sound is 1
# (examples/airfoil/airfoil.json, src/models/euler.cu:401-404).
P_INF = 1.0
T_INF = 1.0 / 1.4

CHANNEL_MACH = (0.5, 0.0, 0.0)


def channel_bcs(mach=CHANNEL_MACH):
    """Channel boundary conditions, in the sorted-key order PhysicsEuler::step
    walks its "bcs" JSON object (src/models/euler.cu:103-135)."""
    ff = ("farfield",)
    return [ff + ("inlet",) + tuple(mach) + (P_INF, T_INF),
            ("slip", "lower"),
            ff + ("outlet",) + tuple(mach) + (P_INF, T_INF),
            ("slip", "sides"),
            ("slip", "upper")]


MESHES = {
    "tet_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="tet"),
    "hex_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="hex"),
    "prism_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="prism"),
    "pyramid_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="pyramid"),
    "mixed_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="mixed"),
    "layered_6x3x2": lambda: meshgen.channel_bump(6, 3, 2, cells="layered"),
    "tet_12x6x2": lambda: meshgen.channel_bump(12, 6, 2, cells="tet"),
    "channel": lambda: meshgen.channel_bump(60, 20, 4, cells="tet"),
}


def element_centres(mesh: meshgen.ElementMesh) -> np.ndarray:
    cs = [mesh.nodes[conn].mean(axis=1) for _, conn in mesh.blocks]
    return np.concatenate(cs)


def synthetic_state(mesh: meshgen.ElementMesh, seed: int = 20261203, noise: float = 0.03):
    """A smooth, non-uniform, physically valid state plus seeded noise, in
    reference cell order (elements, then one ghost per boundary face).

    Returns (rho[n], rhou[n,3], rhoe[n]) as float32 with n = cells + ghosts.
    Ghost values are set too but the boundary conditions overwrite them.
    """
    rng = np.random.default_rng(seed)
    c = element_centres(mesh)
    n = mesh.n_cells + mesh.n_ghosts
    x = np.zeros((n, 3))
    x[: mesh.n_cells] = c
    rho = 1.4 * (1.0 + 0.1 * np.sin(2.0 * x[:, 0]) * np.cos(3.0 * x[:, 1]) + noise * rng.standard_normal(n))
    u = np.stack([0.5 + 0.1 * np.cos(x[:, 1] * 4.0), 0.05 * np.sin(x[:, 0] * 3.0), 0.02 * x[:, 2]], axis=1)
    u += noise * rng.standard_normal((n, 3))
    p = 1.0 + 0.05 * np.cos(x[:, 0] + x[:, 1]) + noise * rng.standard_normal(n)
    rhou = rho[:, None] * u
    rhoe = p / (GAMMA - 1.0) + 0.5 * rho * np.sum(u * u, axis=1)
    return rho.astype(np.float32), rhou.astype(np.float32), rhoe.astype(np.float32)
