"""Headless colour map of a boundary region (gbRenderRegionScalar) against a
numpy restatement of the reference's render kernel."""
import numpy as np
import pytest

import cases
from graphite_b200 import capi
from graphite_b200.euler import EulerCase

pytestmark = pytest.mark.gpu


def _colour(t):
    t = np.clip(t, 0.0, 1.0)
    out = np.zeros(t.shape + (3,))
    a = t <= 0.2
    out[a] = np.stack([0 * t[a], 0 * t[a], 0.5 + t[a] * 0.5 / 0.2], -1)
    b = (t > 0.2) & (t <= 0.4)
    out[b] = np.stack([0 * t[b], (t[b] - 0.2) / 0.2, 1 + 0 * t[b]], -1)
    c = (t > 0.4) & (t <= 0.6)
    out[c] = np.stack([(t[c] - 0.4) / 0.2, 1 + 0 * t[c], 1 - (t[c] - 0.4) / 0.2], -1)
    d = (t > 0.6) & (t <= 0.8)
    out[d] = np.stack([1 + 0 * t[d], 1 - (t[d] - 0.6) / 0.2, 0 * t[d]], -1)
    e = t > 0.8
    out[e] = np.stack([1 - (t[e] - 0.8) * 0.5 / 0.2, 0 * t[e], 0 * t[e]], -1)
    return out


@pytest.mark.parametrize("name,region", [("prism_6x3x2", "lower"), ("hex_6x3x2", "upper")])
def test_region_colours_match_restatement(su2_paths, name, region):
    c = EulerCase(su2_paths(name))
    bcs = cases.channel_bcs()
    c.init(cases.CHANNEL_MACH, cases.P_INF, cases.T_INF)
    c.run(bcs, 0.8, 30)
    c.apply_bcs(bcs)
    c.prepare()                                   # stores gradients + limiters
    rho = c.fields()[0]
    grad, lim = c.gradients()["rho"]
    lib = capi.load()
    rid = lib.cuMeshGetRegionId(c.mesh, region.encode())
    n = lib.gbRenderRegionScalar(c.mesh, rid, c.rho, 1.3, 1.5, None, 0)
    assert n > 0
    out = np.zeros((n, 18), np.float32)
    assert lib.gbRenderRegionScalar(c.mesh, rid, c.rho, 1.3, 1.5, out.ctypes.data, n) == n
    assert lib.gbRenderRegionScalar(c.mesh, rid, c.rho, 1.3, 1.5, out.ctypes.data, n - 1) == -1
    # restatement from the host mirrors, reference order
    b = c.mesh.contents._cpu.contents
    nodes = np.array([[b.nodes[i].x, b.nodes[i].y, b.nodes[i].z] for i in range(b.n_nodes)], np.float64)
    ref = {}
    for k in range(b.ghost_cell_starts[rid], b.ghost_cell_starts[rid + 1]):
        g = b.ghost_cell_ids[k]
        f = b.cell_faces[b.cell_faces_starts[g]]
        i = b.cell_connects[b.cell_faces_starts[g]]
        fn = [b.face_nodes[j] for j in range(b.face_nodes_starts[f], b.face_nodes_starts[f + 1])]
        u = 0.5 * (rho[g] + rho[i])
        for j in range(len(fn) - 2):
            p = nodes[[fn[0], fn[j + 1], fn[j + 2]]]
            cen = p.mean(axis=0)
            uf = (u + (p - cen) @ grad[i] * lim[i] - 1.3) / 0.2
            key = tuple(np.round(p.ravel(), 5))
            ref[key] = np.column_stack([p, _colour(uf)])
    assert len(ref) == n
    for t in out:
        key = tuple(np.round(t.reshape(3, 6)[:, :3].astype(np.float64).ravel(), 5))
        np.testing.assert_allclose(t.reshape(3, 6), ref[key], atol=2e-5)
    c.close()
