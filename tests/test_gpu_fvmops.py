"""The generic finite-volume operators (gbFvmApply) and field gradients
(gbFvmGradient) against their FP64 restatement."""
import ctypes as C

import numpy as np
import pytest

import cases
from graphite_b200 import capi
from oracle.fvmops_oracle import OpMesh
from oracle.pyoracle import OracleMesh

pytestmark = pytest.mark.gpu

OUT = {0: 1, 1: 3, 2: 3, 3: 9, 4: 3, 5: 9, 6: 1, 7: 1, 8: 1, 9: 1, 10: 3}


def _field(lib, mesh, n, comps, name, values):
    f = lib.FvmFieldNew(4 * comps, n, name, 1)
    capi.set_field_values(f, values)
    capi.check(lib.gbVarCpuToGpu(mesh, f), "gbVarCpuToGpu")
    return f


@pytest.mark.parametrize("name", ["tet_6x3x2", "prism_6x3x2", "hex_6x3x2"])
def test_operators_match_restatement(su2_paths, workdir, name):
    lib = capi.load()
    em = cases.MESHES[name]()
    fvm = str(workdir / f"{name}_ops.fvm")
    capi.check(lib.cuMeshFromSu2(su2_paths(name).encode(), fvm.encode()), "cuMeshFromSu2")
    mesh = lib.cuMeshFromFile(fvm.encode())
    n = int(lib.cuMeshGetVarSize(mesh))
    base = mesh.contents._cpu.contents
    x = np.array([[base.cell_centers[i].x, base.cell_centers[i].y, base.cell_centers[i].z] for i in range(n)])
    rng = np.random.default_rng(4)
    s = (np.sin(2 * x[:, 0]) + x[:, 1] ** 2 + 0.05 * rng.standard_normal(n)).astype(np.float32)
    v = np.column_stack([np.cos(x[:, 1]), x[:, 0] * x[:, 2], 1 + 0.1 * rng.standard_normal(n)]).astype(np.float32)
    ph = np.column_stack([1 + 0.2 * x[:, 1], 0.3 * np.ones(n), -0.2 + 0.1 * x[:, 0]]).astype(np.float32)
    fs, fv, fp = _field(lib, mesh, n, 1, b"s", s), _field(lib, mesh, n, 3, b"v", v), _field(lib, mesh, n, 3, b"phi", ph)
    om = OpMesh(OracleMesh(em))
    N = om.N
    # gradients of the scalar and the vector field
    for f, vals, k in ((fs, s, 1), (fv, v, 3)):
        capi.check(lib.gbFvmGradient(mesh, f), "gbFvmGradient")
        lib.VarAllGpuToCpu(f)
        g, l = capi.field_gradients(f)
        gr, lr = om.gradient(vals.astype(np.float64))
        g = g[:N].reshape(N, k, 3)         # host mirror: [cell][component][x, y, z]
        np.testing.assert_allclose(g, gr, atol=2e-5 * np.max(np.abs(gr)))
        np.testing.assert_allclose(np.asarray(l[:N]).reshape(N, k), lr, atol=2e-4)
    gs, ls = om.gradient(s.astype(np.float64))
    phi_c = (0.7, -0.2, 0.4)
    for op, k in OUT.items():
        u = fv if op in (3, 5, 6, 10) else fs
        out = np.zeros((N, k), np.float32)
        capi.check(lib.gbFvmApply(mesh, op, u, fp, capi.vec(phi_c), out.ctypes.data), f"gbFvmApply {op}")
        uu = (v if op in (3, 5, 6, 10) else s).astype(np.float64)
        ref = om.apply(op, uu, grad=gs, lim=ls, phi=ph.astype(np.float64), phi_c=phi_c).reshape(N, k)
        scale = max(np.max(np.abs(ref)), 1e-12)
        assert np.max(np.abs(out - ref)) <= 2e-5 * scale + 1e-6, (op, np.max(np.abs(out - ref)) / scale)
    assert lib.gbFvmApply(mesh, 3, fs, None, capi.vec(phi_c), out.ctypes.data) != 0     # tensor op on a scalar
    assert lib.gbFvmApply(mesh, 11, fs, None, capi.vec(phi_c), out.ctypes.data) != 0
    for f in (fs, fv, fp):
        lib.FvmFieldFree(f)
    lib.cuMeshFree(mesh)


@pytest.mark.parametrize("name", ["tet_6x3x2", "prism_6x3x2", "hex_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2"])
def test_operators_match_reference_operators(su2_paths, workdir, name):
    """gbFvmGradient and gbFvmApply against the reference's own operators and
    gradients (tests/golden/<mesh>_fvmops.npz, made by oracle/ref_fvmops.cu on
    a B200 from the same fields)."""
    from test_oracle_golden import FVMOP_SLOTS, VECTOR_OPS

    lib = capi.load()
    z = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}_fvmops.npz")
    fvm = str(workdir / f"{name}_refops.fvm")
    capi.check(lib.cuMeshFromSu2(su2_paths(name).encode(), fvm.encode()), "cuMeshFromSu2")
    mesh = lib.cuMeshFromFile(fvm.encode())
    n = int(lib.cuMeshGetVarSize(mesh))
    N = int(lib.cuMeshGetnCells(mesh))
    assert n == len(z["s"])
    fs, fv, fp = _field(lib, mesh, n, 1, b"s", z["s"]), _field(lib, mesh, n, 3, b"v", z["v"]), \
        _field(lib, mesh, n, 3, b"phi", z["phi"])
    ops = z["ops"].reshape(N, 35).astype(np.float64)
    for f, key, k in ((fs, "s", 1), (fv, "v", 3)):
        capi.check(lib.gbFvmGradient(mesh, f), "gbFvmGradient")
        lib.VarAllGpuToCpu(f)
        g, l = capi.field_gradients(f)
        ref_g = z[f"{key}.gradient"].reshape(n, -1)[:N]
        ref_l = z[f"{key}.limiter"].reshape(n, -1)[:N]
        assert np.max(np.abs(g[:N] - ref_g)) <= 2e-5 * np.max(np.abs(ref_g)), key
        assert np.max(np.abs(np.asarray(l[:N]).reshape(N, k) - ref_l)) <= 2e-4, key
    pc = tuple(float(c) for c in z["phi_const"])
    for op, (o, k) in FVMOP_SLOTS.items():
        u = fv if op in VECTOR_OPS else fs
        out = np.zeros((N, k), np.float32)
        capi.check(lib.gbFvmApply(mesh, op, u, fp, capi.vec(pc), out.ctypes.data), f"gbFvmApply {op}")
        ref = ops[:, o:o + k]
        scale = max(np.max(np.abs(ref)), 1e-12)
        assert np.max(np.abs(out - ref)) <= 1e-4 * scale, (op, np.max(np.abs(out - ref)) / scale)
    for f in (fs, fv, fp):
        lib.FvmFieldFree(f)
    lib.cuMeshFree(mesh)


SCALAR_TERMS = [(9, -1.0), (0, 0.3), (6, 0.5), (8, 2.0), (7, -0.25)]
VECTOR_TERMS = [(1, 1.0), (4, -1.0), (10, 0.7), (2, 0.2)]


@pytest.mark.parametrize("name", ["tet_6x3x2", "prism_6x3x2", "hex_6x3x2", "pyramid_6x3x2", "mixed_6x3x2", "layered_6x3x2"])
def test_operator_terms_compose_in_one_pass(su2_paths, workdir, name):
    """gbFvmApplyTerms (several operators summed in one pass over the faces,
    into a field on the device) against the same linear combination of the
    reference's own operators (tests/golden/<mesh>_fvmops.npz) and of
    gbFvmApply's single-operator results; and its argument checks."""
    from test_oracle_golden import FVMOP_SLOTS, VECTOR_OPS

    lib = capi.load()
    z = np.load(f"{cases.__file__.rsplit('/', 1)[0]}/{name}_fvmops.npz")
    fvm = str(workdir / f"{name}_terms.fvm")
    capi.check(lib.cuMeshFromSu2(su2_paths(name).encode(), fvm.encode()), "cuMeshFromSu2")
    mesh = lib.cuMeshFromFile(fvm.encode())
    n = int(lib.cuMeshGetVarSize(mesh))
    N = int(lib.cuMeshGetnCells(mesh))
    fs, fv, fp = _field(lib, mesh, n, 1, b"s", z["s"]), _field(lib, mesh, n, 3, b"v", z["v"]), \
        _field(lib, mesh, n, 3, b"phi", z["phi"])
    capi.check(lib.gbFvmGradient(mesh, fs), "gbFvmGradient")
    ops = z["ops"].reshape(N, 35).astype(np.float64)
    pc = capi.vec(tuple(float(c) for c in z["phi_const"]))
    out_s = lib.FvmFieldNew(4, n, b"r", 0)
    out_v = lib.FvmFieldNew(12, n, b"rv", 0)

    def terms(spec):
        arr = (capi.gbFvmTerm * len(spec))()
        for q, (op, coef) in enumerate(spec):
            arr[q] = capi.gbFvmTerm(op, coef, fv if op in VECTOR_OPS else fs, fp if op in (9, 10) else None, pc)
        return arr

    for spec, out, k in ((SCALAR_TERMS, out_s, 1), (VECTOR_TERMS, out_v, 3)):
        capi.check(lib.gbFvmApplyTerms(mesh, len(spec), terms(spec), out), "gbFvmApplyTerms")
        lib.VarGpuToCpu(out)
        got = capi.field_values(out)[:N].reshape(N, k)
        ref = np.zeros((N, k))
        single = np.zeros((N, k))
        scale = 0.0
        for op, coef in spec:
            o, w = FVMOP_SLOTS[op]
            assert w == k
            ref += coef * ops[:, o:o + k]
            scale += abs(coef) * np.max(np.abs(ops[:, o:o + k]))
            one = np.zeros((N, k), np.float32)
            u = fv if op in VECTOR_OPS else fs
            capi.check(lib.gbFvmApply(mesh, op, u, fp, pc, one.ctypes.data), f"gbFvmApply {op}")
            single += coef * one
        assert np.max(np.abs(got - ref)) <= 1e-4 * scale, np.max(np.abs(got - ref)) / scale
        assert np.max(np.abs(got - single)) <= 2e-6 * scale, np.max(np.abs(got - single)) / scale

    # argument checks: every one returns 1 with an error and launches nothing
    bad = [
        (terms([(0, 1.0), (1, 1.0)]), 2, out_s),        # a scalar and a vector operator
        (terms([(3, 1.0)]), 1, out_v),                   # tensor-valued
        (terms([(0, 1.0)]), 1, out_v),                   # scalar terms into a vector field
        (terms([(0, 1.0)]), 1, fs),                      # the output is an input
        (terms([(0, 1.0)]), 0, out_s),                   # no terms
        (terms([(0, 1.0)] * 9), 9, out_s),               # more than 8
        (terms([(11, 1.0)]), 1, out_s),                  # unknown operator
    ]
    no_phi = (capi.gbFvmTerm * 1)()
    no_phi[0] = capi.gbFvmTerm(9, 1.0, fs, None, pc)
    bad.append((no_phi, 1, out_s))                       # convection by a missing velocity field
    for arr, cnt, out in bad:
        assert lib.gbFvmApplyTerms(mesh, cnt, arr, out) == 1
        assert capi.last_error()
    for f in (fs, fv, fp, out_s, out_v):
        lib.FvmFieldFree(f)
    lib.cuMeshFree(mesh)


def test_field_init_and_boundary_conditions(su2_paths, workdir):
    """gbFieldInit, gbFieldBcFixed and gbFieldBcZeroGrad on a mesh of mixed
    elements, in the reference's cell order: every value set (gradients
    zeroed, limiters 1); a region's ghosts set to a value or to their
    interior cells' values, nothing else touched."""
    lib = capi.load()
    fvm = str(workdir / "mixed_fieldbc.fvm")
    capi.check(lib.cuMeshFromSu2(su2_paths("mixed_6x3x2").encode(), fvm.encode()), "cuMeshFromSu2")
    mesh = lib.cuMeshFromFile(fvm.encode())
    n = int(lib.cuMeshGetVarSize(mesh))
    N = int(lib.cuMeshGetnCells(mesh))
    rng = np.random.default_rng(7)
    s = rng.standard_normal(n).astype(np.float32)
    v = rng.standard_normal((n, 3)).astype(np.float32)
    fs, fv = _field(lib, mesh, n, 1, b"s", s), _field(lib, mesh, n, 3, b"v", v)
    capi.check(lib.gbFvmGradient(mesh, fs), "gbFvmGradient")          # the field now has gradients
    capi.check(lib.gbFieldInit(mesh, fs, capi.vec((2.5, 0.0, 0.0))), "gbFieldInit")
    lib.VarAllGpuToCpu(fs)
    assert np.all(capi.field_values(fs) == np.float32(2.5))
    g, l = capi.field_gradients(fs)
    assert np.all(g == 0.0) and np.all(np.asarray(l) == 1.0)
    capi.check(lib.gbFieldInit(mesh, fv, capi.vec((1.0, -2.0, 0.5))), "gbFieldInit")
    lib.VarGpuToCpu(fv)
    assert np.array_equal(capi.field_values(fv), np.tile(np.float32([1.0, -2.0, 0.5]), (n, 1)))

    gid, starts = capi.mesh_array(mesh, "ghost_cell_ids"), capi.mesh_array(mesh, "ghost_cell_starts")
    cfs, cc = capi.mesh_array(mesh, "cell_faces_starts"), capi.mesh_array(mesh, "cell_connects")
    for f, vals in ((fs, s), (fv, v)):
        capi.set_field_values(f, vals)
        capi.check(lib.gbVarCpuToGpu(mesh, f), "gbVarCpuToGpu")
    r_in, r_low = lib.cuMeshGetRegionId(mesh, b"inlet"), lib.cuMeshGetRegionId(mesh, b"lower")
    capi.check(lib.gbFieldBcFixed(mesh, fs, capi.vec((7.0, 0.0, 0.0)), r_in), "gbFieldBcFixed")
    capi.check(lib.gbFieldBcZeroGrad(mesh, fv, r_low), "gbFieldBcZeroGrad")
    capi.check(lib.gbFieldBcZeroGrad(mesh, fs, r_low), "gbFieldBcZeroGrad")
    lib.VarGpuToCpu(fs)
    lib.VarGpuToCpu(fv)
    want_s, want_v = s.copy(), v.copy()
    want_s[gid[starts[r_in]:starts[r_in + 1]]] = 7.0
    low = gid[starts[r_low]:starts[r_low + 1]]
    inner = cc[cfs[low]]
    want_s[low] = s[inner]
    want_v[low] = v[inner]
    assert np.array_equal(capi.field_values(fs), want_s)
    assert np.array_equal(capi.field_values(fv), want_v)
    assert lib.gbFieldBcFixed(mesh, fs, capi.vec((1.0, 0.0, 0.0)), 99) == 1 and capi.last_error()
    for f in (fs, fv):
        lib.FvmFieldFree(f)
    lib.cuMeshFree(mesh)


def test_scalar_transport_built_from_the_operators(su2_paths, workdir):
    """A model assembled from the generic API alone -- zero-gradient ghosts
    (gbFieldBcZeroGrad), the field's gradient (gbFvmGradient), the residual
    -conv(u) + nu lap(u) in one pass (gbFvmApplyTerms) and an explicit update
    (gbFieldAxpy) -- for 50 steps on the mixed-element channel, against the
    same steps of the FP64 operator restatement."""
    lib = capi.load()
    name = "mixed_6x3x2"
    em = cases.MESHES[name]()
    fvm = str(workdir / f"{name}_transport.fvm")
    capi.check(lib.cuMeshFromSu2(su2_paths(name).encode(), fvm.encode()), "cuMeshFromSu2")
    mesh = lib.cuMeshFromFile(fvm.encode())
    n = int(lib.cuMeshGetVarSize(mesh))
    n_regions = int(mesh.contents._cpu.contents.n_regions)
    base = mesh.contents._cpu.contents
    x = np.array([[base.cell_centers[i].x, base.cell_centers[i].y, base.cell_centers[i].z] for i in range(n)])
    u0 = (np.sin(2 * x[:, 0]) + x[:, 1] ** 2).astype(np.float32)
    fu = _field(lib, mesh, n, 1, b"u", u0)
    fr = lib.FvmFieldNew(4, n, b"r", 0)
    phi_c, nu, dt, steps = (0.8, 0.1, 0.05), 0.02, 0.01, 50
    terms = (capi.gbFvmTerm * 2)()
    terms[0] = capi.gbFvmTerm(7, -1.0, fu, None, capi.vec(phi_c))
    terms[1] = capi.gbFvmTerm(0, nu, fu, None, capi.vec(phi_c))
    for _ in range(steps):
        for r in range(n_regions):
            capi.check(lib.gbFieldBcZeroGrad(mesh, fu, r), "gbFieldBcZeroGrad")
        capi.check(lib.gbFvmGradient(mesh, fu), "gbFvmGradient")
        capi.check(lib.gbFvmApplyTerms(mesh, 2, terms, fr), "gbFvmApplyTerms")
        capi.check(lib.gbFieldAxpy(mesh, fu, dt, fr), "gbFieldAxpy")
    lib.VarGpuToCpu(fu)
    got = capi.field_values(fu)
    om = OpMesh(OracleMesh(em))
    N = om.N
    cfs = capi.mesh_array(mesh, "cell_faces_starts")
    cc = capi.mesh_array(mesh, "cell_connects")
    inner = cc[cfs[N:n]]                                 # each ghost's interior cell
    u = u0.astype(np.float64)
    for _ in range(steps):
        u[N:] = u[inner]
        g, lim = om.gradient(u)
        res = -om.apply(7, u, phi_c=phi_c) + nu * om.apply(0, u, grad=g, lim=lim)
        u[:N] += dt * res.reshape(N)
    u[N:] = u[inner]
    err = np.linalg.norm(got[:N] - u[:N]) / np.linalg.norm(u[:N])
    print(f"transport: relative L2 {err:.2e}")
    assert err < 1e-6                                    # measured 1.1e-7
    assert np.max(np.abs(got[:N] - u0[:N])) > 1e-2       # the field did evolve
    assert lib.gbFieldAxpy(mesh, fu, dt, fu) == 1
    lib.FvmFieldFree(fu)
    lib.FvmFieldFree(fr)
    lib.cuMeshFree(mesh)
