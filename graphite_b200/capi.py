"""ctypes binding of libgraphite_b200.so (the C ABI in include/graphite_b200.h).

This is the binding an FFI user of the library writes; the tests and the
benchmark go through it, so every call they make crosses the C ABI.  Loading
fails loudly if the shared library has not been built (``make -C
graphite_b200`` or ``__graft_entry__.build()``): there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgraphite_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "graphite_b200.h")


class gb_vector(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class gb_tensor(C.Structure):
    _fields_ = [("u", gb_vector), ("v", gb_vector), ("w", gb_vector)]


class cuMeshBase(C.Structure):
    _fields_ = [("type", C.c_int), ("allocated", C.c_int),
                ("n_cells", C.c_size_t), ("n_faces", C.c_size_t), ("n_nodes", C.c_size_t),
                ("n_ghosts", C.c_size_t), ("n_regions", C.c_size_t),
                ("cell_faces", C.POINTER(C.c_uint)), ("cell_connects", C.POINTER(C.c_uint)),
                ("cell_faces_starts", C.POINTER(C.c_uint)), ("cell_volumes", C.POINTER(C.c_float)),
                ("cell_centers", C.POINTER(gb_vector)), ("cell_matrices", C.POINTER(gb_tensor)),
                ("face_nodes", C.POINTER(C.c_uint)), ("face_nodes_starts", C.POINTER(C.c_uint)),
                ("face_areas", C.POINTER(C.c_float)), ("face_centers", C.POINTER(gb_vector)),
                ("face_normals", C.POINTER(gb_vector)), ("nodes", C.POINTER(gb_vector)),
                ("ghost_cell_ids", C.POINTER(C.c_uint)), ("ghost_cell_starts", C.POINTER(C.c_uint))]


class cuMesh(C.Structure):
    _fields_ = [("_cpu", C.POINTER(cuMeshBase)), ("_hgpu", C.POINTER(cuMeshBase)), ("_gpu", C.POINTER(cuMeshBase)),
                ("region_names", C.POINTER(C.c_char_p)), ("region_names_alloc", C.c_size_t),
                ("region_names_size", C.c_size_t), ("impl", C.c_void_p)]


class FvmFieldBase(C.Structure):
    _fields_ = [("elem_size", C.c_size_t), ("size", C.c_size_t), ("value", C.c_void_p),
                ("gradient", C.c_void_p), ("limiter", C.c_void_p)]


class FvmField(C.Structure):
    _fields_ = [("_cpu", C.POINTER(FvmFieldBase)), ("_hgpu", C.POINTER(FvmFieldBase)),
                ("_gpu", C.POINTER(FvmFieldBase)), ("name", C.c_char_p), ("impl", C.c_void_p)]


class gbFvmTerm(C.Structure):
    _fields_ = [("op", C.c_int), ("coef", C.c_float), ("u", C.POINTER(FvmField)), ("phi", C.POINTER(FvmField)),
                ("phi_const", gb_vector)]


class gbBc(C.Structure):
    _fields_ = [("type", C.c_int), ("region_id", C.c_uint), ("mach", gb_vector), ("pressure", C.c_float),
                ("temperature", C.c_float)]


class gbBatchInstance(C.Structure):
    _fields_ = [("mesh", C.c_int), ("n_bc", C.c_int), ("bcs", C.POINTER(gbBc))]


MeshP = C.POINTER(cuMesh)
FieldP = C.POINTER(FvmField)

_PROTOS = {
    "cuMeshFromSu2": (C.c_int, [C.c_char_p, C.c_char_p]),
    "cuMeshFromFile": (MeshP, [C.c_char_p]),
    "cuMeshFree": (None, [MeshP]),
    "cuMeshGetVarSize": (C.c_size_t, [MeshP]),
    "cuMeshGetnCells": (C.c_size_t, [MeshP]),
    "cuMeshGetnGhosts": (C.c_size_t, [MeshP]),
    "cuMeshGetnCellsAndGhosts": (C.c_size_t, [MeshP]),
    "cuMeshGetnRegionCells": (C.c_size_t, [MeshP, C.c_uint]),
    "cuMeshGetRegionId": (C.c_uint, [MeshP, C.c_char_p]),
    "cuMeshPrintInfo": (None, [MeshP]),
    "FvmFieldNew": (FieldP, [C.c_size_t, C.c_size_t, C.c_char_p, C.c_int]),
    "FvmFieldFree": (None, [FieldP]),
    "FvmFieldGetType": (C.c_int, [FieldP]),
    "FvmFieldValueIndex": (C.c_void_p, [FieldP, C.c_size_t]),
    "VarGpuToCpu": (None, [FieldP]),
    "VarAllGpuToCpu": (None, [FieldP]),
    "FvmEulerInit": (C.c_int, [MeshP, FieldP, FieldP, FieldP, gb_vector, C.c_float, C.c_float]),
    "FvmEulerSlipBc": (C.c_int, [MeshP, FieldP, FieldP, FieldP, C.c_char_p]),
    "FvmEulerInletOutletBc": (C.c_int, [MeshP, FieldP, FieldP, FieldP, gb_vector, C.c_float, C.c_float, C.c_char_p]),
    "FvmEulerStepPrepare": (C.c_int, [MeshP, FieldP, FieldP, FieldP]),
    "FvmEulerStep": (C.c_int, [MeshP, FieldP, FieldP, FieldP, C.c_float, C.c_char_p, FieldP, FieldP]),
    "FvmFieldReduceSum": (C.c_float, [MeshP, FieldP]),
    "gbGetLastError": (C.c_char_p, []),
    "gbSetStream": (C.c_int, [C.c_void_p]),
    "gbGetStream": (C.c_void_p, []),
    "gbVarCpuToGpu": (C.c_int, [MeshP, FieldP]),
    "gbSetReferenceMomentumReconstruction": (C.c_int, [C.c_int]),
    "gbSetRenumbering": (C.c_int, [C.c_int]),
    "gbMeshFromSu2": (MeshP, [C.c_char_p]),
    "gbEulerRun": (C.c_int64, [MeshP, FieldP, FieldP, FieldP, FieldP, C.c_float, C.c_int64, C.POINTER(gbBc), C.c_int,
                               C.c_double, C.c_int, C.POINTER(C.c_double)]),
    "gbEulerRunDensityResidual": (C.c_int64, [MeshP, FieldP, FieldP, FieldP, FieldP, C.c_float, C.c_int64,
                                              C.POINTER(gbBc), C.c_int, C.c_double, C.c_int,
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "gbKernelLaunchCount": (C.c_uint64, []),
    "gbReduceSumNoAlloc": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "gbBatchCreate": (C.c_void_p, [C.c_int, C.POINTER(MeshP), C.c_int, C.POINTER(gbBatchInstance)]),
    "gbBatchSetResidualScale": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "gbFvmGradient": (C.c_int, [MeshP, FieldP]),
    "gbFvmApply": (C.c_int, [MeshP, C.c_int, FieldP, FieldP, gb_vector, C.c_void_p]),
    "gbFvmApplyTerms": (C.c_int, [MeshP, C.c_int, C.POINTER(gbFvmTerm), FieldP]),
    "gbFieldInit": (C.c_int, [MeshP, FieldP, gb_vector]),
    "gbFieldBcFixed": (C.c_int, [MeshP, FieldP, gb_vector, C.c_uint]),
    "gbFieldBcZeroGrad": (C.c_int, [MeshP, FieldP, C.c_uint]),
    "gbFieldAxpy": (C.c_int, [MeshP, FieldP, C.c_float, FieldP]),
    "gbRenderRegionScalar": (C.c_int64, [MeshP, C.c_uint, FieldP, C.c_float, C.c_float, C.c_void_p, C.c_int64]),
    "FieldsWriteVtu": (C.c_int, [C.c_char_p, MeshP, C.POINTER(FieldP), C.c_size_t]),
    "gbFieldsWriteVtuBinary": (C.c_int, [C.c_char_p, MeshP, C.POINTER(FieldP), C.c_size_t]),
    "gbNSISetConstants": (C.c_int, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int]),
    "FvmNSIInit": (C.c_int, [MeshP, FieldP, FieldP, gb_vector, C.c_float]),
    "FvmNSISlipBc": (C.c_int, [MeshP, FieldP, FieldP, C.c_char_p]),
    "FvmNSIWallBc": (C.c_int, [MeshP, FieldP, FieldP, C.c_char_p]),
    "FvmNSIInletOutletBc": (C.c_int, [MeshP, FieldP, FieldP, gb_vector, C.c_float, C.c_char_p]),
    "FvmNSIStepPrepare": (C.c_int, [MeshP, FieldP, FieldP]),
    "FvmNSIStep": (C.c_int, [MeshP, FieldP, FieldP, C.c_float, C.c_char_p, FieldP, FieldP]),
    "gbNSIRun": (C.c_int64, [MeshP, FieldP, FieldP, FieldP, C.c_float, C.c_int64, C.POINTER(gbBc), C.c_int,
                             C.c_double, C.c_int, C.c_void_p]),
    "gbNSIWallForce": (C.c_int, [MeshP, FieldP, FieldP, C.c_uint, C.c_void_p]),
    "gbWallForce": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint, C.c_void_p]),
    "gbBatchWallForce": (C.c_int, [C.c_void_p, C.c_int, C.c_uint, C.c_void_p]),
    "gbWarmStartCreate": (C.c_void_p, [C.c_void_p, C.c_uint, C.c_uint64]),
    "gbWarmStartFree": (None, [C.c_void_p]),
    "gbWarmStartParamCount": (C.c_int64, []),
    "gbWarmStartGetWeights": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gbWarmStartSetWeights": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gbWarmStartGetScales": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gbWarmStartSetScales": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gbWarmStartGetFeatures": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gbWarmStartAddBatchField": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, gb_vector, C.c_float, C.c_float]),
    "gbWarmStartAddField": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, gb_vector, C.c_float,
                                      C.c_float]),
    "gbWarmStartFieldCount": (C.c_int64, [C.c_void_p]),
    "gbWarmStartTrain": (C.c_int64, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int64]),
    "gbWarmStartPredictBatch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, gb_vector, C.c_float, C.c_float]),
    "gbWarmStartPredict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, gb_vector, C.c_float,
                                     C.c_float]),
    "gbWarmStartGradient": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gbWarmStartForward": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "gbWarmStartSetWaitLimit": (C.c_int, [C.c_void_p, C.c_longlong]),
    "gbBatchInjectBarrierFault": (C.c_int, [C.c_void_p]),
    "gbApplyBoundaryConditions": (C.c_int, [MeshP]),
    "gbBatchFree": (None, [C.c_void_p]),
    "gbBatchInitUniform": (C.c_int, [C.c_void_p, C.c_int, gb_vector, C.c_float, C.c_float]),
    "gbBatchSetState": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gbBatchGetState": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gbBatchSetTuning": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gbBatchGetTuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "gbBatchAutotune": (C.c_int, [C.c_void_p, C.c_float, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "gbBatchRun": (C.c_int64, [C.c_void_p, C.c_float, C.c_int64, C.c_double, C.c_int, C.POINTER(C.c_int64),
                               C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
}

_lib = None


def load():
    """Load the library (raises if it is missing: the CUDA path has no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {HERE}` (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def header_functions() -> List[str]:
    """Names of the functions include/graphite_b200.h declares for the library
    to export (its static inline helpers are defined in the header itself)."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^(?!static\b)[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


class GraphiteError(RuntimeError):
    pass


def last_error() -> str:
    return load().gbGetLastError().decode()


def check(rc, what="call"):
    if rc != 0:
        raise GraphiteError(f"{what} failed: {last_error()}")


def vec(x, y=None, z=None) -> gb_vector:
    if y is None:
        x, y, z = x
    return gb_vector(float(x), float(y), float(z))


def field_values(f: FieldP) -> np.ndarray:
    """Host mirror of a field's values (after VarGpuToCpu), reference order."""
    base = f.contents._cpu.contents
    comps = base.elem_size // 4
    arr = np.ctypeslib.as_array(C.cast(base.value, C.POINTER(C.c_float)), shape=(base.size * comps,))
    return arr.reshape(base.size, comps).copy() if comps > 1 else arr.copy()


def field_gradients(f: FieldP):
    """(gradient, limiter) host mirrors after VarAllGpuToCpu, reference layout."""
    base = f.contents._cpu.contents
    comps = base.elem_size // 4
    g = np.ctypeslib.as_array(C.cast(base.gradient, C.POINTER(C.c_float)), shape=(base.size * comps * 3,)).copy()
    lim = np.ctypeslib.as_array(C.cast(base.limiter, C.POINTER(C.c_float)), shape=(base.size * comps,)).copy()
    if comps == 1:
        return g.reshape(base.size, 3), lim
    return g.reshape(base.size, 9), lim.reshape(base.size, 3)


def set_field_values(f: FieldP, values: np.ndarray) -> None:
    base = f.contents._cpu.contents
    comps = base.elem_size // 4
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    assert v.size == base.size * comps
    C.memmove(base.value, v.ctypes.data, v.nbytes)


def mesh_array(mesh: MeshP, name: str) -> np.ndarray:
    """Copy of a host-mirror mesh array (reference layout and order)."""
    b = mesh.contents._cpu.contents
    N, G, F = b.n_cells, b.n_ghosts, b.n_faces
    NG = N + G
    sizes = {"cell_faces_starts": (NG + 1, 1, C.c_uint), "face_nodes_starts": (F + 1, 1, C.c_uint),
             "cell_volumes": (NG, 1, C.c_float), "cell_centers": (NG, 3, C.c_float),
             "cell_matrices": (N, 9, C.c_float), "face_areas": (F, 1, C.c_float), "face_centers": (F, 3, C.c_float),
             "face_normals": (F, 3, C.c_float), "nodes": (b.n_nodes, 3, C.c_float),
             "ghost_cell_ids": (G, 1, C.c_uint), "ghost_cell_starts": (b.n_regions + 1, 1, C.c_uint)}
    if name in ("cell_faces", "cell_connects"):
        n = b.cell_faces_starts[NG]
        ptr, k, ct = getattr(b, name), 1, C.c_uint
    elif name == "face_nodes":
        n = b.face_nodes_starts[F]
        ptr, k, ct = b.face_nodes, 1, C.c_uint
    else:
        n, k, ct = sizes[name]
        ptr = getattr(b, name)
    a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n * k,)).copy()
    return a.reshape(n, k) if k > 1 else a
