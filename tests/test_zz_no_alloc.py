"""gbReduceSumNoAlloc, the reduction entry point that allocates no device
memory (for callers that cannot call cudaMalloc: hosts that own all device
memory through their own pool, plugins whose device footprint is fixed after
setup).

It is checked through the C ABI against the entry point it mirrors,
FvmFieldReduceSum, on the same values, on two calls in a row (the scratch
array is shared by all calls and keeps the previous call's contents).  This
file is collected last so that a run stopping at the first failure has run
every other test first; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import cases
from graphite_b200 import capi
from graphite_b200.euler import EulerCase

pytestmark = pytest.mark.gpu

# the tolerance the parity tests use for residual sums (relative)
RTOL = 1e-5


def _reduce_no_alloc(lib, values_dev, n, out_dev, stream):
    rc = lib.gbReduceSumNoAlloc(ctypes.c_void_p(values_dev.data_ptr()), n, ctypes.c_void_p(out_dev.data_ptr()),
                                ctypes.c_void_p(stream))
    assert rc == 0, capi.last_error()


def test_no_alloc_sum_matches_field_reduce_sum(su2_paths):
    import torch

    lib = capi.load()
    torch.cuda.init()
    stream = torch.cuda.current_stream().cuda_stream
    lib.gbSetStream(ctypes.c_void_p(stream))
    rng = np.random.default_rng(7)
    with EulerCase(su2_paths("channel")) as c:
        n_all = c.n_cells + c.n_ghosts
        for call in range(2):                     # two calls in a row, different data
            vals = rng.uniform(0.1, 10.0, n_all).astype(np.float32) * (call + 1)
            capi.set_field_values(c.error, vals)
            capi.check(lib.gbVarCpuToGpu(c.mesh, c.error), "gbVarCpuToGpu")
            expected = float(lib.FvmFieldReduceSum(c.mesh, c.error))      # interior cells
            assert expected == expected, capi.last_error()
            dev = torch.from_numpy(vals[: c.n_cells]).cuda()
            out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
            _reduce_no_alloc(lib, dev, c.n_cells, out, stream)
            torch.cuda.synchronize()
            got = float(out.item())
            assert abs(got - expected) <= RTOL * abs(expected), (call, got, expected)
            exact = float(np.sum(vals[: c.n_cells].astype(np.float64)))
            assert abs(got - exact) <= 1e-12 * abs(exact)


def test_no_alloc_limits_and_reuse():
    """Large inputs use many partial sums; the last call's partials must not
    leak into the next call; sizes above the maximum are rejected."""
    import torch

    lib = capi.load()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    big = torch.rand(8_388_608, dtype=torch.float32, device="cuda")
    _reduce_no_alloc(lib, big, big.numel(), out, stream)
    torch.cuda.synchronize()
    ref = float(big.double().sum().item())
    assert abs(out.item() - ref) <= 1e-12 * ref
    small = torch.ones(3000, dtype=torch.float32, device="cuda")
    _reduce_no_alloc(lib, small, small.numel(), out, stream)
    torch.cuda.synchronize()
    assert out.item() == 3000.0
    _reduce_no_alloc(lib, small, 0, out, stream)
    torch.cuda.synchronize()
    assert out.item() == 0.0
    rc = lib.gbReduceSumNoAlloc(ctypes.c_void_p(big.data_ptr()), 8_388_609, ctypes.c_void_p(out.data_ptr()),
                                ctypes.c_void_p(stream))
    assert rc != 0 and "exceed the maximum" in capi.last_error()
    # a host pointer for the result is rejected before any launch
    host = np.zeros(1, np.float64)
    rc = lib.gbReduceSumNoAlloc(ctypes.c_void_p(small.data_ptr()), small.numel(),
                                ctypes.c_void_p(host.ctypes.data), ctypes.c_void_p(stream))
    assert rc != 0 and "device" in capi.last_error() and host[0] == 0.0
    _reduce_no_alloc(lib, small, small.numel(), out, stream)     # and the next call works
    torch.cuda.synchronize()
    assert out.item() == 3000.0
