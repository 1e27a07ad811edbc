"""The allocation-free Pareto filter (pmdd_pareto_filter_noalloc).

Some callers cannot allocate device memory: a library running beside a framework
allocator that has already reserved the device, or a service that forbids cudaMalloc /
cudaFree after start-up because those calls can synchronise the device.  They hand in
their own input and output device buffers; the filter's scratch comes from a fixed
device array in the library.  This checks, through the C ABI, that two calls in a row
(the second reusing the array the first left behind) return exactly the point sets of
the allocating entry point pmdd_pareto_filter and of the oracle's keep rule, that the
largest allowed call (131072 points of 8 objectives) is exact, that a warmed-up call
takes no device memory, and that the size limit is enforced.  The file is named so that
pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from pmdd_b200 import _native

pytestmark = pytest.mark.gpu

MAX_POINTS = 1 << 17


def noalloc_filter(points):
    import torch

    pts = np.ascontiguousarray(points, dtype=np.int32)
    n, d = pts.shape
    d_in = torch.from_numpy(pts).cuda()
    d_out = torch.empty_like(d_in)
    n_out = ctypes.c_int64(-1)
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _native.gpu_lib().pmdd_pareto_filter_noalloc(
        ctypes.c_void_p(d_in.data_ptr()), n, d, ctypes.c_void_p(d_out.data_ptr()), ctypes.byref(n_out),
        ctypes.c_void_p(stream), err, len(err))
    return rc, d_out[: max(n_out.value, 0)].cpu().numpy(), err.value.decode()


def as_set(a):
    a = np.asarray(a, dtype=np.int64)
    return a[np.lexsort(a.T[::-1])] if len(a) > 1 else a


def test_noalloc_matches_allocating_filter_and_oracle_twice():
    rng = np.random.default_rng(2024)
    first = rng.integers(-500, 500, size=(60_000, 3)).astype(np.int32)
    first[10_000:10_100] = first[:100]  # duplicates must collapse to one copy
    second = rng.integers(-30, 30, size=(7_000, 5)).astype(np.int32)
    for pts in (first, second):
        rc, got, err = noalloc_filter(pts)
        assert rc == 0, err
        want = P.pareto_filter(pts)
        assert np.array_equal(as_set(got), as_set(want))
        assert np.array_equal(as_set(got), as_set(pts[oracle.nd_keep(pts)]))


def test_noalloc_largest_call_is_exact_and_allocates_nothing():
    import torch

    rng = np.random.default_rng(77)
    # 131072 points of 8 objectives: the whole scratch array, count word included
    pts = rng.integers(0, 40, size=(MAX_POINTS, 8)).astype(np.int32)
    pts[: MAX_POINTS // 2, 0] = 0  # half the set dominated early, many duplicates
    d_in = torch.from_numpy(pts).cuda()
    d_out = torch.empty_like(d_in)
    lib = _native.gpu_lib()
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        n_out = ctypes.c_int64(-1)
        err = ctypes.create_string_buffer(256)
        rc = lib.pmdd_pareto_filter_noalloc(ctypes.c_void_p(d_in.data_ptr()), MAX_POINTS, 8,
                                            ctypes.c_void_p(d_out.data_ptr()), ctypes.byref(n_out),
                                            ctypes.c_void_p(stream), err, len(err))
        assert rc == 0, err.value
        return d_out[: n_out.value].cpu().numpy()

    got1 = call()  # warm-up: the one-time address look-up and module load
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    got2 = call()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    want = P.pareto_filter(pts)
    assert np.array_equal(as_set(got1), as_set(want))
    assert np.array_equal(as_set(got2), as_set(want))


def test_noalloc_rejects_oversized_sets():
    import torch

    too_many = MAX_POINTS + 1
    d_in = torch.zeros((too_many, 2), dtype=torch.int32, device="cuda")
    d_out = torch.empty_like(d_in)
    n_out = ctypes.c_int64(-1)
    err = ctypes.create_string_buffer(256)
    rc = _native.gpu_lib().pmdd_pareto_filter_noalloc(
        ctypes.c_void_p(d_in.data_ptr()), too_many, 2, ctypes.c_void_p(d_out.data_ptr()), ctypes.byref(n_out),
        None, err, len(err))
    assert rc == 9 and b"131072" in err.value
