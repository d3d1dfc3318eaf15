"""weno_sb_checksum_noalloc: the checksum entry point that allocates nothing.

Some callers cannot allocate device memory -- Fortran drivers whose device
heap belongs to the OpenMP/OpenACC offload runtime (as in MFC), and time-step
loops that must avoid cudaMalloc/cudaFree because those may synchronise the
device.  This entry point keeps its partial sums in a static device array
inside the library.  Here it is called through the C ABI, twice in a row, and
its sums are compared with the allocating entry point weno_sb_checksum_dev
(caller-provided scratch) at the tolerance of the other GPU tests.  This file
is collected last so that a failure here stops a -x run only after every
other test has run; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _reference_sums(L, arrays, dtype):
    import torch
    lib = L.lib()
    out = []
    for t in arrays:
        scratch = torch.empty(int(lib.weno_sb_checksum_scratch_bytes(t.numel())) // 8 + 1,
                              dtype=torch.float64, device="cuda")
        res = torch.empty(1, dtype=torch.float64, device="cuda")
        L.check(lib.weno_sb_checksum_dev(dtype, t.data_ptr(), t.numel(), scratch.data_ptr(),
                                         res.data_ptr(), None))
        out.append(float(res.item()))
    return out


def _noalloc_sums(L, arrays, dtype, stream=None):
    import torch
    lib = L.lib()
    k = len(arrays)
    ptrs = (ctypes.c_void_p * k)(*[t.data_ptr() for t in arrays])
    ns = (ctypes.c_int64 * k)(*[t.numel() for t in arrays])
    res = torch.full((k,), float("nan"), dtype=torch.float64, device="cuda")
    if stream is not None:
        # the inputs and the result buffer were written on the current stream
        stream.wait_stream(torch.cuda.current_stream())
    L.check(lib.weno_sb_checksum_noalloc(dtype, ptrs, ns, k, res.data_ptr(),
                                         None if stream is None else stream.cuda_stream))
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return res.cpu().tolist()


@pytest.mark.parametrize("dtype_name", ["fp64", "fp32"])
def test_noalloc_checksum_matches_allocating_entry(dtype_name):
    import torch
    from wenostandalone_b200 import _lib as L
    tdt = torch.float64 if dtype_name == "fp64" else torch.float32
    dtype = L.FP64 if dtype_name == "fp64" else L.FP32
    g = torch.Generator(device="cuda").manual_seed(5)
    sizes = [1, 1000, 1_000_003, 3_000_000, 0, 17]
    arrays = [torch.randn(s, generator=g, device="cuda", dtype=torch.float64).to(tdt) for s in sizes]
    ref = _reference_sums(L, arrays, dtype)
    for _ in range(2):   # two calls in a row share (and reuse) the static scratch
        got = _noalloc_sums(L, arrays, dtype)
        for a, (x, y) in enumerate(zip(got, ref)):
            assert abs(x - y) <= TOL * max(abs(y), 1e-300), (a, x, y)
    # a second, different batch after the first: no stale partials leak in
    arrays2 = [a.flip(0) * 2 for a in arrays[:3]]
    ref2 = _reference_sums(L, arrays2, dtype)
    got2 = _noalloc_sums(L, arrays2, dtype)
    for x, y in zip(got2, ref2):
        assert abs(x - y) <= TOL * max(abs(y), 1e-300)


def test_noalloc_rejects_more_arrays_than_the_scratch_holds():
    import torch
    from wenostandalone_b200 import _lib as L
    t = torch.ones(10, dtype=torch.float64, device="cuda")
    k = 17
    ptrs = (ctypes.c_void_p * k)(*[t.data_ptr()] * k)
    ns = (ctypes.c_int64 * k)(*[10] * k)
    res = torch.empty(k, dtype=torch.float64, device="cuda")
    rc = L.lib().weno_sb_checksum_noalloc(L.FP64, ptrs, ns, k, res.data_ptr(), None)
    assert rc == L.ERR_ARG
    assert "at most 16" in L.last_error()


def test_noalloc_on_a_non_default_stream():
    """Launched on a caller's stream, the sums are there once that stream
    has been synchronised."""
    import torch
    from wenostandalone_b200 import _lib as L
    g = torch.Generator(device="cuda").manual_seed(9)
    arrays = [torch.randn(s, generator=g, device="cuda", dtype=torch.float64) for s in (5, 777_777, 2_000_001)]
    ref = _reference_sums(L, arrays, L.FP64)
    s = torch.cuda.Stream()
    for _ in range(2):
        got = _noalloc_sums(L, arrays, L.FP64, stream=s)
        for x, y in zip(got, ref):
            assert abs(x - y) <= TOL * max(abs(y), 1e-300), (x, y)


def test_noalloc_rejects_bad_arguments():
    import torch
    from wenostandalone_b200 import _lib as L
    lib = L.lib()
    t = torch.ones(10, dtype=torch.float64, device="cuda")
    res = torch.empty(2, dtype=torch.float64, device="cuda")

    def call(ptr_list, n_list, count):
        k = max(len(ptr_list), 1)
        ptrs = (ctypes.c_void_p * k)(*ptr_list)
        ns = (ctypes.c_int64 * k)(*n_list)
        return lib.weno_sb_checksum_noalloc(L.FP64, ptrs, ns, count, res.data_ptr(), None)

    assert call([t.data_ptr()], [10], 0) == L.ERR_ARG            # count = 0
    assert call([t.data_ptr()], [-1], 1) == L.ERR_ARG            # negative n
    assert "negative" in L.last_error()
    assert call([None, t.data_ptr()], [10, 10], 2) == L.ERR_ARG  # NULL array with n > 0
    assert "NULL" in L.last_error()
    assert call([None], [0], 1) == L.OK                          # NULL is fine for an empty array
    torch.cuda.synchronize()


def test_noalloc_allocates_no_device_memory():
    """After a first call (which looks up the static array's address), later
    calls change neither the device's free memory, nor the reserve of the
    stream-ordered allocator's default pool, nor torch's caching allocator."""
    import torch
    from cuda.bindings import runtime as rt
    from wenostandalone_b200 import _lib as L
    arrays = [torch.rand(1 << 20, device="cuda", dtype=torch.float64) for _ in range(16)]
    _noalloc_sums(L, arrays, L.FP64)          # first call on this device
    torch.cuda.synchronize()

    def state():
        err, free, _ = rt.cudaMemGetInfo()
        assert err == rt.cudaError_t.cudaSuccess
        err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
        assert err == rt.cudaError_t.cudaSuccess
        vals = []
        for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent,
                     rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh):
            err, v = rt.cudaMemPoolGetAttribute(pool, attr)
            assert err == rt.cudaError_t.cudaSuccess
            vals.append(int(v))
        return free, vals, torch.cuda.memory_allocated(), torch.cuda.memory_reserved()

    lib = L.lib()
    k = len(arrays)
    ptrs = (ctypes.c_void_p * k)(*[t.data_ptr() for t in arrays])
    ns = (ctypes.c_int64 * k)(*[t.numel() for t in arrays])
    res = torch.empty(k, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    before = state()
    for _ in range(20):
        L.check(lib.weno_sb_checksum_noalloc(L.FP64, ptrs, ns, k, res.data_ptr(), None))
    torch.cuda.synchronize()
    after = state()
    assert before == after, (before, after)
