"""The allocation-free edge-weights entry point, bcmgx_edge_weights_noalloc.

It exists for callers that cannot let the library allocate device memory (a framework whose
caching allocator already holds the GPU's memory, or a fixed device-memory budget). Its
results must equal those of the allocating entry point, bcmgx_edge_weights, bit for bit (the
same kernels run on the same data), on consecutive calls that reuse the shared static scratch.
This file is collected last so that a run that stops at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 65536
MAX_NNZ = 2097152


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(bx, r, c, v, w, stream):
    import torch
    W = torch.empty_like(v)
    mn = C.c_double()
    rc = bx.lib().bcmgx_edge_weights_noalloc(int(r.numel()) - 1, int(c.numel()), _ptr(r), _ptr(c), _ptr(v), _ptr(w),
                                             _ptr(W), C.byref(mn), C.c_void_p(stream.cuda_stream))
    return rc, W, mn.value


def test_noalloc_matches_allocating_entry_point(bx, cuda):
    import torch
    stream = torch.cuda.current_stream(cuda)
    cases = [(27, (30, 30, 30), 11), (7, (40, 30, 20), 12), (27, (30, 30, 30), 13)]
    for st, dims, seed in cases:   # consecutive calls: the second and third reuse the scratch
        row, col, val = bx.laplacian_3d(st, *dims)
        n = row.size - 1
        assert n <= MAX_ROWS and col.size <= MAX_NNZ
        rng = np.random.default_rng(seed)
        val = val * rng.uniform(0.5, 1.5, val.size)   # non-uniform entries, same pattern
        d = [torch.from_numpy(a).to(cuda) for a in (row, col, val)]
        w = torch.from_numpy(rng.uniform(0.5, 2.0, n)).to(cuda)
        W_ref, mn_ref = bx.edge_weights(d[0], d[1], d[2], w, stream=stream)
        rc, W, mn = _noalloc(bx, d[0], d[1], d[2], w, stream)
        assert rc == 0, bx._lib.last_error()
        torch.cuda.synchronize()
        assert mn == mn_ref
        assert torch.equal(W, W_ref)


def test_noalloc_rejects_oversized_input(bx, cuda):
    import torch
    stream = torch.cuda.current_stream(cuda)
    one = torch.zeros(1, dtype=torch.int32, device=cuda)
    onef = torch.zeros(1, dtype=torch.float64, device=cuda)
    L = bx.lib()
    for n, nnz in [(MAX_ROWS + 1, 10), (10, MAX_NNZ + 1)]:
        mn = C.c_double()
        rc = L.bcmgx_edge_weights_noalloc(n, nnz, _ptr(one), _ptr(one), _ptr(onef), _ptr(onef), _ptr(onef),
                                          C.byref(mn), C.c_void_p(stream.cuda_stream))
        assert rc == -1
        assert "too large for the allocation-free entry point" in bx._lib.last_error()


def test_noalloc_takes_no_device_memory(bx, cuda):
    """After the first call (which commits the static scratch), repeated calls leave the device's
    free memory and the default memory pool's usage unchanged: nothing is allocated."""
    import torch
    from cuda.bindings import runtime as rt
    stream = torch.cuda.current_stream(cuda)
    row, col, val = bx.laplacian_3d(27, 20, 20, 20)
    n = row.size - 1
    d = [torch.from_numpy(a).to(cuda) for a in (row, col, val)]
    w = torch.ones(n, dtype=torch.float64, device=cuda)
    W = torch.empty_like(d[2])
    mn = C.c_double()
    L = bx.lib()

    def call():
        rc = L.bcmgx_edge_weights_noalloc(n, int(d[1].numel()), _ptr(d[0]), _ptr(d[1]), _ptr(d[2]), _ptr(w), _ptr(W),
                                          C.byref(mn), C.c_void_p(stream.cuda_stream))
        assert rc == 0, bx._lib.last_error()

    def pool_used():
        err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
        assert err == rt.cudaError_t.cudaSuccess
        err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
        assert err == rt.cudaError_t.cudaSuccess
        return int(v)

    call()
    torch.cuda.synchronize()
    free0, used0 = torch.cuda.mem_get_info(cuda)[0], pool_used()
    for _ in range(5):
        call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free0
    assert pool_used() == used0
