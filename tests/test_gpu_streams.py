"""Stream ordering of device-resident inputs: the library runs on its own non-blocking stream and
must read buffers that the caller's queued work is still writing only after that work ends.
Each test queues a GPU sleep (a bounded spin of a few ms) and then the write of the input on the
caller's stream, and calls the library at once, with no synchronisation in between."""
import numpy as np
import pytest

from test_gpu_parity import as_csr, to_dev

pytestmark = pytest.mark.gpu

SLEEP_CYCLES = 20_000_000   # about 10 ms at the B200's clock


def _late_copy(torch, dst, src):
    torch.cuda._sleep(SLEEP_CYCLES)
    dst.copy_(src)


@pytest.mark.parametrize("side_stream", [False, True])
def test_solve_waits_for_the_callers_rhs(bx, cuda, side_stream):
    import torch
    A = as_csr(bx, ("lap27", (24, 24, 24)))
    b = A @ np.random.default_rng(11).uniform(-1, 1, A.shape[0])
    h = bx.prec_setup(A.indptr, A.indices, A.data, bx.params_default(solver="FCG", rtol=1e-10, dispnorm=0))
    x_ref, _ = h.solve(b)
    src = torch.from_numpy(b).to(cuda)
    bd = torch.zeros_like(src)
    xd = torch.full_like(src, 1e300)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    with torch.cuda.stream(stream):
        _late_copy(torch, bd, src)
        xd.zero_()
        h.solve(bd, x0=xd)
    torch.cuda.synchronize()
    assert np.array_equal(xd.cpu().numpy(), x_ref)


def test_setup_waits_for_the_callers_values(bx, cuda):
    import torch
    A = as_csr(bx, ("diff", (16, 2)))
    b = np.ones(A.shape[0])
    p = bx.params_default(solver="FCG", rtol=1e-10, dispnorm=0)
    x_ref, i_ref = bx.prec_setup(A.indptr, A.indices, A.data, p).solve(b)
    row, col, val = to_dev(torch, A, cuda)
    late = torch.zeros_like(val)
    torch.cuda.synchronize()
    _late_copy(torch, late, val)
    h = bx.Hierarchy(row, col, late, p)
    x, info = h.solve(b)
    assert info["niter"] == i_ref["niter"]
    assert np.array_equal(x, x_ref)


def test_prec_apply_and_multi_wait_for_the_caller(bx, cuda):
    import torch
    A = as_csr(bx, ("lap7", (20, 20, 20)))
    n = A.shape[0]
    rng = np.random.default_rng(12)
    r = rng.uniform(-1, 1, n)
    B = rng.uniform(-1, 1, (n, 4))
    h = bx.prec_setup(A.indptr, A.indices, A.data, bx.params_default(solver="FCG", rtol=1e-9, dispnorm=0))
    v_ref = h.prec_apply(r)
    X_ref, _ = h.solve_multi(B)
    rs, Bs = torch.from_numpy(r).to(cuda), torch.from_numpy(B).to(cuda)
    rd, Bd = torch.zeros_like(rs), torch.zeros_like(Bs)
    torch.cuda.synchronize()
    _late_copy(torch, rd, rs)
    v = h.prec_apply(rd)
    _late_copy(torch, Bd, Bs)
    X, _ = h.solve_multi(Bd)
    assert np.array_equal(v.cpu().numpy(), v_ref)
    assert np.array_equal(X.cpu().numpy(), X_ref)
