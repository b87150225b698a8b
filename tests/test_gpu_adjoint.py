"""Differentiated solve: the adjoint path (bcmgx_solve_adjoint) and its torch.autograd binding,
checked against exact dense gradients, FP64 central finite differences, and the gradient of a
fresh plain-FP64 solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(bx, n, seed):
    from bootcmatchgx_b200 import problems
    theta = problems.gaussian_random_field((n, n, n), length=3.0, sigma=1.0, seed=seed)
    return theta


def test_adjoint_matches_dense_gradient(bx, cuda):
    """Tiny system: dL/db = A^{-1} g and dL/dA_ij = -lambda_i x_j against dense numpy."""
    import torch
    row, col, val = bx.laplacian_3d(7, 6, 5, 4)
    n = row.size - 1
    rng = np.random.default_rng(0)
    val = val * (1 + 0.1 * rng.random(val.size))
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    A = (A + A.T) * 0.5 + sp.diags(np.full(n, 1.0))
    A.sort_indices()
    b = rng.uniform(-1, 1, n)
    g = rng.uniform(-1, 1, n)
    h = bx.prec_setup(A.indptr, A.indices, A.data, bx.params_default(solver="FCG", preconditioner="BCMG",
                                                                    rtol=1e-13, dispnorm=0))
    x, _ = h.solve(b)
    lam, dA, _ = h.adjoint(g, x)
    D = A.toarray()
    lam_ref = np.linalg.solve(D, g)
    x_ref = np.linalg.solve(D, b)
    assert np.linalg.norm(lam - lam_ref) / np.linalg.norm(lam_ref) < 1e-10
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    dA_ref = -lam_ref[rows] * x_ref[A.indices]
    assert np.linalg.norm(dA - dA_ref) / np.linalg.norm(dA_ref) < 1e-10


def test_autograd_vs_central_differences(bx, cuda):
    """L = 0.5 ||x(theta) - x_obs||^2 on 7-point FV diffusion, kappa = exp(theta): the autograd
    gradient along random directions against FP64 central differences (step 1e-6)."""
    import torch
    from bootcmatchgx_b200 import autograd, problems
    n = 14
    theta0 = torch.from_numpy(_problem(bx, n, 5).reshape(-1)).to(cuda)
    asm = problems.DiffusionAssembler(n, n, n, cuda)
    rng = np.random.default_rng(1)
    b = torch.from_numpy(rng.uniform(0, 1, n ** 3)).to(cuda)
    prm = autograd.default_params(rtol=1e-13)
    with torch.no_grad():
        x_obs = autograd.solve(asm.row, asm.col, asm.values(torch.exp(theta0)), b, prm)
        x_obs = x_obs + 1e-3 * torch.from_numpy(rng.standard_normal(n ** 3)).to(cuda)
    theta = (theta0 + 0.3 * torch.from_numpy(rng.standard_normal(n ** 3)).to(cuda)).requires_grad_(True)

    def loss(th):
        x = autograd.solve(asm.row, asm.col, asm.values(torch.exp(th)), b, prm)
        return 0.5 * ((x - x_obs) ** 2).sum()

    L = loss(theta)
    (grad,) = torch.autograd.grad(L, theta)
    h = 1e-6
    errs = []
    for k in range(6):
        d = torch.from_numpy(rng.standard_normal(n ** 3)).to(cuda)
        with torch.no_grad():
            fd = (loss(theta + h * d) - loss(theta - h * d)) / (2 * h)
        ad = (grad * d).sum()
        errs.append(abs(float(fd - ad)) / abs(float(fd)))
    assert max(errs) < 1e-5, errs


def test_fp32_vcycle_gradient_vs_fresh_fp64(bx, cuda):
    """The gradient through the FP32 V-cycle equals the one from a fresh FP64 hierarchy."""
    import torch
    from bootcmatchgx_b200 import autograd, problems
    n = 16
    theta = torch.from_numpy(_problem(bx, n, 7).reshape(-1)).to(cuda).requires_grad_(True)
    asm = problems.DiffusionAssembler(n, n, n, cuda)
    b = torch.from_numpy(np.random.default_rng(2).uniform(0, 1, n ** 3)).to(cuda)
    grads = {}
    for prec in ("FP32", "FP64"):
        prm = autograd.default_params(rtol=1e-12, vcycle_precision=prec)
        x = autograd.solve(asm.row, asm.col, asm.values(torch.exp(theta)), b, prm)
        (g,) = torch.autograd.grad(0.5 * (x ** 2).sum(), theta)
        grads[prec] = g
    rel = float((grads["FP32"] - grads["FP64"]).norm() / grads["FP64"].norm())
    assert rel < 1e-8, rel
