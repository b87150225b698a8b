"""Synthetic problems of the benchmark configurations (host-side input generation).

* poisson(stencil, grid, seed): 7/27-point Laplacian (the reference's generators), x* uniform[-1,1]
  from numpy default_rng(seed), b = A x*.
* gaussian_random_field(shape, length, sigma, seed): a field with squared-exponential covariance
  sigma^2 exp(-d^2 / (2 length^2)), made by filtering white noise (default_rng(seed)) with a
  Gaussian of standard deviation length / sqrt(2) (periodic boundaries) and scaling to variance
  sigma^2.
* diffusion(...): 7-point finite-volume matrix for kappa = exp(theta) with harmonic-mean faces
  (bcmgx_diffusion_7p), and DiffusionAssembler, which rebuilds the same values from kappa with
  torch operations so that gradients flow from the CSR values back to theta.
"""
from __future__ import annotations

import numpy as np

from . import api


def poisson(stencil, grid, seed, P=(1, 1, 1)):
    import scipy.sparse as sp
    row, col, val = api.laplacian_3d(stencil, *grid, *P)
    n = row.size - 1
    xs = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    b = sp.csr_matrix((val, col, row), shape=(n, n)) @ xs
    return row, col, val, xs, b


def gaussian_random_field(shape, length=8.0, sigma=2.0, seed=0):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    s = length / np.sqrt(2.0)
    f = gaussian_filter(w, s, mode="wrap")
    delta = np.zeros(shape)
    delta[tuple(k // 2 for k in shape)] = 1.0
    g = gaussian_filter(delta, s, mode="wrap")
    return sigma * f / np.sqrt((g * g).sum())


def diffusion(nx, ny, nz, kappa):
    return api.diffusion_7p(nx, ny, nz, np.ascontiguousarray(kappa, dtype=np.float64).reshape(-1))


class DiffusionAssembler:
    """Index maps of the 7-point FV pattern, to assemble its values from kappa in torch.

    Off-diagonal entry (i, j): -2 k_i k_j / (k_i + k_j). Diagonal of cell i: the sum of its face
    coefficients plus 2 k_i for every boundary face (Dirichlet), as bcmgx_diffusion_7p.
    """

    def __init__(self, nx, ny, nz, device):
        import torch
        self.shape = (nx, ny, nz)
        n = nx * ny * nz
        row, col, _ = api.diffusion_7p(nx, ny, nz, np.ones(n))
        rows = np.repeat(np.arange(n), np.diff(row))
        off = col != rows
        self.row = torch.from_numpy(row).to(device)
        self.col = torch.from_numpy(col).to(device)
        self.nnz = col.size
        self.off_e = torch.from_numpy(np.nonzero(off)[0]).to(device)
        self.off_i = torch.from_numpy(rows[off]).to(device)
        self.off_j = torch.from_numpy(col[off].astype(np.int64)).to(device)
        self.diag_e = torch.from_numpy(np.nonzero(~off)[0]).to(device)
        nb = 6 - np.bincount(rows[off], minlength=n)
        self.nbound = torch.from_numpy(nb.astype(np.float64)).to(device)
        self.n = n

    def values(self, kappa):
        import torch
        k = kappa.reshape(-1)
        ki, kj = k[self.off_i], k[self.off_j]
        t = 2.0 * ki * kj / (ki + kj)
        diag = torch.zeros(self.n, dtype=k.dtype, device=k.device).index_add(0, self.off_i, t) + 2.0 * k * self.nbound
        val = torch.zeros(self.nnz, dtype=k.dtype, device=k.device)
        val = val.index_put((self.off_e,), -t).index_put((self.diag_e,), diag)
        return val
