"""Synthetic test matrices (the reference's bench/matrices.jl plus the
workloads of the multifrontal benchmark).

Grid Laplacians use the reference's exact index order (bench/matrices.jl:5-44),
so their CSC arrays are identical to the reference's.  Random matrices cannot
reproduce Julia's MersenneTwister / ``sprand`` streams; they use numpy's
seeded ``default_rng`` with the reference generator's shape and value
distribution, and parity is defined on identical inputs.
"""

from __future__ import annotations

import numpy as np

from .sparse import SparseCSC


def poisson2d(k: int) -> SparseCSC:
    """5-point Laplacian on a k x k grid, n = k^2 (bench/matrices.jl:5-22)."""
    n = k * k
    jj, ii = np.meshgrid(np.arange(1, k + 1), np.arange(1, k + 1), indexing="ij")
    i = ii.ravel()
    j = jj.ravel()
    c = (j - 1) * k + i
    I = [c]
    J = [c]
    V = [np.full(n, 4.0)]
    for cond, nb in ((i > 1, c - 1), (i < k, c + 1), (j > 1, c - k), (j < k, c + k)):
        I.append(c[cond])
        J.append(nb[cond])
        V.append(np.full(int(cond.sum()), -1.0))
    return SparseCSC.from_coo(np.concatenate(I), np.concatenate(J), np.concatenate(V), n, n)


def poisson3d(k: int) -> SparseCSC:
    """7-point Laplacian on a k x k x k grid, n = k^3 (bench/matrices.jl:25-44)."""
    n = k ** 3
    ll, jj, ii = np.meshgrid(np.arange(1, k + 1), np.arange(1, k + 1), np.arange(1, k + 1), indexing="ij")
    i, j, l = ii.ravel(), jj.ravel(), ll.ravel()
    c = ((l - 1) * k + (j - 1)) * k + i
    I = [c]
    J = [c]
    V = [np.full(n, 6.0)]
    for cond, nb in ((i > 1, c - 1), (i < k, c + 1), (j > 1, c - k), (j < k, c + k), (l > 1, c - k * k),
                     (l < k, c + k * k)):
        I.append(c[cond])
        J.append(nb[cond])
        V.append(np.full(int(cond.sum()), -1.0))
    return SparseCSC.from_coo(np.concatenate(I), np.concatenate(J), np.concatenate(V), n, n)


def randmat(n: int, deg: int, seed: int = 1) -> SparseCSC:
    """Random unsymmetric matrix with ~deg entries per column plus (deg+1) I
    (shape of bench/matrices.jl:47-51; numpy stream, not Julia's)."""
    rng = np.random.default_rng(seed)
    nz = rng.binomial(n * n, deg / n) if n > 0 else 0
    lin = np.unique(rng.choice(n * n, size=min(nz, n * n), replace=False))
    I = lin % n + 1
    J = lin // n + 1
    V = rng.random(len(lin))
    A = SparseCSC.from_coo(I, J, V, n, n)
    return A.add_diagonal(deg + 1.0)


def arrowband(n: int, bw: int, seed: int = 3) -> SparseCSC:
    """Arrowhead + band unsymmetric matrix (shape of bench/matrices.jl:54-86)."""
    rng = np.random.default_rng(seed)
    I, J, V = [], [], []
    for j in range(1, n + 1):
        I.append(j); J.append(j); V.append(float(n))
        for d in range(1, bw + 1):
            if j + d <= n:
                I += [j, j + d]
                J += [j + d, j]
                V += [rng.standard_normal(), rng.standard_normal()]
    for j in range(1, n + 1):
        if rng.random() < 0.3:
            I += [1, j]
            J += [j, 1]
            V += [rng.standard_normal(), rng.standard_normal()]
    return SparseCSC.from_coo(I, J, V, n, n)


def convdiff3d(k: int, velocity=(1.0, 0.5, 0.25), peclet: float = 10.0) -> SparseCSC:
    """7-point Laplacian plus first-order upwind convection on a k^3 grid.

    Cell Peclet number ``peclet`` scales the velocity: with unit grid spacing
    the convective coefficient on axis d is ``peclet * v_d / max(v)`` times the
    diffusion coefficient 1.  Upwinding puts the convective flux on the
    upstream neighbour, which makes the matrix unsymmetric in value but
    structurally symmetric.
    """
    n = k ** 3
    v = np.asarray(velocity, dtype=np.float64)
    a = peclet * v / np.max(np.abs(v))
    ll, jj, ii = np.meshgrid(np.arange(1, k + 1), np.arange(1, k + 1), np.arange(1, k + 1), indexing="ij")
    i, j, l = ii.ravel(), jj.ravel(), ll.ravel()
    c = ((l - 1) * k + (j - 1)) * k + i
    diag = np.full(n, 6.0 + float(np.sum(np.abs(a))))
    I = [c]
    J = [c]
    V = [diag]
    strides = (1, k, k * k)
    coords = (i, j, l)
    for d in range(3):
        s, x, ad = strides[d], coords[d], a[d]
        # upstream neighbour (x-1 for positive velocity) carries -1 - a_d
        up = -1.0 - max(ad, 0.0)
        dn = -1.0 - max(-ad, 0.0)
        m1 = x > 1
        I.append(c[m1]); J.append(c[m1] - s); V.append(np.full(int(m1.sum()), up))
        m2 = x < k
        I.append(c[m2]); J.append(c[m2] + s); V.append(np.full(int(m2.sum()), dn))
    return SparseCSC.from_coo(np.concatenate(I), np.concatenate(J), np.concatenate(V), n, n)


def grid3d_random(k: int, offdiag: float = 0.5, seed: int = 1) -> SparseCSC:
    """7-point grid pattern (poisson3d's) with random values: diagonal
    U[1, 2], off-diagonals N(0, offdiag^2), unsymmetric in value.  Partial
    pivoting inside the pivot blocks then makes row interchanges with clear
    margins and modest element growth."""
    A = poisson3d(k)
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(A.nnz()) * offdiag
    diag = (A.rowval - 1) == A.colind()
    v[diag] = 1.0 + rng.random(int(diag.sum()))
    return SparseCSC(A.m, A.n, A.colptr, A.rowval, v)


def random_unsym(n: int = 20000, per_col: int = 5, shift: float = 10.0, seed: int = 0) -> SparseCSC:
    """n x n, ``per_col`` entries per column at uniform random rows, N(0,1)
    values, plus ``shift`` * I."""
    rng = np.random.default_rng(seed)
    J = np.repeat(np.arange(1, n + 1), per_col)
    I = rng.integers(1, n + 1, size=n * per_col)
    V = rng.standard_normal(n * per_col)
    A = SparseCSC.from_coo(I, J, V, n, n)
    return A.add_diagonal(shift)


def batched_set(count: int = 1024, seed: int = 0, nrhs: int = 4):
    """Independent shifted grid Laplacians: half 2-D with side U[16,64], half
    3-D with side U[8,20], each plus shift*I with shift ~ U[0,1], and nrhs
    N(0,1) right-hand sides.  Returns a list of (A, B)."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        if t < count // 2:
            A = poisson2d(int(rng.integers(16, 65)))
        else:
            A = poisson3d(int(rng.integers(8, 21)))
        A = A.add_diagonal(float(rng.random()))
        B = rng.standard_normal((A.n, nrhs))
        out.append((A, np.asfortranarray(B)))
    return out


def rhs(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    """Seeded N(0,1) right-hand side(s) (numpy stream)."""
    rng = np.random.default_rng(seed)
    if nrhs == 1:
        return rng.standard_normal(n)
    return np.asfortranarray(rng.standard_normal((n, nrhs)))
