"""SparseCSC: the host-side matrix type, laid out as Julia's SparseMatrixCSC.

``colptr`` (n+1) and ``rowval`` (nnz) are 1-based Int64, ``nzval`` is Float64
(or Float32 when given Float32 values, as ``SparseMatrixCSC{Float32,Int64}``),
rows ascend within each column, exactly the layout ``SparseMatrixCSC`` hands
to ``ccall`` -- so buffers pass to the C ABI without conversion.
"""

from __future__ import annotations

import numpy as np


class SparseCSC:
    __slots__ = ("m", "n", "colptr", "rowval", "nzval")

    def __init__(self, m: int, n: int, colptr, rowval, nzval):
        self.m = int(m)
        self.n = int(n)
        self.colptr = np.ascontiguousarray(colptr, dtype=np.int64)
        self.rowval = np.ascontiguousarray(rowval, dtype=np.int64)
        nzval = np.asarray(nzval)
        dt = np.float32 if nzval.dtype == np.float32 else (np.complex128 if np.iscomplexobj(nzval) else np.float64)
        self.nzval = np.ascontiguousarray(nzval, dtype=dt)
        if self.colptr.shape != (self.n + 1,):
            raise ValueError("colptr must have n+1 entries")
        if self.colptr[0] != 1 or self.colptr[-1] - 1 != len(self.rowval) or len(self.rowval) != len(self.nzval):
            raise ValueError("inconsistent CSC arrays")

    # -- construction ------------------------------------------------------
    @staticmethod
    def from_coo(I, J, V, m: int, n: int) -> "SparseCSC":
        """Julia's ``sparse(I, J, V, m, n)``: 1-based triplets, rows sorted
        within each column, duplicate entries summed."""
        I = np.asarray(I, dtype=np.int64)
        J = np.asarray(J, dtype=np.int64)
        V = np.asarray(V, dtype=np.float64)
        order = np.lexsort((I, J))
        I, J, V = I[order], J[order], V[order]
        if len(I):
            key = (J - 1) * m + (I - 1)
            first = np.ones(len(key), dtype=bool)
            first[1:] = key[1:] != key[:-1]
            grp = np.cumsum(first) - 1
            Vs = np.zeros(int(grp[-1]) + 1)
            np.add.at(Vs, grp, V)
            I, J, V = I[first], J[first], Vs
        counts = np.bincount(J - 1, minlength=n) if len(J) else np.zeros(n, np.int64)
        colptr = np.empty(n + 1, np.int64)
        colptr[0] = 1
        np.cumsum(counts, out=colptr[1:])
        colptr[1:] += 1
        return SparseCSC(m, n, colptr, I, V)

    @staticmethod
    def from_scipy(S) -> "SparseCSC":
        S = S.tocsc()
        S.sort_indices()
        S.sum_duplicates()
        dt = np.float32 if S.dtype == np.float32 else (np.complex128 if np.iscomplexobj(S.data) else np.float64)
        return SparseCSC(S.shape[0], S.shape[1], S.indptr.astype(np.int64) + 1, S.indices.astype(np.int64) + 1,
                         S.data.astype(dt))

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.nzval, self.rowval - 1, self.colptr - 1), shape=(self.m, self.n))

    # -- queries -----------------------------------------------------------
    @property
    def shape(self):
        return (self.m, self.n)

    @property
    def eltype(self):
        """Element type of the stored values (numpy float64, float32 or complex128)."""
        return self.nzval.dtype.type

    def astype(self, dtype) -> "SparseCSC":
        """Copy with values converted to ``dtype`` (Float64, Float32 or ComplexF64)."""
        return SparseCSC(self.m, self.n, self.colptr.copy(), self.rowval.copy(), self.nzval.astype(dtype))

    def nnz(self) -> int:
        return int(len(self.rowval))

    def copy(self) -> "SparseCSC":
        return SparseCSC(self.m, self.n, self.colptr.copy(), self.rowval.copy(), self.nzval.copy())

    def colind(self) -> np.ndarray:
        """0-based column of every stored entry."""
        return np.repeat(np.arange(self.n, dtype=np.int64), np.diff(self.colptr))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """A * x (x may be n x k)."""
        return self.to_scipy() @ x

    def __add__(self, other: "SparseCSC") -> "SparseCSC":
        a, b = self.to_scipy(), other.to_scipy()
        return SparseCSC.from_scipy(a + b)

    def transpose(self) -> "SparseCSC":
        return SparseCSC.from_scipy(self.to_scipy().T)

    def add_diagonal(self, d) -> "SparseCSC":
        """A + Diagonal(d) (d scalar or length-n); the diagonal is made structural."""
        d = np.broadcast_to(np.asarray(d, dtype=np.float64), (self.n,))
        i = np.arange(1, self.n + 1, dtype=np.int64)
        I = np.concatenate([self.rowval, i])
        J = np.concatenate([self.colind() + 1, i])
        V = np.concatenate([self.nzval, d])
        return SparseCSC.from_coo(I, J, V, self.m, self.n)

    def __repr__(self):
        return f"SparseCSC({self.m}x{self.n}, nnz={self.nnz()})"
