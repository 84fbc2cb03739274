"""ctypes front end of the CPU oracle (``oracle/mf_oracle.cpp``).

TEST INFRASTRUCTURE ONLY.  Tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this module as the checker / reference
timing.  The shipped package never imports it.

Every function mirrors one piece of the reference (PureUMFPACK.jl) and keeps
its 1-based Int64 index convention:

* ``row_scaling``        src/scaling.jl:92-115
* ``amd_order_sym``      src/amd.jl:141-148
* ``colamd_order``       src/amd.jl:183-188
* ``symbolic_mf``        src/symbolic.jl:211-226
* ``multifrontal_lu``    src/multifrontal.jl:146-358
* ``solve``              src/interface.jl:170-177 (with ``_solve_factor`` :123-138)
* ``gplu``, ``splu_gplu`` src/gplu.jl:173-303 and splu(A; method=:gplu,
  ordering) (src/interface.jl:93-120): Gilbert-Peierls left-looking LU with
  threshold partial pivoting
* ``*_f32``              the same for the reference's generic Tv = Float32: row
  scaling, the numeric phase (sgetrf / strsm / sgemm fronts) and the solve
  with its refinement, all in Float32 arithmetic
* ``*_c64``              the same for Tv = ComplexF64 (``ComplexCSC`` values):
  real row scaling from |z| = hypot(re, im), zgetrf / ztrsm / zgemm fronts
  (pivot of largest |re| + |im|, LAPACK's rule, as Julia's lu! uses), complex
  solves and refinement
"""

from __future__ import annotations

import ctypes
import glob
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmforacle.so")
_lib = None

SCALE_NONE, SCALE_SUM, SCALE_MAX = 0, 1, 2

_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)


def openblas_path() -> str:
    """Path of numpy's bundled ILP64 OpenBLAS (exports scipy_dgetrf_64_ etc.)."""
    import numpy

    libs = os.path.join(os.path.dirname(os.path.dirname(numpy.__file__)), "numpy.libs")
    hits = sorted(glob.glob(os.path.join(libs, "libscipy_openblas64_*.so")))
    if not hits:
        raise RuntimeError("numpy's bundled OpenBLAS (libscipy_openblas64_) not found")
    return hits[0]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "mf_oracle.cpp")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_blas.argtypes = [ctypes.c_char_p]
        L.orc_blas_threads.argtypes = [ctypes.c_int]
        L.orc_symbolic.restype = ctypes.c_void_p
        L.orc_symbolic.argtypes = [ctypes.c_int64, _i64p, _i64p, _i64p]
        L.orc_symbolic_free.argtypes = [ctypes.c_void_p]
        L.orc_symbolic_sizes.argtypes = [ctypes.c_void_p, _i64p]
        L.orc_symbolic_get.argtypes = [ctypes.c_void_p] + [_i64p] * 7
        L.orc_multifrontal_lu.restype = ctypes.c_void_p
        L.orc_multifrontal_lu.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, _i64p, ctypes.c_int, _i64p]
        L.orc_numeric.restype = ctypes.c_void_p
        L.orc_gplu.restype = ctypes.c_void_p
        L.orc_gplu.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, _i64p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                               _i64p]
        L.orc_gplu_f32.restype = ctypes.c_void_p
        L.orc_gplu_f32.argtypes = [ctypes.c_int64, _i64p, _i64p, _f32p, _i64p, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, _i64p]
        L.orc_gplu_c64.restype = ctypes.c_void_p
        L.orc_gplu_c64.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, _i64p, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, _i64p]
        L.orc_gplu_solve_c64.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int64, _i64p, _i64p, _f64p, ctypes.c_int64,
                                         _f64p, _f64p, ctypes.c_int]
        L.orc_numeric.argtypes = [ctypes.c_void_p, _f64p, _i64p, _i64p, ctypes.c_int, _i64p]
        L.orc_factor_free.argtypes = [ctypes.c_void_p]
        L.orc_factor_sizes.argtypes = [ctypes.c_void_p, _i64p]
        L.orc_factor_get.argtypes = [ctypes.c_void_p, _i64p, _i64p, _f64p, _i64p, _i64p, _f64p, _i64p, _i64p, _i64p]
        L.orc_solve_factor.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p]
        L.orc_solve.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int64, _i64p, _i64p, _f64p, ctypes.c_int64,
                                _f64p, _f64p, ctypes.c_int]
        L.orc_row_scaling.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, ctypes.c_int, _f64p]
        L.orc_amd_order_sym.argtypes = [ctypes.c_int64, _i64p, _i64p, ctypes.c_double, _i64p]
        L.orc_colamd_order.argtypes = [ctypes.c_int64, ctypes.c_int64, _i64p, _i64p, ctypes.c_double, _i64p]
        L.orc_row_scaling_f32.argtypes = [ctypes.c_int64, _i64p, _i64p, _f32p, ctypes.c_int, _f32p]
        L.orc_multifrontal_lu_f32.restype = ctypes.c_void_p
        L.orc_multifrontal_lu_f32.argtypes = [ctypes.c_int64, _i64p, _i64p, _f32p, _i64p, ctypes.c_int, _i64p]
        L.orc_solve_f32.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, _i64p, _i64p, _f32p, ctypes.c_int64,
                                    _f32p, _f32p, ctypes.c_int]
        L.orc_row_scaling_c64.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, ctypes.c_int, _f64p]
        L.orc_multifrontal_lu_c64.restype = ctypes.c_void_p
        L.orc_multifrontal_lu_c64.argtypes = [ctypes.c_int64, _i64p, _i64p, _f64p, _i64p, ctypes.c_int, _i64p]
        L.orc_factor_free_c64.argtypes = [ctypes.c_void_p]
        L.orc_factor_sizes_c64.argtypes = [ctypes.c_void_p, _i64p]
        L.orc_factor_get_c64.argtypes = [ctypes.c_void_p, _i64p, _i64p, _f64p, _i64p, _i64p, _f64p, _i64p, _i64p,
                                         _i64p]
        L.orc_solve_c64.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int64, _i64p, _i64p, _f64p, ctypes.c_int64,
                                    _f64p, _f64p, ctypes.c_int]
        rc = L.orc_set_blas(openblas_path().encode())
        if rc != 0:
            raise RuntimeError("oracle: cannot load OpenBLAS: " + L.orc_last_error().decode())
        _lib = L
    return _lib


def _p(a, ty=_i64p):
    return a.ctypes.data_as(ty) if a is not None else None


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def blas_threads(k: int = 0) -> int:
    """Set (k > 0) and return OpenBLAS's thread count."""
    return int(lib().orc_blas_threads(int(k)))


def row_scaling(A, kind: int) -> np.ndarray:
    n = A.m
    Rs = np.empty(n)
    lib().orc_row_scaling(n, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_f(A.nzval), _f64p), int(kind), _p(Rs, _f64p))
    return Rs


def apply_row_scaling(A, Rs):
    """Diagonal(Rs) * A with the same pattern (scaling.jl:118-126)."""
    B = A.copy()
    B.nzval = B.nzval * Rs[B.rowval - 1]
    return B


def amd_order_sym(A, dense: float = 10.0) -> np.ndarray:
    n = A.n
    perm = np.empty(n, dtype=np.int64)
    lib().orc_amd_order_sym(n, _p(_i(A.colptr)), _p(_i(A.rowval)), float(dense), _p(perm))
    return perm


def colamd_order(A, dense: float = 10.0) -> np.ndarray:
    n = A.n
    perm = np.empty(n, dtype=np.int64)
    lib().orc_colamd_order(A.m, n, _p(_i(A.colptr)), _p(_i(A.rowval)), float(dense), _p(perm))
    return perm


@dataclass
class Symbolic:
    """SymbolicMF (symbolic.jl:203-209), flattened; all indices 1-based."""

    qf: np.ndarray
    parent: np.ndarray          # 0 = root
    cs_ptr: np.ndarray          # colstruct[j] = cs_idx[cs_ptr[j]-1 : cs_ptr[j+1]-1]
    cs_idx: np.ndarray
    sstart: np.ndarray
    ch_ptr: np.ndarray
    ch_idx: np.ndarray
    handle: int = 0

    def colstruct(self, j: int) -> np.ndarray:   # j 1-based
        return self.cs_idx[self.cs_ptr[j - 1] - 1 : self.cs_ptr[j] - 1]

    def childsupers(self, s: int) -> np.ndarray:  # s 1-based
        return self.ch_idx[self.ch_ptr[s - 1] - 1 : self.ch_ptr[s] - 1]

    @property
    def nsuper(self) -> int:
        return len(self.sstart) - 1

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.orc_symbolic_free(ctypes.c_void_p(self.handle))
            self.handle = 0


def predicted_fill(S: Symbolic) -> int:
    """symbolic.jl:230-237."""
    n = len(S.qf)
    return 2 * (n + int(S.cs_ptr[-1] - 1))


def symbolic_mf(A, q=None) -> Symbolic:
    n = A.n
    qa = _i(q) if q is not None else None
    h = lib().orc_symbolic(n, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(qa))
    sz = np.empty(4, dtype=np.int64)
    lib().orc_symbolic_sizes(ctypes.c_void_p(h), _p(sz))
    ns, ncs, nch = int(sz[1]), int(sz[2]), int(sz[3])
    qf = np.empty(n, np.int64)
    parent = np.empty(n, np.int64)
    cs_ptr = np.empty(n + 1, np.int64)
    cs_idx = np.empty(ncs, np.int64)
    sstart = np.empty(ns + 1, np.int64)
    ch_ptr = np.empty(ns + 1, np.int64)
    ch_idx = np.empty(nch, np.int64)
    lib().orc_symbolic_get(ctypes.c_void_p(h), _p(qf), _p(parent), _p(cs_ptr), _p(cs_idx), _p(sstart), _p(ch_ptr),
                           _p(ch_idx))
    return Symbolic(qf, parent, cs_ptr, cs_idx, sstart, ch_ptr, ch_idx, handle=h)


class SingularException(Exception):
    """Julia's LinearAlgebra.SingularException(info)."""

    def __init__(self, info: int):
        super().__init__(f"SingularException({info})")
        self.info = info


@dataclass
class Factor:
    """GPLUFactorization (gplu.jl:45-51) from the oracle; 1-based."""

    Lcolptr: np.ndarray
    Lrowval: np.ndarray
    Lnzval: np.ndarray
    Ucolptr: np.ndarray
    Urowval: np.ndarray
    Unzval: np.ndarray
    p: np.ndarray
    q: np.ndarray
    pinv: np.ndarray
    handle: int = 0

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.orc_factor_free(ctypes.c_void_p(self.handle))
            self.handle = 0


def _extract(h) -> Factor:
    sz = np.empty(3, dtype=np.int64)
    lib().orc_factor_sizes(ctypes.c_void_p(h), _p(sz))
    n, nl, nu = (int(v) for v in sz)
    Lp = np.empty(n + 1, np.int64)
    Up = np.empty(n + 1, np.int64)
    Li = np.empty(nl, np.int64)
    Ui = np.empty(nu, np.int64)
    Lx = np.empty(nl)
    Ux = np.empty(nu)
    p = np.empty(n, np.int64)
    q = np.empty(n, np.int64)
    pinv = np.empty(n, np.int64)
    lib().orc_factor_get(ctypes.c_void_p(h), _p(Lp), _p(Li), _p(Lx, _f64p), _p(Up), _p(Ui), _p(Ux, _f64p), _p(p),
                         _p(q), _p(pinv))
    return Factor(Lp, Li, Lx, Up, Ui, Ux, p, q, pinv, handle=h)


def multifrontal_lu(A, q=None, check: bool = True) -> Factor:
    """multifrontal.jl:146-358 on the matrix as given (no scaling)."""
    n = A.n
    st = np.zeros(1, np.int64)
    qa = _i(q) if q is not None else None
    h = lib().orc_multifrontal_lu(n, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_f(A.nzval), _f64p), _p(qa),
                                  int(check), _p(st))
    if st[0] < 0:
        lib().orc_factor_free(ctypes.c_void_p(h))
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())
    if st[0] > 0:
        lib().orc_factor_free(ctypes.c_void_p(h))
        raise SingularException(int(st[0]))
    return _extract(h)


def gplu(A, q=None, tol: float = 0.1, check: bool = True, sort_factors: bool = True):
    """gplu(A; q, tol, check, sort_factors) (gplu.jl:173-303), A as given:
    Float64, Float32 (values returned widened to Float64, exactly) or
    ComplexF64 (a ``ComplexCSC``; returns a ``FactorC``)."""
    if A.m != A.n:
        raise ValueError("DimensionMismatch: gplu requires a square matrix")
    st = np.zeros(1, np.int64)
    qa = _i(q) if q is not None else None
    pat = (A.n, _p(_i(A.colptr)), _p(_i(A.rowval)))
    cz = np.iscomplexobj(A.nzval)
    if cz:
        h = lib().orc_gplu_c64(*pat, _p(_ri(A.nzval), _f64p), _p(qa), float(tol), int(check), int(sort_factors),
                               _p(st))
    elif A.nzval.dtype == np.float32:
        h = lib().orc_gplu_f32(*pat, _p(_f32(A.nzval), _f32p), _p(qa), float(tol), int(check), int(sort_factors),
                               _p(st))
    else:
        h = lib().orc_gplu(*pat, _p(_f(A.nzval), _f64p), _p(qa), float(tol), int(check), int(sort_factors), _p(st))
    free = lib().orc_factor_free_c64 if cz else lib().orc_factor_free
    if st[0] < 0:
        free(ctypes.c_void_p(h))
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())
    if st[0] > 0:
        free(ctypes.c_void_p(h))
        raise SingularException(int(st[0]))
    if cz:
        return _extract_c64(h)
    F = _extract(h)
    F.f32 = A.nzval.dtype == np.float32
    return F


def gplu_order(A, ordering: str) -> np.ndarray:
    """The column order splu(A; method=:gplu, ordering) factors in
    (interface.jl:108-116), 1-based."""
    if ordering == "natural":
        return np.arange(1, A.n + 1, dtype=np.int64)
    if ordering == "amd":
        return amd_order_sym(A)
    if ordering == "colamd":
        return colamd_order(A)
    raise ValueError(f"ArgumentError: unknown ordering {ordering}")


def numeric(S: Symbolic, A, check: bool = True) -> Factor:
    """Numeric phase only, on a precomputed symbolic object."""
    st = np.zeros(1, np.int64)
    h = lib().orc_numeric(ctypes.c_void_p(S.handle), _p(_f(A.nzval), _f64p), _p(_i(A.colptr)), _p(_i(A.rowval)),
                          int(check), _p(st))
    if st[0] != 0:
        lib().orc_factor_free(ctypes.c_void_p(h))
        raise SingularException(int(st[0])) if st[0] > 0 else RuntimeError("oracle numeric failed")
    return _extract(h)


@dataclass
class PureLU:
    """interface.jl:38-48: (Rs .* A)[p, q] == L * U."""

    F: Factor
    Rs: np.ndarray
    A: object


def splu(A, scale: int = SCALE_SUM, check: bool = True, q=None) -> PureLU:
    """splu(A; method=:multifrontal, scale) (interface.jl:93-105).

    ``q`` (not part of ``splu``) routes a caller order through
    ``multifrontal_lu(As; q)`` as ``multifrontal.jl:152`` allows.
    """
    if A.m != A.n:
        raise ValueError("DimensionMismatch: splu requires a square matrix")
    Rs = row_scaling(A, scale)
    As = A if scale == SCALE_NONE else apply_row_scaling(A, Rs)
    F = multifrontal_lu(As, q=q, check=check)
    return PureLU(F, Rs, A)


def splu_gplu(A, ordering: str = "amd", tol: float = 0.1, scale: int = SCALE_SUM, check: bool = True) -> PureLU:
    """splu(A; method=:gplu, ordering, tol, scale, check) (interface.jl:93-120)
    for Float64, Float32 and ComplexF64 values."""
    if A.m != A.n:
        raise ValueError("DimensionMismatch: splu requires a square matrix")
    if np.iscomplexobj(A.nzval):
        Rs = row_scaling_c64(A, scale)
        As = A if scale == SCALE_NONE else apply_row_scaling_c64(A, Rs)
    elif A.nzval.dtype == np.float32:
        Rs = row_scaling_f32(A, scale)
        As = A.copy()
        if scale != SCALE_NONE:
            As.nzval = (_f32(As.nzval) * Rs[As.rowval - 1]).astype(np.float32)
    else:
        Rs = row_scaling(A, scale)
        As = A if scale == SCALE_NONE else apply_row_scaling(A, Rs)
    q = gplu_order(A, ordering)
    return PureLU(gplu(As, q=q, tol=tol, check=check), Rs, A)


def solve_gplu(F, b, refine: int = 0):
    """solve(F, b; refine) over Gilbert-Peierls factors in the factors' own
    element type: F a PureLU (row scaling, refinement against F.A), or a raw
    factor (F \\ b, refine 0)."""
    if isinstance(F, PureLU):
        Fo, Rs, A = F.F, F.Rs, F.A
    else:
        Fo, Rs, A = F, None, None
        if refine:
            raise ValueError("refinement needs a PureLU")
    n = len(Fo.p)
    cp = _i(A.colptr) if A is not None else np.ones(n + 1, np.int64)
    rv = _i(A.rowval) if A is not None else np.zeros(0, np.int64)
    if isinstance(Fo, FactorC):
        B = np.asfortranarray(b, dtype=np.complex128)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        Bri = np.ascontiguousarray(B.ravel(order="F")).view(np.float64)
        Xri = np.empty_like(Bri)
        nz = _ri(A.nzval) if A is not None else np.zeros(0)
        lib().orc_gplu_solve_c64(ctypes.c_void_p(Fo.handle), _p(_f(Rs), _f64p) if Rs is not None else None, n,
                                 _p(cp), _p(rv), _p(nz, _f64p), nrhs, _p(Bri, _f64p), _p(Xri, _f64p), int(refine))
        return Xri.view(np.complex128).reshape(B.shape, order="F")
    if getattr(Fo, "f32", False):
        B = np.asfortranarray(b, dtype=np.float32)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        X = np.empty_like(B)
        nz = _f32(A.nzval) if A is not None else np.zeros(0, np.float32)
        lib().orc_solve_f32(ctypes.c_void_p(Fo.handle), _p(_f32(Rs), _f32p) if Rs is not None else None, n, _p(cp),
                            _p(rv), _p(nz, _f32p), nrhs, _p(B, _f32p), _p(X, _f32p), int(refine))
        return X
    return solve(F, b, refine=refine) if Rs is not None else solve_raw(Fo, b)


def solve(F: PureLU, b: np.ndarray, refine: int = 0) -> np.ndarray:
    """solve(F::PureLU, b; refine) (interface.jl:170-177); b may be n x k."""
    A = F.A
    B = np.asfortranarray(b, dtype=np.float64)
    nrhs = 1 if B.ndim == 1 else B.shape[1]
    X = np.empty_like(B)
    lib().orc_solve(ctypes.c_void_p(F.F.handle), _p(_f(F.Rs), _f64p), A.n, _p(_i(A.colptr)), _p(_i(A.rowval)),
                    _p(_f(A.nzval), _f64p), nrhs, _p(B, _f64p), _p(X, _f64p), int(refine))
    return X


def solve_raw(F: Factor, b: np.ndarray) -> np.ndarray:
    """solve(F::GPLUFactorization, b) (solve.jl:66-77)."""
    x = np.empty(len(b))
    bb = _f(b)
    lib().orc_solve_factor(ctypes.c_void_p(F.handle), None, _p(bb, _f64p), _p(x, _f64p))
    return x


# ---------------------------------------------------------------------------
# Float32 (the reference's generic Tv = Float32)
# ---------------------------------------------------------------------------
def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def row_scaling_f32(A, kind: int) -> np.ndarray:
    """row_scaling of a Float32 matrix, in Float32 (scaling.jl:92-115)."""
    Rs = np.empty(A.m, np.float32)
    lib().orc_row_scaling_f32(A.m, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_f32(A.nzval), _f32p), int(kind),
                              _p(Rs, _f32p))
    return Rs


def multifrontal_lu_f32(A, q=None, check: bool = True) -> Factor:
    """multifrontal_lu of a Float32 matrix: every front operation in Float32
    (values returned widened to Float64, exactly)."""
    st = np.zeros(1, np.int64)
    qa = _i(q) if q is not None else None
    h = lib().orc_multifrontal_lu_f32(A.n, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_f32(A.nzval), _f32p), _p(qa),
                                      int(check), _p(st))
    if st[0] < 0:
        lib().orc_factor_free(ctypes.c_void_p(h))
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())
    if st[0] > 0:
        lib().orc_factor_free(ctypes.c_void_p(h))
        raise SingularException(int(st[0]))
    return _extract(h)


def splu_f32(A, scale: int = SCALE_SUM, check: bool = True, q=None) -> PureLU:
    """splu(A::SparseMatrixCSC{Float32}; method=:multifrontal, scale)."""
    Rs = row_scaling_f32(A, scale)
    As = A.copy()
    if scale != SCALE_NONE:
        As.nzval = (_f32(As.nzval) * Rs[As.rowval - 1]).astype(np.float32)
    F = multifrontal_lu_f32(As, q=q, check=check)
    return PureLU(F, Rs, A)


def solve_f32(F: PureLU, b: np.ndarray, refine: int = 0) -> np.ndarray:
    """solve(F::PureLU{Float32}, b::Vector{Float32}; refine), all in Float32."""
    A = F.A
    B = np.asfortranarray(b, dtype=np.float32)
    nrhs = 1 if B.ndim == 1 else B.shape[1]
    X = np.empty_like(B)
    lib().orc_solve_f32(ctypes.c_void_p(F.F.handle), _p(_f32(F.Rs), _f32p), A.n, _p(_i(A.colptr)),
                        _p(_i(A.rowval)), _p(_f32(A.nzval), _f32p), nrhs, _p(B, _f32p), _p(X, _f32p), int(refine))
    return X


# ---------------------------------------------------------------------------
# ComplexF64 (the reference's generic Tv = ComplexF64)
# ---------------------------------------------------------------------------
@dataclass
class ComplexCSC:
    """SparseMatrixCSC{ComplexF64, Int64}: 1-based pattern, complex values."""

    m: int
    n: int
    colptr: np.ndarray
    rowval: np.ndarray
    nzval: np.ndarray

    @staticmethod
    def from_scipy(S) -> "ComplexCSC":
        S = S.tocsc()
        S.sort_indices()
        S.sum_duplicates()
        return ComplexCSC(S.shape[0], S.shape[1], S.indptr.astype(np.int64) + 1, S.indices.astype(np.int64) + 1,
                          np.ascontiguousarray(S.data, dtype=np.complex128))

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.nzval, self.rowval - 1, self.colptr - 1), shape=(self.m, self.n))

    def nnz(self) -> int:
        return len(self.rowval)


def _ri(z) -> np.ndarray:
    """Complex values as interleaved (re, im) doubles."""
    return np.ascontiguousarray(z, dtype=np.complex128).view(np.float64)


@dataclass
class FactorC(Factor):
    """Factor of a ComplexF64 matrix (complex Lnzval / Unzval)."""

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.orc_factor_free_c64(ctypes.c_void_p(self.handle))
            self.handle = 0


def row_scaling_c64(A: ComplexCSC, kind: int) -> np.ndarray:
    """row_scaling of a ComplexF64 matrix: Float64 Rs from |z| = hypot(re, im)
    (scaling.jl:92-115 with R = real(Tv))."""
    Rs = np.empty(A.m)
    lib().orc_row_scaling_c64(A.m, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_ri(A.nzval), _f64p), int(kind),
                              _p(Rs, _f64p))
    return Rs


def multifrontal_lu_c64(A: ComplexCSC, q=None, check: bool = True) -> FactorC:
    """multifrontal_lu of a ComplexF64 matrix (multifrontal.jl:146-358 with
    Tv = ComplexF64): every front operation in complex double."""
    st = np.zeros(1, np.int64)
    qa = _i(q) if q is not None else None
    h = lib().orc_multifrontal_lu_c64(A.n, _p(_i(A.colptr)), _p(_i(A.rowval)), _p(_ri(A.nzval), _f64p), _p(qa),
                                      int(check), _p(st))
    if st[0] != 0:
        lib().orc_factor_free_c64(ctypes.c_void_p(h))
        if st[0] > 0:
            raise SingularException(int(st[0]))
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())
    sz = np.empty(3, dtype=np.int64)
    lib().orc_factor_sizes_c64(ctypes.c_void_p(h), _p(sz))
    n, nl, nu = (int(v) for v in sz)
    Lp, Up = np.empty(n + 1, np.int64), np.empty(n + 1, np.int64)
    Li, Ui = np.empty(nl, np.int64), np.empty(nu, np.int64)
    Lx, Ux = np.empty(nl, np.complex128), np.empty(nu, np.complex128)
    p, qq, pinv = np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64)
    lib().orc_factor_get_c64(ctypes.c_void_p(h), _p(Lp), _p(Li), _p(Lx.view(np.float64), _f64p), _p(Up), _p(Ui),
                             _p(Ux.view(np.float64), _f64p), _p(p), _p(qq), _p(pinv))
    return FactorC(Lp, Li, Lx, Up, Ui, Ux, p, qq, pinv, handle=h)


def _extract_c64(h) -> FactorC:
    sz = np.empty(3, dtype=np.int64)
    lib().orc_factor_sizes_c64(ctypes.c_void_p(h), _p(sz))
    n, nl, nu = (int(v) for v in sz)
    Lp, Up = np.empty(n + 1, np.int64), np.empty(n + 1, np.int64)
    Li, Ui = np.empty(nl, np.int64), np.empty(nu, np.int64)
    Lx, Ux = np.empty(nl, np.complex128), np.empty(nu, np.complex128)
    p, qq, pinv = np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64)
    lib().orc_factor_get_c64(ctypes.c_void_p(h), _p(Lp), _p(Li), _p(Lx.view(np.float64), _f64p), _p(Up), _p(Ui),
                             _p(Ux.view(np.float64), _f64p), _p(p), _p(qq), _p(pinv))
    return FactorC(Lp, Li, Lx, Up, Ui, Ux, p, qq, pinv, handle=h)


def apply_row_scaling_c64(A: ComplexCSC, Rs) -> ComplexCSC:
    """Rs .* A: each part of a value times its row's real factor."""
    r = np.asarray(Rs, dtype=np.float64)[A.rowval - 1]
    z = np.empty(len(A.nzval), np.complex128)
    z.real = A.nzval.real * r
    z.imag = A.nzval.imag * r
    return ComplexCSC(A.m, A.n, A.colptr.copy(), A.rowval.copy(), z)


def splu_c64(A: ComplexCSC, scale: int = SCALE_SUM, check: bool = True, q=None) -> PureLU:
    """splu(A::SparseMatrixCSC{ComplexF64}; method=:multifrontal, scale)."""
    if A.m != A.n:
        raise ValueError("DimensionMismatch: splu requires a square matrix")
    Rs = row_scaling_c64(A, scale)
    As = A if scale == SCALE_NONE else apply_row_scaling_c64(A, Rs)
    return PureLU(multifrontal_lu_c64(As, q=q, check=check), Rs, A)


def solve_c64(F: PureLU, b: np.ndarray, refine: int = 0) -> np.ndarray:
    """solve(F::PureLU{ComplexF64}, b; refine) (interface.jl:170-177)."""
    A = F.A
    B = np.asfortranarray(b, dtype=np.complex128)
    nrhs = 1 if B.ndim == 1 else B.shape[1]
    X = np.empty_like(B)
    lib().orc_solve_c64(ctypes.c_void_p(F.F.handle), _p(_f(F.Rs), _f64p), A.n, _p(_i(A.colptr)), _p(_i(A.rowval)),
                        _p(_ri(A.nzval), _f64p), nrhs, _p(B.ravel(order="F").view(np.float64), _f64p),
                        _p(X.ravel(order="F").view(np.float64), _f64p), int(refine))
    return X
