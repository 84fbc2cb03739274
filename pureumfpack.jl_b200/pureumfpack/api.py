"""The reference's public API for the multifrontal path, over libmfgpu.

Mirrors PureUMFPACK.jl (names, argument meaning, errors):

* ``splu(A; method, ordering, tol, scale, check)`` -> ``PureLU``
  (src/interface.jl:93-120), ``method=:multifrontal`` or ``:gplu``
* ``gplu(A; q, tol, check, sort_factors)`` -> ``GPLUFactorization``
  (src/gplu.jl:173-303), one warp per system on the GPU
* ``multifrontal_lu(A; q, tol, check)`` -> ``GPLUFactorization``
  (src/multifrontal.jl:146-358)
* ``solve(F, b; refine)`` (src/interface.jl:170-177), ``F \\ b`` as
  ``F.ldiv(b)`` / ``solve(F, b)`` (src/interface.jl:179, src/solve.jl:66-79)
* ``row_scaling`` / ``apply_row_scaling`` / ``SCALE_*`` (src/scaling.jl)
* ``amd_order_sym`` / ``colamd_order`` (src/amd.jl:141-188)
* ``symbolic_mf`` / ``predicted_fill`` (src/symbolic.jl:203-237)

Indices are 1-based Int64 as in Julia.  Every numeric step (scaling applied
to the values, assembly, factorization, solves, refinement) runs on the GPU
through libmfgpu; ordering and symbolic analysis are the library's host code,
whose output is identical to the reference's.
"""

from __future__ import annotations

import ctypes
import json
import os
from concurrent.futures import ThreadPoolExecutor
from enum import IntEnum

import numpy as np

from . import _lib as L
from .sparse import SparseCSC


class ScaleKind(IntEnum):
    """@enum ScaleKind (src/scaling.jl:11)."""

    SCALE_NONE = 0
    SCALE_SUM = 1
    SCALE_MAX = 2


SCALE_NONE = ScaleKind.SCALE_NONE
SCALE_SUM = ScaleKind.SCALE_SUM
SCALE_MAX = ScaleKind.SCALE_MAX

PRECISION_FP64 = 0
PRECISION_MIXED = 1
FLAG_NO_TENSOR_CORES = 1   # mfgpu_options.flags: SIMT FP32 Schur updates in the mixed form
FLAG_PERSISTENT_SOLVE = 2  # mfgpu_options.flags: one persistent cooperative launch per solve pass
FLAG_TF32_SPLIT = 4        # mfgpu_options.flags: 3xTF32 instead of BF16x3 tensor-core products
FLAG_STEP_SOLVE = 8        # mfgpu_options.flags: one launch per solve step, whatever the rhs count
FLAG_LEAN_FRONTS = 16      # mfgpu_options.flags: reuse front memory by lifetime (compact panel pool)
FLAG_NO_FRONT_MERGE = 32   # mfgpu_options.flags: one front per supernode (no merged supernode chains)


class ArgumentError(ValueError):
    """Julia's ArgumentError."""


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch."""


class SingularException(Exception):
    """LinearAlgebra.SingularException(info): zero pivot at factor column info."""

    def __init__(self, info: int):
        super().__init__(f"SingularException({info})")
        self.info = int(info)


class MfgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libmfgpu error {code}: {msg}")
        self.code = code


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _z(a):
    """ComplexF64 values as interleaved (re, im) doubles (Julia's layout)."""
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _check_host(rc: int):
    if rc != 0:
        msg = L.lib().mfgpu_host_last_error().decode()
        if rc == -1:
            raise ArgumentError(msg or "invalid argument")
        raise MfgpuError(rc, msg)


# ---------------------------------------------------------------------------
# scaling, ordering, symbolic (host code of libmfgpu)
# ---------------------------------------------------------------------------
def row_scaling(A: SparseCSC, kind: ScaleKind) -> np.ndarray:
    """Rs with row i of A multiplied by Rs[i]; empty rows get 1."""
    if A.m != A.n:
        # the reference computes Rs for any m x n; libmfgpu's square-only ABI
        acc = np.zeros(A.m)
        if kind == SCALE_SUM:
            np.add.at(acc, A.rowval - 1, np.abs(A.nzval))
        elif kind == SCALE_MAX:
            np.maximum.at(acc, A.rowval - 1, np.abs(A.nzval))
        return np.where(acc > 0, 1.0 / np.where(acc > 0, acc, 1.0), 1.0) if kind != SCALE_NONE else np.ones(A.m)
    if np.iscomplexobj(A.nzval):      # ComplexF64 matrix: Float64 Rs from |z| (R = real(Tv))
        rs = np.empty(A.n)
        _check_host(L.lib().mfgpu_row_scaling_c64(A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)),
                                                  L.ptr(_z(A.nzval), L.f64p), int(kind), L.ptr(rs, L.f64p)))
        return rs
    if A.nzval.dtype == np.float32:   # Float32 matrix: Float32 arithmetic (R = real(Tv))
        rs = np.empty(A.n, np.float32)
        _check_host(L.lib().mfgpu_row_scaling_f32(A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)),
                                                  L.ptr(np.ascontiguousarray(A.nzval), L.f32p), int(kind),
                                                  L.ptr(rs, L.f32p)))
        return rs
    rs = np.empty(A.n)
    _check_host(L.lib().mfgpu_row_scaling(A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)),
                                          L.ptr(_f(A.nzval), L.f64p), int(kind), L.ptr(rs, L.f64p)))
    return rs


def apply_row_scaling(A: SparseCSC, Rs) -> SparseCSC:
    """Diagonal(Rs) * A with the same pattern (src/scaling.jl:118-126)."""
    B = A.copy()
    B.nzval = B.nzval * np.asarray(Rs, dtype=B.nzval.dtype)[B.rowval - 1]
    return B


def amd_order_sym(A: SparseCSC, dense: float = 10.0) -> np.ndarray:
    if A.m != A.n:
        raise DimensionMismatch("amd requires a square matrix")
    perm = np.empty(A.n, dtype=np.int64)
    _check_host(L.lib().mfgpu_amd_order(A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)), float(dense), L.ptr(perm)))
    return perm


def colamd_order(A: SparseCSC, dense: float = 10.0) -> np.ndarray:
    perm = np.empty(A.n, dtype=np.int64)
    _check_host(L.lib().mfgpu_colamd_order(A.m, A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)), float(dense),
                                           L.ptr(perm)))
    return perm


class SymbolicMF:
    """SymbolicMF (src/symbolic.jl:203-209); 1-based.

    ``colstruct[j]`` (L's below-diagonal rows of column j) is derived on
    demand from the supernode partition and the update sets: within a
    fundamental supernode the structures nest, so column j of supernode s
    holds rows j+1..last(s) followed by upd(s).
    """

    def __init__(self, handle, n, qf, parent, colcount, sstart, upd_ptr, upd_idx, child_ptr, child_idx):
        self._h = handle
        self.n = n
        self.qf = qf
        self.parent = parent
        self.colcount = colcount
        self.sstart = sstart
        self.upd_ptr = upd_ptr
        self.upd_idx = upd_idx
        self.child_ptr = child_ptr
        self.child_idx = child_idx
        self._super_of = None

    @property
    def nsuper(self) -> int:
        return len(self.sstart) - 1

    def update_set(self, s: int) -> np.ndarray:
        """colstruct[last column of supernode s] (s 1-based)."""
        return self.upd_idx[self.upd_ptr[s - 1] - 1: self.upd_ptr[s] - 1]

    @property
    def childsupers(self):
        return [self.child_idx[self.child_ptr[s] - 1: self.child_ptr[s + 1] - 1] for s in range(self.nsuper)]

    def colstruct(self, j: int) -> np.ndarray:
        if self._super_of is None:
            self._super_of = np.repeat(np.arange(1, self.nsuper + 1), np.diff(self.sstart))
        s = int(self._super_of[j - 1])
        last = int(self.sstart[s]) - 1
        return np.concatenate([np.arange(j + 1, last + 1, dtype=np.int64), self.update_set(s)])

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                L.lib().mfgpu_symbolic_destroy(self._h)
            except Exception:
                pass
            self._h = None


def symbolic_mf(A: SparseCSC, q=None, relax: bool = False) -> SymbolicMF:
    """symbolic_mf(A; q) (src/symbolic.jl:211-226).  ``relax`` (not in the
    reference) adds relaxed amalgamation: fewer, larger supernodes whose
    factors store explicit zeros."""
    if A.m != A.n:
        raise DimensionMismatch("symbolic analysis requires a square matrix")
    lib = L.lib()
    h = ctypes.c_void_p()
    qa = _i(q) if q is not None else None
    if qa is not None and len(qa) != A.n:   # q reaches the C ABI as a bare pointer
        raise DimensionMismatch("length(q) must equal size(A, 2)")
    _check_host(lib.mfgpu_symbolic_create(A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)), L.ptr(qa), ctypes.byref(h)))
    if relax:
        _check_host(lib.mfgpu_symbolic_relax(h))
    return _symbolic_from_handle(h)


def symbolic_batch(As, ordering: str = "amd") -> SymbolicMF:
    """Symbolic analysis of independent square systems as one block-diagonal
    forest: each system ordered (AMD or COLAMD) and analysed by symbolic_mf
    on its own, on all host cores, then concatenated -- equal to
    symbolic_mf of the block-diagonal matrix with the concatenated orders."""
    lib = L.lib()
    cps = [_i(A.colptr) for A in As]
    rvs = [_i(A.rowval) for A in As]
    ns = np.array([A.n for A in As], dtype=np.int64)
    h = ctypes.c_void_p()
    _check_host(lib.mfgpu_symbolic_create_batch(len(As), L.ptr(ns), L.ptr_array(cps), L.ptr_array(rvs),
                                                {"amd": 0, "colamd": 1}[ordering], ctypes.byref(h)))
    return _symbolic_from_handle(h)


def _symbolic_from_handle(h) -> SymbolicMF:
    lib = L.lib()
    sz = np.empty(4, np.int64)
    lib.mfgpu_symbolic_sizes(h, L.ptr(sz))
    n, ns, nupd, nch = (int(v) for v in sz)
    qf = np.empty(n, np.int64)
    parent = np.empty(n, np.int64)
    colcount = np.empty(n, np.int64)
    sstart = np.empty(ns + 1, np.int64)
    upd_ptr = np.empty(ns + 1, np.int64)
    upd_idx = np.empty(nupd, np.int64)
    child_ptr = np.empty(ns + 1, np.int64)
    child_idx = np.empty(nch, np.int64)
    lib.mfgpu_symbolic_get(h, L.ptr(qf), L.ptr(parent), L.ptr(colcount), L.ptr(sstart), L.ptr(upd_ptr),
                           L.ptr(upd_idx), L.ptr(child_ptr), L.ptr(child_idx))
    return SymbolicMF(h, n, qf, parent, colcount, sstart, upd_ptr, upd_idx, child_ptr, child_idx)


def predicted_fill(S: SymbolicMF) -> int:
    """nnz(L) + nnz(U) with both diagonals (src/symbolic.jl:230-237)."""
    return 2 * (S.n + int(np.sum(S.colcount)))


# ---------------------------------------------------------------------------
# GPU context
# ---------------------------------------------------------------------------
class GpuContext:
    """One libmfgpu handle: analysis, resident factors, solves."""

    def __init__(self, device: int = 0, precision: int = PRECISION_FP64, tensor_cores: bool = True,
                 persistent_solve: bool | None = None, tf32_split: bool = False, lean_fronts: bool = False,
                 merge_fronts: bool = True):
        """persistent_solve: True / False forces the solve mode; None lets the
        library choose by right-hand-side count.  merge_fronts: factor chains
        of supernodes as merged fronts (pivots and factor structure stay the
        original supernodes')."""
        self._lib = L.lib()
        flags = ((0 if tensor_cores else FLAG_NO_TENSOR_CORES) | (FLAG_TF32_SPLIT if tf32_split else 0)
                 | {None: 0, True: FLAG_PERSISTENT_SOLVE, False: FLAG_STEP_SOLVE}[persistent_solve]
                 | (FLAG_LEAN_FRONTS if lean_fronts else 0) | (0 if merge_fronts else FLAG_NO_FRONT_MERGE))
        opts = L.MfOptions(device, precision, flags, 0)
        h = ctypes.c_void_p()
        rc = self._lib.mfgpu_create(ctypes.byref(opts), ctypes.byref(h))
        if rc != 0:
            raise MfgpuError(rc, "mfgpu_create failed (needs a B200 / sm_100 device)")
        self._h = h
        self.n = 0
        self.precision = precision
        self.f32 = False   # the last factorization is of a Float32 matrix
        self.c64 = False   # the last factorization is of a ComplexF64 matrix

    def _check(self, rc: int):
        if rc < 0:
            msg = self._lib.mfgpu_last_error(self._h).decode()
            if rc == -1:
                raise ArgumentError(msg)
            if rc == -6:
                raise DimensionMismatch(msg)
            raise MfgpuError(rc, msg)
        return rc

    def set_precision(self, precision: int):
        self._check(self._lib.mfgpu_set_precision(self._h, int(precision)))
        self.precision = precision

    def set_growth_limit(self, limit: float):
        """Mixed form: refactor in FP64 when the FP32 factors' element growth
        max|U| / max|Rs .* A| exceeds ``limit``."""
        self._check(self._lib.mfgpu_set_growth_limit(self._h, float(limit)))

    def set_wait_limit(self, seconds: float):
        """Bound on every device-side wait of this handle's kernels (default
        4 s); a wait that runs out makes the call raise MfgpuError(-5)."""
        self._check(self._lib.mfgpu_set_wait_limit(self._h, ctypes.c_double(seconds)))

    def test_stall(self, on: bool):
        """Test hook: the kernels' bounded waits run out (mfgpu_test_stall)."""
        self._check(self._lib.mfgpu_test_stall(self._h, int(bool(on))))

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.mfgpu_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def analyze(self, A: SparseCSC, S: SymbolicMF):
        self._check(self._lib.mfgpu_analyze_symbolic(self._h, A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)), S._h))
        self.n = A.n
        self.nnz = A.nnz()

    def _values(self, nzval, Rs):
        """The factor calls copy nnz values and n row factors from bare
        pointers: check the lengths against the analyzed pattern first."""
        if getattr(self, "nnz", None) is not None and len(nzval) != self.nnz:
            raise DimensionMismatch("nzval must hold one value per entry of the analyzed pattern")
        if Rs is not None and len(Rs) != self.n:
            raise DimensionMismatch("length(Rs) must equal size(A, 1)")

    def analyze_arrays(self, A: SparseCSC, qf, parent, sstart, upd_ptr, upd_idx):
        """mfgpu_analyze with the reference's own symbolic arrays (1-based)."""
        ns = len(sstart) - 1
        if (len(qf) != A.n or len(parent) != A.n or ns < 0 or len(upd_ptr) != ns + 1
                or len(upd_idx) < int(upd_ptr[-1]) - 1):
            raise ArgumentError("symbolic arrays do not match n and the supernode count")
        self._check(self._lib.mfgpu_analyze(self._h, A.n, L.ptr(_i(A.colptr)), L.ptr(_i(A.rowval)), L.ptr(_i(qf)),
                                            L.ptr(_i(parent)), ns, L.ptr(_i(sstart)), L.ptr(_i(upd_ptr)),
                                            L.ptr(_i(upd_idx))))
        self.n = A.n
        self.nnz = A.nnz()

    def factor(self, nzval, Rs=None, check: bool = True) -> int:
        self._values(nzval, Rs)
        rs = _f(Rs) if Rs is not None else None
        self.f32 = self.c64 = False
        return self._check(self._lib.mfgpu_factor(self._h, L.ptr(_f(nzval), L.f64p), L.ptr(rs, L.f64p), int(check)))

    def factor_f32(self, nzval, Rs=None, check: bool = True) -> int:
        """Factorization of a Float32 matrix: Float32 fronts, Float32 factors."""
        self._values(nzval, Rs)
        v = np.ascontiguousarray(nzval, dtype=np.float32)
        rs = np.ascontiguousarray(Rs, dtype=np.float32) if Rs is not None else None
        self.f32, self.c64 = True, False
        return self._check(self._lib.mfgpu_factor_f32(self._h, L.ptr(v, L.f32p), L.ptr(rs, L.f32p), int(check)))

    def factor_c64(self, nzval, Rs=None, check: bool = True) -> int:
        """Factorization of a ComplexF64 matrix: complex fronts, complex factors."""
        self._values(nzval, Rs)
        rs = _f(Rs) if Rs is not None else None
        self.f32, self.c64 = False, True
        return self._check(self._lib.mfgpu_factor_c64(self._h, L.ptr(_z(nzval), L.f64p), L.ptr(rs, L.f64p),
                                                      int(check)))

    def factor_scaled(self, nzval, scale, check: bool = True) -> int:
        """Row scaling of kind ``scale`` computed on the device, then the
        factorization of Diagonal(Rs) * A."""
        self._values(nzval, None)
        return self._check(self._lib.mfgpu_factor_scaled(self._h, L.ptr(_f(nzval), L.f64p), int(scale), int(check)))

    def row_scaling(self) -> np.ndarray:
        """Rs of the last factorization (ones without scaling)."""
        rs = np.empty(self.n)
        self._check(self._lib.mfgpu_get_row_scaling(self._h, L.ptr(rs, L.f64p)))
        return rs

    def factor_device(self, nzval_ptr: int, rs_ptr: int | None, check: bool = True) -> int:
        return self._check(self._lib.mfgpu_factor_device(self._h, ctypes.c_void_p(nzval_ptr),
                                                         ctypes.c_void_p(rs_ptr) if rs_ptr else None, int(check)))

    def sizes(self):
        out = np.empty(3, np.int64)
        self._check(self._lib.mfgpu_factor_sizes(self._h, L.ptr(out)))
        return int(out[0]), int(out[1]), int(out[2])

    def factors(self):
        n, nl, nu = self.sizes()
        if getattr(self, "c64", False):
            return self._factors_c64(n, nl, nu)
        f32 = getattr(self, "f32", False)
        dt, vp = (np.float32, L.f32p) if f32 else (np.float64, L.f64p)
        Lp = np.empty(n + 1, np.int64)
        Li = np.empty(nl, np.int64)
        Lx = np.empty(nl, dt)
        Up = np.empty(n + 1, np.int64)
        Ui = np.empty(nu, np.int64)
        Ux = np.empty(nu, dt)
        p = np.empty(n, np.int64)
        q = np.empty(n, np.int64)
        pinv = np.empty(n, np.int64)
        get = self._lib.mfgpu_get_factors_f32 if f32 else self._lib.mfgpu_get_factors
        self._check(get(self._h, L.ptr(Lp), L.ptr(Li), L.ptr(Lx, vp), L.ptr(Up), L.ptr(Ui), L.ptr(Ux, vp), L.ptr(p),
                        L.ptr(q), L.ptr(pinv)))
        return SparseCSC(n, n, Lp, Li, Lx), SparseCSC(n, n, Up, Ui, Ux), p, q, pinv

    def _factors_c64(self, n, nl, nu):
        Lp, Li, Lx = np.empty(n + 1, np.int64), np.empty(nl, np.int64), np.empty(nl, np.complex128)
        Up, Ui, Ux = np.empty(n + 1, np.int64), np.empty(nu, np.int64), np.empty(nu, np.complex128)
        p, q, pinv = np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64)
        self._check(self._lib.mfgpu_get_factors_c64(self._h, L.ptr(Lp), L.ptr(Li), L.ptr(Lx.view(np.float64), L.f64p),
                                                    L.ptr(Up), L.ptr(Ui), L.ptr(Ux.view(np.float64), L.f64p),
                                                    L.ptr(p), L.ptr(q), L.ptr(pinv)))
        return SparseCSC(n, n, Lp, Li, Lx), SparseCSC(n, n, Up, Ui, Ux), p, q, pinv

    def solve(self, b, refine: int = 0) -> np.ndarray:
        if getattr(self, "c64", False):
            B = np.asfortranarray(b, dtype=np.complex128)
            X = np.empty_like(B)
            nrhs = 1 if B.ndim == 1 else B.shape[1]
            self._check(self._lib.mfgpu_solve_c64(self._h, nrhs, L.ptr(B.reshape(-1, order="F").view(np.float64),
                                                                       L.f64p),
                                                  L.ptr(X.reshape(-1, order="F").view(np.float64), L.f64p),
                                                  int(refine)))
            return X
        if getattr(self, "f32", False):
            B = np.asfortranarray(b, dtype=np.float32)
            X = np.empty_like(B)
            nrhs = 1 if B.ndim == 1 else B.shape[1]
            self._check(self._lib.mfgpu_solve_f32(self._h, nrhs, L.ptr(B, L.f32p), L.ptr(X, L.f32p), int(refine)))
            return X
        B = np.asfortranarray(b, dtype=np.float64)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        X = np.empty_like(B)
        n = B.shape[0]
        self._check(self._lib.mfgpu_solve(self._h, nrhs, L.ptr(B, L.f64p), n, L.ptr(X, L.f64p), n, int(refine)))
        return X

    def factor_solve(self, nzval, Rs, b, refine: int = 0, check: bool = True):
        """factor(nzval, Rs) then solve(b, refine) in one call, the
        right-hand sides' copy overlapped with the factorization.  Returns
        (status, x); x is None when the factorization found a singular column."""
        self._values(nzval, Rs)
        rs = _f(Rs) if Rs is not None else None
        B = np.asfortranarray(b, dtype=np.float64)
        nrhs = 1 if B.ndim == 1 else B.shape[1]
        X = np.empty_like(B)
        self.f32 = self.c64 = False
        st = self._check(self._lib.mfgpu_factor_solve(self._h, L.ptr(_f(nzval), L.f64p), L.ptr(rs, L.f64p),
                                                      int(check), nrhs, L.ptr(B, L.f64p), B.shape[0],
                                                      L.ptr(X, L.f64p), B.shape[0], int(refine)))
        return st, (X if st == 0 else None)

    def solve_device(self, nrhs: int, b_ptr: int, ldb: int, x_ptr: int, ldx: int, refine: int = 0):
        self._check(self._lib.mfgpu_solve_device(self._h, nrhs, ctypes.c_void_p(b_ptr), ldb, ctypes.c_void_p(x_ptr),
                                                 ldx, int(refine)))

    def backward_error_device(self, nrhs: int, b_ptr: int, ldb: int, x_ptr: int, ldx: int) -> float:
        out = ctypes.c_double()
        self._check(self._lib.mfgpu_backward_error_device(self._h, nrhs, ctypes.c_void_p(b_ptr), ldb,
                                                          ctypes.c_void_p(x_ptr), ldx, ctypes.byref(out)))
        return out.value

    def stats(self) -> dict:
        buf = ctypes.create_string_buffer(16384)
        self._check(self._lib.mfgpu_stats_json(self._h, buf, 16384))
        return json.loads(buf.value.decode())

    def set_profiling(self, on: bool):
        self._check(self._lib.mfgpu_set_profiling(self._h, int(bool(on))))

    def launch_records(self) -> list:
        """Profiled launches: [kernel class, level, tasks, ms, flops, bytes,
        tunable GEMM index or -1]."""
        cap = 1 << 20
        while True:
            buf = ctypes.create_string_buffer(cap)
            rc = self._lib.mfgpu_launch_records(self._h, buf, cap)
            if rc == 0:
                return json.loads(buf.value.decode())
            if rc < 0:
                self._check(rc)
            cap = rc + 16

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                self._lib.mfgpu_destroy(self._h)
            except Exception:
                pass
            self._h = None


# ---------------------------------------------------------------------------
# factorization objects
# ---------------------------------------------------------------------------
class _Factors:
    """Lazily copied CSC factors of a GPU factorization."""

    def __init__(self, ctx: GpuContext):
        self._ctx = ctx
        self._cache = None

    def _get(self):
        if self._cache is None:
            self._cache = self._ctx.factors()
        return self._cache


class GPLUFactorization:
    """src/gplu.jl:45-51: A[p, q] == L * U (factors resident on the GPU)."""

    def __init__(self, ctx: GpuContext, symbolic: SymbolicMF | None = None):
        self.ctx = ctx
        self.symbolic = symbolic
        self._f = _Factors(ctx)

    L = property(lambda self: self._f._get()[0])
    U = property(lambda self: self._f._get()[1])
    p = property(lambda self: self._f._get()[2])
    q = property(lambda self: self._f._get()[3])
    pinv = property(lambda self: self._f._get()[4])

    def size(self, i: int | None = None):
        s = (self.ctx.n, self.ctx.n)
        return s if i is None else s[i - 1]

    def ldiv(self, b):
        """F \\ b (src/solve.jl:66-79): no scaling, no refinement."""
        return self.ctx.solve(b, 0)


class PureLU:
    """src/interface.jl:38-48: (Rs .* A)[p, q] == L * U."""

    def __init__(self, ctx: GpuContext, Rs: np.ndarray, A: SparseCSC, symbolic: SymbolicMF | None = None):
        self.ctx = ctx
        self.Rs = Rs
        self.A = A
        self.symbolic = symbolic
        self._f = _Factors(ctx)

    L = property(lambda self: self._f._get()[0])
    U = property(lambda self: self._f._get()[1])
    p = property(lambda self: self._f._get()[2])
    q = property(lambda self: self._f._get()[3])

    def size(self, i: int | None = None):
        s = (self.A.n, self.A.n)
        return s if i is None else s[i - 1]

    def ldiv(self, b):
        """F \\ b = solve(F, b) with refine = 0 (src/interface.jl:179)."""
        return solve(self, b)


def _factor(A: SparseCSC, q, check: bool, Rs, device: int, precision: int, relax: bool = False):
    S = symbolic_mf(A, q=q, relax=relax)
    ctx = GpuContext(device=device, precision=precision)
    ctx.analyze(A, S)
    # a Float32 (ComplexF64) matrix is factored in Float32 (ComplexF64), the
    # reference's generic Tv
    fac = (ctx.factor_c64 if np.iscomplexobj(A.nzval) else
           ctx.factor_f32 if A.nzval.dtype == np.float32 else ctx.factor)
    status = fac(A.nzval, Rs, check)
    if status > 0:
        raise SingularException(status)
    return ctx, S


def multifrontal_lu(A: SparseCSC, q=None, tol=None, check: bool = True, device: int = 0,
                    precision: int = PRECISION_FP64) -> GPLUFactorization:
    """Supernodal multifrontal LU of A as given (no scaling); ``tol`` is
    accepted and ignored, as in the reference (src/multifrontal.jl:121,147)."""
    if A.m != A.n:
        raise DimensionMismatch("multifrontal_lu requires a square matrix")
    ctx, S = _factor(A, q, check, None, device, precision)
    return GPLUFactorization(ctx, S)


def splu(A: SparseCSC, method: str = "gplu", ordering: str = "amd", tol: float = 0.1, scale=SCALE_SUM,
         check: bool = True, device: int = 0, precision: int = PRECISION_FP64, relax: bool = False) -> PureLU:
    """splu(A; method, ordering, tol, scale, check) (src/interface.jl:93-120).

    ``method="multifrontal"`` factors with the multifrontal kernels; as in
    the reference it ignores ``ordering`` and ``tol`` (AMD + postorder).
    ``method="gplu"`` (the reference's default) orders the columns by
    ``ordering`` (``"amd"``, ``"colamd"`` or ``"natural"``) and runs the
    Gilbert-Peierls factorization on the GPU with threshold ``tol``
    (``gplu``): the reference's exact results, but a chain of column steps
    that one warp runs, far slower than ``method="multifrontal"`` on large
    systems.  ``precision`` and ``relax`` apply to the multifrontal method.
    """
    method = method.lstrip(":") if isinstance(method, str) else method
    if A.m != A.n:
        raise DimensionMismatch("splu requires a square matrix")
    scale = ScaleKind(int(scale))
    if method == "multifrontal":
        Rs = row_scaling(A, scale)
        ctx, S = _factor(A, None, check, None if scale == SCALE_NONE else Rs, device, precision, relax)
        return PureLU(ctx, Rs, A, S)
    if method != "gplu":
        raise ArgumentError(f"unknown method {method}")
    if ordering == "natural":
        q = np.arange(1, A.n + 1, dtype=np.int64)
    elif ordering == "amd":
        q = amd_order_sym(A)
    elif ordering == "colamd":
        q = colamd_order(A)
    else:
        raise ArgumentError(f"unknown ordering {ordering}")
    Rs = row_scaling(A, scale)
    ctx = GpluContext(device)
    st = ctx.factor([A], [q], None if scale == SCALE_NONE else [Rs], tol=tol, check=check)
    if st[0] > 0:
        raise SingularException(int(st[0]))
    return PureLU(ctx, Rs, A)


def splu_q(A: SparseCSC, q, scale=SCALE_SUM, check: bool = True, device: int = 0,
           precision: int = PRECISION_FP64) -> PureLU:
    """``PureLU`` of ``multifrontal_lu(apply_row_scaling(A, Rs); q)`` -- the
    route by which a COLAMD (or any caller) order reaches the multifrontal
    kernel in the reference (src/multifrontal.jl:152)."""
    scale = ScaleKind(int(scale))
    Rs = row_scaling(A, scale)
    ctx, S = _factor(A, q, check, None if scale == SCALE_NONE else Rs, device, precision)
    return PureLU(ctx, Rs, A, S)


# ---------------------------------------------------------------------------
# Gilbert-Peierls LU (src/gplu.jl)
# ---------------------------------------------------------------------------
class GpluContext:
    """One libmfgpu Gilbert-Peierls handle: the factors of one or many
    independent systems, resident on the GPU (one warp factors one system)."""

    def __init__(self, device: int = 0):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.mfgpu_gplu_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise MfgpuError(rc, "mfgpu_gplu_create failed (needs a B200 / sm_100 device)")
        self._h = h
        self.n = 0
        self.sizes = []

    def _check(self, rc: int):
        if rc < 0:
            msg = self._lib.mfgpu_gplu_last_error(self._h).decode()
            if rc == -1:
                raise ArgumentError(msg)
            if rc == -6:
                raise DimensionMismatch(msg)
            raise MfgpuError(rc, msg)
        return rc

    def set_initial_capacity(self, entries: int):
        """Entries of L and of U each system gets before it first overflows
        (0: sized from the symbolic fill)."""
        self._check(self._lib.mfgpu_gplu_set_initial_capacity(self._h, int(entries)))

    def factor(self, As, qs=None, Rs=None, tol: float = 0.1, check: bool = True,
               sort_factors: bool = True) -> np.ndarray:
        """gplu(Rs_i .* A_i; q = qs[i], tol, check, sort_factors) for every
        system; returns the per-system status (0, or the singular column).
        The values' type (Float64, Float32 or ComplexF64, the same for every
        system) is the arithmetic's, as the reference's generic Tv."""
        for A in As:
            if A.m != A.n:
                raise DimensionMismatch("gplu requires a square matrix")
        for arrs, what in ((qs, "q"), (Rs, "Rs")):
            if arrs is None:
                continue
            if len(arrs) != len(As):
                raise DimensionMismatch(f"one {what} per system")
            for A, a in zip(As, arrs):
                if a is not None and len(a) != A.n:
                    raise DimensionMismatch(f"length({what}) must equal size(A, 1)")
        kind = ("c64" if np.iscomplexobj(As[0].nzval) else "f32" if As[0].nzval.dtype == np.float32 else "f64") \
            if As else "f64"
        for A in As:
            k = "c64" if np.iscomplexobj(A.nzval) else "f32" if A.nzval.dtype == np.float32 else "f64"
            if k != kind:
                raise ArgumentError("every system of a batch needs the same element type")
        vt = {"f64": np.float64, "f32": np.float32, "c64": np.complex128}[kind]
        rt = np.float32 if kind == "f32" else np.float64
        cps = [_i(A.colptr) for A in As]
        rvs = [_i(A.rowval) for A in As]
        nzs = [np.ascontiguousarray(A.nzval, dtype=vt) for A in As]
        n = np.array([A.n for A in As], np.int64)
        qa = None if qs is None else [_i(q) if q is not None else None for q in qs]
        ra = None if Rs is None else [np.ascontiguousarray(r, dtype=rt) if r is not None else None for r in Rs]

        def parr(arrs):
            if arrs is None:
                return None
            return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data if a is not None else None for a in arrs])

        fn = {"f64": self._lib.mfgpu_gplu_factor, "f32": self._lib.mfgpu_gplu_factor_f32,
              "c64": self._lib.mfgpu_gplu_factor_c64}[kind]
        status = np.zeros(len(As), np.int64)
        self._check(fn(self._h, len(As), L.ptr(n), parr(cps), parr(rvs), parr(nzs), parr(qa), parr(ra), float(tol),
                       int(bool(check)), int(bool(sort_factors)), L.ptr(status)))
        self.kind = kind
        self.sizes = [A.n for A in As]
        self.n = As[0].n if len(As) == 1 else 0
        return status

    def factors(self, sys: int = 0):
        """(L, U, p, q, pinv) of system sys: A_i[p, q] == L * U, values in
        the factored element type."""
        sz = np.empty(3, np.int64)
        self._check(self._lib.mfgpu_gplu_sizes(self._h, int(sys), L.ptr(sz)))
        n, nl, nu = (int(v) for v in sz)
        kind = getattr(self, "kind", "f64")
        vt = {"f64": np.float64, "f32": np.float32, "c64": np.complex128}[kind]
        Lp, Li, Lx = np.empty(n + 1, np.int64), np.empty(nl, np.int64), np.empty(nl, vt)
        Up, Ui, Ux = np.empty(n + 1, np.int64), np.empty(nu, np.int64), np.empty(nu, vt)
        p, q, pinv = np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64)
        fn, vp = {"f64": (self._lib.mfgpu_gplu_get_factors, L.f64p),
                  "f32": (self._lib.mfgpu_gplu_get_factors_f32, L.f32p),
                  "c64": (self._lib.mfgpu_gplu_get_factors_c64, L.f64p)}[kind]
        lx = Lx.view(np.float64) if kind == "c64" else Lx
        ux = Ux.view(np.float64) if kind == "c64" else Ux
        self._check(fn(self._h, int(sys), L.ptr(Lp), L.ptr(Li), L.ptr(lx, vp), L.ptr(Up), L.ptr(Ui), L.ptr(ux, vp),
                       L.ptr(p), L.ptr(q), L.ptr(pinv)))
        return SparseCSC(n, n, Lp, Li, Lx), SparseCSC(n, n, Up, Ui, Ux), p, q, pinv

    def solve_batch(self, Bs, refine: int = 0):
        """x_i for every system's b_i (vectors, or n_i x k with one k), in
        the factored element type."""
        kind = getattr(self, "kind", "f64")
        vt = {"f64": np.float64, "f32": np.float32, "c64": np.complex128}[kind]
        Bs = [np.asfortranarray(b, dtype=vt) for b in Bs]
        if len(Bs) != len(self.sizes):
            raise DimensionMismatch("one right-hand side block per system")
        k = 1 if Bs[0].ndim == 1 else Bs[0].shape[1]
        for n, b in zip(self.sizes, Bs):
            if b.shape[0] != n or (1 if b.ndim == 1 else b.shape[1]) != k:
                raise DimensionMismatch("right-hand side block does not match its system")
        Xs = [np.empty_like(b) for b in Bs]
        fn = {"f64": self._lib.mfgpu_gplu_solve, "f32": self._lib.mfgpu_gplu_solve_f32,
              "c64": self._lib.mfgpu_gplu_solve_c64}[kind]
        self._check(fn(self._h, k, L.ptr_array(Bs), L.ptr_array(Xs), int(refine)))
        return Xs

    def solve(self, b, refine: int = 0) -> np.ndarray:
        """The single system's solve(F, b; refine); b a vector or n x k."""
        return self.solve_batch([b], refine)[0]

    def timings(self) -> dict:
        out = np.zeros(5)
        self._check(self._lib.mfgpu_gplu_timings(self._h, L.ptr(out, L.f64p)))
        return {"factor_ms": out[0], "finish_ms": out[1], "solve_ms": out[2], "factor_launches": int(out[3]),
                "reruns": int(out[4])}

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                self._lib.mfgpu_gplu_destroy(self._h)
            except Exception:
                pass
            self._h = None


def gplu(A: SparseCSC, q=None, tol: float = 0.1, check: bool = True, sort_factors: bool = True,
         device: int = 0) -> GPLUFactorization:
    """gplu(A; q, tol, check, sort_factors) (src/gplu.jl:173-303) on the GPU:
    A[p, q] == L * U with threshold partial pivoting; factors, pivots and
    F \\ b are bit for bit the reference's."""
    if A.m != A.n:
        raise DimensionMismatch("gplu requires a square matrix")
    ctx = GpluContext(device)
    st = ctx.factor([A], None if q is None else [q], None, tol=tol, check=check, sort_factors=sort_factors)
    if st[0] > 0:
        raise SingularException(int(st[0]))
    return GPLUFactorization(ctx)


class BatchGPLU:
    """splu(A_i; method=:gplu, ordering, tol, scale) of many independent
    systems in one call: one warp per system, all systems side by side."""

    def __init__(self, As, ordering: str = "amd", tol: float = 0.1, scale=SCALE_SUM, check: bool = True,
                 device: int = 0, initial_capacity: int = 0):
        self.As = list(As)
        order = {"natural": lambda A: np.arange(1, A.n + 1, dtype=np.int64), "amd": amd_order_sym,
                 "colamd": colamd_order}
        if ordering not in order:
            raise ArgumentError(f"unknown ordering {ordering}")
        scale = ScaleKind(int(scale))
        # the host orderings and scalings of the systems, side by side (the
        # library's host code releases the interpreter and keeps no shared state)
        with ThreadPoolExecutor(max_workers=max(1, min(len(self.As), os.cpu_count() or 1))) as ex:
            qs = list(ex.map(order[ordering], self.As))
            self.Rs = list(ex.map(lambda A: row_scaling(A, scale), self.As))
        self.ctx = GpluContext(device)
        if initial_capacity:
            self.ctx.set_initial_capacity(initial_capacity)
        self.status = self.ctx.factor(self.As, qs, None if scale == SCALE_NONE else self.Rs, tol=tol, check=check)

    def __len__(self):
        return len(self.As)

    def solve(self, Bs, refine: int = 0):
        return self.ctx.solve_batch(Bs, refine)

    def factors(self, i: int):
        """(L, U, p, q, pinv) of system i: (Rs_i .* A_i)[p, q] == L * U."""
        return self.ctx.factors(i)


# ---------------------------------------------------------------------------
# batched systems
# ---------------------------------------------------------------------------
ORDER_AMD = 0
ORDER_COLAMD = 1


class BatchLU:
    """Factors of many independent systems held by one GPU handle.

    System ``i`` behaves as ``splu(As[i]; method=:multifrontal, scale)``
    (src/interface.jl:93-120), or with ``ordering="colamd"`` as
    ``multifrontal_lu(Rs .* As[i]; q=colamd_order(As[i]))``
    (src/multifrontal.jl:152); all systems are factored by one launch
    sequence whose level-batched kernels take the fronts of every system at a
    tree level together."""

    def __init__(self, ctx: GpuContext, As, Rs, status):
        self.ctx = ctx
        self.As = list(As)
        self.Rs = Rs
        self.status = status
        nsys = ctypes.c_int64()
        col_off = np.empty(len(self.As) + 1, np.int64)
        nz_off = np.empty(len(self.As) + 1, np.int64)
        ctx._check(ctx._lib.mfgpu_batch_layout(ctx._h, ctypes.byref(nsys), L.ptr(col_off), L.ptr(nz_off)))
        self.col_off, self.nz_off = col_off, nz_off

    def __len__(self):
        return len(self.As)

    def solve(self, Bs, refine: int = 0):
        """solve(F_i, b_i; refine) for every system; each b_i is a vector or
        an n_i x k matrix with the same k for all systems."""
        Bs = [np.asfortranarray(b, dtype=np.float64) for b in Bs]
        if len(Bs) != len(self.As):
            raise DimensionMismatch("one right-hand side block per system")
        k = 1 if Bs[0].ndim == 1 else Bs[0].shape[1]
        for A, b in zip(self.As, Bs):
            if b.shape[0] != A.n or (1 if b.ndim == 1 else b.shape[1]) != k:
                raise DimensionMismatch("right-hand side block does not match its system")
        Xs = [np.empty_like(b) for b in Bs]
        self.ctx._check(self.ctx._lib.mfgpu_batch_solve(self.ctx._h, k, L.ptr_array(Bs), L.ptr_array(Xs),
                                                        int(refine)))
        return Xs

    def factors(self, i: int):
        """(L, U, p, q, pinv) of system i: (Rs_i .* A_i)[p, q] == L * U."""
        ctx = self.ctx
        sz = np.empty(3, np.int64)
        ctx._check(ctx._lib.mfgpu_batch_factor_sizes(ctx._h, int(i), L.ptr(sz)))
        n, nl, nu = (int(v) for v in sz)
        Lp, Li, Lx = np.empty(n + 1, np.int64), np.empty(nl, np.int64), np.empty(nl)
        Up, Ui, Ux = np.empty(n + 1, np.int64), np.empty(nu, np.int64), np.empty(nu)
        p, q, pinv = np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64)
        ctx._check(ctx._lib.mfgpu_batch_get_factors(ctx._h, int(i), L.ptr(Lp), L.ptr(Li), L.ptr(Lx, L.f64p),
                                                    L.ptr(Up), L.ptr(Ui), L.ptr(Ux, L.f64p), L.ptr(p), L.ptr(q),
                                                    L.ptr(pinv)))
        return SparseCSC(n, n, Lp, Li, Lx), SparseCSC(n, n, Up, Ui, Ux), p, q, pinv


def analyze_batch(As, ordering: str = "amd", device: int = 0, precision: int = PRECISION_FP64) -> GpuContext:
    """A GPU handle analyzed for the systems ``As`` (patterns only)."""
    As = list(As)
    if not As:
        raise ArgumentError("empty batch")
    for A in As:
        if A.m != A.n:
            raise DimensionMismatch("every system of a batch must be square")
    order = {"amd": ORDER_AMD, "colamd": ORDER_COLAMD}.get(str(ordering).lstrip(":"))
    if order is None:
        raise ArgumentError(f"unknown ordering {ordering}")
    ctx = GpuContext(device=device, precision=precision)
    ns = np.array([A.n for A in As], np.int64)
    cps = [_i(A.colptr) for A in As]
    rvs = [_i(A.rowval) if A.nnz() else np.ones(1, np.int64) for A in As]
    ctx._check(ctx._lib.mfgpu_batch_analyze(ctx._h, len(As), L.ptr(ns), L.ptr_array(cps), L.ptr_array(rvs), order))
    ctx.n = int(ns.sum())
    return ctx


def splu_batch(As, scale=SCALE_SUM, ordering: str = "amd", check: bool = True, device: int = 0,
               precision: int = PRECISION_FP64, ctx: GpuContext | None = None) -> BatchLU:
    """Factor many independent systems in one batched call.  With ``check``
    a singular system raises SingularException for the first such system
    (``BatchLU.status`` lists every system's first singular column)."""
    As = list(As)
    scale = ScaleKind(int(scale))
    if ctx is None:
        ctx = analyze_batch(As, ordering, device, precision)
    status = np.zeros(len(As), np.int64)
    vals = [_f(A.nzval) if A.nnz() else np.zeros(1) for A in As]
    ctx._check(ctx._lib.mfgpu_batch_factor(ctx._h, L.ptr_array(vals), int(scale), 0, L.ptr(status)))
    if check and np.any(status):
        raise SingularException(int(status[np.flatnonzero(status)[0]]))
    Rs = [row_scaling(A, scale) for A in As]
    return BatchLU(ctx, As, Rs, status)


def solve(F, b, refine: int = 0) -> np.ndarray:
    """solve(F::PureLU, b; refine) (src/interface.jl:170-177): x = F \\ b, then
    ``refine`` steps of x += F \\ (b - A x) with the unscaled A, all on the GPU.
    ``b`` may be a vector or an n x k matrix (k right-hand sides)."""
    if isinstance(F, GPLUFactorization):
        if refine:
            raise ArgumentError("refinement needs a PureLU (it keeps A and Rs)")
        return F.ldiv(b)
    dt = np.complex128 if np.iscomplexobj(F.A.nzval) else (np.float32 if F.A.nzval.dtype == np.float32 else np.float64)
    b = np.asarray(b, dtype=dt)
    if b.shape[0] != F.A.n:
        raise DimensionMismatch("length(b) must equal size(F, 1)")
    return F.ctx.solve(b, refine)
