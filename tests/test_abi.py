"""The C ABI library loads on a host without a GPU and exports every symbol
declared in include/mfgpu.h; GPU entry points fail cleanly without a device."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mfgpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mfgpu_\w+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("mfgpu_create", "mfgpu_analyze", "mfgpu_factor", "mfgpu_get_factors", "mfgpu_solve",
                 "mfgpu_destroy", "mfgpu_amd_order", "mfgpu_symbolic_create"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from pureumfpack import _lib

    L = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared_functions()) == bound


def test_gpu_entry_points_fail_cleanly_without_device(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    from pureumfpack import _lib

    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.mfgpu_create(None, ctypes.byref(h))
    assert rc == -8 and not h.value
    assert L.mfgpu_factor(None, None, None, 1) == -1
    assert L.mfgpu_solve(None, 1, None, 1, None, 1, 0) == -1


def test_gplu_entry_points_fail_cleanly_without_device(has_gpu):
    """The Gilbert-Peierls handle needs a B200; without one it is refused and
    the Python entry points raise instead of computing anywhere else."""
    if has_gpu:
        pytest.skip("a GPU is present")
    from pureumfpack import MfgpuError, SparseCSC, _lib, gplu, splu

    L = _lib.lib()
    g = ctypes.c_void_p()
    assert L.mfgpu_gplu_create(0, ctypes.byref(g)) == -8 and not g.value
    assert L.mfgpu_gplu_create(0, None) == -1
    assert L.mfgpu_gplu_factor(None, 0, None, None, None, None, None, None, 0.1, 1, 1, None) == -1
    assert L.mfgpu_gplu_solve(None, 1, None, None, 0) == -1
    assert L.mfgpu_gplu_solve_c64(None, 1, None, None, 0) == -1
    A = SparseCSC.from_coo([1, 2], [1, 2], [2.0, 3.0], 2, 2)
    with pytest.raises(MfgpuError):
        gplu(A)
    with pytest.raises(MfgpuError):
        splu(A)   # the default method is :gplu


def test_gplu_wrapper_checks_lengths_before_the_library():
    """q and Rs reach the C ABI as bare pointers, so the Python wrapper
    checks their lengths first (DimensionMismatch, no library call)."""
    import numpy as np

    from pureumfpack import DimensionMismatch, SparseCSC
    from pureumfpack.api import GpluContext

    A = SparseCSC.from_coo([1, 2, 3], [1, 2, 3], [1.0, 2.0, 3.0], 3, 3)
    ctx = GpluContext.__new__(GpluContext)   # no device needed: the checks come first
    with pytest.raises(DimensionMismatch):
        ctx.factor([A], [np.array([1, 2])])
    with pytest.raises(DimensionMismatch):
        ctx.factor([A], None, [np.ones(2)])
    with pytest.raises(DimensionMismatch):
        ctx.factor([A, A], [np.array([1, 2, 3])])


def test_factor_wrapper_checks_value_lengths():
    """The factor calls copy nnz values and n row factors from bare
    pointers; the Python wrapper checks both against the analyzed pattern."""
    import numpy as np

    from pureumfpack import DimensionMismatch, GpuContext

    ctx = GpuContext.__new__(GpuContext)   # no device needed: the checks come first
    ctx.n, ctx.nnz = 3, 7
    ctx._values(np.ones(7), np.ones(3))
    with pytest.raises(DimensionMismatch):
        ctx._values(np.ones(6), None)
    with pytest.raises(DimensionMismatch):
        ctx._values(np.ones(7), np.ones(2))
    for call in (ctx.factor, ctx.factor_f32, ctx.factor_c64):
        with pytest.raises(DimensionMismatch):
            call(np.ones(5), None)
