"""pureumfpack -- B200 multifrontal sparse LU behind PureUMFPACK.jl's API.

The numeric multifrontal factorization, the Gilbert-Peierls factorization
and the triangular solves of PureUMFPACK.jl run on one B200 through libmfgpu.so (hand-written sm_100a
kernels behind a C ABI, include/mfgpu.h).  This package is the host side:
the reference's entry points with the same names, arguments and errors.
"""

from .api import (
    PRECISION_FP64,
    PRECISION_MIXED,
    SCALE_MAX,
    SCALE_NONE,
    SCALE_SUM,
    ArgumentError,
    BatchGPLU,
    BatchLU,
    DimensionMismatch,
    GPLUFactorization,
    GpluContext,
    GpuContext,
    MfgpuError,
    PureLU,
    ScaleKind,
    SingularException,
    SymbolicMF,
    amd_order_sym,
    analyze_batch,
    apply_row_scaling,
    colamd_order,
    gplu,
    multifrontal_lu,
    predicted_fill,
    row_scaling,
    solve,
    splu,
    splu_batch,
    splu_q,
    symbolic_mf,
)
from .sparse import SparseCSC

__all__ = [
    "PRECISION_FP64", "PRECISION_MIXED", "SCALE_MAX", "SCALE_NONE", "SCALE_SUM", "ArgumentError", "BatchGPLU",
    "BatchLU", "DimensionMismatch", "GPLUFactorization", "GpluContext", "GpuContext", "MfgpuError", "PureLU", "ScaleKind",
    "SingularException", "SymbolicMF", "SparseCSC", "amd_order_sym", "analyze_batch", "apply_row_scaling", "colamd_order",
    "gplu", "multifrontal_lu", "predicted_fill", "row_scaling", "solve", "splu", "splu_batch", "splu_q", "symbolic_mf",
]
