"""GPU parity of the numeric multifrontal factorization against the oracle.

Mirrors test/multifrontal_test.jl of the reference: structure (fill, L/U
patterns, permutations) must be bit-identical to the oracle's restatement of
multifrontal_lu; values agree to 1e-12 (tests/helpers.py states the rule);
reconstruction A[p,q] = L U holds to 1e-9 * max(1, ||A||_F).  Everything is
called through libmfgpu's C ABI.
"""

import numpy as np
import pytest

from helpers import assert_close_values, assert_same_structure, reconstruction_error
from oracle import oracle as O
from pureumfpack import (
    SCALE_MAX,
    SCALE_NONE,
    SCALE_SUM,
    SingularException,
    SparseCSC,
    apply_row_scaling,
    colamd_order,
    multifrontal_lu,
    row_scaling,
    splu,
    splu_q,
)
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def spd6():
    rng = np.random.default_rng(2024)
    X = rng.standard_normal((6, 6))
    return SparseCSC.from_scipy(__import__("scipy.sparse", fromlist=["csc_matrix"]).csc_matrix(X @ X.T + 6 * np.eye(6)))


CASES = [
    ("spd6", spd6),
    ("poisson2d-8", lambda: M.poisson2d(8)),
    ("poisson2d-24", lambda: M.poisson2d(24)),
    ("poisson2d-100", lambda: M.poisson2d(100)),
    ("poisson3d-6", lambda: M.poisson3d(6)),
    ("poisson3d-10", lambda: M.poisson3d(10)),
    ("poisson3d-16", lambda: M.poisson3d(16)),
    ("randmat-500", lambda: M.randmat(500, 6)),
    ("arrowband-400", lambda: M.arrowband(400, 4)),
    ("convdiff-10", lambda: M.convdiff3d(10)),
    ("random-2000", lambda: M.random_unsym(2000, 5, 10.0, seed=3)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_multifrontal_lu_matches_oracle(name, make):
    A = make()
    fo = O.multifrontal_lu(A, check=False)
    F = multifrontal_lu(A, check=False)
    L, U, p, q, pinv = F.L, F.U, F.p, F.q, F.pinv
    assert_same_structure(fo, L, U, p, q, pinv)
    assert_close_values(fo, L, U)
    assert reconstruction_error(A, L, U, p, q) <= 1e-9
    # unit lower L with its diagonal first, U upper with its diagonal last
    assert np.all(L.nzval[L.colptr[:-1] - 1] == 1.0)
    assert np.all(L.rowval[L.colptr[:-1] - 1] == np.arange(1, A.n + 1))
    assert np.all(U.rowval[U.colptr[1:] - 2] == np.arange(1, A.n + 1))


@pytest.mark.parametrize("scale", [SCALE_NONE, SCALE_SUM, SCALE_MAX])
def test_splu_scaled_factors(scale):
    A = M.convdiff3d(8)
    Rs = O.row_scaling(A, int(scale))
    As = A if scale == SCALE_NONE else O.apply_row_scaling(A, Rs)
    fo = O.multifrontal_lu(As, check=False)
    F = splu(A, method="multifrontal", scale=scale, check=False)
    np.testing.assert_array_equal(F.Rs, Rs)
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert_close_values(fo, F.L, F.U)
    assert reconstruction_error(A, F.L, F.U, F.p, F.q, Rs=F.Rs) <= 1e-9


def test_colamd_route():
    """multifrontal_lu(As; q=colamd_order(A)): the COLAMD path (multifrontal.jl:152)."""
    A = M.random_unsym(3000, 5, 10.0, seed=7)
    qc = colamd_order(A)
    np.testing.assert_array_equal(qc, O.colamd_order(A))
    Rs = O.row_scaling(A, 2)
    fo = O.multifrontal_lu(O.apply_row_scaling(A, Rs), q=qc, check=False)
    F = splu_q(A, qc, scale=SCALE_MAX, check=False)
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert_close_values(fo, F.L, F.U)


@pytest.mark.parametrize("k,off", [(12, 0.5), (16, 0.4)])
def test_pivoting_in_large_fronts(k, off):
    """Random values on a 3-D grid pattern: row interchanges inside the pivot
    blocks of large fronts (shared-memory panels; at k=16 the top pivot block
    has 298 rows, so the speculative panel meets a larger row and the
    factorization is redone with global-memory partial pivoting)."""
    A = M.grid3d_random(k, off, seed=1)
    fo = O.multifrontal_lu(A, check=False)
    F = multifrontal_lu(A, check=False)
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F.pinv)
    # element growth max|U| / max|A| is about 5 (k=12) and 30 (k=14-16) here
    assert_close_values(fo, F.L, F.U, entry_rtol=1e-10)
    assert np.sum(F.p != F.q) > 5, "case meant to exercise row interchanges"
    # partial pivoting inside the blocks: |L11| <= 1
    S = F.symbolic
    sup_last = np.repeat(S.sstart[1:] - 1, np.diff(S.sstart))
    cols = np.repeat(np.arange(1, A.n + 1), np.diff(F.L.colptr))
    inblock = (F.L.rowval > cols) & (F.L.rowval <= sup_last[cols - 1])
    assert np.max(np.abs(F.L.nzval[inblock])) <= 1.0


def test_pivoting_small_fronts_fixture():
    """Committed oracle fixture with interchanges in small fronts."""
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "factors.npz"))
    name = "pivoting-200"
    A = SparseCSC(int(d[name + "/n"]), int(d[name + "/n"]), d[name + "/colptr"], d[name + "/rowval"],
                  d[name + "/nzval"])
    F = multifrontal_lu(A, check=False)
    np.testing.assert_array_equal(F.L.rowval, d[name + "/Lrowval"])
    np.testing.assert_array_equal(F.U.rowval, d[name + "/Urowval"])
    np.testing.assert_array_equal(F.p, d[name + "/p"])
    # ill-conditioned (shift 0.3): growth amplifies rounding; normwise 1e-9
    from helpers import column_value_errors

    assert column_value_errors(np.asarray(F.L.colptr), d[name + "/Lnzval"], F.L.nzval)[0] <= 1e-9
    assert column_value_errors(np.asarray(F.U.colptr), d[name + "/Unzval"], F.U.nzval)[0] <= 1e-9


def test_singular_exception_column():
    # structurally nonsingular, numerically singular: a stored zero diagonal
    A = SparseCSC.from_coo([1, 2, 3, 4, 1], [1, 2, 3, 4, 2], [2.0, 3.0, 0.0, 7.0, 1.0], 4, 4)
    with pytest.raises(O.SingularException) as eo:
        O.multifrontal_lu(A, check=True)
    with pytest.raises(SingularException) as eg:
        multifrontal_lu(A, check=True)
    assert eg.value.info == eo.value.info


def test_edge_cases():
    # test/multifrontal_test.jl:77-83
    F = splu(SparseCSC.from_coo([1], [1], [4.0], 1, 1), method="multifrontal")
    assert np.allclose(F.ldiv(np.array([8.0])), [2.0])
    D = SparseCSC.from_coo([1, 2, 3, 4], [1, 2, 3, 4], [2.0, 3.0, 5.0, 7.0], 4, 4)
    x = splu(D, method="multifrontal").ldiv(np.array([2.0, 6.0, 15.0, 28.0]))
    assert np.allclose(x, [1.0, 2.0, 3.0, 4.0])
    from pureumfpack import ArgumentError, DimensionMismatch

    with pytest.raises(ArgumentError):
        splu(D, method="nonsense")
    with pytest.raises(DimensionMismatch):
        splu(SparseCSC.from_coo([1, 2], [1, 1], [1.0, 1.0], 2, 1), method="multifrontal")


def test_doctest_known_answer():
    # src/multifrontal.jl:138-144, src/interface.jl:85-91
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [2.0, 1.0, 1.0, 2.0], 2, 2)
    x = multifrontal_lu(A).ldiv(np.array([1.0, 0.0]))
    assert np.allclose(x, [0.6666666666666666, -0.3333333333333333], rtol=0, atol=1e-16)
    x = splu(A, method="multifrontal").ldiv(np.array([1.0, 0.0]))
    assert np.allclose(x, [0.6666666666666666, -0.3333333333333333], rtol=0, atol=1e-16)


@pytest.mark.parametrize("scale", [SCALE_NONE, SCALE_SUM, SCALE_MAX])
def test_device_row_scaling_is_bitwise_the_host_one(scale):
    """mfgpu_factor_scaled computes Rs on the device in the host's summation
    order: Rs and the factors equal the host-scaled factorization exactly."""
    from pureumfpack import GpuContext, symbolic_mf

    A = M.convdiff3d(9)
    S = symbolic_mf(A)
    Rs = row_scaling(A, scale)
    host = GpuContext()
    host.analyze(A, S)
    assert host.factor(A.nzval, None if scale == SCALE_NONE else Rs, True) == 0
    dev = GpuContext()
    dev.analyze(A, S)
    assert dev.factor_scaled(A.nzval, scale, True) == 0
    np.testing.assert_array_equal(dev.row_scaling(), Rs if scale != SCALE_NONE else np.ones(A.n))
    L0, U0 = host.factors()[:2]
    L1, U1 = dev.factors()[:2]
    np.testing.assert_array_equal(L1.nzval, L0.nzval)
    np.testing.assert_array_equal(U1.nzval, U0.nzval)
