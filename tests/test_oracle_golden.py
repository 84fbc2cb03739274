"""The oracle against the reference's golden values (CPU).

Pins: the published fill counts of AMD + symbolic analysis
(results/SUMMARY.md:32-36,56), the published supernode counts
(results/SCALING_DIAGNOSIS.md:24-26), the doctests of src/scaling.jl:86-90
and src/multifrontal.jl:138-144, and the reconstruction / residual bounds of
test/multifrontal_test.jl.  The committed fixtures in tests/golden/ hold these
values with their sources.
"""

import json
import os

import numpy as np
import pytest

from helpers import reconstruction_error
from oracle import oracle as O
from pureumfpack import SparseCSC
from pureumfpack import matrices as M

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat.json")))


@pytest.mark.parametrize("case", GOLDEN["fill"], ids=[c["matrix"] for c in GOLDEN["fill"]])
def test_published_fill(case):
    kind, k = case["matrix"].split("-")
    A = (M.poisson2d if kind == "poisson2d" else M.poisson3d)(int(k))
    S = O.symbolic_mf(A)
    assert O.predicted_fill(S) == case["fill"]
    if "nsuper" in case:
        assert S.nsuper == case["nsuper"]


def test_scaling_doctest():
    A = SparseCSC.from_coo([1, 1, 2], [1, 2, 2], [1.0, 2.0, 4.0], 2, 2)
    np.testing.assert_array_equal(O.row_scaling(A, O.SCALE_SUM), GOLDEN["row_scaling_sum"])


def test_solve_doctest():
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [2.0, 1.0, 1.0, 2.0], 2, 2)
    x = O.solve(O.splu(A), np.array([1.0, 0.0]), refine=1)
    np.testing.assert_allclose(x, GOLDEN["solve_2x2"], rtol=0, atol=1e-16)


@pytest.mark.parametrize("make", [lambda: M.poisson2d(24), lambda: M.poisson3d(10), lambda: M.randmat(500, 6),
                                  lambda: M.arrowband(400, 4)])
def test_oracle_reconstruction(make):
    A = make()
    F = O.multifrontal_lu(A, check=False)
    L = SparseCSC(A.n, A.n, F.Lcolptr, F.Lrowval, F.Lnzval)
    U = SparseCSC(A.n, A.n, F.Ucolptr, F.Urowval, F.Unzval)
    assert reconstruction_error(A, L, U, F.p, F.q) <= 1e-9
    assert np.array_equal(np.sort(F.p), np.arange(1, A.n + 1))
    # fill of the numeric factor == predicted fill (test/multifrontal_test.jl:43-51)
    assert len(F.Lrowval) + len(F.Urowval) == O.predicted_fill(O.symbolic_mf(A))


def test_oracle_fixtures():
    """Small factorizations committed under tests/golden (made by make_golden.py)."""
    data = np.load(os.path.join(os.path.dirname(__file__), "golden", "factors.npz"))
    for name in GOLDEN["fixtures"]:
        A = SparseCSC(int(data[name + "/n"]), int(data[name + "/n"]), data[name + "/colptr"], data[name + "/rowval"],
                      data[name + "/nzval"])
        F = O.multifrontal_lu(A, check=False)
        np.testing.assert_array_equal(F.Lrowval, data[name + "/Lrowval"])
        np.testing.assert_array_equal(F.Urowval, data[name + "/Urowval"])
        np.testing.assert_array_equal(F.p, data[name + "/p"])
        np.testing.assert_allclose(F.Lnzval, data[name + "/Lnzval"], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(F.Unzval, data[name + "/Unzval"], rtol=1e-13, atol=1e-15)
