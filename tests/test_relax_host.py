"""Relaxed amalgamation (opt-in, host symbolic): a valid supernodal
structure for the numeric phase.  Each merged supernode's update set holds
its children's update rows, the column counts match the supernodes, and the
fill grows only by the explicit zeros the merges store."""

import numpy as np
import pytest

from pureumfpack import matrices as M
from pureumfpack import predicted_fill, symbolic_mf


@pytest.mark.parametrize("name,make", [("poisson3d-12", lambda: M.poisson3d(12)),
                                       ("poisson2d-40", lambda: M.poisson2d(40)),
                                       ("convdiff-8", lambda: M.convdiff3d(8))])
def test_relaxed_structure_is_consistent(name, make):
    A = make()
    S0 = symbolic_mf(A)
    S = symbolic_mf(A, relax=True)
    np.testing.assert_array_equal(S.qf, S0.qf)          # same order, coarser partition
    assert S.nsuper < S0.nsuper
    assert set(S.sstart.tolist()) <= set(S0.sstart.tolist())
    assert predicted_fill(S) >= predicted_fill(S0)
    for s in range(1, S.nsuper + 1):
        c1, c2 = int(S.sstart[s - 1]), int(S.sstart[s]) - 1   # 1-based columns
        upd = S.update_set(s)
        assert np.all(np.diff(upd) > 0) and (len(upd) == 0 or upd[0] > c2)
        for j in range(c1, c2 + 1):
            assert S.colcount[j - 1] == (c2 - j) + len(upd)
        rows = set(range(c1, c2 + 1)) | set(upd.tolist())
        for c in S.childsupers[s - 1]:
            assert set(S.update_set(int(c)).tolist()) <= rows
