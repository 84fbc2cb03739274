"""Regenerate the committed golden fixtures of tests/golden/.

    python tests/golden/make_golden.py

kat.json holds the reference's own published values (with their sources);
factors.npz holds small factorizations computed by the oracle (which the KATs
pin) so the GPU parity tests also have fixed, committed expectations.
The reference itself is Julia and cannot run here, so there are no fixtures
produced by it directly.
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "pureumfpack.jl_b200")]

from oracle import oracle as O  # noqa: E402
from pureumfpack import matrices as M  # noqa: E402

KAT = {
    "fill": [
        {"matrix": "poisson2d-32", "fill": 23800, "source": "results/SUMMARY.md:32"},
        {"matrix": "poisson2d-64", "fill": 134400, "source": "results/SUMMARY.md:33"},
        {"matrix": "poisson2d-100", "fill": 412664, "source": "results/SUMMARY.md:34,53"},
        {"matrix": "poisson3d-16", "fill": 562028, "nsuper": 2792,
         "source": "results/SUMMARY.md:35; nsuper results/SCALING_DIAGNOSIS.md:25"},
        {"matrix": "poisson3d-20", "fill": 1684564, "nsuper": 5445,
         "source": "results/SUMMARY.md:36; nsuper results/SCALING_DIAGNOSIS.md:26"},
        {"matrix": "poisson3d-24", "fill": 3749118, "nsuper": 9348,
         "source": "results/SUMMARY.md:56; nsuper results/SCALING_DIAGNOSIS.md:27"},
    ],
    "row_scaling_sum": [0.3333333333333333, 0.25],
    "row_scaling_source": "src/scaling.jl:86-90",
    "solve_2x2": [0.6666666666666666, -0.3333333333333333],
    "solve_2x2_source": "src/multifrontal.jl:138-144, src/interface.jl:85-91",
    "fixtures": ["poisson2d-6", "arrowband-60", "pivoting-200", "convdiff-5"],
}


def fixture_mats():
    return {
        "poisson2d-6": M.poisson2d(6),
        "arrowband-60": M.arrowband(60, 3),
        "pivoting-200": M.random_unsym(200, 4, 0.3, seed=5),
        "convdiff-5": M.convdiff3d(5),
    }


def main():
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(KAT, f, indent=1)
    arrays = {}
    for name, A in fixture_mats().items():
        F = O.multifrontal_lu(A, check=False)
        arrays.update({f"{name}/n": np.int64(A.n), f"{name}/colptr": A.colptr, f"{name}/rowval": A.rowval,
                       f"{name}/nzval": A.nzval, f"{name}/Lrowval": F.Lrowval, f"{name}/Urowval": F.Urowval,
                       f"{name}/p": F.p, f"{name}/Lnzval": F.Lnzval, f"{name}/Unzval": F.Unzval})
    np.savez_compressed(os.path.join(HERE, "factors.npz"), **arrays)


if __name__ == "__main__":
    main()
