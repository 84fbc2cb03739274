"""A model of k_gplu_factor's warp algorithm against the oracle (CPU).

The device factorization keeps the reference's depth-first order while
reading each column of L in 32-row chunks (four chunks per step), finishing
rows without edges as the scan meets them, and choosing the pivot by a
butterfly reduction over 32 lanes.  This test runs the same steps on the
host -- the chunked scans and ballots as list operations, the reduction
lane by lane -- and requires the result to be the oracle's unsorted factors
(src/gplu.jl:70-291) bit for bit: the argument for the kernel's exactness,
checked without a GPU.  Arithmetic is Float64 in Python, whose operations
round separately, as the kernel's intrinsics do.
"""

import numpy as np
import pytest

from oracle import oracle as O
from pureumfpack import SparseCSC
from pureumfpack import matrices as M

LANES, CHUNKS = 32, 4


def warp_model(A, q, tol):
    n = A.n
    cp, ri, av = A.colptr - 1, A.rowval - 1, A.nzval
    pinv = np.full(n, -1)
    mark = np.zeros(n, np.int64)
    x = np.zeros(n)
    xi = np.zeros(n, np.int64)
    stack = np.zeros(n, np.int64)
    pstack = np.zeros(n, np.int64)
    lp, up, li, lx, ui, ux = [0], [0], [], [], [], []

    def dfs(j0, J0, stamp, top):
        head, j, J, pp = 0, j0, J0, lp[J0]
        stack[0] = j0
        mark[j0] = stamp
        while head >= 0:
            pend = lp[J + 1]
            pushed = False
            while pp < pend and not pushed:
                # CHUNKS chunks of LANES rows: rows, marks and pivot steps loaded together
                chunks = []
                for c in range(CHUNKS):
                    rows = [li[p] if p < pend else -1 for p in range(pp + LANES * c, pp + LANES * (c + 1))]
                    unm = [r >= 0 and r != j and mark[r] != stamp for r in rows]
                    jv = [pinv[r] if u else -1 for r, u in zip(rows, unm)]
                    chunks.append((rows, unm, jv))
                for c, (rows, unm, jv) in enumerate(chunks):
                    piv = [u and v >= 0 for u, v in zip(unm, jv)]
                    f = piv.index(True) if any(piv) else LANES
                    leaves = [t for t in range(f) if unm[t] and jv[t] < 0]
                    for rank, t in enumerate(leaves):      # ballot ranks: scan order
                        xi[top - 1 - rank] = rows[t]
                        mark[rows[t]] = stamp
                    top -= len(leaves)
                    if f < LANES:
                        inext, Jnext = rows[f], jv[f]
                        pp += LANES * c + f
                        pushed = True
                        break
                if not pushed:
                    pp += LANES * CHUNKS
            if pushed:
                pstack[head] = pp
                stack[head + 1] = inext
                mark[inext] = stamp
                head, j, J, pp = head + 1, inext, Jnext, lp[Jnext]
            else:
                top -= 1
                xi[top] = j
                head -= 1
                if head >= 0:
                    j, pp = stack[head], pstack[head]
                    J = pinv[j]
        return top

    for k in range(n):
        col, stamp, top = q[k], k + 1, n
        for pa in range(cp[col], cp[col + 1]):
            b = ri[pa]
            if mark[b] == stamp:
                continue
            if pinv[b] < 0:
                top -= 1
                mark[b] = stamp
                xi[top] = b
            else:
                top = dfs(b, pinv[b], stamp, top)
        for pa in range(cp[col], cp[col + 1]):
            x[ri[pa]] = av[pa]
        for px in range(top, n):
            J = pinv[xi[px]]
            if J < 0 or lp[J] + 1 >= lp[J + 1]:
                continue
            xj = x[xi[px]]
            for p in range(lp[J] + 1, lp[J + 1]):
                x[li[p]] -= lx[p] * xj
        # lanes' strided scans (strict >), then a butterfly (larger value, or
        # equal value at the earlier position)
        best = [-1.0] * LANES
        bpos = [np.iinfo(np.int64).max] * LANES
        for px in range(top, n):
            i = xi[px]
            if pinv[i] >= 0:
                ui.append(pinv[i])
                ux.append(x[i])
            else:
                lane = (px - top) % LANES
                t = abs(x[i])
                if t > best[lane]:
                    best[lane], bpos[lane] = t, px
        off = LANES // 2
        while off:
            nb, npos = best[:], bpos[:]
            for lane in range(LANES):
                ob, op = best[lane ^ off], bpos[lane ^ off]
                if ob > best[lane] or (ob == best[lane] and op < bpos[lane]):
                    nb[lane], npos[lane] = ob, op
            best, bpos, off = nb, npos, off // 2
        assert len(set(best)) == 1 and len(set(bpos)) == 1
        a = best[0]
        ipiv = -1 if bpos[0] == np.iinfo(np.int64).max else xi[bpos[0]]
        assert ipiv >= 0 and a > 0
        if pinv[col] < 0 and abs(x[col]) >= tol * a:
            ipiv = col
        pivot = x[ipiv]
        ui.append(k)
        ux.append(pivot)
        up.append(len(ui))
        pinv[ipiv] = k
        li.append(ipiv)
        lx.append(1.0)
        for px in range(top, n):
            i = xi[px]
            if pinv[i] < 0:
                li.append(i)
                lx.append(x[i] / pivot)
            x[i] = 0.0
        lp.append(len(li))
    return np.array(lp), np.array(li), np.array(lx), np.array(up), np.array(ui), np.array(ux), pinv


def sprand_plus(n, density, shift, seed):
    rng = np.random.default_rng(seed)
    idx = rng.choice(n * n, size=int(round(density * n * n)), replace=False)
    d = np.arange(1, n + 1)
    return SparseCSC.from_coo(np.concatenate([idx % n + 1, d]), np.concatenate([idx // n + 1, d]),
                              np.concatenate([rng.random(len(idx)), np.full(n, shift)]), n, n)


CASES = [
    ("poisson2d-12", lambda: M.poisson2d(12), 0.1),
    ("poisson3d-6", lambda: M.poisson3d(6), 0.1),
    ("grid3d-random-5", lambda: M.grid3d_random(5), 1.0),
    ("convdiff-6", lambda: M.convdiff3d(6), 0.1),
    ("sprand-150", lambda: sprand_plus(150, 12 / 150, 1.0, 5), 1.0),
    ("dense-columns-180", lambda: sprand_plus(180, 0.4, 2.0, 6), 1.0),   # columns of L longer than 4 x 32 rows
]


@pytest.mark.parametrize("name,make,tol", CASES, ids=[c[0] for c in CASES])
def test_warp_model_is_the_reference_order(name, make, tol):
    A = make()
    q = O.colamd_order(A)
    Fo = O.gplu(A, q=q, tol=tol, sort_factors=False)
    lp, li, lx, up, ui, ux, pinv = warp_model(A, q - 1, tol)
    np.testing.assert_array_equal(lp + 1, Fo.Lcolptr)
    np.testing.assert_array_equal(pinv[li] + 1, Fo.Lrowval)
    np.testing.assert_array_equal(lx, Fo.Lnzval)
    np.testing.assert_array_equal(up + 1, Fo.Ucolptr)
    np.testing.assert_array_equal(ui + 1, Fo.Urowval)
    np.testing.assert_array_equal(ux, Fo.Unzval)
    np.testing.assert_array_equal(pinv + 1, Fo.pinv)
