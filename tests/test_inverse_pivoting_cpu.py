"""The pivoting of the register-resident overlap inverse (gj_inverse_reg_kernel), restated in numpy.

The kernel never interchanges rows: step k takes the eligible row p (not pivoted before) of largest
|re| + |im| in column k, ties going to the row that the interchanging elimination would hold at the
lowest position (tracked as pos[row] / row_at[position]); the stored result E then satisfies
E[p_j][k] = inv(S)[j][p_k], undone on write-out.  Checked here against the interchanging Gauss-Jordan
elimination (LU's partial pivoting, then the column interchanges in reverse order): the same
inverse bit for bit, the same pivots and interchange count (so the same determinant), on random
matrices and on integer matrices whose pivot candidates tie exactly.  Test infrastructure only.
"""
import numpy as np


def abs1(z):
    return np.abs(z.real) + np.abs(z.imag)


def gj_interchanging(S):
    A = S.astype(complex).copy()
    N = len(A)
    perm, pivots, nswap = [], [], 0
    for k in range(N):
        p = k + int(np.argmax(abs1(A[k:, k])))  # first index of the maximum
        if p != k:
            A[[k, p]] = A[[p, k]]
            nswap += 1
        perm.append(p)
        piv = A[k, k]
        pivots.append(piv)
        inv = 1.0 / piv
        rowk = A[k] * inv
        rowk[k] = inv
        colk = A[:, k].copy()
        for i in range(N):
            if i == k:
                A[i] = rowk
            else:
                a = A[i].copy()
                a[k] = 0.0
                A[i] = a - colk[i] * rowk
    for k in range(N - 1, -1, -1):
        p = perm[k]
        if p != k:
            A[:, [k, p]] = A[:, [p, k]]
    return A, pivots, nswap


def gj_implicit(S):
    A = S.astype(complex).copy()
    N = len(A)
    pos, row_at = list(range(N)), list(range(N))
    step_of_row, piv_row = [0] * N, [0] * N
    pivots, nswap = [], 0
    for k in range(N):
        best, brow = -1.0, None
        for r in range(N):
            if pos[r] >= k:
                v = abs1(A[r, k])
                if v > best or (v == best and pos[r] < pos[brow]):
                    best, brow = v, r
        p = brow
        pp = pos[p]
        if pp != k:
            q = row_at[k]
            row_at[pp], pos[q] = q, pp
            row_at[k], pos[p] = p, k
            nswap += 1
        step_of_row[p], piv_row[k] = k, p
        piv = A[p, k]
        pivots.append(piv)
        inv = 1.0 / piv
        rowk = A[p] * inv
        rowk[k] = inv
        colk = A[:, k].copy()
        for i in range(N):
            if i == p:
                A[i] = rowk
            else:
                a = A[i].copy()
                a[k] = 0.0
                A[i] = a - colk[i] * rowk
    out = np.empty_like(A)
    for r in range(N):
        for c in range(N):
            out[step_of_row[r], piv_row[c]] = A[r, c]
    return out, pivots, nswap


def test_implicit_pivoting_matches_the_interchanging_form():
    rng = np.random.default_rng(11)
    cases = [rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) for n in (3, 8, 21)]
    # exact ties among the candidates: small integer entries
    cases += [(rng.integers(-2, 3, size=(n, n)) + 1j * rng.integers(-2, 3, size=(n, n))).astype(complex)
              for n in (6, 12)]
    # partial pivoting has to act: a permuted upper-triangular matrix
    T = np.triu(rng.normal(size=(9, 9)) + 1j * rng.normal(size=(9, 9))) + 3 * np.eye(9)
    cases.append(T[rng.permutation(9)])
    for S in cases:
        if abs(np.linalg.det(S)) < 1e-9:
            continue
        A1, p1, s1 = gj_interchanging(S)
        A2, p2, s2 = gj_implicit(S)
        assert np.array_equal(A1, A2)
        assert np.array_equal(np.array(p1), np.array(p2)) and s1 == s2
        det = np.prod(p2) * (-1) ** s2
        assert abs(det - np.linalg.det(S)) <= 1e-10 * abs(det)
        assert np.abs(A2 @ S - np.eye(len(S))).max() <= 1e-10
