"""CPU check of the dataflow LU's algorithm (csrc/lu.cu, k_gj_dataflow), as a
numpy restatement of its steps, against LAPACK (scipy.linalg.lu_factor,
numpy.linalg): the reference computes log det and inverse with
LAPACKE_dgetrf + LAPACKE_dgetri (simulation/organic_dense_matrix.c:580-595).

The kernel never moves rows.  Per panel of 8 columns it runs a Gauss-Jordan
sweep restricted to the panel: each step picks the largest |a| among rows
not yet used as pivots, ties to the smallest logical position (the row's
place in LAPACK's order after the interchanges so far), scales the pivot row
and eliminates the column from every other row.  The other columns then take
the block update A(P,c) <- K(P,:) A(P,c), A(r,c) += K(r,:) A(P,c), with K the
swept panel and P its pivot rows.  Rows only carry logical positions; the
pivot of step j is the logical position swapped with j (LAPACK's ipiv), and
the inverse is X(lpos(r), P_j) = Y(r, j) with Y the final array.

This restatement follows the kernel's arithmetic step by step but not its
fused multiply-adds, so the comparisons are to rounding; the pivot sequences
are compared exactly.  The GPU tests (test_gpu_eval.py) run the kernel itself
on the same kinds of matrices."""
import numpy as np
import pytest

NB = 8


def dataflow_lu(A):
    """Inverse (LAPACK view X(r, c)), 0-based pivots, log|det| and sign."""
    A = np.array(A, dtype=np.float64)
    V = A.shape[0]
    a = A.copy()
    lpos = np.arange(V)
    ipiv = np.zeros(V, dtype=np.int64)
    diag = np.zeros(V)
    own = np.zeros(V, dtype=np.int64)
    for j0 in range(0, V, NB):
        nbc = min(NB, V - j0)
        blk = a[:, j0:j0 + nbc].copy()
        for jj in range(nbc):
            j = j0 + jj
            cand = lpos >= j
            key = np.where(cand, np.abs(blk[:, jj]), -1.0)
            best = key.max()
            rows = np.flatnonzero(cand & (key == best))
            p = rows[np.argmin(lpos[rows])]
            lb = lpos[p]
            d = blk[p, jj]
            inv = 0.0 if d == 0 else 1.0 / d
            prs = blk[p, :] * inv
            prs[jj] = inv
            f = blk[:, jj].copy()
            new = blk - np.outer(f, prs)
            new[:, jj] = -f * prs[jj]
            new[p, :] = prs
            blk = new
            at_j, at_lb = lpos == j, lpos == lb
            lpos[at_j], lpos[at_lb] = lb, j
            ipiv[j], diag[j], own[j] = lb, d, p
        P = np.array([np.flatnonzero(lpos == j0 + m)[0] for m in range(nbc)])
        other = np.r_[0:j0, j0 + nbc:V]
        Cp = a[np.ix_(P, other)]
        upd = blk @ Cp
        is_p = np.zeros(V, dtype=bool)
        is_p[P] = True
        a[:, other] = np.where(is_p[:, None], upd, a[:, other] + upd)
        a[:, j0:j0 + nbc] = blk
    X = np.empty_like(a)
    X[np.ix_(lpos, own)] = a
    logdet = float(np.sum(np.log(np.abs(diag))))
    neg = int(np.sum(diag <= 0) + np.sum(ipiv != np.arange(V))) & 1
    return X, ipiv, logdet, -1 if neg else 1


def _check(A, inv_tol=1e-10):
    import scipy.linalg as sl
    X, ipiv, ld, sg = dataflow_lu(A)
    _, piv = sl.lu_factor(A)
    assert np.array_equal(ipiv, piv)
    s_np, ld_np = np.linalg.slogdet(A)
    assert sg == int(s_np)
    assert abs(ld - ld_np) <= 1e-12 * max(1.0, abs(ld_np))
    ref = np.linalg.inv(A)
    assert np.max(np.abs(X - ref)) <= inv_tol * np.max(np.abs(ref))


@pytest.mark.parametrize("V", [5, 8, 20, 37, 64])
def test_random_matrices(V):
    rng = np.random.default_rng(V)
    _check(rng.standard_normal((V, V)))


@pytest.mark.parametrize("V", [16, 37])
def test_permutation_matrix(V):
    rng = np.random.default_rng(3)
    A = np.eye(V)[rng.permutation(V)]
    _check(A, inv_tol=0)


@pytest.mark.parametrize("V", [12, 24])
def test_ones_minus_identity_ties(V):
    """Column 0 is 0 above V-1 equal ones: the first step's pivot is decided
    by the tie-break (the first row in LAPACK's current order)."""
    _check(np.ones((V, V)) - np.eye(V))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_sign_matrix_ties(seed):
    """Random +-1 matrices: every entry of column 0 ties, and the eliminated
    entries stay small integers (0, +-2, ...), so ties recur at later steps."""
    rng = np.random.default_rng(seed)
    A = rng.choice([-1.0, 1.0], size=(20, 20))
    assert abs(np.linalg.det(A)) > 0.5
    _check(A)
