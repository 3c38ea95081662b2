"""CPU restatement of the coarsest-level inversion of the multigrid solver
(platoanalyze_b200/csrc/pa_mg.cu: k_gj_pivot, k_gj_panels, k_gj_update),
block step by block step, checked on the kinds of matrices that level
produces: symmetric positive definite elastic operators with identity rows and
columns on Dirichlet and padding dofs, and singular ones that must be flagged
(the solver then keeps the Chebyshev coarse solve)."""
import numpy as np

NB = 64  # elimination block (kGJ)


def pivot_block(P, diag0):
    """In-place Gauss-Jordan of one NB x NB block without pivoting, as the
    one-CTA kernel: returns P^-1 and whether a pivot was not above 1e-12 of
    its row's original diagonal."""
    P = P.copy()
    flagged = False
    for p in range(P.shape[0]):
        row, col = P[p, :].copy(), P[:, p].copy()
        pv = row[p]
        if not pv > 1e-12 * diag0[p]:
            flagged = True
        ip = 1.0 / pv
        P -= np.outer(col, row) * ip
        P[p, :] = row * ip
        P[:, p] = -col * ip
        P[p, p] = ip
    return P, flagged


def invert_blocked(A):
    """The host loop over block steps: pivot block, panels W = P^-1 A[K,:] and
    Cp = A[:,K], then the four-case update of every 64 x 64 tile."""
    n = A.shape[0]
    assert n % NB == 0
    A = A.copy()
    diag0 = np.diag(A).copy()
    flagged = False
    for k0 in range(0, n, NB):
        K = slice(k0, k0 + NB)
        Pinv, f = pivot_block(A[K, K], diag0[K])
        flagged |= f
        W = Pinv @ A[K, :]
        Cp = A[:, K].copy()
        out = A - Cp @ W
        out[:, K] = -Cp @ Pinv
        out[K, :] = W
        out[K, K] = Pinv
        A = out
    return A, flagged


def coarse_operator(n3, nd, fixed, seed):
    """An SPD matrix of n3 dofs padded to nd, identity on `fixed` and padding."""
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n3, n3))
    K = M @ M.T / n3 + np.diag(rng.uniform(0.5, 2.0, n3))
    A = np.zeros((nd, nd))
    A[:n3, :n3] = K
    for d in list(fixed) + list(range(n3, nd)):
        A[d, :] = 0.0
        A[:, d] = 0.0
        A[d, d] = 1.0
    return A


def test_blocked_inverse_of_padded_operators():
    # 135 dofs (the 4x2x2 coarsest box: 3 blocks) and 300 dofs (5 blocks); the
    # 1,188-dof bottom level of 160x80x80 runs in the GPU multigrid tests
    for n3, seed in ((135, 1), (300, 2)):
        nd = (n3 + NB - 1) // NB * NB
        A = coarse_operator(n3, nd, fixed=range(0, n3, 7), seed=seed)
        Ainv, flagged = invert_blocked(A)
        assert not flagged
        assert np.abs(Ainv @ A - np.eye(nd)).max() < 1e-10
        # the V-cycle's use: x = A^-1 b with b zero on Dirichlet dofs gives x zero there
        b = np.random.default_rng(seed).standard_normal(nd)
        b[list(range(0, n3, 7)) + list(range(n3, nd))] = 0.0
        x = Ainv @ b
        assert np.abs(x[list(range(0, n3, 7))]).max() == 0.0


def test_high_contrast_operator_is_inverted_accurately():
    """Void-like dofs (stiffness 1e-8 of the solid's) keep pivots far above the
    1e-12 relative threshold of their own rows."""
    n3, nd = 120, 128
    A = coarse_operator(n3, nd, fixed=range(0, 12), seed=3)
    s = np.ones(nd)
    s[60:n3] = 1e-4  # a scaling by 1e-4 makes those rows/columns 1e-8 softer
    A = A * np.outer(s, s)
    Ainv, flagged = invert_blocked(A)
    assert not flagged
    assert np.abs(Ainv @ A - np.eye(nd)).max() < 1e-8


def test_singular_operator_is_flagged():
    """No Dirichlet dofs: a free chain of springs (per component) has a
    translation null vector; its Schur pivots are 1, ..., 1 and then exactly 0,
    so the last pivot of each chain is flagged and the solve falls back.  (A
    null vector that rounding lifts above 1e-12 of the diagonal is not caught;
    the outer CG's check of the true residual then decides the outcome.)"""
    n3, nd = 96, 128
    L = np.zeros((n3, n3))
    for i in range(n3 - 1):
        L[i, i] += 1.0
        L[i + 1, i + 1] += 1.0
        L[i, i + 1] -= 1.0
        L[i + 1, i] -= 1.0
    A = np.eye(nd)
    A[:n3, :n3] = L
    with np.errstate(divide="ignore", invalid="ignore"):  # the zero pivot is divided by, as on the GPU
        _, flagged = invert_blocked(A)
    assert flagged
    # one fixed end (a Dirichlet dof) removes the null vector
    A[0, :] = 0.0
    A[:, 0] = 0.0
    A[0, 0] = 1.0
    Ainv, flagged = invert_blocked(A)
    assert not flagged
    assert np.abs(Ainv @ A - np.eye(nd)).max() < 1e-9
