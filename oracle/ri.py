"""Test infrastructure only: numpy restatement of the RI-JK contractions from their definitions, on
three- and two-centre integrals produced by the reference itself (oracle/ref.py: RefStructure.eri3,
RefStructure.eri2, i.e. lible::ints::eri3 / eri2, src/lible/ints/twoel/eri3.cpp:7-48 and
eri2.cpp:27-72).  The reference has no RI driver; the formulas are

    J_mn = sum_PQ (mn|P) [M^-1]_PQ (Q|ls) D_ls,   K_mn = sum_PQ (ml|P) [M^-1]_PQ (Q|ns) D_ls,

with M = (P|Q).  M^-1 follows the same policy as the library's metric factorisation: Cholesky;
failing that, Cholesky of M + 1e-11 max(diag M) I; failing that, the eigendecomposition with the
eigenpairs below 1e-12 of the largest dropped.  Used by tests/ and tests/golden/make_golden.py only."""
import numpy as np


def metric_factor(M):
    """(F, method) with M^-1 = F^T F: F = L^-1 for the Cholesky factor L (method 0, or 2 after the
    diagonal shift), or F = diag(w^-1/2) V^T over the kept eigenpairs (method 1)."""
    from scipy.linalg import solve_triangular

    n = M.shape[0]
    eye = np.eye(n)
    for method, shift in ((0, 0.0), (2, 1e-11 * np.max(np.diag(M)))):
        try:
            L = np.linalg.cholesky(M + shift * eye)
            return solve_triangular(L, eye, lower=True), method
        except np.linalg.LinAlgError:
            pass
    w, V = np.linalg.eigh(M)
    keep = w > 1e-12 * w.max()
    return (V[:, keep] / np.sqrt(w[keep])).T, 1


def ri_exchange(B3, M, D):
    """K from the reference layout B3[m][n][P] = (mn|P), M[P][Q] = (P|Q), symmetric D:
    W_R = sum_P F_RP (..|P), K = sum_R W_R D W_R^T."""
    n, na = B3.shape[0], B3.shape[2]
    F, _ = metric_factor(M)
    W = (F @ B3.reshape(n * n, na).T).reshape(-1, n, n)
    return np.einsum("Rml,ls,Rns->mn", W, D, W, optimize=True)


def ri_coulomb(B3, M, D):
    """RI-J from the same integrals: gamma = (mn|P) D_mn, J = (mn|P) M^-1 gamma."""
    F, _ = metric_factor(M)
    gamma = np.einsum("mnP,mn->P", B3, D, optimize=True)
    return np.einsum("mnP,P->mn", B3, F.T @ (F @ gamma), optimize=True)
