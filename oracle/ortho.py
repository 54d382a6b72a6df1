"""Oracle: PairCalculator products and the Ortho S -> T iteration (FP64).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* S (symmetric PC) = 2 * psi_r^T psi_r over the real view of the packed
  coefficients with Gx=0 rows scaled by 1/sqrt(2): ckPairCalculator.C:682-751
  (alpha = 2 for double pack), scaling CP_State_GSpacePlane.C:3120-3123.
  Equivalent: S_ij = sum_p wpt_p Re(conj psi_i(p) psi_j(p)), wpt = 1 on Gx=0.
* lambda (asymmetric PC) = psi_r^T F_r: that PairCalculator runs without the
  double-pack factor (cpaimd.C:2527, alpha = 1), and the 1/sqrt(2) scaling of
  psi and sqrt(2) scaling of F on Gx=0 (CP_State_GSpacePlane.C:1933-1954)
  cancel: lambda_ji = sum_p Re(conj psi_j(p) F_i(p)) with no weights.
* Schulz iteration: CPORTHOG::get_iter_Tmat (cp_lowdin.C:180-265) and its
  distributed twin Ortho::do_iteration/step_2/step_3/tolerance_check
  (ortho.C:862-985): A = I, B = S/2; C = 3I - A B; B <- B C / 2; A <- C A / 2;
  stop when rms(A_old - A_new) <= 1e-15, fail after 10 iterations.
* back-multiply psi_new = psi T (ckPairCalculator.C:1314, 'N','N').
"""
import numpy as np


def weights(kx):
    return np.where(np.asarray(kx) == 0, 1.0, 2.0)


def real_view(c):
    return np.stack([c.real, c.imag], axis=-1).reshape(c.shape[0], -1)


def pc_overlap(a, b, kx):
    """2 * a_r^T b_r with the Gx=0 weights: [S, S] (rows of a against rows of b)."""
    w = np.repeat(weights(kx), 2)
    return (real_view(a) * w[None]) @ real_view(b).T


def schulz_tmat(S, tol=1e-15, max_iter=10):
    """T = (S/2)^(-1/2) by the reference's coupled Schulz iteration.

    Returns (T, iterations, final rms); raises RuntimeError on non-convergence
    (the reference prints an error and exits, cp_lowdin.C:243-250).
    """
    n = S.shape[0]
    B = S / 2.0
    A = np.eye(n)
    it, tol_now = 0, 1.0
    while tol_now > tol and it < max_iter:
        it += 1
        C = 3.0 * np.eye(n) - A @ B.T
        B = 0.5 * (B @ C.T)
        A_old = A
        A = 0.5 * (C @ A_old.T)
        tol_now = np.sqrt(np.sum((A_old - A) ** 2) / (n * n))
    if tol_now > tol:
        raise RuntimeError("Schulz S^-1/2 iteration failed in %d iterations (rms %g)"
                           % (it, tol_now))
    return A, it, tol_now


def back_multiply(psi, T):
    """psi_new[i] = sum_j T[j, i] psi[j]  (psi . T in the reference's column view)."""
    return T.T @ psi
