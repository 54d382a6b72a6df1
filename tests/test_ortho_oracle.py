"""The oracle's Schulz iteration against the reference's get_iter_Tmat."""
import os

import numpy as np
import pytest

from oracle import ortho as OO
from conftest import ref_lib

HERE = os.path.dirname(os.path.abspath(__file__))


def test_schulz_matches_reference_golden():
    g = np.load(os.path.join(HERE, "golden", "schulz_n48.npz"))
    T, it, tol = OO.schulz_tmat(g["S"])
    assert np.max(np.abs(T - g["T"])) < 1e-13


def test_schulz_matches_compiled_reference_live():
    import ctypes
    L = ref_lib()
    if L is None:
        pytest.skip("oracle/_ref/libref.so not built")
    DP = ctypes.POINTER(ctypes.c_double)
    L.ref_get_iter_Tmat.argtypes = [DP, DP, ctypes.c_int]
    rng = np.random.default_rng(11)
    n = 32
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    S = (Q * rng.uniform(1.7, 2.3, n)) @ Q.T
    S = np.ascontiguousarray(0.5 * (S + S.T))
    T = np.zeros_like(S)
    L.ref_get_iter_Tmat(S.ctypes.data_as(DP), T.ctypes.data_as(DP), n)
    To, _, _ = OO.schulz_tmat(S)
    assert np.max(np.abs(T - To)) < 1e-13
    # and it is the inverse square root of S/2
    assert np.max(np.abs(To @ (S / 2) @ To - np.eye(n))) < 1e-12


def test_schulz_reports_non_convergence():
    S = np.diag([0.05, 2.0, 5.0])  # B = S/2 has an eigenvalue above 2: diverges
    with pytest.raises(RuntimeError):
        OO.schulz_tmat(S)
