"""PairCalculator products and the Ortho S -> T iteration on the GPU vs the oracle."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pc():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.layout import StateLayout
    from openatom_b200.system import make_psi
    lay = StateLayout(12.0, 30.0)
    S = 37  # not a tile multiple
    psi = make_psi(lay, S, seed=21, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(2)
    f = (torch.randn((S, lay.npts), generator=g, dtype=torch.float64)
         + 1j * torch.randn((S, lay.npts), generator=g, dtype=torch.float64)).to(torch.complex128).cuda()
    ctx = StepContext(lay, S, precision="fp64")
    yield dict(lay=lay, psi=psi, f=f, ctx=ctx, S=S)
    ctx.close()


def colmajor(t):
    return t.cpu().numpy().T  # tensors hold column-major matrices as [ncol][ld]


def test_overlap_symmetric_matches_oracle(pc):
    from oracle import ortho as OO
    out = pc["ctx"].pc_overlap(pc["psi"], pc["psi"])
    ref = OO.pc_overlap(pc["psi"].cpu().numpy(), pc["psi"].cpu().numpy(), pc["lay"].kx)
    assert np.max(np.abs(colmajor(out) - ref)) < 1e-12
    # orthonormalised input: S = 2 I
    assert np.max(np.abs(ref - 2.0 * np.eye(pc["S"]))) < 1e-10


def test_overlap_asymmetric_lambda_matches_oracle(pc):
    from oracle import ortho as OO
    out = pc["ctx"].pc_overlap(pc["psi"], pc["f"])
    ref = OO.pc_overlap(pc["psi"].cpu().numpy(), pc["f"].cpu().numpy(), pc["lay"].kx)
    assert np.max(np.abs(colmajor(out) - ref)) / np.max(np.abs(ref)) < 1e-13


def test_overlap_alpha_beta(pc):
    from oracle import ortho as OO
    import torch
    c0 = torch.ones((pc["S"], pc["S"]), dtype=torch.float64, device="cuda")
    out = pc["ctx"].pc_overlap(pc["psi"], pc["f"], alpha=-0.5, beta=2.0, out=c0)
    ref = -0.5 * OO.pc_overlap(pc["psi"].cpu().numpy(), pc["f"].cpu().numpy(), pc["lay"].kx) + 2.0
    assert np.max(np.abs(colmajor(out) - ref)) < 1e-11


def test_backmultiply_matches_oracle(pc):
    import torch
    S = pc["S"]
    rng = np.random.default_rng(4)
    M = rng.standard_normal((S, S))  # column-major matrix M(j,i) = M[j, i]
    Mt = torch.from_numpy(np.ascontiguousarray(M.T)).cuda()  # [col][row] storage
    out = pc["ctx"].pc_backmultiply(Mt, pc["psi"], alpha=1.0, beta=0.0)
    ref = M.T @ pc["psi"].cpu().numpy()
    assert np.max(np.abs(out.cpu().numpy() - ref)) / np.max(np.abs(ref)) < 1e-13
    out2 = pc["ctx"].pc_backmultiply(Mt, pc["psi"], alpha=-1.0, beta=1.0, out=pc["f"].clone())
    ref2 = pc["f"].cpu().numpy() - ref
    assert np.max(np.abs(out2.cpu().numpy() - ref2)) / np.max(np.abs(ref2)) < 1e-13


def test_dgemm_all_transposes(pc):
    import torch
    rng = np.random.default_rng(8)
    m, n, k = 45, 70, 33
    for ta in "NT":
        for tb in "NT":
            A = rng.standard_normal((m, k) if ta == "N" else (k, m))
            B = rng.standard_normal((k, n) if tb == "N" else (n, k))
            C = rng.standard_normal((m, n))
            opA = A if ta == "N" else A.T
            opB = B if tb == "N" else B.T
            ref = 1.5 * opA @ opB - 0.5 * C
            dA = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()
            dB = torch.from_numpy(np.asfortranarray(B).T.copy()).cuda()
            dC = torch.from_numpy(np.asfortranarray(C).T.copy()).cuda()
            pc["ctx"].dgemm(ta, tb, m, n, k, 1.5, dA, A.shape[0], dB, B.shape[0], -0.5, dC, m)
            assert np.max(np.abs(dC.cpu().numpy().T - ref)) < 1e-12


@pytest.mark.parametrize("n,lo,hi", [(37, 1.7, 2.3), (128, 0.5, 2.0)])
def test_ortho_fp64_matches_oracle(pc, n, lo, hi):
    import torch
    from oracle import ortho as OO
    rng = np.random.default_rng(n)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    S = (Q * np.exp(rng.uniform(np.log(lo), np.log(hi), n))) @ Q.T
    S = 0.5 * (S + S.T)
    T, it, rms = pc["ctx"].ortho_tmat(torch.from_numpy(S).cuda(), tol=1e-14, max_iter=12)
    To, ito, _ = OO.schulz_tmat(S, tol=1e-14, max_iter=12)
    T = T.cpu().numpy()
    assert np.max(np.abs(T - To)) < 1e-12
    assert np.max(np.abs(T @ (S / 2) @ T - np.eye(n))) < 1e-12


@pytest.mark.parametrize("lo,hi,scale", [(1.6, 2.4, False), (0.5, 2.0, False), (0.05, 5.0, True)])
def test_ortho_mixed_is_orthonormal_to_fp64(pc, lo, hi, scale):
    import torch
    n = 96
    rng = np.random.default_rng(7)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    S = (Q * np.exp(rng.uniform(np.log(lo), np.log(hi), n))) @ Q.T
    S = 0.5 * (S + S.T)
    T, it, rms = pc["ctx"].ortho_tmat(torch.from_numpy(S).cuda(), mixed=True, scale=scale,
                                      tol=2e-6, max_iter=40)
    T = T.cpu().numpy()
    # |T^T (S/2) T - I| at FP64 rounding after the FP64 correction
    assert np.max(np.abs(T.T @ (S / 2) @ T - np.eye(n))) < 1e-12
    w, V = np.linalg.eigh(S / 2)
    Z = (V * w ** -0.5) @ V.T
    assert np.max(np.abs(T - Z)) < 1e-4


def test_ortho_reports_non_convergence(pc):
    import torch
    from openatom_b200 import _lib
    S = torch.diag(torch.tensor([0.05, 2.0, 5.0], dtype=torch.float64)).cuda()
    with pytest.raises(_lib.CpstepError) as e:
        pc["ctx"].ortho_tmat(S)
    assert e.value.code == _lib.CPSTEP_ERR_NOCONV
