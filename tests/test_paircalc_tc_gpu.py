"""Tensor-core (split-BF16, tcgen05) PairCalculator products of the mixed
context against the FP64 products of an FP64 context and numpy.

The mixed context sends cpstep_pc_overlap / cpstep_pc_backmultiply to the
tcgen05 kernels: every FP64 element rounded to FP32 and split into three BF16
levels, six level products accumulated in FP32 over 128-real groups, the
groups, slabs and epilogue summed in FP64; the diagonal of S = psi^T psi and
the diagonal of the back-multiplied matrix in FP64.  Overlaps of 256 states
or more split both operands once in global memory into their BF16 levels
and stream them through the tensor cores (the six level products in one
accumulator, FP64 folds every 128 reals; the diagonal of S still in FP64).  Tolerances (relative to
the largest entry of the FP64 result): S 1e-7, lambda 1e-6, psi.T 2e-9
(T near I: the error scales with T - diag T), psi.M 1e-6 for a random M.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


def _ctxs(lay, S):
    from openatom_b200.context import StepContext
    return StepContext(lay, S, precision="fp64"), StepContext(lay, S, precision="mixed")


def _psi(lay, S, seed, pert=0.01):
    import torch
    from openatom_b200.system import make_psi
    psi = make_psi(lay, S, seed=seed, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(seed)
    noise = (torch.randn((S, lay.npts), generator=g, dtype=torch.float64)
             + 1j * torch.randn((S, lay.npts), generator=g, dtype=torch.float64)).cuda()
    f = (torch.randn((S, lay.npts), generator=g, dtype=torch.float64)
         + 1j * torch.randn((S, lay.npts), generator=g, dtype=torch.float64)).cuda()
    return psi + pert * noise * psi.abs().mean(), f


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.fixture(scope="module")
def small():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200.layout import StateLayout
    return StateLayout(12.0, 30.0)


@pytest.mark.parametrize("S", [37, 128, 300])
def test_overlap_tensor_cores_vs_fp64(small, S):
    psi, f = _psi(small, S, seed=S)
    c64, cm = _ctxs(small, S)
    try:
        S64, Stc = c64.pc_overlap(psi, psi), cm.pc_overlap(psi, psi)
        assert _rel(Stc, S64) < 1e-7
        # exactly symmetric, FP64 diagonal
        assert float((Stc - Stc.T).abs().max()) == 0.0
        assert float((Stc.diagonal() - S64.diagonal()).abs().max()) < 1e-13
        L64, Ltc = c64.pc_overlap(psi, f), cm.pc_overlap(psi, f)
        assert _rel(Ltc, L64) < 1e-6
        # alpha / beta
        import torch
        c0 = torch.ones((S, S), dtype=torch.float64, device="cuda")
        o64 = c64.pc_overlap(psi, f, alpha=-0.5, beta=2.0, out=c0.clone())
        otc = cm.pc_overlap(psi, f, alpha=-0.5, beta=2.0, out=c0.clone())
        assert _rel(otc, o64) < 1e-6
        assert cm.device_errors() == 0
    finally:
        c64.close()
        cm.close()


@pytest.mark.parametrize("S,nout", [(128, 128), (300, 300), (128, 96), (40, 40), (72, 56)])
def test_backmultiply_tensor_cores_vs_fp64(small, S, nout):
    import torch
    psi, f = _psi(small, S, seed=7 + S)
    c64, cm = _ctxs(small, S)
    try:
        Sm = c64.pc_overlap(psi, psi)
        T, _, _ = c64.ortho_tmat(Sm, tol=1e-13, max_iter=30)
        T = T[:nout].contiguous()  # columns 0..nout-1 of the column-major T
        o64 = c64.pc_backmultiply(T, psi, nout=nout)
        otc = cm.pc_backmultiply(T, psi, nout=nout)
        assert _rel(otc, o64) < 2e-9
        rng = np.random.default_rng(S)
        M = torch.from_numpy(rng.standard_normal((nout, S))).cuda()
        o64 = c64.pc_backmultiply(M, psi, nout=nout, alpha=-0.5, beta=1.0, out=f[:nout].clone())
        otc = cm.pc_backmultiply(M, psi, nout=nout, alpha=-0.5, beta=1.0, out=f[:nout].clone())
        assert _rel(otc, o64) < 1e-6
        assert cm.device_errors() == 0
    finally:
        c64.close()
        cm.close()


def test_gemm_path_switch_gives_fp64_products(small):
    psi, f = _psi(small, 64, seed=3)
    c64, cm = _ctxs(small, 64)
    try:
        cm.set_gemm_path(False)
        assert float((cm.pc_overlap(psi, f) - c64.pc_overlap(psi, f)).abs().max()) == 0.0
        cm.set_gemm_path(True)
        assert float((cm.pc_overlap(psi, f) - c64.pc_overlap(psi, f)).abs().max()) > 0.0
    finally:
        c64.close()
        cm.close()


@pytest.mark.parametrize("lo,hi", [(0.5, 2.0), (0.05, 5.0)])
def test_standalone_paircalc_ortho_512_states(lo, hi):
    """512 states x 59,536 real coefficients (a 29,768-point half sphere),
    S with eigenvalues log-uniform in [lo, hi]: tensor-core S, lambda and
    psi.T against FP64, and the mixed Ortho (FP32 iteration + FP64 correction)
    on the tensor-core S checked for |T^T S T / 2 - I|."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.layout import StateLayout
    lay = StateLayout(18.0, 70.0)
    n = 512
    rng = np.random.default_rng(int(hi * 100))
    # orthonormal rows (S = 2 I) by QR of a Gaussian block, then rotated and
    # scaled so that S = Q diag(2 s) Q^T with s log-uniform in [lo, hi]
    K = 2 * lay.npts
    w = np.where(lay.kx == 0, 1.0, 2.0)
    G = rng.standard_normal((K, n)) * np.exp(-np.arange(K) / K)[:, None]
    Qg, _ = np.linalg.qr(G * np.sqrt(np.repeat(w, 2))[:, None])
    X = (Qg / np.sqrt(np.repeat(w, 2))[:, None]).T * np.sqrt(2.0)      # S = 2 I
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    X = (Q * np.sqrt(s)) @ Q.T @ X
    psi = torch.from_numpy(np.ascontiguousarray(X)).cuda().view(torch.complex128)
    f = torch.from_numpy(rng.standard_normal((n, K))).cuda().view(torch.complex128)
    c64, cm = _ctxs(lay, n)
    try:
        S64, Stc = c64.pc_overlap(psi, psi), cm.pc_overlap(psi, psi)
        ev = np.linalg.eigvalsh(S64.cpu().numpy() / 2)
        assert ev.min() > 0.9 * lo and ev.max() < 1.1 * hi
        assert _rel(Stc, S64) < 1e-7
        assert _rel(cm.pc_overlap(psi, f), c64.pc_overlap(psi, f)) < 1e-6
        T, it, _ = cm.ortho_tmat(Stc, mixed=True, scale=hi > 2.5, tol=2e-6, max_iter=60)
        Sn = S64.cpu().numpy()
        Tn = T.cpu().numpy()
        # T is exact for the tensor-core S; against the FP64 S the error is S's
        assert np.max(np.abs(Tn.T @ (Stc.cpu().numpy() / 2) @ Tn - np.eye(n))) < 1e-11
        assert np.max(np.abs(Tn.T @ (Sn / 2) @ Tn - np.eye(n))) < 1e-6
        o64 = c64.pc_backmultiply(T, psi)
        otc = cm.pc_backmultiply(T, psi)
        assert _rel(otc, o64) < 1e-6
        assert cm.device_errors() == 0
    finally:
        c64.close()
        cm.close()
