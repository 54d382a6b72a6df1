"""The allocation-free overlap entry point against the context-based one.

cpstep_pc_overlap_noalloc serves callers that must not allocate device
memory (their memory is owned by a pool or a fixed budget, or they run where
cudaMalloc is not allowed); its scratch is a fixed array inside the library.
This file is collected last so that a failure here comes after every other
test has run; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, same FP64 arithmetic with a possibly different K split


def _noalloc(a, b, w, out, alpha=1.0, beta=0.0):
    import torch
    from openatom_b200 import _lib
    na, nb = a.shape[0], b.shape[0]
    s = torch.cuda.current_stream().cuda_stream
    _lib.call("cpstep_pc_overlap_noalloc", _lib.ptr(a), _lib.ptr(b), na, nb, a.shape[1],
              _lib.ptr(w), float(alpha), float(beta), _lib.ptr(out), na, ctypes.c_void_p(s))
    return out


def test_noalloc_overlap_matches_context_entry_twice():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.layout import StateLayout
    from openatom_b200.system import make_psi
    lay = StateLayout(12.0, 30.0)
    S = 40
    psi = make_psi(lay, S, seed=3, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(5)
    f = (torch.randn((S, lay.npts), generator=g, dtype=torch.float64)
         + 1j * torch.randn((S, lay.npts), generator=g, dtype=torch.float64)).cuda()
    w = torch.from_numpy(np.where(lay.kx == 0, 1.0, 2.0)).cuda()
    ctx = StepContext(lay, S, precision="fp64")
    try:
        # first call: S = overlap(psi, psi) with the Gx=0 weights
        ref1 = ctx.pc_overlap(psi, psi)
        out1 = _noalloc(psi, psi, w, torch.zeros((S, S), dtype=torch.float64, device="cuda"))
        # second call in a row, other inputs, alpha/beta: lambda-like product
        c0 = torch.ones((S, S), dtype=torch.float64, device="cuda")
        ref2 = ctx.pc_overlap(psi, f, alpha=-0.5, beta=2.0, out=c0.clone())
        out2 = _noalloc(psi, f, w, c0.clone(), alpha=-0.5, beta=2.0)
        torch.cuda.synchronize()
        for out, ref in ((out1, ref1), (out2, ref2)):
            r = ref.cpu().numpy()
            assert np.max(np.abs(out.cpu().numpy() - r)) <= TOL * np.max(np.abs(r))
        # the first result is untouched by the second call (the caller owns it)
        assert np.max(np.abs(out1.cpu().numpy() - ref1.cpu().numpy())) <= TOL * 2.0
    finally:
        ctx.close()


@pytest.mark.parametrize("na,nb", [(1024, 1024), (1000, 1048)])
def test_noalloc_at_its_scratch_limit(na, nb):
    """Products just inside the fixed scratch (na nb <= 2^20): the split-K
    width is bounded by the array there (one slab at 1024 x 1024), and every
    partial tile must stay inside it."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.layout import StateLayout
    lay = StateLayout(9.0, 20.0)
    g = torch.Generator(device="cpu").manual_seed(11)

    def rnd(n):
        return (torch.randn((n, lay.npts), generator=g, dtype=torch.float64)
                + 1j * torch.randn((n, lay.npts), generator=g, dtype=torch.float64)).cuda()
    a, b = rnd(na), rnd(nb)
    w = torch.from_numpy(np.where(lay.kx == 0, 1.0, 2.0)).cuda()
    ctx = StepContext(lay, max(na, nb), precision="fp64")
    try:
        ref = ctx.pc_overlap(a, b)
        out = _noalloc(a, b, w, torch.zeros((nb, na), dtype=torch.float64, device="cuda"))
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        assert np.max(np.abs(out.cpu().numpy() - r)) <= TOL * np.max(np.abs(r))
        assert ctx.device_errors() == 0
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200 import _lib
    n = 1100  # 1100 * 1100 > 2^20 partial doubles
    a = torch.zeros((n, 8), dtype=torch.complex128, device="cuda")
    out = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.CpstepError) as e:
        _noalloc(a, a, None, out)
    assert e.value.code == _lib.CPSTEP_ERR_ARG
