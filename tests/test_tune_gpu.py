"""The autotuner: it keeps a valid candidate for every choice, get/set round
trip, and a step with the tuned choices agrees with the default-choice step
to rounding (FP64) or to the mixed path's accuracy."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


def _setup(precision):
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 16, {"O": 4, "H": 8}, nfft=48, seed=9)
    ctx = StepContext(sysm.layout, sysm.nstates, precision=precision)
    ctx.set_atoms(sysm)
    ctx.set_nonlocal(sysm)
    ctx.set_cp_mass(25.0, 30.0)
    ctx.set_constraint("ortho_t", 1.0)  # cp_norb_tol above this step's deviation
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    return sysm, ctx, occ


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_choices_and_step(precision):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    sysm, ctx, occ = _setup(precision)
    ref_sys, ref, _ = _setup(precision)
    try:
        default = ctx.tune_get()
        choice, ms = ctx.autotune(sysm.psi(), occ)
        assert choice["plane_shfl"] in (0, 1, 2)  # Stockham, shuffles, two-stage (FP32)
        if precision == "fp64":
            assert choice["plane_shfl"] in (0, 1)
        assert choice["plane_waves"] in (1, 2, 3, 6)
        assert choice["nl_blocks"] in (3, 6, 12)
        assert choice["pc_split"] in (1, 2)
        assert ms["plane_shfl"] > 0 and ms["plane_waves"] > 0 and ms["pc_split"] > 0
        assert choice["ees_gspace"] in (0, 1)
        if precision == "mixed":
            assert ms["tensor_cores"] > 0
        ctx.tune_set(default)
        assert ctx.tune_get() == default
        ctx.tune_set(choice)
        assert ctx.tune_get() == choice
        psi, v = sysm.psi(), None
        p2 = ref_sys.psi()
        v1, v2 = torch.zeros_like(psi), torch.zeros_like(p2)
        e1, f1 = ctx.cp_step(psi, v1, occ, 5.0, 1)
        e2, f2 = ref.cp_step(p2, v2, occ, 5.0, 1)
        e1, e2 = e1.cpu().numpy(), e2.cpu().numpy()
        tol = 1e-10 if precision == "fp64" else 1e-6
        assert abs(e1[8] - e2[8]) <= tol * abs(e2[8])
        assert ctx.device_errors() == 0
    finally:
        ctx.close()
        ref.close()
