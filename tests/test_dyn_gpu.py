"""The reference's CP dynamics constraint on the GPU against the oracle.

Four steps of cpstep_cp_step with CPSTEP_CONSTRAINT_ORTHO_T (the default):
gamma = orthoT lambda, F_c = F.orthoT - W psi.gamma, Verlet on the
non-orthogonal coefficients, the norb check and the PsiV reset.  Two regimes:
cp_norb_tol above every deviation (no reset: psi_no and orthoT carried over
all steps) and cp_norb_tol just above the first step's deviation (a reset on
every later step).
FP64: energies 1e-10 relative, psi and v 1e-9, psi_no and orthoT (read back
with cpstep_dyn_state) 1e-9, the reset count equal.
Mixed: energy <= 1e-6 Ha/atom and atom forces <= 1e-5 Ha/bohr against the
FP64 oracle, the same resets.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0
NSTEP = 4


@pytest.fixture(scope="module")
def dsys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import density as OD
    from oracle import layout as OL
    from oracle import step as OS
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 16, {"O": 4, "H": 8}, nfft=48)
    lay = OL.Layout(12.0, 30.0, grid=48)
    dlay = OD.density_layout(12.0, 30.0, 48)
    psi = sysm.psi()
    cmass = OS.cp_mass(lay, 25.0, 30.0)
    pn = psi.cpu().numpy()
    occ = np.ones(sysm.nstates)
    _, _, _, _, a = OS.cp_step(pn, np.zeros_like(pn), occ, sysm, lay, dlay, cmass, DT, 1,
                               tol_norb=1.0)
    tols = {"none": 1.0, "reset": 1.5 * a["dyn"]["dev"]}
    ref = {}
    for regime, tol in tols.items():
        p, v, dyn, out = pn, np.zeros_like(pn), None, []
        for it in range(1, NSTEP + 1):
            p, v, en, f, aux = OS.cp_step(p, v, occ, sysm, lay, dlay, cmass, DT, it,
                                          tol_norb=tol, dyn=dyn)
            dyn = aux["dyn"]
            out.append((p, v, en, f, dyn))
        ref[regime] = out
    assert ref["none"][-1][4]["resets"] == 0 and ref["reset"][-1][4]["resets"] == NSTEP - 1
    return dict(sys=sysm, psi=psi, occ=torch.ones(sysm.nstates, dtype=torch.float64,
                                                  device="cuda"), tols=tols, ref=ref)


def _ctx(dsys, precision, tol):
    from openatom_b200.context import StepContext
    s = dsys["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    ctx.set_atoms(s)
    ctx.set_cp_mass(25.0, 30.0)
    ctx.set_constraint("ortho_t", tol)
    return ctx


NAMES = [("EXC", 0), ("EHART", 2), ("EEXT", 3), ("EKE", 6), ("ETOT", 8), ("FICT", 9)]


@pytest.mark.parametrize("regime", ["none", "reset"])
def test_fp64_dynamics_matches_oracle(dsys, regime):
    import torch
    ctx = _ctx(dsys, "fp64", dsys["tols"][regime])
    try:
        psi = dsys["psi"].clone()
        v = torch.zeros_like(psi)
        for it, (pr, vr, er, fr, dyn) in enumerate(dsys["ref"][regime], start=1):
            e, f = ctx.cp_step(psi, v, dsys["occ"], DT, it)
            _, ok = ctx.step_status()
            assert ok
            e = e.cpu().numpy()
            for name, slot in NAMES:
                assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), (it, name)
            assert np.max(np.abs(psi.cpu().numpy() - pr)) < 1e-9, it
            assert np.max(np.abs(v.cpu().numpy() - vr)) < 1e-9 * max(1.0, np.max(np.abs(vr)))
            assert np.max(np.abs(f.cpu().numpy() - fr)) < 1e-9 * max(1.0, np.max(np.abs(fr)))
            pno, tm, half = ctx.dyn_state()
            assert half == (0 if dyn["half_reset"] else 1), it
            assert np.max(np.abs(pno.cpu().numpy() - dyn["psi_no"])) < 1e-9, it
            assert np.max(np.abs(tm.cpu().numpy() - dyn["T"])) < 1e-9, it
            dev, resets = ctx.dyn_status()
            assert resets == dyn["resets"], it
            assert abs(dev - dyn["dev"]) <= 1e-9 * max(1.0, dyn["dev"])
    finally:
        ctx.close()


@pytest.mark.parametrize("regime", ["none", "reset"])
def test_mixed_dynamics_within_budget(dsys, regime):
    import torch
    ctx = _ctx(dsys, "mixed", dsys["tols"][regime])
    natm = dsys["sys"].natm
    try:
        psi = dsys["psi"].clone()
        v = torch.zeros_like(psi)
        for it, (pr, vr, er, fr, dyn) in enumerate(dsys["ref"][regime], start=1):
            e, f = ctx.cp_step(psi, v, dsys["occ"], DT, it)
            _, ok = ctx.step_status()
            assert ok
            e = e.cpu().numpy()
            assert abs(e[8] - er["ETOT"]) / natm <= 1e-6, it
            assert np.max(np.abs(f.cpu().numpy() - fr)) <= 1e-5, it
            assert ctx.dyn_status()[1] == dyn["resets"], it
            pno, _, half = ctx.dyn_state()
            assert half == (0 if dyn["half_reset"] else 1), it
            if dyn["half_reset"]:  # the reset's psi_no is this step's psi, bit for bit
                assert torch.equal(pno, psi), it
                assert np.max(np.abs(v.cpu().numpy() - vr)) <= 1e-4 * max(1.0, np.max(np.abs(vr)))
    finally:
        ctx.close()


def test_first_step_norb_failure_is_an_error(dsys):
    import torch
    from openatom_b200 import _lib
    ctx = _ctx(dsys, "fp64", 1e-8)
    try:
        psi = dsys["psi"].clone()
        v = torch.zeros_like(psi)
        with pytest.raises(RuntimeError) as ei:
            ctx.cp_step(psi, v, dsys["occ"], DT, 1)
        assert "cp_norb_tol" in str(ei.value) and ei.value.code == _lib.CPSTEP_ERR_NORB
        # iteration > 1 with no carried state is refused, not guessed
        ctx.set_constraint("ortho_t", 1.0)
        with pytest.raises(RuntimeError):
            ctx.cp_step(psi, v, dsys["occ"], DT, 2)
        assert _lib.CPSTEP_ERR_NORB == 6
    finally:
        ctx.close()


def test_loaded_state_continues_the_trajectory(dsys):
    """Read psi_no and orthoT after two steps, load them into a fresh context
    with the same psi and v: its next step equals the original context's."""
    import torch
    a = _ctx(dsys, "fp64", 1.0)
    b = _ctx(dsys, "fp64", 1.0)
    try:
        psi = dsys["psi"].clone()
        v = torch.zeros_like(psi)
        for it in (1, 2):
            a.cp_step(psi, v, dsys["occ"], DT, it)
        pno, tm, half = a.dyn_state()
        psi_b, v_b = psi.clone(), v.clone()
        b.dyn_state(pno, tm, half)
        ea, _ = a.cp_step(psi, v, dsys["occ"], DT, 3)
        eb, _ = b.cp_step(psi_b, v_b, dsys["occ"], DT, 3)
        torch.cuda.synchronize()
        assert bool((psi == psi_b).all()) and bool((v == v_b).all())
        assert bool((ea == eb).all())
    finally:
        a.close()
        b.close()
