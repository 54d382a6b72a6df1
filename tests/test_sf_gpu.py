"""The structure-factor (non-EES) nonlocal path on the GPU against the oracle
(oracle/sf.py, pinned to the reference's cp_struct_fact.C, cp_nlmat.C and
cp_nl_energy_forc.C): the pass alone in both precisions, and a step."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0


@pytest.fixture(scope="module")
def sfsys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200.system import System
    return System(12.0, 30.0, 8, {"O": 3, "H": 6}, nfft=48, seed=2)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-6)])
def test_sf_pass_matches_oracle(sfsys, precision, tol):
    import torch
    from oracle import sf as OSF
    from openatom_b200.context import StepContext
    s = sfsys
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal_sf(s)
        psi = s.psi()
        occ_h = np.linspace(2.0, 1.0, s.nstates)
        occ = torch.from_numpy(occ_h).cuda()
        fpsi, e, f = ctx.sf_nonlocal(psi, occ)
        enl, fa, fp = OSF.sf_pass(psi.cpu().numpy(), occ_h, s)
        assert enl > 0.0
        assert abs(float(e[7]) - enl) <= tol * abs(enl)
        assert np.max(np.abs(f.cpu().numpy() - fa)) <= tol * np.max(np.abs(fa))
        assert np.max(np.abs(fpsi.cpu().numpy() - fp)) <= tol * np.max(np.abs(fp))
        # accumulates into the given psi force
        fpsi2, _, _ = ctx.sf_nonlocal(psi, occ, fpsi=fpsi.clone())
        assert np.max(np.abs(fpsi2.cpu().numpy() - 2 * fp)) <= 2 * tol * np.max(np.abs(fp))
    finally:
        ctx.close()


def test_sf_and_ees_setups_exclude_each_other(sfsys):
    import torch
    from openatom_b200.context import StepContext
    s = sfsys
    ctx = StepContext(s.layout, s.nstates, precision="fp64")
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal_sf(s)
        ctx.set_nonlocal(s)   # EES replaces the structure-factor path
        occ = torch.ones(s.nstates, dtype=torch.float64, device="cuda")
        from openatom_b200 import _lib
        with pytest.raises(_lib.CpstepError):
            ctx.sf_nonlocal(s.psi(), occ)
    finally:
        ctx.close()


@pytest.fixture(scope="module")
def sfstep():
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
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    cmass = OS.cp_mass(lay, 25.0, 30.0)
    pn = psi.cpu().numpy()
    p1, v1, en1, f1, _ = OS.cp_step(pn, np.zeros_like(pn), np.ones(sysm.nstates), sysm, lay,
                                    dlay, cmass, DT, 1, nonlocal_sf=True, tol_norb=1.0)
    return dict(sys=sysm, psi=psi, occ=occ, ref=(p1, v1, en1, f1))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_with_sf_nonlocal_matches_oracle(sfstep, precision):
    import torch
    from openatom_b200.context import StepContext
    s = sfstep["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal_sf(s)
        ctx.set_cp_mass(25.0, 30.0)
        ctx.set_constraint("ortho_t", 1.0)  # cp_norb_tol above this step's deviation
        psi = sfstep["psi"].clone()
        v = torch.zeros_like(psi)
        e, f = ctx.cp_step(psi, v, sfstep["occ"], DT, 1)
        _, ok = ctx.step_status()
        assert ok
        pr, vr, er, fr = sfstep["ref"]
        e = e.cpu().numpy()
        assert er["ENL"] > 0.0
        if precision == "fp64":
            for name, slot in (("ENL", 7), ("EKE", 6), ("ETOT", 8)):
                assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), name
            assert np.max(np.abs(psi.cpu().numpy() - pr)) < 1e-9
            assert np.max(np.abs(f.cpu().numpy() - fr)) < 1e-9 * max(1.0, np.max(np.abs(fr)))
        else:
            assert abs(e[8] - er["ETOT"]) / s.natm <= 1e-6
            assert np.max(np.abs(f.cpu().numpy() - fr)) <= 1e-5
    finally:
        ctx.close()
