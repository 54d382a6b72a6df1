"""EES non-local on the GPU (cpstep_ees_nonlocal and inside cpstep_cp_step)
against the FP64 oracle (oracle/ees.py, itself pinned to the reference's
cp_ees_nonlocal.C routines by tests/test_ees_oracle.py).

FP64 path: E_NL to 1e-11 relative, psi force and atom forces to 1e-10 of
their largest entry.  Mixed path (FP32 NL FFTs, FP64 sums): E_NL to 1e-5
relative, forces to 1e-5 of their largest entry, both for the NL-grid FFT
form and for the G-space form (the same stencil sums by Parseval, evaluated
as split-BF16 tensor-core products with the separable B-spline transforms);
inside the step, energy per atom <= 1e-6 Ha and atom forces <= 1e-5 Ha/bohr.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0


@pytest.fixture(scope="module")
def nlsys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import ees as OE
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 16, {"O": 4, "H": 8}, nfft=48, seed=21)
    psi = sysm.psi()
    occ_np = np.where(np.arange(sysm.nstates) % 3 == 0, 1.0, 2.0)
    occ = torch.from_numpy(occ_np).cuda()
    nkf = OE.nl_grid_size(sysm.layout.kmax)
    e, fpsi, fatm = OE.nonlocal_ees(psi.cpu().numpy(), sysm.layout, occ_np, sysm.box_len ** 3,
                                    sysm.hmati(), dict(pos=sysm.pos, typ=sysm.typ),
                                    sysm.channels, sysm.tab, nkf)
    return dict(sys=sysm, psi=psi, occ=occ, nkf=nkf, ref=(e, fpsi, fatm))


def _run(nlsys, precision, gspace=None):
    from openatom_b200.context import StepContext
    s = nlsys["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        nkf = ctx.set_nonlocal(s)
        if gspace is not None:
            ctx.tune_set({"ees_gspace": int(gspace)})
        assert nkf == nlsys["nkf"]
        fpsi, e, f = ctx.ees_nonlocal(nlsys["psi"], nlsys["occ"])
        return e.cpu().numpy()[7], fpsi.cpu().numpy(), f.cpu().numpy()
    finally:
        ctx.close()


def test_nl_grid_size_entry():
    from openatom_b200 import _lib
    from oracle import ees as OE
    L = _lib.lib()
    for kmax in (6, 10, 31, 49):
        assert L.cpstep_nl_grid_size(kmax, 1.2, 8) == OE.nl_grid_size(kmax)


def test_fp64_ees_matches_oracle(nlsys):
    e, fpsi, f = _run(nlsys, "fp64")
    er, fr, far = nlsys["ref"]
    assert er > 0.0
    assert abs(e - er) <= 1e-11 * abs(er)
    assert np.max(np.abs(fpsi - fr)) <= 1e-10 * np.max(np.abs(fr))
    assert np.max(np.abs(f - far)) <= 1e-10 * np.max(np.abs(far))


@pytest.mark.parametrize("gspace", [True, False])
def test_mixed_ees_within_budget(nlsys, gspace):
    """Mixed contexts: the G-space form on the tensor cores (gspace) and the
    NL-grid FFT form."""
    e, fpsi, f = _run(nlsys, "mixed", gspace)
    er, fr, far = nlsys["ref"]
    assert abs(e - er) <= 1e-5 * abs(er)
    assert np.max(np.abs(fpsi - fr)) <= 1e-5 * np.max(np.abs(fr))
    assert np.max(np.abs(f - far)) <= 1e-5 * np.max(np.abs(far))


def test_ees_accumulates_into_the_force(nlsys):
    import torch
    from openatom_b200.context import StepContext
    s = nlsys["sys"]
    ctx = StepContext(s.layout, s.nstates, precision="fp64")
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal(s)
        base = torch.full_like(nlsys["psi"], 0.25 - 0.5j)
        fpsi, _, _ = ctx.ees_nonlocal(nlsys["psi"], nlsys["occ"], fpsi=base.clone())
        _, fr, _ = nlsys["ref"]
        got = fpsi.cpu().numpy() - base.cpu().numpy()
        assert np.max(np.abs(got - fr)) <= 1e-10 * np.max(np.abs(fr))
    finally:
        ctx.close()


@pytest.fixture(scope="module")
def nlstep(nlsys):
    from oracle import density as OD
    from oracle import layout as OL
    from oracle import step as OS
    s = nlsys["sys"]
    lay = OL.Layout(12.0, 30.0, grid=48)
    dlay = OD.density_layout(12.0, 30.0, 48)
    cmass = OS.cp_mass(lay, 25.0, 30.0)
    pn = nlsys["psi"].cpu().numpy()
    occ = nlsys["occ"].cpu().numpy()
    p1, v1, en1, f1, _ = OS.cp_step(pn, np.zeros_like(pn), occ, s, lay, dlay, cmass, DT, 1,
                                    nonlocal_on=True, nkf=nlsys["nkf"], tol_norb=1.0)
    return (p1, v1, en1, f1)


def _step(nlsys, precision):
    import torch
    from openatom_b200.context import StepContext
    s = nlsys["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal(s)
        ctx.set_cp_mass(25.0, 30.0)
        ctx.set_constraint("ortho_t", 1.0)  # cp_norb_tol above this step's deviation
        psi = nlsys["psi"].clone()
        v = torch.zeros_like(psi)
        e, f = ctx.cp_step(psi, v, nlsys["occ"], DT, 1)
        _, ok = ctx.step_status()
        return psi.cpu().numpy(), v.cpu().numpy(), e.cpu().numpy(), f.cpu().numpy(), ok
    finally:
        ctx.close()


def test_fp64_step_with_nonlocal(nlsys, nlstep):
    p, v, e, f, ok = _step(nlsys, "fp64")
    pr, vr, er, fr = nlstep
    assert ok
    for name, slot in (("ENL", 7), ("EKE", 6), ("ETOT", 8)):
        assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), name
    assert np.max(np.abs(p - pr)) < 1e-9
    assert np.max(np.abs(f - fr)) < 1e-9 * max(1.0, np.max(np.abs(fr)))


def test_mixed_step_with_nonlocal(nlsys, nlstep):
    p, v, e, f, ok = _step(nlsys, "mixed")
    pr, vr, er, fr = nlstep
    natm = nlsys["sys"].natm
    assert ok
    assert abs(e[8] - er["ETOT"]) / natm <= 1e-6
    assert np.max(np.abs(f - fr)) <= 1e-5
