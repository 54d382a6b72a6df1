"""The EES form of the Hartree + local + Ewald pass (cpstep_set_local_ees,
the reference's cp_eext_ees_opt) on the GPU against the oracle
(oracle/eext_ees.py, pinned to the compiled cp_hart_ext.C routines).

* the pass alone (cpstep_hart_eext) on two systems: vks(G), energies 1e-11
  relative, atom forces 1e-10;
* switching back to the explicit structure factors restores that form;
* two FP64 steps (orthoT constraint, EES non-local on) against two oracle
  steps in the EES form: energies 1e-10, psi 1e-9; the mixed path within the
  energy (1e-6 Ha/atom) and force (1e-5 Ha/bohr) budget.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

CASES = [(12.0, 30.0, {"O": 3, "H": 6}, 48), (9.0, 20.0, {"O": 1, "H": 2}, 28)]
DT = 5.0
TOL = 1.0


def _rho(sysm, ctx):
    import torch
    from oracle import density as OD
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    rho = ctx.density(sysm.psi(), occ).cpu().numpy()
    o = OD.density_layout(sysm.box_len, sysm.ecut_ry, sysm.layout.n)
    return OD.rho_to_g(rho, o, sysm.box_len ** 3), o


@pytest.mark.parametrize("box,ecut,counts,grid", CASES)
def test_ees_local_pass_matches_oracle(box, ecut, counts, grid):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import density as OD
    from oracle import eext_ees as OX
    from oracle import layout as OL
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(box, ecut, 6, counts, nfft=grid)
    ctx = StepContext(sysm.layout, sysm.nstates, precision="fp64")
    try:
        ctx.set_atoms(sysm)
        rg, o = _rho(sysm, ctx)
        ng = ctx.set_local_ees(True)
        assert ng == OX.eext_grid_size(OL.calc_kmax(box, ecut))
        v, e, f = ctx.hart_eext(torch.from_numpy(rg).cuda())
        vr, eh, ee, ew, fr = OX.hart_eext_ees(rg, o.kx, o.ky, o.kz, box, 0.5 * ecut,
                                              sysm.atoms_dict(), sysm.tab, sysm.alp_ewd, ng)
        e = e.cpu().numpy()
        assert np.max(np.abs(v.cpu().numpy() - vr)) < 1e-11 * np.max(np.abs(vr))
        assert abs(e[2] - eh) < 1e-11 * abs(eh)
        assert abs(e[3] - ee) < 1e-11 * abs(ee)
        assert abs(e[4] - ew) < 1e-11 * abs(ew)
        assert np.max(np.abs(f.cpu().numpy() - fr)) < 1e-10 * np.max(np.abs(fr))
        # back to the explicit structure factors
        ctx.set_local_ees(False)
        v2, e2, f2 = ctx.hart_eext(torch.from_numpy(rg).cuda())
        vx, ehx, eex, ewx, fx = OD.hart_eext(rg, o.kx, o.ky, o.kz, box, 0.5 * ecut,
                                             sysm.atoms_dict(), sysm.tab, sysm.alp_ewd)
        assert abs(e2.cpu().numpy()[3] - eex) < 1e-11 * abs(eex)
        assert np.max(np.abs(f2.cpu().numpy() - fx)) < 1e-10 * np.max(np.abs(fx))
        assert ctx.device_errors() == 0
    finally:
        ctx.close()


def test_ees_local_rejects_other_orders():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200 import _lib
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(9.0, 20.0, 4, {"O": 1, "H": 2}, nfft=28)
    ctx = StepContext(sysm.layout, sysm.nstates, precision="fp64")
    try:
        with pytest.raises(_lib.CpstepError):
            ctx.set_local_ees(True, n_interp=8)  # no atoms yet
        ctx.set_atoms(sysm)
        with pytest.raises(_lib.CpstepError) as ei:
            ctx.set_local_ees(True, ngrid=32, n_interp=6)
        assert ei.value.code == _lib.CPSTEP_ERR_ARG
    finally:
        ctx.close()


@pytest.fixture(scope="module")
def ees_steps():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from oracle import density as OD
    from oracle import eext_ees as OX
    from oracle import layout as OL
    from oracle import step as OS
    from openatom_b200.system import System
    box, ecut, grid = 12.0, 30.0, 48
    sysm = System(box, ecut, 12, {"O": 4, "H": 8}, nfft=grid)
    lay = OL.Layout(box, ecut, grid=grid)
    dlay = OD.density_layout(box, ecut, grid)
    ng = OX.eext_grid_size(OL.calc_kmax(box, ecut))
    psi0 = sysm.psi(device="cpu")
    cmass = OS.cp_mass(lay, 25.0, ecut)
    p, v, dyn, ref = psi0.numpy(), np.zeros(tuple(psi0.shape), complex), None, []
    for it in (1, 2):
        p, v, en, f, aux = OS.cp_step(p, v, np.ones(sysm.nstates), sysm, lay, dlay, cmass, DT, it,
                                      nonlocal_on=True, tol_norb=TOL, dyn=dyn, eext_ees=ng)
        dyn = aux["dyn"]
        ref.append((en, f, p, v))
    return dict(sys=sysm, psi0=psi0, ref=ref, ecut=ecut)


def _run(d, precision):
    import torch
    from openatom_b200.context import StepContext
    s = d["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal(s)
        ctx.set_cp_mass(25.0, d["ecut"])
        ctx.set_constraint("ortho_t", TOL)
        ctx.set_local_ees(True)
        psi = d["psi0"].to("cuda", copy=True)
        v = torch.zeros_like(psi)
        occ = torch.ones(s.nstates, dtype=torch.float64, device="cuda")
        out = []
        for it in (1, 2):
            e, f = ctx.cp_step(psi, v, occ, DT, it)
            out.append((e.cpu().numpy().copy(), f.cpu().numpy().copy(), psi.cpu().numpy(),
                        v.cpu().numpy()))
        assert ctx.device_errors() == 0
        return out
    finally:
        ctx.close()


SLOTS = {"EXC": 0, "EHART": 2, "EEXT": 3, "EWD": 4, "EKE": 6, "ENL": 7, "ETOT": 8}


def test_fp64_steps_with_ees_local_match_oracle(ees_steps):
    out = _run(ees_steps, "fp64")
    for (e, f, p, v), (er, fr, pr, vr) in zip(out, ees_steps["ref"]):
        for name, slot in SLOTS.items():
            assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), name
        assert np.max(np.abs(f - fr)) <= 1e-9 * max(1.0, np.max(np.abs(fr)))
        assert np.max(np.abs(p - pr)) <= 1e-9


def test_mixed_steps_with_ees_local_within_budget(ees_steps):
    natm = ees_steps["sys"].natm
    out = _run(ees_steps, "mixed")
    for (e, f, p, v), (er, fr, pr, vr) in zip(out, ees_steps["ref"]):
        assert abs(e[8] - er["ETOT"]) / natm <= 1e-6
        assert np.max(np.abs(f - fr)) <= 1e-5
