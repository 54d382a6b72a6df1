"""BLYP on the GPU (cpstep_set_xc, cpstep_gga_functional, the density side
and the step with BLYP) against the oracle (oracle/xc.py, pinned to the
reference's cp_becke.C / cp_grad_rho_ctrl.C / cp_pz_lda.C)."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0


@pytest.fixture(scope="module")
def bsys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 8, {"O": 3, "H": 6}, nfft=48)
    ctx = StepContext(sysm.layout, sysm.nstates, precision="fp64")
    ctx.set_atoms(sysm)
    ctx.set_xc("blyp")
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    rho = ctx.density(sysm.psi(), occ)
    yield dict(sys=sysm, ctx=ctx, rho=rho)
    ctx.close()


def test_gga_functional_matches_oracle(bsys):
    import torch
    from oracle import xc as OX
    rho = bsys["rho"]
    rng = np.random.default_rng(7)
    g = [torch.from_numpy(rng.standard_normal(rho.shape) * 0.05).cuda() for _ in range(3)]
    vks0 = torch.from_numpy(rng.standard_normal(rho.shape)).cuda()
    v, ux, uy, uz, e = bsys["ctx"].gga_functional(rho, *g, vks0)
    dv, ox, oy, oz, oe = OX.gga_functional(rho.cpu().numpy(), *(a.cpu().numpy() for a in g),
                                           bsys["sys"].box_len ** 3)
    d = (v - vks0).cpu().numpy().ravel()
    assert np.max(np.abs(d - dv)) < 1e-12 * np.max(np.abs(dv))
    for a, b in ((ux, ox), (uy, oy), (uz, oz)):
        assert np.max(np.abs(a.cpu().numpy().ravel() - b)) < 1e-12 * np.max(np.abs(b))
    assert abs(float(e[10]) - oe) < 1e-12 * abs(oe)


def test_blyp_lda_part_is_slater_exchange(bsys):
    from oracle import xc as OX
    v, e = bsys["ctx"].exc(bsys["rho"])
    vr, er, mr = OX.slater_lda(bsys["rho"].cpu().numpy(), bsys["sys"].box_len ** 3)
    assert np.max(np.abs(v.cpu().numpy() - vr)) < 1e-13 * np.max(np.abs(vr))
    assert abs(float(e[0]) - er) < 1e-12 * abs(er)
    assert abs(float(e[1]) - mr) < 1e-12 * abs(mr)


def test_blyp_vks_chain_matches_oracle(bsys):
    """Slater exchange, density gradients, CP_getGGAFunctional, White-Bird and
    Hartree/local: V_KS(r), EEXC (LDA + GGA) and EXC_GGA."""
    from oracle import density as OD
    from oracle import xc as OX
    s = bsys["sys"]
    o = OD.density_layout(s.box_len, s.ecut_ry, s.layout.n)
    rho = bsys["rho"].cpu().numpy()
    vol = s.box_len ** 3
    v, e, f = bsys["ctx"].vks_from_rho(bsys["rho"])
    vxc, exc, mu, egga = OX.blyp_vxc(rho, o, vol)
    rg = OD.rho_to_g(rho, o, vol)
    vg, eh, ee, ew, fr = OD.hart_eext(rg, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry,
                                      s.atoms_dict(), s.tab, s.alp_ewd)
    vref = vxc + OD.vg_to_r(vg, o)
    e = e.cpu().numpy()
    assert egga != 0.0
    assert np.max(np.abs(v.cpu().numpy() - vref)) < 1e-11 * np.max(np.abs(vref))
    assert abs(e[0] - exc) < 1e-11 * abs(exc)
    assert abs(e[10] - egga) < 1e-11 * abs(egga)


@pytest.fixture(scope="module")
def bstep():
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
                                    dlay, cmass, DT, 1, xc="blyp", tol_norb=1.0)
    return dict(sys=sysm, psi=psi, occ=occ, ref=(p1, v1, en1, f1))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_blyp_step_matches_oracle(bstep, precision):
    import torch
    from openatom_b200.context import StepContext
    s = bstep["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_cp_mass(25.0, 30.0)
        ctx.set_xc("blyp")
        ctx.set_constraint("ortho_t", 1.0)  # cp_norb_tol above this step's deviation
        psi = bstep["psi"].clone()
        v = torch.zeros_like(psi)
        e, f = ctx.cp_step(psi, v, bstep["occ"], DT, 1)
        _, ok = ctx.step_status()
        assert ok
        pr, vr, er, fr = bstep["ref"]
        e = e.cpu().numpy()
        if precision == "fp64":
            for name, slot in (("EXC", 0), ("EHART", 2), ("EEXT", 3), ("EKE", 6), ("ETOT", 8)):
                assert abs(e[slot] - er[name]) <= 1e-10 * max(1.0, abs(er[name])), name
            assert np.max(np.abs(psi.cpu().numpy() - pr)) < 1e-9
        else:
            assert abs(e[8] - er["ETOT"]) / s.natm <= 1e-6
            assert np.max(np.abs(f.cpu().numpy() - fr)) <= 1e-5
    finally:
        ctx.close()
