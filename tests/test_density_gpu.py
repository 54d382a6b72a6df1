"""Density side on the GPU (XC, density FFT, Hartree/local/Ewald, V_KS) vs the oracle."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dsys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 8, {"O": 3, "H": 6}, nfft=48)
    psi = sysm.psi()
    ctx = StepContext(sysm.layout, sysm.nstates, precision="fp64")
    ctx.set_atoms(sysm)
    import torch
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    rho = ctx.density(psi, occ)
    yield dict(sys=sysm, ctx=ctx, rho=rho)
    ctx.close()


def _olay(d):
    from oracle import density as OD
    s = d["sys"]
    return OD.density_layout(s.box_len, s.ecut_ry, s.layout.n)


def test_density_layout_matches_oracle(dsys):
    kx, ky, kz = dsys["ctx"].rho_layout()
    o = _olay(dsys)
    assert np.array_equal(kx, o.kx) and np.array_equal(ky, o.ky) and np.array_equal(kz, o.kz)


def test_xc_matches_oracle(dsys):
    from oracle import density as OD
    v, e = dsys["ctx"].exc(dsys["rho"])
    vr, exc, mu = OD.pz_lda(dsys["rho"].cpu().numpy(), dsys["sys"].box_len ** 3)
    assert np.max(np.abs(v.cpu().numpy() - vr)) < 1e-12 * np.max(np.abs(vr))
    e = e.cpu().numpy()
    assert abs(e[0] - exc) < 1e-11 * abs(exc)
    assert abs(e[1] - mu) < 1e-11 * abs(mu)


def test_rho_fft_matches_oracle(dsys):
    from oracle import density as OD
    rg = dsys["ctx"].rho_r2g(dsys["rho"]).cpu().numpy()
    ref = OD.rho_to_g(dsys["rho"].cpu().numpy(), _olay(dsys), dsys["sys"].box_len ** 3)
    assert np.max(np.abs(rg - ref)) < 1e-12 * np.max(np.abs(ref))
    # G = 0 term is the electron count (2 per state)
    i0 = np.nonzero((_olay(dsys).kx == 0) & (_olay(dsys).ky == 0) & (_olay(dsys).kz == 0))[0][0]
    assert abs(ref[i0].real - 2.0 * dsys["sys"].nstates) < 1e-9


def test_hart_eext_matches_oracle(dsys):
    from oracle import density as OD
    s = dsys["sys"]
    o = _olay(dsys)
    rg = OD.rho_to_g(dsys["rho"].cpu().numpy(), o, s.box_len ** 3)
    import torch
    v, e, f = dsys["ctx"].hart_eext(torch.from_numpy(rg).cuda())
    vr, eh, ee, ew, fr = OD.hart_eext(rg, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry,
                                      s.atoms_dict(), s.tab, s.alp_ewd)
    e = e.cpu().numpy()
    assert np.max(np.abs(v.cpu().numpy() - vr)) < 1e-12 * np.max(np.abs(vr))
    assert abs(e[2] - eh) < 1e-11 * abs(eh)
    assert abs(e[3] - ee) < 1e-11 * abs(ee)
    assert abs(e[4] - ew) < 1e-11 * abs(ew)
    assert np.max(np.abs(f.cpu().numpy() - fr)) < 1e-10 * np.max(np.abs(fr))


def test_vks_chain_matches_oracle(dsys):
    from oracle import density as OD
    s = dsys["sys"]
    o = _olay(dsys)
    rho = dsys["rho"].cpu().numpy()
    v, e, f = dsys["ctx"].vks_from_rho(dsys["rho"])
    vxc, exc, mu = OD.pz_lda(rho, s.box_len ** 3)
    rg = OD.rho_to_g(rho, o, s.box_len ** 3)
    vg, eh, ee, ew, fr = OD.hart_eext(rg, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry,
                                      s.atoms_dict(), s.tab, s.alp_ewd)
    vref = vxc + OD.vg_to_r(vg, o)
    assert np.max(np.abs(v.cpu().numpy() - vref)) < 1e-11 * np.max(np.abs(vref))


def test_local_force_is_minus_energy_gradient(dsys):
    """Finite difference of E_ext + E_ewd in one atom coordinate (fixed rho)."""
    from oracle import density as OD
    s = dsys["sys"]
    o = _olay(dsys)
    rg = OD.rho_to_g(dsys["rho"].cpu().numpy(), o, s.box_len ** 3)
    a = s.atoms_dict()
    _, _, _, _, f = OD.hart_eext(rg, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry, a, s.tab, s.alp_ewd)
    h = 1e-4
    for d in range(3):
        ep, em = [], []
        for sgn, lst in ((1, ep), (-1, em)):
            pos = a["pos"].copy()
            pos[0, d] += sgn * h
            b = dict(a, pos=pos)
            _, _, ee, ew, _ = OD.hart_eext(rg, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry, b,
                                           s.tab, s.alp_ewd)
            lst.append(ee + ew)
        fd = -(ep[0] - em[0]) / (2 * h)
        assert abs(fd - f[0, d]) < 1e-6 * max(1.0, abs(fd))


@pytest.fixture(scope="module")
def big():
    """The 768-atom box and grid (L = 37.2 bohr, 70 Ry, 200^3) with a few states:
    the density sphere's plane (99 columns of 201 FP64 complex) does not fit in
    a block's shared memory, so the split plane passes run."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(37.2, 70.0, 4, {"O": 4, "H": 8}, nfft=200, seed=3)
    ctx = StepContext(sysm.layout, sysm.nstates, precision="fp64")
    ctx.set_atoms(sysm)
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    rho = ctx.density(sysm.psi(), occ)
    yield dict(sys=sysm, ctx=ctx, rho=rho, occ=occ)
    ctx.close()


def test_split_plane_passes_at_200(big):
    from oracle import density as OD
    s = big["sys"]
    o = OD.density_layout(s.box_len, s.ecut_ry, 200)
    assert int(o.kx.max()) + 1 == 99  # the plane that needs the split passes
    rho = big["rho"].cpu().numpy()
    rg = big["ctx"].rho_r2g(big["rho"]).cpu().numpy()
    ref = OD.rho_to_g(rho, o, s.box_len ** 3)
    assert np.max(np.abs(rg - ref)) < 1e-12 * np.max(np.abs(ref))
    v, e, f = big["ctx"].vks_from_rho(big["rho"])
    vxc, exc, mu = OD.pz_lda(rho, s.box_len ** 3)
    vg, eh, ee, ew, fr = OD.hart_eext(ref, o.kx, o.ky, o.kz, s.box_len, 0.5 * s.ecut_ry,
                                      s.atoms_dict(), s.tab, s.alp_ewd)
    vref = vxc + OD.vg_to_r(vg, o)
    assert np.max(np.abs(v.cpu().numpy() - vref)) < 1e-11 * np.max(np.abs(vref))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_runs_at_200(big, precision):
    import torch
    from openatom_b200.context import StepContext
    s = big["sys"]
    ctx = StepContext(s.layout, s.nstates, precision=precision)
    try:
        ctx.set_atoms(s)
        ctx.set_nonlocal(s)
        ctx.set_cp_mass(25.0, 70.0)
        ctx.set_constraint("ortho_t", 1.0)  # cp_norb_tol above this step's deviation
        psi = s.psi()
        v = torch.zeros_like(psi)
        e, f = ctx.cp_step(psi, v, big["occ"], 5.0, 1)
        it, ok = ctx.step_status()
        assert ok and np.isfinite(e.cpu().numpy()).all()
    finally:
        ctx.close()
