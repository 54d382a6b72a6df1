"""The isokinetic NHC thermostat of the CP coefficients on the GPU against the
oracle (oracle/isokin.py, pinned to the reference's cp_isokin.C and
cp_dynamics.C): the integrator alone over several steps with sampled chain
states, and thermostatted steps of the whole electronic step."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

DT = 5.0


@pytest.fixture(scope="module")
def lay():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from oracle import layout as OL
    from openatom_b200.layout import StateLayout
    return StateLayout(10.0, 24.0, nfft=40), OL.Layout(10.0, 24.0, grid=40)


def _states(OK, p, nstates, seed):
    rng = np.random.default_rng(seed)
    return [OK.sample_state(p, rng) for _ in range(nstates)]


def _pack(states, key):
    return np.stack([st[key] for st in states])


@pytest.mark.parametrize("num,nck,nres,nyosh", [(2, 1, 4, 9), (3, 3, 2, 5)])
def test_integrate_matches_oracle(lay, num, nck, nres, nyosh):
    import torch
    from oracle import isokin as OK
    from oracle import step as OS
    from openatom_b200.context import StepContext
    glay, olay = lay
    S = 6
    rng = np.random.default_rng(7)
    n = olay.npts
    cls, ridx, rsrc = OS.point_classes(olay)
    ncoef = int(np.sum(cls != 0))
    p = OK.init_nhc(ncoef, 1, num, nck, 300.0, 25.0)
    states = _states(OK, p, S, 11)
    cmass = OS.cp_mass(olay, 25.0, 24.0)
    psi = rng.standard_normal((S, n)) + 1j * rng.standard_normal((S, n))
    v = 1e-3 * (rng.standard_normal((S, n)) + 1j * rng.standard_normal((S, n)))
    v[:, cls == 1] = v[:, cls == 1].real   # a G=0 velocity is real (get_fictKE would count it)
    ctx = StepContext(glay, S, precision="fp64")
    try:
        ctx.set_cp_mass(25.0, 24.0)
        ctx.set_cp_thermostat(300.0, 25.0, num, nck, nres, nyosh)
        x0, xp0, v0 = ctx.cp_thermostat_state()
        np.testing.assert_allclose(v0[..., 0], np.sqrt(p["kT"] / p["m"][0]), rtol=1e-14)
        ctx.cp_thermostat_state(_pack(states, "x"), _pack(states, "xp"), _pack(states, "vn"))
        dpsi = torch.from_numpy(psi.copy()).cuda()
        dv = torch.from_numpy(v.copy()).cuda()
        for it in (1, 2, 3):
            F = 1e-2 * (1.0 + 0.2 * it) * (rng.standard_normal((S, n))
                                           + 1j * rng.standard_normal((S, n)))
            ke = ctx.cp_integrate(torch.from_numpy(F).cuda(), dpsi, dv, DT, it)
            psi, v, kr, _, _ = OK.integrate_nhc(F, psi, v, cmass, cls, ridx, rsrc, p, states, DT,
                                                it, nres, nyosh)
            assert abs(float(ke) - kr) <= 1e-12 * abs(kr)
            assert np.max(np.abs(dpsi.cpu().numpy() - psi)) <= 1e-12
            assert np.max(np.abs(dv.cpu().numpy() - v)) <= 1e-12 * np.max(np.abs(v))
            x, xp, vn = ctx.cp_thermostat_state()
            assert np.max(np.abs(vn - _pack(states, "vn"))) <= 1e-11 * np.max(np.abs(vn))
            assert np.max(np.abs(x - _pack(states, "x"))) <= 1e-11 * max(1.0, np.max(np.abs(x)))
            en = p["m"][0] * vn[..., 0] ** 2 + p["m"][1] * vn[..., 1] ** 2
            np.testing.assert_allclose(en, p["kT"], rtol=1e-12)   # isokinetic constraint
    finally:
        ctx.close()


def test_thermostat_off_restores_plain_verlet(lay):
    import torch
    from oracle import step as OS
    from openatom_b200.context import StepContext
    glay, olay = lay
    S, n = 4, olay.npts
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((S, n)) + 1j * rng.standard_normal((S, n))
    v = 1e-3 * (rng.standard_normal((S, n)) + 1j * rng.standard_normal((S, n)))
    F = 1e-2 * (rng.standard_normal((S, n)) + 1j * rng.standard_normal((S, n)))
    ctx = StepContext(glay, S, precision="fp64")
    try:
        ctx.set_cp_mass(25.0, 24.0)
        ctx.set_cp_thermostat(300.0)
        ctx.set_cp_thermostat(0.0)
        dpsi, dv = torch.from_numpy(psi.copy()).cuda(), torch.from_numpy(v.copy()).cuda()
        ctx.cp_integrate(torch.from_numpy(F).cuda(), dpsi, dv, DT, 2)
        pr, vr, _ = OS.integrate(F, psi, v, OS.cp_mass(olay, 25.0, 24.0), olay, DT, 2)
        assert np.max(np.abs(dpsi.cpu().numpy() - pr)) <= 1e-13
        from openatom_b200 import _lib
        with pytest.raises(_lib.CpstepError):
            ctx.cp_thermostat_state()
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("reset", [False, True])
def test_thermostatted_steps_match_oracle(precision, reset):
    """Three thermostatted steps of the orthoT form against the oracle; with
    reset, cp_norb_tol sits just above the first step's deviation so the
    later steps take the PsiV reset (no second half kick and no NHC update
    of that half after it)."""
    import copy
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import density as OD
    from oracle import isokin as OK
    from oracle import layout as OL
    from oracle import step as OS
    from openatom_b200.context import StepContext
    from openatom_b200.system import System
    sysm = System(12.0, 30.0, 8, {"O": 2, "H": 4}, nfft=48)
    lay = OL.Layout(12.0, 30.0, grid=48)
    dlay = OD.density_layout(12.0, 30.0, 48)
    cls, _, _ = OS.point_classes(lay)
    p = OK.init_nhc(int(np.sum(cls != 0)), 1, 2, 1, 300.0, 25.0)
    states = _states(OK, p, sysm.nstates, 3)
    cmass = OS.cp_mass(lay, 25.0, 30.0)
    psi = sysm.psi()
    occ = torch.ones(sysm.nstates, dtype=torch.float64, device="cuda")
    pn = psi.cpu().numpy()
    vn = np.zeros_like(pn)
    tol = 1.0
    if reset:  # probe the first step's max |S - 2I|
        _, _, _, _, aux = OS.cp_step(pn, vn, np.ones(sysm.nstates), sysm, lay, dlay, cmass, DT,
                                     1, nhc=(p, copy.deepcopy(states), 4, 9), tol_norb=1.0)
        tol = 1.5 * aux["dyn"]["dev"]
    ctx = StepContext(sysm.layout, sysm.nstates, precision=precision)
    try:
        ctx.set_atoms(sysm)
        ctx.set_cp_mass(25.0, 30.0)
        ctx.set_cp_thermostat(300.0)
        ctx.set_constraint("ortho_t", tol)
        ctx.cp_thermostat_state(_pack(states, "x"), _pack(states, "xp"), _pack(states, "vn"))
        dpsi, dv = psi.clone(), torch.zeros_like(psi)
        dyn = None
        for it in (1, 2, 3):
            e, _ = ctx.cp_step(dpsi, dv, occ, DT, it)
            pn, vn, er, _, aux = OS.cp_step(pn, vn, np.ones(sysm.nstates), sysm, lay, dlay, cmass,
                                            DT, it, nhc=(p, states, 4, 9), tol_norb=tol, dyn=dyn)
            dyn = aux["dyn"]
            assert ctx.dyn_status()[1] == dyn["resets"]
            e = e.cpu().numpy()
            if precision == "fp64":
                for name, slot in (("ETOT", 8), ("FICT", 9), ("NHC_KE", 12), ("NHC_POT", 13)):
                    assert abs(e[slot] - er[name]) <= 1e-9 * max(1e-6, abs(er[name])), name
                assert np.max(np.abs(dpsi.cpu().numpy() - pn)) < 1e-9
            else:
                assert abs(e[8] - er["ETOT"]) / sysm.natm <= 1e-6
                assert abs(e[12] - er["NHC_KE"]) <= 1e-6 * abs(er["NHC_KE"])
    finally:
        ctx.close()
