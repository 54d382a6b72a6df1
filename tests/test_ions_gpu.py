"""Ions on the GPU: real-space Ewald forces and energy (cpstep_ion_forces)
and the NVE atom step (cpstep_atoms_integrate) against the oracle
(oracle/ions.py, pinned to the reference's CP_getionforce), and the
context's positions following the integrator."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def isys():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from openatom_b200.system import System
    return System(12.0, 30.0, 8, {"O": 4, "H": 8}, nfft=48, seed=4)


def _cell(L):
    h = np.zeros(9)
    h[0] = h[4] = h[8] = L
    hi = np.zeros(9)
    hi[0] = hi[4] = hi[8] = 1.0 / L
    return h, hi


def _q(s):
    a = s.atoms_dict()
    return np.asarray(a["q"], dtype=np.float64)[np.asarray(s.typ)]


def test_ion_forces_match_oracle(isys):
    import torch
    from oracle import ions as OI
    from openatom_b200.context import StepContext
    s = isys
    ctx = StepContext(s.layout, s.nstates, precision="fp64")
    try:
        ctx.set_atoms(s)
        f0 = torch.ones((s.natm, 3), dtype=torch.float64, device="cuda")
        f, e = ctx.ion_forces(f0.clone())
        h, hi = _cell(s.box_len)
        pot, vs, vb, fr = OI.ewald_rs(s.pos, _q(s), h, hi, s.box_len ** 3, s.alp_ewd,
                                      4.0 * 0.5 * s.ecut_ry)
        assert abs(float(e[11]) - (pot + vs + vb)) < 1e-11 * abs(pot + vs + vb)
        assert np.max(np.abs(f.cpu().numpy() - 1.0 - fr)) < 1e-11 * np.max(np.abs(fr))
    finally:
        ctx.close()


def test_atoms_integrate_matches_oracle_and_moves_the_context(isys):
    import torch
    from oracle import ions as OI
    from openatom_b200.context import StepContext
    s = isys
    rng = np.random.default_rng(5)
    ctx = StepContext(s.layout, s.nstates, precision="fp64")
    ref = StepContext(s.layout, s.nstates, precision="fp64")
    try:
        ctx.set_atoms(s)
        pos = torch.from_numpy(np.ascontiguousarray(s.pos)).cuda()
        vel = torch.from_numpy(rng.standard_normal((s.natm, 3)) * 1e-4).cuda()
        frc = torch.from_numpy(rng.standard_normal((s.natm, 3)) * 1e-2).cuda()
        mass = torch.from_numpy(np.where(np.asarray(s.typ) == 0, 29156.9, 1837.15)).cuda()
        p0, v0 = pos.cpu().numpy(), vel.cpu().numpy()
        pr, vr, ekr = OI.nve_step(1, p0, v0, frc.cpu().numpy(), mass.cpu().numpy(), 20.0)
        ek = ctx.atoms_integrate(1, pos, vel, frc, mass, 20.0)
        assert abs(ek - ekr) < 1e-12 * ekr
        assert np.max(np.abs(pos.cpu().numpy() - pr)) < 1e-13
        assert np.max(np.abs(vel.cpu().numpy() - vr)) < 1e-15
        # the context now sees the moved atoms: same local/Ewald energies as a
        # context set up at the new positions
        occ = torch.ones(s.nstates, dtype=torch.float64, device="cuda")
        rho = ctx.density(s.psi(), occ)
        _, e1, f1 = ctx.vks_from_rho(rho)
        ref.set_atoms(s)
        ref.set_positions(pr)
        _, e2, f2 = ref.vks_from_rho(rho)
        assert np.allclose(e1.cpu().numpy()[2:5], e2.cpu().numpy()[2:5], rtol=1e-12, atol=0.0)
        assert np.max(np.abs(f1.cpu().numpy() - f2.cpu().numpy())) < 1e-12 * np.max(np.abs(f2.cpu().numpy()))
    finally:
        ctx.close()
        ref.close()


@pytest.mark.parametrize("L,nres,nyosh", [(4, 1, 1), (2, 4, 9)])
def test_atoms_nvt_matches_oracle(isys, L, nres, nyosh):
    """The massive-NHC NVT atom step against oracle/ions.py nvt_step (pinned to
    integration_drivers.C) over three steps, chains loaded from a sample."""
    import torch
    from oracle import ions as OI
    from openatom_b200.context import StepContext
    s = isys
    n = s.natm
    rng = np.random.default_rng(L * 7 + nyosh)
    mass = np.where(np.asarray(s.typ) == s.typ[0], 29164.0, 1837.0).astype(np.float64)
    kT = np.full(n, 300.0 / 315777.0)
    mnhc = kT[:, None] * (200.0 / 0.0241888) ** 2 * (1.0 + 0.1 * np.arange(L))[None, :]
    vn = rng.standard_normal((n, 3, L)) * np.sqrt(kT[:, None, None] / mnhc[:, None, :])
    pkt = np.zeros(n)
    pos_h = np.array(s.pos, dtype=np.float64)
    vel_h = rng.standard_normal((n, 3)) * np.sqrt(kT[:, None] / mass[:, None])
    ctx = StepContext(s.layout, s.nstates, precision="fp64")
    try:
        ctx.set_atoms(s)
        ctx.set_atom_thermostat(L, kT, mnhc, nres, nyosh)
        ctx.atom_thermostat_state(vn, pkt)
        pos = torch.from_numpy(pos_h.copy()).cuda()
        vel = torch.from_numpy(vel_h.copy()).cuda()
        dm = torch.from_numpy(mass).cuda()
        for it in range(3):
            f = 1e-3 * rng.standard_normal((n, 3))
            ek = ctx.atoms_integrate(it, pos, vel, torch.from_numpy(f).cuda(), dm, 20.0)
            pos_h, vel_h, ekr, eknr, potr = OI.nvt_step(it, pos_h, vel_h, f, mass, kT, mnhc, vn,
                                                        pkt, 20.0, nres, nyosh)
            gvn, gpk, ge = ctx.atom_thermostat_state()
            assert abs(ek - ekr) <= 1e-12 * ekr
            assert abs(ge[0] - eknr) <= 1e-12 * eknr
            assert abs(ge[1] - potr) <= 1e-12 * max(1e-12, abs(potr))
            assert np.max(np.abs(vel.cpu().numpy() - vel_h)) <= 1e-12 * np.max(np.abs(vel_h))
            assert np.max(np.abs(gvn - vn)) <= 1e-12 * np.max(np.abs(vn))
            assert np.max(np.abs(pos.cpu().numpy() - pos_h)) <= 1e-12
        ctx.set_atom_thermostat(0)
        from openatom_b200 import _lib
        with pytest.raises(_lib.CpstepError):
            ctx.atom_thermostat_state()
    finally:
        ctx.close()
