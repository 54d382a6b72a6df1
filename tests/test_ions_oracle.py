"""Real-space ion-ion forces and the NVE atom step: the oracle (oracle/ions.py)
against the reference's CP_getionforce compiled from cp_rspace_ion.C
(oracle/_ref, ref_ion.cpp), and the forces against finite differences of the
energy.  Host only."""
import ctypes

import numpy as np
import pytest

from oracle import ions as OI


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _cell(L):
    h = np.zeros(9)
    h[0] = h[4] = h[8] = L
    hi = np.zeros(9)
    hi[0] = hi[4] = hi[8] = 1.0 / L
    return h, hi


def _atoms(n, L, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.2 * L, 1.2 * L, (n, 3))   # some outside the cell: minimum image
    q = rng.choice([6.0, 1.0], n)
    return pos, q


@pytest.fixture(scope="module")
def ref():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_ionforce"):
        pytest.skip("oracle/_ref/libref.so with CP_getionforce is not built")
    lib.ref_ionforce.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    return lib


def test_ewald_rs_matches_reference(ref):
    L, alp, ecut = 12.0, 0.45, 60.0
    pos, q = _atoms(24, L, 1)
    h, hi = _cell(L)
    pot, vs, vb, f = OI.ewald_rs(pos, q, h, hi, L ** 3, alp, ecut)
    rf = np.zeros((24, 3))
    out = np.zeros(3)
    ref.ref_ionforce(24, _p(np.ascontiguousarray(pos)), _p(q), _p(h), _p(hi), L ** 3, alp, ecut,
                     _p(rf), _p(out))
    assert abs(pot - out[0]) < 1e-12 * abs(out[0])
    assert abs(vs - out[1]) < 1e-13 * abs(out[1]) and abs(vb - out[2]) < 1e-13 * abs(out[2])
    assert np.max(np.abs(f - rf)) < 1e-12 * np.max(np.abs(rf))


def test_ewald_rs_force_is_minus_energy_gradient():
    L, alp = 12.0, 0.45
    pos, q = _atoms(10, L, 2)
    h, hi = _cell(L)
    _, _, _, f = OI.ewald_rs(pos, q, h, hi, L ** 3, alp, 60.0)
    eps = 1e-5
    for i in (0, 3):
        for d in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[i, d] += eps
            pm[i, d] -= eps
            ep = OI.ewald_rs(pp, q, h, hi, L ** 3, alp, 60.0)[0]
            em = OI.ewald_rs(pm, q, h, hi, L ** 3, alp, 60.0)[0]
            # the polynomial erfc is not exactly the derivative pair of its own
            # derivative polynomial: agreement to the approximation's accuracy
            assert abs(-(ep - em) / (2 * eps) - f[i, d]) < 2e-6 * max(1.0, abs(f[i, d]))


def test_nve_step_is_velocity_verlet():
    rng = np.random.default_rng(3)
    pos, vel, f = rng.standard_normal((3, 5, 3))
    m = rng.uniform(1e3, 3e4, 5)
    p1, v1, ek0 = OI.nve_step(0, pos, vel, f, m, 2.0)
    assert np.allclose(v1, vel + 2.0 * f / m[:, None] * 0.5)
    assert np.allclose(p1, pos + 2.0 * v1)
    assert abs(ek0 - 0.5 * np.sum(m[:, None] * vel * vel)) < 1e-12 * ek0
    p2, v2, ek1 = OI.nve_step(1, p1, v1, f, m, 2.0)
    vh = v1 + f / m[:, None]
    assert abs(ek1 - 0.5 * np.sum(m[:, None] * vh * vh)) < 1e-12 * ek1


@pytest.mark.parametrize("L,nres,nyosh", [(4, 1, 1), (3, 2, 3), (2, 4, 9)])
def test_nvt_step_matches_reference(L, nres, nyosh):
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_atom_nvt_step"):
        pytest.skip("oracle/_ref/libref.so with integration_drivers.C is not built")
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.ref_atom_nvt_step.argtypes = [i, i, i] + [vp] * 8 + [d, i, i, vp]
    rng = np.random.default_rng(L)
    n, dt = 9, 20.0
    pos = rng.uniform(0.0, 10.0, (n, 3))
    mass = rng.choice([29164.0, 1837.0], n)
    kT = np.full(n, 300.0 / 315777.0)
    vel = rng.standard_normal((n, 3)) * np.sqrt(kT[:, None] / mass[:, None])
    mnhc = kT[:, None] * (200.0 / 0.0241888) ** 2 * (1.0 + 0.1 * np.arange(L))[None, :]
    vn = rng.standard_normal((n, 3, L)) * np.sqrt(kT[:, None, None] / mnhc[:, None, :])
    pkt = np.zeros(n)
    rp, rv, rvn, rpk = pos.copy(), vel.copy(), vn.copy(), pkt.copy()
    for it in range(3):
        f = 1e-3 * rng.standard_normal((n, 3))
        out = np.zeros(3)
        lib.ref_atom_nvt_step(n, L, it, _p(rp), _p(rv), _p(f), _p(mass), _p(kT), _p(mnhc),
                              _p(rvn), _p(rpk), dt, nres, nyosh, _p(out))
        pos, vel, ek, ekn, pot = OI.nvt_step(it, pos, vel, f, mass, kT, mnhc, vn, pkt, dt, nres,
                                             nyosh)
        assert abs(ek - out[0]) <= 1e-13 * abs(out[0])
        assert abs(ekn - out[1]) <= 1e-13 * abs(out[1])
        assert abs(pot - out[2]) <= 1e-12 * max(1e-12, abs(out[2]))
        np.testing.assert_allclose(vel, rv, rtol=1e-13, atol=1e-18)
        np.testing.assert_allclose(vn, rvn, rtol=1e-13, atol=1e-18)
        assert np.max(np.abs(pos - rp)) <= 1e-12
