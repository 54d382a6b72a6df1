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
