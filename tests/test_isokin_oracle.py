"""The CP velocity Verlet with isokinetic Nose-Hoover chains: the oracle
(oracle/isokin.py) against the reference's initCPNHC / cp_isoNHC_update /
CP_integrate_dyn compiled from cp_isokin.C and cp_dynamics.C (oracle/_ref,
ref_isokin.cpp), over several steps; and the constraint the thermostat keeps.
Host only."""
import ctypes

import numpy as np
import pytest

from oracle import isokin as OK

DT = 5.0


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def ref():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_cp_integrate_dyn"):
        pytest.skip("oracle/_ref/libref.so with cp_isokin.C / cp_dynamics.C is not built")
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.ref_init_cpnhc.argtypes = [i, i, i, i, d, d] + [vp] * 7
    lib.ref_cp_integrate_dyn.argtypes = [i, i, vp, vp, vp, vp, i, i, i, i, i, vp, vp, vp, d, i, i,
                                         d, d, vp]
    return lib


@pytest.mark.parametrize("num,nck", [(2, 1), (3, 4)])
def test_init_matches_reference(ref, num, nck):
    p = OK.init_nhc(1001, 1, num, nck, 300.0, 25.0)
    out = np.zeros(6)
    v0, a2, a4, dfs = (np.zeros(n) for n in (num, num, num, nck))
    istr, iend = np.zeros(nck, dtype=np.int32), np.zeros(nck, dtype=np.int32)
    ref.ref_init_cpnhc(1001, 1, num, nck, 300.0, 25.0, _p(out), _p(v0), _p(a2), _p(a4), _p(dfs),
                       _p(istr), _p(iend))
    assert out[0] == p["kT"]
    np.testing.assert_allclose(out[4:6], p["m"], rtol=1e-15)
    for a, b in ((v0, p["v0"]), (a2, p["a2"]), (a4, p["a4"]), (dfs, p["dfs"])):
        np.testing.assert_allclose(a, b, rtol=1e-15)
    assert list(istr) == p["istr"] and list(iend) == p["iend"]


def _chare(rng, n, nred, nuni):
    """A chare's packed arrays: nred redundant points first (left alone), G = 0,
    nuni - 1 unique Gx = 0 points, the rest; masses like set_cpmass."""
    psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    v = 1e-3 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    f = 1e-2 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    m = 400.0 * (1.0 + rng.uniform(0.0, 3.0, n))
    m[nred] = 200.0
    v[nred] = v[nred].real
    return psi, v, f, m


@pytest.mark.parametrize("num,nck,nres,nyosh", [(2, 1, 4, 9), (2, 3, 2, 5), (3, 2, 1, 7)])
def test_integrate_matches_reference(ref, num, nck, nres, nyosh):
    rng = np.random.default_rng(num * 10 + nck)
    n, nred, nuni = 700, 12, 13
    psi, v, f, m = _chare(rng, n, nred, nuni)
    te, tau = 300.0, 25.0
    p = OK.init_nhc(n - nred, 1, num, nck, te, tau)
    st = OK.sample_state(p, rng)
    rst = {k: np.ascontiguousarray(a.copy()) for k, a in st.items()}
    rpsi, rv = psi.copy(), v.copy()
    opsi, ov = psi[nred:].copy(), v[nred:].copy()
    for it in (1, 2, 3, 4):
        fr = f * (1.0 + 0.1 * it)
        rf = fr.copy()
        mm = m.copy()
        out = np.zeros(3)
        ref.ref_cp_integrate_dyn(n, it, _p(rf), _p(rv), _p(rpsi), _p(mm), nred, nuni, 1, num,
                                 nck, _p(rst["x"]), _p(rst["xp"]), _p(rst["vn"]), DT, nres, nyosh,
                                 te, tau, _p(out))
        opsi, ov, ke, ekn, pot = OK.integrate_dyn_chare(opsi, ov, fr[nred:], m[nred:], 1, nuni,
                                                        p, st, DT, it, nres, nyosh)
        assert abs(ke - out[0]) <= 1e-12 * abs(out[0])
        assert abs(ekn - out[1]) <= 1e-12 * abs(out[1])
        assert abs(pot - out[2]) <= 1e-10 * max(1e-3, abs(out[2]))
        assert np.max(np.abs(opsi - rpsi[nred:])) <= 1e-12
        assert np.max(np.abs(ov - rv[nred:])) <= 1e-12 * np.max(np.abs(rv))
        for k in ("x", "vn"):
            assert np.max(np.abs(st[k] - rst[k])) <= 1e-11 * max(1.0, np.max(np.abs(rst[k]))), k


def test_isokinetic_constraint_holds():
    rng = np.random.default_rng(3)
    p = OK.init_nhc(500, 1, 2, 2, 300.0, 25.0)
    st = OK.sample_state(p, rng)
    v = 1e-3 * (rng.standard_normal(500) + 1j * rng.standard_normal(500))
    m = np.full(500, 400.0)
    for _ in range(3):
        OK.iso_update(v, m, p, st, DT, 4, 9)
        en = p["m"][0] * st["vn"][..., 0] ** 2 + p["m"][1] * st["vn"][..., 1] ** 2
        np.testing.assert_allclose(en, p["kT"], rtol=1e-13)
