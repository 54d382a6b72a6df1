"""BLYP exchange-correlation oracle (oracle/xc.py) against the reference's own
routines compiled from cp_becke.C, cp_grad_rho_ctrl.C and cp_pz_lda.C
(oracle/_ref, ref_xc.cpp), and the BLYP potential against finite differences
of the BLYP energy.  Host only."""
import ctypes
import math

import numpy as np
import pytest

from oracle import xc as OX


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def ref():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_gga_functional"):
        pytest.skip("oracle/_ref/libref.so with the XC routines is not built")
    lib.ref_becke.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    lib.ref_lyp.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    lib.ref_gga_functional.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_double,
                                                            ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 6
    lib.ref_exc_calc.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.c_int] + \
        [ctypes.c_void_p] * 4
    return lib


def _samples(seed=0, n=400):
    rng = np.random.default_rng(seed)
    rho = 10.0 ** rng.uniform(-5, 1, n)
    g2 = 10.0 ** rng.uniform(-10, 2, n)
    return rho, g2


def test_becke_and_lyp_match_reference(ref):
    rho, g2 = _samples()
    out = np.zeros(3)
    fb = np.array(OX.becke(rho, g2)).T
    fl = np.array(OX.lyp(rho, g2)).T
    for i in range(len(rho)):
        ref.ref_becke(rho[i], g2[i], OX.BECKE_BETA, _p(out))
        assert np.allclose(fb[i], out, rtol=1e-13, atol=0.0)
        ref.ref_lyp(rho[i], g2[i], _p(out))
        assert np.allclose(fl[i], out, rtol=1e-12, atol=1e-300)


def _grid_density(shape, seed):
    rng = np.random.default_rng(seed)
    rho = np.exp(rng.uniform(np.log(1e-7), np.log(2.0), shape))
    grads = [rng.standard_normal(shape) * 0.3 for _ in range(3)]
    return rho, grads


@pytest.mark.parametrize("shape", [(4, 5, 6), (6, 4, 7)])
def test_gga_functional_matches_reference(ref, shape):
    """The pointwise driver on an odd/even mix of grid sizes (row padding),
    including points below rho_cut and inside the switching band."""
    nf3, nf2, nf1 = shape
    rho, (gx, gy, gz) = _grid_density(shape, 3)
    rho.flat[:5] = [1e-7, 4e-6, 5e-6, 2e-5, 1.9e-4]        # below, at and inside the switch
    vol = 123.4
    vks0 = np.random.default_rng(4).standard_normal(shape)
    dv, ux, uy, uz, e = OX.gga_functional(rho, gx, gy, gz, vol)
    rx, ry, rz, rv = (np.ascontiguousarray(a.copy()) for a in (gx, gy, gz, vks0))
    exc = np.zeros(1)
    ref.ref_gga_functional(nf1, nf2, nf3, vol, OX.GGA_CUT, 1, 1, _p(np.ascontiguousarray(rho)),
                           _p(rx), _p(ry), _p(rz), _p(rv), _p(exc))
    assert abs(e - exc[0]) < 1e-13 * abs(exc[0])
    assert np.allclose(vks0.ravel() + dv, rv.ravel(), rtol=1e-13, atol=1e-15)
    for a, b in ((ux, rx), (uy, ry), (uz, rz)):
        assert np.allclose(a, b.ravel(), rtol=1e-13, atol=1e-15)


def test_slater_part_matches_reference(ref):
    shape = (5, 6, 7)
    rho, _ = _grid_density(shape, 5)
    vol = 77.0
    v, e, mu = OX.slater_lda(rho, vol)
    rv = np.zeros(shape)
    exc, muxc = np.zeros(1), np.zeros(1)
    ref.ref_exc_calc(7, 6, 5, vol, 1, _p(np.ascontiguousarray(rho)), _p(rv), _p(exc), _p(muxc))
    assert np.allclose(v, rv, rtol=1e-14, atol=0.0)
    assert abs(e - exc[0]) < 1e-13 * abs(exc[0]) and abs(mu - muxc[0]) < 1e-13 * abs(muxc[0])


@pytest.mark.parametrize("shape", [(5, 6, 7), (8, 8, 8)])
def test_pz_lda_matches_reference(ref, shape):
    """The benchmark's functional: CP_exc_calc with cp_lyp = 0 (Perdew-Zunger
    correlation on both sides of rs = 1, Slater exchange) against the oracle's
    pz_lda, densities from 1e-12 (rs ~ 6e3) to 2 (rs ~ 0.5).  At exactly zero
    density the reference's potential is NaN (rs = inf) where the oracle and
    the GPU put 0; a density of occupied states is positive everywhere."""
    from oracle import density as OD
    nf3, nf2, nf1 = shape
    rho, _ = _grid_density(shape, 7)
    rho.flat[0] = 1e-12
    vol = 91.0
    v, e, mu = OD.pz_lda(rho, vol)
    rv = np.zeros(shape)
    exc, muxc = np.zeros(1), np.zeros(1)
    ref.ref_exc_calc(nf1, nf2, nf3, vol, 0, _p(np.ascontiguousarray(rho)), _p(rv), _p(exc),
                     _p(muxc))
    assert np.allclose(np.asarray(v).reshape(shape), rv, rtol=1e-13, atol=0.0)
    assert abs(e - exc[0]) < 1e-13 * abs(exc[0]) and abs(mu - muxc[0]) < 1e-13 * abs(muxc[0])


@pytest.fixture(scope="module")
def dens():
    """A positive density band-limited inside the density sphere of a small box."""
    from oracle import density as OD
    box, ecut, n = 10.0, 12.0, 24
    lay = OD.density_layout(box, ecut, n)
    x = np.arange(n) * box / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    k = 2.0 * math.pi / box
    rho = 0.02 * (1.0 + 0.5 * np.cos(k * X) * np.cos(k * Y) + 0.3 * np.sin(2 * k * Z)
                  + 0.2 * np.cos(k * (X + Y - Z)))
    # project once onto the sphere so rho is exactly band-limited there
    rho = OD.vg_to_r(OD.rho_to_g(rho, lay, box ** 3) / box ** 3, lay).reshape(n, n, n)
    return dict(lay=lay, rho=rho.real, vol=box ** 3, n=n, box=box)


def test_density_gradient_is_the_analytic_gradient(dens):
    """grad of a single plane wave inside the sphere."""
    from oracle import density as OD
    n, box, lay = dens["n"], dens["box"], dens["lay"]
    x = np.arange(n) * box / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    k = 2.0 * math.pi / box
    f = 1.0 + 0.1 * np.cos(k * X + 2 * k * Y - k * Z)
    g = OX.density_gradient(f, lay, box ** 3)
    # the oracle's transforms keep the grid's axis order; find which array axis is x
    want = [-0.1 * k * np.sin(k * X + 2 * k * Y - k * Z) * c for c in (1, 2, -1)]
    err = min(max(np.max(np.abs(g[i] - want[p[i]])) for i in range(3))
              for p in [(0, 1, 2), (2, 1, 0)])
    assert err < 1e-12


def test_blyp_potential_is_the_energy_derivative(dens):
    """dE_xc/deps along a band-limited perturbation equals sum V_xc delta dV
    (the White-Bird term's sign and scale included)."""
    from oracle import density as OD
    rho, lay, vol, n = dens["rho"], dens["lay"], dens["vol"], dens["n"]
    rng = np.random.default_rng(9)
    d = rng.standard_normal(rho.shape)
    d = OD.vg_to_r(OD.rho_to_g(d, lay, vol) / vol, lay).reshape(rho.shape).real
    d *= 0.05 * np.max(rho) / np.max(np.abs(d))
    v, e, _, e_gga = OX.blyp_vxc(rho, lay, vol)
    assert e_gga != 0.0
    h = 1e-3
    ep = OX.blyp_vxc(rho + h * d, lay, vol)[1]
    em = OX.blyp_vxc(rho - h * d, lay, vol)[1]
    fd = (ep - em) / (2 * h)
    an = np.sum(v * d) * vol / rho.size
    assert abs(fd - an) < 1e-7 * abs(an)
