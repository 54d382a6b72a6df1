"""Pins of the oracle's kinetic term, G-space expand/pack and Hartree +
local pseudopotential + reciprocal Ewald routine against the reference's own
code compiled from source into oracle/_ref (oracle/build_ref.sh,
oracle/ref_local.cpp):

* CPNONLOCAL::CP_eke_calc            cp_nonlocal/cp_eke.C:30-140
* FFTcache::expandGSpace/packGSpace  fft_slab_ctrl/fftCache.C:460-553
* CPLOCAL::CP_hart_eext_calc         cp_local/cp_hart_ext.C:56-405

Host only; tolerances 1e-12 relative (the reference advances its structure
factors along kz by products, the oracle evaluates them directly) and exact
for the copies of expand/pack.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import density as OD
from oracle import fftpath as OF
from oracle import layout as OL

VP = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(VP)


@pytest.fixture(scope="module")
def ref():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_hart_eext"):
        pytest.skip("oracle/_ref/libref.so with cp_eke.C / cp_hart_ext.C is not built")
    lib.ref_eke.argtypes = [ctypes.c_int, ctypes.c_int, VP, VP, VP, VP, VP, VP, ctypes.c_int,
                            ctypes.c_double, ctypes.c_int, VP, VP]
    lib.ref_hart_eext.argtypes = ([ctypes.c_int, VP, VP, VP, VP, ctypes.c_double, VP, VP,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   VP, VP, VP, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   VP, VP, VP, VP, VP])
    lib.ref_expand.argtypes = [VP, VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.ref_pack.argtypes = [VP, VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    return lib


@pytest.fixture(scope="module")
def sysm():
    from openatom_b200.system import System
    return System(12.0, 30.0, 6, {"O": 4, "H": 8}, nfft=48, seed=11)


def _cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("box,ecut,grid", [(12.0, 30.0, 48), (9.0, 20.0, 28)])
def test_expand_pack_match_reference(ref, box, ecut, grid):
    lay = OL.Layout(box, ecut, grid=grid)
    rng = np.random.default_rng(1)
    psi = _cplx(rng, (2, lay.npts))
    runs = np.ascontiguousarray(lay.runs.reshape(-1, 7), dtype=np.int32)
    nruns = runs.shape[0]
    ex = OF.expand(psi, lay)
    for s in range(2):
        out = np.full((nruns // 2, lay.n), 7.0 + 7.0j)   # the routine zeroes first
        p = np.ascontiguousarray(psi[s])
        ref.ref_expand(_p(out), _p(p), _p(runs), nruns, lay.npts, lay.n)
        assert np.array_equal(out, ex[s])
        back = np.zeros(lay.npts, complex)
        lines = np.ascontiguousarray(_cplx(rng, (nruns // 2, lay.n)))
        ref.ref_pack(_p(lines), _p(back), _p(runs), nruns, lay.npts, lay.n)
        assert np.array_equal(back, OF.pack(lines[None], lay)[0])


def test_eke_matches_reference(ref, sysm):
    lay = OL.Layout(12.0, 30.0, grid=48)
    rng = np.random.default_rng(2)
    S = 3
    psi = _cplx(rng, (S, lay.npts)) * np.exp(-lay.g2 / 8.0)[None]
    force = _cplx(rng, (S, lay.npts))
    occ = np.array([2.0, 1.0, 0.5])
    # a cutoff inside the sphere so the zeroing branch is taken too
    ecut = 0.8 * float(np.max(lay.g2))
    f_or, e_or = OF.eke(force, psi, lay, occ, ecut)
    # the routine expects a chare's Gx=0 points first
    order = np.concatenate([np.nonzero(lay.kx == 0)[0], np.nonzero(lay.kx != 0)[0]])
    nkx0 = int(np.sum(lay.kx == 0))
    kx, ky, kz = (np.ascontiguousarray(a[order], dtype=np.int32)
                  for a in (lay.kx, lay.ky, lay.kz))
    g2 = np.ascontiguousarray(lay.g2[order])
    for s in range(S):
        f = np.ascontiguousarray(force[s, order])
        p = np.ascontiguousarray(psi[s, order])
        e = np.zeros(1)
        ref.ref_eke(lay.npts, s, _p(f), _p(p), _p(kx), _p(ky), _p(kz), _p(g2), nkx0, ecut, S,
                    _p(occ), _p(e))
        back = np.empty_like(f)
        back[order] = f
        assert np.allclose(back, f_or[s], rtol=1e-13, atol=1e-13 * np.max(np.abs(f_or[s])))
        assert abs(e[0] - e_or[s]) <= 1e-13 * abs(e_or[s])


@pytest.mark.parametrize("alp_ewd", [0.35, 0.6])
def test_hart_eext_matches_reference(ref, sysm, alp_ewd):
    box, ecut_ry = 12.0, 30.0
    dlay = OD.density_layout(box, ecut_ry, 48)
    rng = np.random.default_rng(3)
    tpi = 2.0 * math.pi / box
    g2 = (dlay.kx * tpi) ** 2 + (dlay.ky * tpi) ** 2 + (dlay.kz * tpi) ** 2
    rho = _cplx(rng, dlay.npts) * np.exp(-g2 / 20.0)
    rho[g2 == 0] = 24.0
    atoms = sysm.atoms_dict()
    tab = sysm.tab
    vks, eh, ee, ew, f = OD.hart_eext(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut_ry, atoms,
                                      tab, alp_ewd)
    typ = np.ascontiguousarray(atoms["typ"], dtype=np.int32)
    natm = len(typ)
    q = np.ascontiguousarray(np.asarray(atoms["q"], dtype=np.float64)[typ])
    xyz = np.ascontiguousarray(np.asarray(atoms["pos"], dtype=np.float64))
    vloc = np.ascontiguousarray(np.asarray(tab["vps"], dtype=np.float64))
    ntyp, _, nspl = vloc.shape
    gz = np.ascontiguousarray(np.asarray(tab["gzvps"], dtype=np.float64))
    hmat = np.eye(3) * box
    hmati = np.eye(3) / box
    kx, ky, kz = (np.ascontiguousarray(a, dtype=np.int32) for a in (dlay.kx, dlay.ky, dlay.kz))
    rv = np.zeros(dlay.npts, complex)
    e = np.zeros(3)
    fr = np.zeros((natm, 3))
    r = np.ascontiguousarray(rho)
    ref.ref_hart_eext(dlay.npts, _p(kx), _p(ky), _p(kz), _p(r), 0.5 * ecut_ry, _p(hmat),
                      _p(hmati), box ** 3, alp_ewd, natm, ntyp, _p(typ), _p(xyz), _p(q), nspl,
                      float(tab["gmin"]), float(tab["dg"]), _p(vloc), _p(gz), _p(rv), _p(e),
                      _p(fr))
    assert abs(e[0] - eh) <= 1e-12 * abs(eh)
    assert abs(e[1] - ee) <= 1e-12 * abs(ee)
    assert abs(e[2] - ew) <= 1e-12 * abs(ew)
    assert np.max(np.abs(rv - vks)) <= 1e-12 * np.max(np.abs(vks))
    assert np.max(np.abs(fr - f)) <= 1e-11 * np.max(np.abs(f))
