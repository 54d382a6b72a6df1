"""The oracle's EES form of the Hartree + local + Ewald pass (oracle/eext_ees.py)
against the reference's own routines compiled from cp_local/cp_hart_ext.C
into oracle/_ref (oracle/build_ref.sh, oracle/ref_local.cpp), stage by stage:

* eesAtmBsplineRgrp + eesPackGridRchare   the spread grid of every type, exact
* eesSetEesWghtGgrp + eesHartEextGchare + eesEwaldGchare
                                          energies, vks(G), the force terms, 1e-12
* eesAtmForceRchare                       the atom forces from the back-
                                          transformed grids, 1e-12

and, for the two transforms between the stages (Charm-FFT in the reference):
the whole pass reproduces the explicit structure-factor form (oracle/density.py,
itself pinned to CP_hart_eext_calc) to the interpolation error, and its forces
are the derivative of its energy (central differences, 1e-8 relative).
Host only.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import density as OD
from oracle import ees as OE
from oracle import eext_ees as OX
from oracle import layout as OL
from oracle import synth as OSY

VP = ctypes.c_void_p
CASES = [(9.0, 20.0, {"O": 1, "H": 2}, 28), (12.0, 30.0, {"O": 4, "H": 8}, 48)]


def _p(a):
    return a.ctypes.data_as(VP)


@pytest.fixture(scope="module")
def ref():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_eext_ees_gspace"):
        pytest.skip("oracle/_ref/libref.so with the EES local routines is not built")
    I, D = ctypes.c_int, ctypes.c_double
    lib.ref_eext_ees_spread.argtypes = [I, I, VP, VP, VP, D, I, I, VP]
    lib.ref_eext_ees_gspace.argtypes = [I, VP, VP, VP, VP, D, VP, D, D, I, I, I, VP, I, D, D,
                                        VP, VP, VP, VP, VP, VP]
    lib.ref_eext_ees_force.argtypes = [I, I, VP, VP, VP, VP, D, I, I, VP, VP]
    return lib


def _setup(box, ecut, counts, grid, seed=7):
    sysm = OSY.System(box, ecut, 4, counts, nfft=grid, seed=seed)
    dlay = OD.density_layout(box, ecut, grid)
    rng = np.random.default_rng(seed)
    tpi = 2.0 * math.pi / box
    g2 = (dlay.kx * tpi) ** 2 + (dlay.ky * tpi) ** 2 + (dlay.kz * tpi) ** 2
    rho = (rng.standard_normal(dlay.npts) + 1j * rng.standard_normal(dlay.npts)) * np.exp(-g2 / 20)
    rho[dlay.kx == 0] = 0.0
    # the Gx = 0 plane Hermitian, as the density of a real rho(r) is
    sel = np.nonzero(dlay.kx == 0)[0]
    key = {(int(dlay.ky[i]), int(dlay.kz[i])): int(i) for i in sel}
    for i in sel:
        j = key[(-int(dlay.ky[i]), -int(dlay.kz[i]))]
        if i <= j:
            v = rng.standard_normal() + 1j * rng.standard_normal()
            v *= math.exp(-g2[i] / 20)
            rho[i] = v if i != j else v.real
            rho[j] = np.conj(rho[i])
    rho[g2 == 0] = float(sum(counts.values()))
    kmax = OL.calc_kmax(box, ecut)
    ngrid = OX.eext_grid_size(kmax)
    return sysm, dlay, rho, ngrid


def _atoms(sysm):
    a = sysm.atoms_dict()
    typ = np.ascontiguousarray(a["typ"], dtype=np.int32)
    xyz = np.ascontiguousarray(np.asarray(a["pos"], dtype=np.float64))
    qt = np.ascontiguousarray(np.asarray(a["q"], dtype=np.float64))
    return a, typ, xyz, qt


@pytest.mark.parametrize("box,ecut,counts,grid", CASES)
def test_ees_local_stages_match_reference(ref, box, ecut, counts, grid):
    sysm, dlay, rho, ng = _setup(box, ecut, counts, grid)
    a, typ, xyz, qt = _atoms(sysm)
    natm, ntyp = len(typ), len(qt)
    hmati = (np.eye(3) / box).reshape(-1)
    vol = box ** 3
    n_interp = OE.N_INTERP
    bs = OE.atom_bsplines(xyz, hmati, ng, n_interp)
    # spread
    row = 2 * (ng // 2 + 1)
    grids = np.zeros((ntyp, ng, ng, row))
    ref.ref_eext_ees_spread(natm, ntyp, _p(typ), _p(xyz), _p(hmati), vol, ng, n_interp,
                            _p(grids))
    spread = [OX.spread(bs, typ == t, ng) for t in range(ntyp)]
    for t in range(ntyp):
        assert np.array_equal(grids[t][:, :, :ng], spread[t]), t
    # G pass
    kx, ky, kz = (np.ascontiguousarray(v, dtype=np.int32) for v in (dlay.kx, dlay.ky, dlay.kz))
    sf = np.array([OX.forward(spread[t], dlay.kx, dlay.ky, dlay.kz) for t in range(ntyp)])
    b = OX.ees_b(dlay.kx, dlay.ky, dlay.kz, ng, n_interp)
    tab = sysm.tab
    vks, eh, ee, ew, backs, ewt = OX.gpass(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, sf,
                                           qt, tab, sysm.alp_ewd, b)
    vloc = np.ascontiguousarray(np.asarray(tab["vps"], dtype=np.float64))
    nspl = vloc.shape[2]
    gz = np.ascontiguousarray(np.asarray(tab["gzvps"], dtype=np.float64))
    sfr = np.ascontiguousarray(sf.copy())
    stot = np.zeros(dlay.npts, complex)
    vr = np.zeros(dlay.npts, complex)
    e = np.zeros(3)
    r = np.ascontiguousarray(rho)
    ref.ref_eext_ees_gspace(dlay.npts, _p(kx), _p(ky), _p(kz), _p(r), 0.5 * ecut, _p(hmati), vol,
                            sysm.alp_ewd, ng, n_interp, ntyp, _p(qt), nspl, float(tab["gmin"]),
                            float(tab["dg"]), _p(vloc), _p(gz), _p(sfr), _p(stot), _p(vr), _p(e))
    assert abs(e[0] - eh) <= 1e-12 * abs(eh)
    assert abs(e[1] - ee) <= 1e-12 * abs(ee)
    assert abs(e[2] - ew) <= 1e-12 * abs(ew)
    assert np.max(np.abs(vr - vks)) <= 1e-12 * np.max(np.abs(vks))
    assert np.max(np.abs(sfr - backs)) <= 1e-12 * np.max(np.abs(backs))
    assert np.max(np.abs(stot - ewt)) <= 1e-12 * np.max(np.abs(ewt))
    # forces from the back-transformed grids
    rg = np.zeros((ntyp + 1, ng, ng, row))
    for t in range(ntyp):
        rg[t][:, :, :ng] = OX.backward(backs[t], dlay.kx, dlay.ky, dlay.kz, ng)
    rg[ntyp][:, :, :ng] = OX.backward(ewt, dlay.kx, dlay.ky, dlay.kz, ng)
    q = np.ascontiguousarray(qt[typ])
    fr = np.zeros((natm, 3))
    ref.ref_eext_ees_force(natm, ntyp, _p(typ), _p(xyz), _p(q), _p(hmati), vol, ng, n_interp,
                           _p(rg), _p(fr))
    _, _, _, _, f = OX.hart_eext_ees(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, a, tab,
                                     sysm.alp_ewd, ng, n_interp)
    assert np.max(np.abs(fr - f)) <= 1e-12 * np.max(np.abs(f))


@pytest.mark.parametrize("box,ecut,counts,grid", CASES)
def test_ees_local_reproduces_explicit_form(box, ecut, counts, grid):
    sysm, dlay, rho, ng = _setup(box, ecut, counts, grid)
    a = sysm.atoms_dict()
    v1, eh1, ee1, ew1, f1 = OD.hart_eext(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, a,
                                         sysm.tab, sysm.alp_ewd)
    v2, eh2, ee2, ew2, f2 = OX.hart_eext_ees(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, a,
                                             sysm.tab, sysm.alp_ewd, ng)
    assert abs(eh2 - eh1) <= 1e-13 * abs(eh1)  # the same sum, in another order
    # B-spline order 8 on a grid of 2.4 (2 kmax + 1): interpolation errors
    # near 1e-5 of the terms; a wrong transform sign or scale is off by O(1)
    assert abs(ee2 - ee1) <= 1e-4 * abs(ee1)
    assert abs(ew2 - ew1) <= 1e-6 * abs(ew1)
    assert np.max(np.abs(v2 - v1)) <= 1e-4 * np.max(np.abs(v1))
    assert np.max(np.abs(f2 - f1)) <= 1e-3 * np.max(np.abs(f1))


def test_ees_local_forces_are_the_energy_derivative():
    box, ecut, counts, grid = CASES[0]
    sysm, dlay, rho, ng = _setup(box, ecut, counts, grid)
    a = sysm.atoms_dict()

    def energy(pos):
        b = dict(a)
        b["pos"] = pos
        _, _, ee, ew, _ = OX.hart_eext_ees(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, b,
                                           sysm.tab, sysm.alp_ewd, ng)
        return ee + ew

    _, _, _, _, f = OX.hart_eext_ees(rho, dlay.kx, dlay.ky, dlay.kz, box, 0.5 * ecut, a, sysm.tab,
                                     sysm.alp_ewd, ng)
    h = 1e-5
    pos = np.asarray(a["pos"], dtype=np.float64)
    fd = np.zeros_like(f)
    for i in range(len(pos)):
        for d in range(3):
            p = pos.copy()
            p[i, d] += h
            ep = energy(p)
            p[i, d] -= 2 * h
            fd[i, d] = -(ep - energy(p)) / (2 * h)
    assert np.max(np.abs(fd - f)) <= 1e-8 * max(1.0, np.max(np.abs(f)))
