"""The EES non-local oracle (oracle/ees.py) pinned to the reference's own
cp_ees_nonlocal.C / set_cp_ewald.C routines, compiled from their sources by
oracle/build_ref.sh into oracle/_ref/libref.so.

Stage by stage: NL grid size, B-spline weights b(G), spline look-up, atom
B-splines on every plane, projector x psi, and then the whole non-local pass
(Z matrix, energy, atom forces, scatter, psi force) assembled from the
reference routines around the oracle's FFTs, against oracle.ees.nonlocal_ees.
"""
import ctypes

import numpy as np
import pytest

from oracle import ees as OE
from oracle import fftpath as OF

REL = 1e-12


def _c(a, t):
    return np.ascontiguousarray(a, dtype=t)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def ref_lib():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_ees_setup"):
        pytest.skip("oracle/_ref/libref.so with the EES routines is not built")
    return lib


@pytest.fixture(scope="module")
def small():
    from openatom_b200.system import System
    sysm = System(9.0, 20.0, 3, {"O": 2, "H": 3}, seed=11)
    return sysm


def _setup(ref, sysm, nkf, channels, occ):
    spl = sysm.tab
    ntyp = len(sysm.species)
    lmax = 1
    vnl = np.zeros((ntyp, lmax + 1, 4, spl["nspl"]))
    gz = np.zeros(ntyp)
    vn = np.zeros((ntyp, lmax + 1))
    for ch in channels:
        vnl[ch["type"], ch["l"]] = ch["vnl"]
        vn[ch["type"], ch["l"]] = ch["vnorm"]
        if ch["l"] == 0:
            gz[ch["type"]] = ch["gzvps0"]
    ct = _c([c["type"] for c in channels], np.int32)
    cl = _c([c["l"] for c in channels], np.int32)
    cm = _c([c["m"] for c in channels], np.int32)
    hm = _c(sysm.hmati(), np.float64)
    vnl, gz, vn = _c(vnl, np.float64), _c(gz, np.float64), _c(vn, np.float64)
    typ = _c(sysm.typ, np.int32)
    occ = _c(occ, np.float64)
    ref.ref_ees_setup(nkf, OE.N_INTERP, _p(hm), ctypes.c_double(sysm.box_len ** 3),
                      spl["nspl"], ctypes.c_double(spl["gmin"]), ctypes.c_double(spl["dg"]),
                      ntyp, lmax, _p(vnl), _p(gz), _p(vn), sysm.natm, _p(typ), len(channels),
                      _p(ct), _p(cl), _p(cm), len(occ), _p(occ))
    return (hm, vnl, gz, vn, typ, occ, ct, cl, cm)  # keep alive


def test_nl_grid_size_matches_reference(ref_lib):
    ref_lib.ref_nl_grid_size.restype = ctypes.c_int
    for kmax in list(range(3, 64)) + [80, 99]:
        want = ref_lib.ref_nl_grid_size(kmax, ctypes.c_double(1.2), OE.N_INTERP)
        assert OE.nl_grid_size(kmax) == want, kmax


def test_weights_spline_bsplines_projector(ref_lib, small):
    ref = ref_lib
    sysm = small
    lay = sysm.layout
    nkf = OE.nl_grid_size(lay.kmax)
    occ = np.full(sysm.nstates, 2.0)
    keep = _setup(ref, sysm, nkf, sysm.channels, occ)
    n = lay.npts
    ka, kb, kc = _c(lay.kx, np.int32), _c(lay.ky, np.int32), _c(lay.kz, np.int32)
    hm = sysm.hmati()
    # b(G)
    bre, bim = np.zeros(n), np.zeros(n)
    ref.ref_ees_weights(n, _p(ka), _p(kb), _p(kc), _p(bre), _p(bim))
    ore, oim = OE.ees_weights(lay.kx, lay.ky, lay.kz, nkf)
    assert np.max(np.abs(ore - bre)) <= REL * np.max(np.abs(bre))
    assert np.max(np.abs(oim - bim)) <= REL * np.max(np.abs(bre))
    # spline look-up: index bit-exact, offset to rounding
    h, ind = np.zeros(n), np.zeros(n, dtype=np.int32)
    ref.ref_ees_spline(n, _p(ka), _p(kb), _p(kc), _p(h), _p(ind))
    xk, yk, zk = OE.gvec(lay.kx, lay.ky, lay.kz, hm)
    oi, oh = OE.spline_lookup(np.sqrt(xk * xk + yk * yk + zk * zk), sysm.tab["gmin"],
                              sysm.tab["dg"], sysm.tab["nspl"])
    assert np.array_equal(oi, ind)
    assert np.max(np.abs(oh - h)) <= 1e-14
    # atom B-splines on every plane (reference order: atoms in type order)
    natm, n2 = sysm.natm, OE.N_INTERP ** 2
    xyz = _c(sysm.pos, np.float64)
    pidx = np.zeros((nkf, natm), dtype=np.int32)
    ig = np.zeros((nkf, natm, n2), dtype=np.int32)
    mn, dx, dy, dz = (np.zeros((nkf, natm, n2)) for _ in range(4))
    ref.ref_ees_bspline(_p(xyz), _p(pidx), _p(ig), _p(mn), _p(dx), _p(dy), _p(dz))
    bs = OE.atom_bsplines(sysm.pos, hm, nkf)
    order = np.argsort(sysm.typ, kind="stable")
    for nlidx, i in enumerate(order):
        (c, b, a), omn, odx, ody, odz = OE.stencil(bs, i, hm, nkf)
        for jc in range(OE.N_INTERP):
            plane = int(c[jc, 0, 0])
            assert pidx[plane, nlidx] == jc + 1
            flat = (a[jc] + b[jc] * (nkf + 2)).reshape(-1)
            assert np.array_equal(flat, ig[plane, nlidx])
            for o, r in ((omn, mn), (odx, dx), (ody, dy), (odz, dz)):
                scale = max(1.0, np.max(np.abs(r[plane, nlidx])))
                assert np.max(np.abs(o[jc].reshape(-1) - r[plane, nlidx])) <= REL * scale
    # projector x psi for every channel
    psi = sysm.psi(device="cpu").numpy()
    g0 = int(np.nonzero((lay.kx == 0) & (lay.ky == 0) & (lay.kz == 0))[0][0])
    for it, ch in enumerate(sysm.channels):
        dre, dim = bre.copy(), bim.copy()
        dyr, dyi = np.zeros(n), np.zeros(n)
        proj = np.zeros(2 * n)
        ps = _c(psi[0].view(np.float64), np.float64)
        ref.ref_ees_proj(n, _p(ps), _p(ka), _p(kb), _p(kc), g0, it, _p(dre), _p(dim),
                         _p(ind), _p(h), _p(dyr), _p(dyi), _p(proj))
        dyp = OE.channel_dyp(ch, lay, hm, nkf, sysm.tab)
        sc = np.max(np.abs(dyr + 1j * dyi))
        assert np.max(np.abs(dyp - (dyr + 1j * dyi))) <= REL * sc
        pj = proj.view(np.complex128)
        assert np.max(np.abs(np.conj(dyp * psi[0]) - pj)) <= REL * np.max(np.abs(pj))
    del keep


def test_nonlocal_pass_against_reference_routines(ref_lib, small):
    ref = ref_lib
    ref.ref_ees_energy_force.restype = ctypes.c_double
    sysm = small
    lay = sysm.layout
    nkf = OE.nl_grid_size(lay.kmax)
    S = sysm.nstates
    occ = np.array([2.0, 2.0, 1.0])[:S]
    keep = _setup(ref, sysm, nkf, sysm.channels, occ)
    hm = sysm.hmati()
    vol = sysm.box_len ** 3
    psi = sysm.psi(device="cpu").numpy()
    n = lay.npts
    ka, kb, kc = _c(lay.kx, np.int32), _c(lay.ky, np.int32), _c(lay.kz, np.int32)
    g0 = int(np.nonzero((lay.kx == 0) & (lay.ky == 0) & (lay.kz == 0))[0][0])
    # the reference's per-chunk "first nkx0 points have weight 1" is the kx == 0 set;
    # the layout keeps them first in every chunk, so pass them in that order
    kx0 = np.nonzero(lay.kx == 0)[0]
    rest = np.nonzero(lay.kx != 0)[0]
    perm = np.concatenate([kx0, rest])
    natm, n2 = sysm.natm, OE.N_INTERP ** 2
    xyz = _c(sysm.pos, np.float64)
    pidx = np.zeros((nkf, natm), dtype=np.int32)
    ig = np.zeros((nkf, natm, n2), dtype=np.int32)
    mn, dx, dy, dz = (np.zeros((nkf, natm, n2)) for _ in range(4))
    ref.ref_ees_bspline(_p(xyz), _p(pidx), _p(ig), _p(mn), _p(dx), _p(dy), _p(dz))
    bre, bim = np.zeros(n), np.zeros(n)
    ref.ref_ees_weights(n, _p(ka), _p(kb), _p(kc), _p(bre), _p(bim))
    h, ind = np.zeros(n), np.zeros(n, dtype=np.int32)
    ref.ref_ees_spline(n, _p(ka), _p(kb), _p(kc), _p(h), _p(ind))
    grid = OE.NLGrid(lay, nkf)
    e_ref = 0.0
    f_ref = np.zeros((natm, 3))
    fpsi_ref = np.zeros((S, n), dtype=np.complex128)
    for it, ch in enumerate(sysm.channels):
        na = int(np.sum(sysm.typ == ch["type"]))
        for s in range(S):
            dre, dim = bre.copy(), bim.copy()
            dyr, dyi = np.zeros(n), np.zeros(n)
            proj = np.zeros(2 * n)
            ps = _c(psi[s].view(np.float64), np.float64)
            ref.ref_ees_proj(n, _p(ps), _p(ka), _p(kb), _p(kc), g0, it, _p(dre), _p(dim),
                             _p(ind), _p(h), _p(dyr), _p(dyi), _p(proj))
            pr = OF.state_g_to_r(proj.view(np.complex128)[None, :], grid)[0]   # [c, b, a]
            pad = np.zeros((nkf, nkf, nkf + 2))
            pad[:, :, :nkf] = pr
            pad = _c(pad, np.float64)
            z = np.zeros(na)
            ref.ref_ees_zmat(_p(pad), it, s, _p(z))
            scr = np.zeros((nkf, nkf, nkf + 2))
            fa = np.zeros((natm, 3))
            e_ref += ref.ref_ees_energy_force(_p(z), _p(pad), it, s, _p(fa), _p(scr))
            f_ref += fa
            pg = OF.state_r_to_g(scr[None, :, :, :nkf], grid)[0]
            pgp = _c(pg[perm].view(np.float64), np.float64)
            fp = np.zeros(2 * n)
            dyrp, dyip = _c(dyr[perm], np.float64), _c(dyi[perm], np.float64)
            g0p = int(np.nonzero(perm == g0)[0][0])
            kap, kbp, kcp = (_c(k[perm], np.int32) for k in (lay.kx, lay.ky, lay.kz))
            ref.ref_ees_psi_force(n, g0p, len(kx0), _p(pgp), _p(fp), _p(dyrp), _p(dyip),
                                  _p(kap), _p(kbp), _p(kcp))
            fpsi_ref[s, perm] += fp.view(np.complex128)
    atoms = dict(pos=sysm.pos, typ=sysm.typ)
    e, fpsi, fatm = OE.nonlocal_ees(psi, lay, occ, vol, hm, atoms, sysm.channels, sysm.tab, nkf)
    assert e > 0.0
    assert abs(e - e_ref) <= REL * abs(e_ref)
    assert np.max(np.abs(fatm - f_ref)) <= 1e-11 * np.max(np.abs(f_ref))
    assert np.max(np.abs(fpsi - fpsi_ref)) <= 1e-11 * np.max(np.abs(fpsi_ref))
    del keep
