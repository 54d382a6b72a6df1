"""The structure-factor (non-EES) nonlocal oracle (oracle/sf.py) against the
reference's own CP_calc_Struct_Fact, CP_enl_matrix_calc, CP_enl_atm_forc_calc
and CP_enl_force_calc compiled from cp_struct_fact.C, cp_nlmat.C and
cp_nl_energy_forc.C (oracle/_ref, ref_sf.cpp).  Host only."""
import ctypes
import math

import numpy as np
import pytest

from oracle import ees as OE
from oracle import sf as OS

REL = 1e-12


def _c(a, t):
    return np.ascontiguousarray(a, dtype=t)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def ref_lib():
    from conftest import ref_lib as load
    lib = load()
    if lib is None or not hasattr(lib, "ref_sf_struct_fact"):
        pytest.skip("oracle/_ref/libref.so with the structure-factor routines is not built")
    lib.ref_sf_atm_forc.restype = ctypes.c_double
    return lib


@pytest.fixture(scope="module")
def small():
    from openatom_b200.system import System
    return System(9.0, 20.0, 3, {"O": 2, "H": 3}, seed=11)


def _l0(sysm):
    order, proj, vn0 = OS.system_tables(sysm)
    ch0 = {c["type"]: c for c in sysm.channels if c["l"] == 0}
    return order, proj, vn0, [ch0[t] for t in sorted(ch0)]


def test_structure_factor_path_against_reference(ref_lib, small):
    from test_ees_oracle import _setup
    ref = ref_lib
    sysm = small
    lay = sysm.layout
    S = sysm.nstates
    occ = np.array([2.0, 1.5, 1.0])[:S]
    order, proj, vn0, chans = _l0(sysm)
    keep = _setup(ref, sysm, OE.nl_grid_size(lay.kmax), chans, occ)
    ntyp = len(sysm.species)
    xyz = _c(sysm.pos, np.float64)
    vnc = _c(vn0, np.float64)
    ref.ref_sf_setup(ntyp, _p(vnc), _p(xyz))
    n, natm = lay.npts, sysm.natm
    ka, kb, kc = _c(lay.kx, np.int32), _c(lay.ky, np.int32), _c(lay.kz, np.int32)
    rs = [np.zeros((natm, n), dtype=np.complex128) for _ in range(4)]
    ref.ref_sf_struct_fact(n, _p(ka), _p(kb), _p(kc), *(_p(a) for a in rs))
    s, sd = OS.struct_fact(lay.kx, lay.ky, lay.kz, sysm.box_len,
                           sysm.pos[order] / sysm.box_len, proj)
    for o, r in zip([s, sd[0], sd[1], sd[2]], rs):
        assert np.max(np.abs(o - r)) <= REL * np.max(np.abs(r))
    psi = sysm.psi(device="cpu").numpy()
    e_ref = 0.0
    fpsi_ref = np.zeros((S, n), dtype=np.complex128)
    for st in range(S):
        z = [np.zeros(natm, dtype=np.complex128) for _ in range(4)]
        ps = _c(psi[st], np.complex128)
        ref.ref_sf_zmat(n, _p(ps), _p(ka), _p(kb), _p(kc), *(_p(a) for a in rs),
                        *(_p(a) for a in z), st)
        e_ref += ref.ref_sf_atm_forc(*(_p(a) for a in z), st)
        fp = np.zeros(n, dtype=np.complex128)
        ref.ref_sf_psi_force(_p(z[0]), n, _p(ka), _p(kb), _p(kc), _p(rs[0]), _p(fp), st)
        fpsi_ref[st] = fp
    f_ref = np.zeros((natm, 3))
    ref.ref_sf_forces(_p(f_ref))
    enl, f, fpsi = OS.sf_nonlocal(psi, occ, sysm.box_len ** 3, s, sd, vn0)
    assert abs(enl - e_ref) <= REL * abs(e_ref)
    f_orig = np.zeros_like(f)
    f_orig[order] = f
    assert np.max(np.abs(f_orig - f_ref)) <= REL * np.max(np.abs(f_ref))
    assert np.max(np.abs(fpsi - fpsi_ref)) <= REL * np.max(np.abs(fpsi_ref))
    del keep
