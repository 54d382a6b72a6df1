"""G-vector layout: oracle vs the reference's compiled routines, product vs oracle.

Bit-exact integer work: every comparison is array_equal.
"""
import glob
import os

import numpy as np
import pytest

from oracle import layout as OL
from conftest import ref_lib

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(glob.glob(os.path.join(HERE, "golden", "layout_*.npz")))


def test_golden_fixtures_present():
    assert len(GOLD) >= 5


@pytest.mark.parametrize("path", GOLD, ids=os.path.basename)
def test_oracle_matches_reference_golden(path):
    g = np.load(path)
    lay = OL.Layout(float(g["box"]), float(g["ecut"]), nchareG=int(g["nchareG"]))
    assert lay.n == int(g["n"]) and lay.kmax == int(g["kmax"])
    assert np.array_equal(lay.kx, g["kx"])
    assert np.array_equal(lay.ky, g["ky"])
    assert np.array_equal(lay.kz, g["kz"])
    assert np.array_equal(lay.runs, g["runs"])
    assert lay.decomp["nline_lgrp"] == list(g["nline_lgrp"])


@pytest.mark.parametrize("path", GOLD, ids=os.path.basename)
def test_product_matches_reference_golden(path):
    from openatom_b200.layout import StateLayout
    g = np.load(path)
    lay = StateLayout(float(g["box"]), float(g["ecut"]), nchareG=int(g["nchareG"]))
    assert lay.n == int(g["n"])
    assert np.array_equal(lay.kx, g["kx"])
    assert np.array_equal(lay.ky, g["ky"])
    assert np.array_equal(lay.kz, g["kz"])
    assert np.array_equal(lay.runs, g["runs"])


def test_reference_sizes_of_the_benchmark_systems():
    # half-sphere counts / packed points / z-lines / radixme grids
    for box, ecut, nk, npts, nl, n in [(12.0, 30.0, 2400, 2575, 185, 42),
                                      (23.5, 70.0, 64197, 65736, 1570, 128)]:
        lay = OL.Layout(box, ecut)
        assert (lay.nktot, lay.npts, lay.nlines, lay.n) == (nk, npts, nl, n)


def test_flip_matches_compiled_reference():
    import ctypes
    L = ref_lib()
    if L is None:
        pytest.skip("oracle/_ref/libref.so not built (reference tree absent)")
    IP = ctypes.POINTER(ctypes.c_int)
    L.ref_flip_data_set.argtypes = [ctypes.c_int, IP, IP, IP]
    L.ref_flip_data_set.restype = ctypes.c_int
    for box, ecut in [(7.0, 12.0), (10.0, 25.0), (13.7, 33.0)]:
        kmax = OL.calc_kmax(box, ecut)
        ka, kb, kc = OL.setkvec3d_sm(0.5 * ecut, kmax, box)
        fx, fy, fz, _ = OL.flip_data_set(ka, kb, kc)
        n = len(ka)
        cap = len(fx)
        ax, ay, az = (np.zeros(cap, np.int32) for _ in range(3))
        ax[:n], ay[:n], az[:n] = ka, kb, kc
        m = L.ref_flip_data_set(n, ax.ctypes.data_as(IP), ay.ctypes.data_as(IP),
                                az.ctypes.data_as(IP))
        assert m == cap
        assert np.array_equal(ax, fx) and np.array_equal(ay, fy) and np.array_equal(az, fz)


def test_chunk_params_match_compiled_reference():
    import ctypes
    L = ref_lib()
    if L is None:
        pytest.skip("oracle/_ref/libref.so not built (reference tree absent)")
    IP = ctypes.POINTER(ctypes.c_int)
    L.ref_get_chareG_line_prms.argtypes = [ctypes.c_int] * 3 + [IP] * 5
    rng = np.random.default_rng(3)
    for nline, nch in [(40, 5), (185, 11), (300, 17), (64, 64)]:
        npts = rng.integers(1, 60, nline).astype(np.int32)
        nk = int(npts.sum())
        out = [np.zeros(nch, np.int32) for _ in range(4)]
        L.ref_get_chareG_line_prms(nk, nch, nline, npts.ctypes.data_as(IP),
                                   *[o.ctypes.data_as(IP) for o in out])
        ist, ien, npg, nlg = OL.get_chareG_line_prms(nk, nch, npts)
        assert list(out[2]) == npg and list(out[3]) == nlg
        assert list(out[0]) == ist and list(out[1]) == ien


def test_product_layout_random_boxes_match_oracle():
    from openatom_b200.layout import StateLayout
    for box, ecut, nch in [(8.3, 18.0, 0), (11.1, 26.0, 5), (14.2, 35.0, 0)]:
        a = StateLayout(box, ecut, nchareG=nch)
        b = OL.Layout(box, ecut, nchareG=(nch or None))
        assert np.array_equal(a.kx, b.kx) and np.array_equal(a.ky, b.ky)
        assert np.array_equal(a.kz, b.kz) and np.array_equal(a.runs, b.runs)


def test_runs_cover_lines_and_gx0_partner_symmetry():
    lay = OL.Layout(12.0, 30.0)
    t = lay.line_tables()
    assert int(np.sum(t["nneg"] + t["npos"])) == lay.npts
    # every Gx=0 point has its (0,-ky,-kz) partner stored (flip_data_set)
    s = set(zip(lay.ky[lay.kx == 0].tolist(), lay.kz[lay.kx == 0].tolist()))
    assert all((-y, -z) in s for (y, z) in s)


def test_bad_grid_is_rejected():
    from openatom_b200 import _lib
    from openatom_b200.layout import StateLayout
    with pytest.raises(_lib.CpstepError):
        StateLayout(12.0, 30.0, nfft=20)
