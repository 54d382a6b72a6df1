"""Generate the golden fixtures of tests/golden from the reference's own code.

Runs the reference routines compiled from their sources by oracle/build_ref.sh
(oracle/_ref/libref.so):
  flip_data_set, get_chareG_line_prms (src_charm_driver/utility/para_grp_parse.C),
  sort_commence (src_mathlib/lst_sort_clean.C) -- composed into processState's
  order as util.C:1331-1642 composes them -- and CPORTHOG::get_iter_Tmat
  (src_piny_physics_v1.0/abinito_physics/cp_orthog/cp_lowdin.C).
The half sphere fed to flip_data_set is setkvec3d_sm's order (restated in
oracle/layout.py; its counts are checked against the reference's sizes).

Usage: python tests/golden/make_golden.py   (needs oracle/_ref/libref.so)
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import layout as OL  # noqa: E402

IP = ctypes.POINTER(ctypes.c_int)
DP = ctypes.POINTER(ctypes.c_double)

# (box bohr, ecut Ry, nchareG or 0 for gExpandFact = 1)
CASES = [(9.0, 20.0, 0), (12.0, 30.0, 0), (12.0, 30.0, 7), (15.3, 40.0, 0), (23.5, 70.0, 0)]


def lib():
    p = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    L = ctypes.CDLL(p)
    L.ref_flip_data_set.argtypes = [ctypes.c_int, IP, IP, IP]
    L.ref_flip_data_set.restype = ctypes.c_int
    L.ref_get_chareG_line_prms.argtypes = [ctypes.c_int] * 3 + [IP] * 5
    L.ref_sort_commence.argtypes = [ctypes.c_int, IP, IP]
    L.ref_get_iter_Tmat.argtypes = [DP, DP, ctypes.c_int]
    return L


def ip(a):
    return a.ctypes.data_as(IP)


def ref_layout(L, box, ecut, nchareG):
    kmax = OL.calc_kmax(box, ecut)
    n = OL.radix_size(kmax)
    ka, kb, kc = OL.setkvec3d_sm(0.5 * ecut, kmax, box)
    nk = len(ka)
    nplane0 = int(np.count_nonzero(ka == 0))
    cap = nk + nplane0
    kx = np.zeros(cap, np.int32); ky = np.zeros(cap, np.int32); kz = np.zeros(cap, np.int32)
    kx[:nk], ky[:nk], kz[:nk] = ka, kb, kc
    npk = L.ref_flip_data_set(nk, ip(kx), ip(ky), ip(kz))
    kx, ky, kz = kx[:npk], ky[:npk], kz[:npk]
    if nchareG == 0:
        nchareG = int(kx.max()) + 1
    # processState (util.C:1433-1458): round-robin deal of the lines
    brk = np.nonzero((np.diff(kx) != 0) | (np.diff(ky) != 0))[0] + 1
    st = np.concatenate([[0], brk]); en = np.concatenate([brk, [npk]])
    nline = len(st)
    order = [j for i in range(nchareG) for j in range(i, nline, nchareG)]
    perm = np.concatenate([np.arange(st[j], en[j]) for j in order])
    kx1, ky1, kz1 = kx[perm], ky[perm], kz[perm]
    brk = np.nonzero((np.diff(kx1) != 0) | (np.diff(ky1) != 0))[0] + 1
    st1 = np.concatenate([[0], brk]); en1 = np.concatenate([brk, [npk]])
    npts_line = (en1 - st1).astype(np.int32)
    istrt = np.zeros(nchareG, np.int32); iend = np.zeros(nchareG, np.int32)
    nptsg = np.zeros(nchareG, np.int32); nlineg = np.zeros(nchareG, np.int32)
    L.ref_get_chareG_line_prms(npk, nchareG, nline, ip(npts_line), ip(istrt), ip(iend),
                               ip(nptsg), ip(nlineg))
    # per chunk: sort_kxky (util.C:2223-2247) with the reference sort_commence
    perm2 = []
    loff = 0
    for c in range(nchareG):
        m = int(nlineg[c])
        lx = kx1[st1[loff:loff + m]].astype(np.int32).copy()
        ly = ky1[st1[loff:loff + m]].astype(np.int32).copy()
        idx = np.arange(m, dtype=np.int32)
        if m > 1:
            L.ref_sort_commence(m, ip(lx), ip(idx))
            ly = ly[idx].copy()
            kmin, kmaxx = int(lx[0]), int(lx[-1])
            cnt = np.bincount(lx - kmin, minlength=kmaxx - kmin + 1)
            off = 0
            for q in cnt:
                q = int(q)
                if q > 1:
                    sub_y = ly[off:off + q].copy()
                    sub_i = idx[off:off + q].copy()
                    L.ref_sort_commence(q, ip(sub_y), ip(sub_i))
                    ly[off:off + q] = sub_y
                    idx[off:off + q] = sub_i
                off += q
        for l in idx:
            perm2.append(np.arange(st1[loff + l], en1[loff + l]))
        loff += m
    perm2 = np.concatenate(perm2)
    kx2, ky2, kz2 = kx1[perm2], ky1[perm2], kz1[perm2]
    runs = OL.runs_from_kvecs(kx2, ky2, kz2, n, n, n)
    return dict(kx=kx2.astype(np.int32), ky=ky2.astype(np.int32), kz=kz2.astype(np.int32),
                runs=runs, n=n, kmax=kmax, nchareG=nchareG,
                nline_lgrp=nlineg, npts_lgrp=nptsg)


def ref_tmat(L, n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    S = (Q * ev) @ Q.T
    S = 0.5 * (S + S.T)
    T = np.zeros_like(S)
    Sc = np.ascontiguousarray(S)
    L.ref_get_iter_Tmat(Sc.ctypes.data_as(DP), T.ctypes.data_as(DP), n)
    return S, T


def main():
    L = lib()
    for box, ecut, nch in CASES:
        d = ref_layout(L, box, ecut, nch)
        name = "layout_L%g_E%g_C%d.npz" % (box, ecut, nch)
        np.savez_compressed(os.path.join(HERE, name), box=box, ecut=ecut, **d)
        print(name, len(d["kx"]), d["n"])
    S, T = ref_tmat(L, 48, 7, 1.6, 2.4)
    np.savez_compressed(os.path.join(HERE, "schulz_n48.npz"), S=S, T=T)
    print("schulz_n48.npz")


if __name__ == "__main__":
    main()
