"""Oracle: the EES form of the Hartree + local pseudopotential + Ewald pass
(cp_eext_ees_opt on) in FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows src_piny_physics_v1.0/abinito_physics/cp_local/cp_hart_ext.C and the
density chares that drive it (src_charm_driver/cp_density_ctrl/):

* EES grid           init_eext_ees (interface/cp_ewald/set_cp_ewald.C:1419-1497):
                     the next FFT size >= 2 scale (2 kmax_cp + 1)
* b(G)               CPLOCAL::eesSetEesWghtGgrp :521-630 with get_bspline_wght1d
                     (set_cp_ewald.C:1237-1322), separable per axis
* atom B-splines     CPLOCAL::eesAtmBsplineRgrp :641-915 (the recursion and the
                     grid-index rule of the non-local form, oracle/ees.py)
* spread per type    CPLOCAL::eesPackGridRchare :925-990
                     (CP_Rho_RHartExt::computeAtmSF, CP_Rho_RHartExt.C:264-325)
* R -> G             the forward transform of the spread grid:
                     S_t(G) = sum_r grid_t(r) e^{+iG.r}, unnormalised
* G pass             CPLOCAL::eesHartEextGchare :1005-1230 for t = 1..ntyp in
                     order (Hartree with t = 1), then eesEwaldGchare :1241-1345
                     (CP_Rho_GHartExt::getHartEextEes, CP_Rho_GHartExt.C:653-720)
* G -> R             the backward transform of the per-type and total terms:
                     R(r) = sum_{G in the full sphere} X(G) e^{-iG.r}
* atom forces        CPLOCAL::eesAtmForceRchare :1357-1470 (flag 0 per type,
                     flag 1 with the charges for the Ewald term)

The two transforms are Charm-FFT calls in the reference (absent).  Their
signs and normalisations here are the ones under which S_t(G) b(G)
approximates the exact structure factor sum_a e^{iG.R_a} (the explicit form
of oracle/density.py, which it must reproduce to the interpolation error)
and under which the forces are the exact derivative of the EES energy; the
tests check both.  Everything else is pinned to the compiled routines.

rho_g is the reference's rho(G) = (vol/N) sum_r rho(r) e^{-iG.r} on the
packed density sphere (the Gx = 0 plane whole, Gx > 0 once, weight 2).
"""
import math

import numpy as np

from . import ees as OE
from . import layout as OL

SCALE = 1.2  # cp_pseudo_ees_scale default (set_sim_dict.C, keyword 37)


def eext_grid_size(kmax, scale=SCALE, n_interp=OE.N_INTERP):
    """init_eext_ees for a cubic box with the states' kmax_cp."""
    nk = 2 * kmax + 1
    nkf = int(2.0 * scale * float(nk))
    if nkf < 2 * nk:
        nkf += 1
    for k in OL.FFT_SIZES:
        if k >= nkf:
            if k < n_interp:
                raise ValueError("n_interp larger than the EES grid")
            return k
    raise ValueError("EES grid size too large for the radix table")


def axis_weights(ngrid, n_interp=OE.N_INTERP):
    """bden(k) of one axis as a complex array over k mod ngrid."""
    tr, ti = OE.bspline_wght1d(n_interp, ngrid)
    return tr + 1j * ti


def spread(bs, sel, ngrid):
    """eesPackGridRchare: sum of the atoms' Mn stencils, grid[c][b][a]."""
    grid = np.zeros((ngrid, ngrid, ngrid))
    n = bs["ia"].shape[1]
    for i in np.nonzero(sel)[0]:
        # jc outer, jb, ja inner: the order the reference adds them in
        mc = bs["mn_c"][i]
        mb = bs["mn_b"][i]
        ma = bs["mn_a"][i]
        for jc in range(n):
            for jb in range(n):
                grid[bs["ic"][i][jc], bs["ib"][i][jb], bs["ia"][i]] += ma * mb[jb] * mc[jc]
    return grid


def forward(grid, kx, ky, kz):
    """S(G) = sum_r grid(r) e^{+iG.r} at the sphere points."""
    n = grid.shape[0]
    f = np.fft.ifftn(grid) * float(n) ** 3
    return f[np.mod(kz, n), np.mod(ky, n), np.mod(kx, n)]


def backward(x, kx, ky, kz, n):
    """R(r) = sum over the full sphere of X(G) e^{-iG.r}: the stored half
    (Gx = 0 plane whole) plus the conjugates at -G for Gx > 0."""
    full = np.zeros((n, n, n), dtype=np.complex128)
    full[np.mod(kz, n), np.mod(ky, n), np.mod(kx, n)] = x
    h = kx > 0
    full[np.mod(-kz[h], n), np.mod(-ky[h], n), np.mod(-kx[h], n)] = np.conj(x[h])
    return np.fft.fftn(full).real


def gather(bs, i, hmati, ngrid, r):
    """eesAtmForceRchare for one atom: sum over its stencil of dMn R."""
    (c, b, a), _, dx, dy, dz = OE.stencil(bs, i, hmati, ngrid)
    v = r[c, b, a]
    return np.array([np.sum(dx * v), np.sum(dy * v), np.sum(dz * v)])


def ees_b(kx, ky, kz, ngrid, n_interp=OE.N_INTERP):
    """eesSetEesWghtGgrp: b(G) = bden(kx) bden(ky) bden(kz), G = 0 real."""
    bd = axis_weights(ngrid, n_interp)
    b = bd[np.mod(kx, ngrid)] * bd[np.mod(ky, ngrid)] * bd[np.mod(kz, ngrid)]
    g0 = (kx == 0) & (ky == 0) & (kz == 0)
    return np.where(g0, bd[0].real ** 3 + 0j, b)


def gpass(rho_g, kx, ky, kz, box_len, ecut_ha, sf, qt, tab, alp_ewd, b):
    """eesHartEextGchare for every type in order, then eesEwaldGchare.

    sf [ntyp][npts]: the transformed spread grids.  Returns (vks, ehart, eext,
    ewd, back [ntyp][npts] (the per-type force terms), ewald term [npts])."""
    from .density import spline_eval
    vol = box_len ** 3
    tpi = 2.0 * math.pi / box_len
    g2 = (kx * tpi) ** 2 + (ky * tpi) ** 2 + (kz * tpi) ** 2
    ecut4 = 8.0 * ecut_ha
    g0 = g2 == 0
    sel = (g2 <= ecut4) & ~g0
    w = np.where(kx == 0, 1.0, 2.0)
    vt_all = spline_eval(tab, np.sqrt(g2)) / vol             # [ntyp, npts]
    vks = np.zeros(len(kx), dtype=np.complex128)
    stot = np.zeros(len(kx), dtype=np.complex128)
    ehart = eext = 0.0
    backs = []
    i0 = np.nonzero(g0)[0][0] if g0.any() else -1
    for t in range(len(qt)):
        st = sf[t]
        if t == 0:
            hf = np.where(sel, 4.0 * math.pi / np.where(sel, g2, 1.0) / vol, 0.0)
            ehart = 0.5 * np.sum(hf * np.abs(rho_g) ** 2 * w)
            vks += rho_g * hf
        vt = np.where(sel, vt_all[t], 0.0)
        vext = st * b * vt
        eext += np.sum(np.where(sel, (rho_g * vext).real * w, 0.0))
        vks += np.where(sel, np.conj(vext), 0.0)
        stot = np.where(sel, stot + st * qt[t], np.where(g0, stot.real + st.real * qt[t], 0.0))
        back = np.where(sel, vt * np.conj(rho_g * b), 0.0)
        if i0 >= 0:
            v0 = tab["gzvps"][t] / vol
            vext0 = v0 * (st[i0].real * b[i0].real)
            eext += rho_g[i0].real * vext0
            vks[i0] = vks[i0].real + vext0
            back[i0] = v0 * (rho_g[i0].real * b[i0].real)
        backs.append(back)
    nz = ~g0
    preg = np.where(nz, 4.0 * math.pi * np.exp(-g2 / (4.0 * alp_ewd ** 2))
                    / np.where(nz, g2, 1.0) / vol, 0.0)
    bmag = np.abs(b) ** 2
    ewd = 0.5 * np.sum(np.where(nz, bmag * np.abs(stot) ** 2 * preg * w, 0.0))
    vks = np.where(sel | g0, vks, 0.0)
    return vks, ehart, eext, ewd, np.array(backs), np.where(nz, stot * preg * bmag, 0.0)


def hart_eext_ees(rho_g, kx, ky, kz, box_len, ecut_ha, atoms, tab, alp_ewd, ngrid,
                  n_interp=OE.N_INTERP):
    """The EES pass on packed density-sphere points.

    Arguments as oracle.density.hart_eext, plus the EES grid size and order.
    Returns (vks [npts] complex, ehart, eext, ewd, force [natm, 3]).
    """
    kx, ky, kz = np.asarray(kx), np.asarray(ky), np.asarray(kz)
    hmati = (np.eye(3) / box_len).reshape(-1)
    pos = np.asarray(atoms["pos"], dtype=np.float64)
    typ = np.asarray(atoms["typ"])
    qt = np.asarray(atoms["q"], dtype=np.float64)
    bs = OE.atom_bsplines(pos, hmati, ngrid, n_interp)
    sf = [forward(spread(bs, typ == t, ngrid), kx, ky, kz) for t in range(len(qt))]
    b = ees_b(kx, ky, kz, ngrid, n_interp)
    vks, ehart, eext, ewd, backs, ewt = gpass(rho_g, kx, ky, kz, box_len, ecut_ha, sf, qt, tab,
                                             alp_ewd, b)
    force = np.zeros((len(typ), 3))
    for t in range(len(qt)):
        r = backward(backs[t], kx, ky, kz, ngrid)
        for i in np.nonzero(typ == t)[0]:
            force[i] -= gather(bs, i, hmati, ngrid, r)
    r = backward(ewt, kx, ky, kz, ngrid)
    q = qt[typ]
    for i in range(len(typ)):
        force[i] -= q[i] * gather(bs, i, hmati, ngrid, r)
    return vks, ehart, eext, ewd, force
