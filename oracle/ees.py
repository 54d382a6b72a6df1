"""Oracle: EES non-local pseudopotential (energy, psi forces, atom forces) in FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_ees_nonlocal.C:

* B-spline Euler weights b(G)      eesSetEesWghtGgrp :60-169 with get_bspline_wght1d
                                   (interface/cp_ewald/set_cp_ewald.C:1237-1322)
* spline look-up per point         eesSplProjectorGgrp :182-240
* atom B-splines on the NL grid    eesAtmBsplineRgrp :256-580
* projector x psi                  eesProjGchare :594-724, eesYlmOnD :735-1236 (l = 0, 1)
* Z matrix                         eesZmatRchare :1238-1346 (+ the sum over planes)
* energy, atom forces, scatter     eesEnergyAtmForcRchare :1480-1700
* psi force                        eesPsiForcGspace :2000-2064
* NL grid size                     init_nonlocal_ees (set_cp_ewald.C:1329-1400)
* NL FFTs                          FFTcache::doNlFFT* (fftCache.C:562-809): the state
                                   transform conventions on the NL grid, unscaled.

A channel is (type, l, m), one iteration of the reference's iter_nl loop
(lang_v / mang_v / ityp_v).  Per channel and state:
  projPsiG = conj(dyp psi),  dyp = Ylm b(G) v_tl(|G|)   (G = 0: l = 0 -> b y00 gzvps0, else 0)
  projPsiR = FFT_G->R(projPsiG) on the NL grid
  Z_a      = sum_{8x8x8 stencil} projPsiR Mn,  E_NL += Z_a^2 vnorm/vol occ
  Z_a     *= 2 vnorm/vol occ;  F_a -= Z_a sum projPsiR dMn
  scr      = sum_a Z_a Mn;  fpsi += -w conj(dyp FFT_R->G(scr))   (w = 1 on Gx = 0, else 2)
"""
import math

import numpy as np

from . import fftpath as OF
from . import layout as OL

N_INTERP = 8
EES_SCALE = 1.2  # cp_pseudo_ees_scale (fft_size_scale)


def nl_grid_size(kmax, scale=EES_SCALE, n_interp=N_INTERP):
    """init_nonlocal_ees (set_cp_ewald.C:1329-1400) for a cubic box of kmax_cp."""
    nk = kmax + 1
    nkf = int(2.0 * scale * float(nk))
    if nkf < 2 * nk:
        nkf += 1
    for k in OL.FFT_SIZES:
        if k >= nkf:
            if k < n_interp:
                raise ValueError("n_interp larger than the NL grid")
            return k
    raise ValueError("NL FFT size too large for the radix table")


def bspline_wght1d(n_interp, ngrid):
    """get_bspline_wght1d (set_cp_ewald.C:1237-1322): complex 1/b per grid index m-1."""
    rn = np.arange(1, n_interp + 1, dtype=np.float64)           # rn[j] = j
    rn1 = np.zeros(n_interp)
    rn1[1:] = 1.0 / np.arange(1, n_interp, dtype=np.float64)    # rn1[j] = 1/(j-1)
    uk = np.arange(1, n_interp + 1, dtype=np.float64)
    mn = np.zeros(n_interp)
    mn[0] = 1.0
    for n in range(3, n_interp + 1):
        for k in range(n, 1, -1):
            mn[k - 1] = (uk[k - 1] * mn[k - 1] + (rn[n - 1] - uk[k - 1]) * mn[k - 2]) * rn1[n - 1]
        mn[0] = uk[0] * mn[0] * rn1[n - 1]
    grid = float(ngrid)
    m = np.arange(ngrid, dtype=np.float64)
    tpi_n = 2.0 * math.pi / grid
    br = np.zeros(ngrid)
    bi = np.zeros(ngrid)
    for k in range(1, n_interp):
        arg = tpi_n * ((k - 1) * m)
        br += np.cos(arg) * mn[k - 1]
        bi += np.sin(arg) * mn[k - 1]
    arg = 2.0 * math.pi * float(n_interp - 1) / grid * m
    nr, ni = np.cos(arg), np.sin(arg)
    den = br * br + bi * bi
    tr = (nr * br + ni * bi) / den
    ti = (ni * br - nr * bi) / den
    return tr, ti


def ees_weights(kx, ky, kz, nkf, n_interp=N_INTERP):
    """eesSetEesWghtGgrp: b(G) = bden_a(ka) bden_b(kb) bden_c(kc), G = 0 real."""
    ar, ai = bspline_wght1d(n_interp, nkf)
    ia, ib, ic = np.mod(kx, nkf), np.mod(ky, nkf), np.mod(kz, nkf)
    abr = ar[ia] * ar[ib] - ai[ia] * ai[ib]
    abi = ai[ia] * ar[ib] + ar[ia] * ai[ib]
    bre = abr * ar[ic] - abi * ai[ic]
    bim = abi * ar[ic] + abr * ai[ic]
    g0 = (kx == 0) & (ky == 0) & (kz == 0)
    bre = np.where(g0, ar[0] * ar[0] * ar[0], bre)
    bim = np.where(g0, 0.0, bim)
    return bre, bim


def gvec(kx, ky, kz, hmati):
    """(gx, gy, gz) = 2 pi hmati^T k (hmati column-major, 0-based)."""
    tpi = 2.0 * math.pi
    h = hmati
    xk = (kx * h[0] + ky * h[1] + kz * h[2]) * tpi
    yk = (kx * h[3] + ky * h[4] + kz * h[5]) * tpi
    zk = (kx * h[6] + ky * h[7] + kz * h[8]) * tpi
    return xk, yk, zk


def spline_lookup(g, gmin, dg, nspl):
    """eesSplProjectorGgrp: 1-based index and offset h (g < 1e-12: 1, 0)."""
    iii = ((g - gmin) / dg + 1.0).astype(np.int64)
    iii = np.clip(iii, 1, nspl)
    h = g - ((iii - 1) * dg + gmin)
    small = g < 1.0e-12
    return np.where(small, 1, iii), np.where(small, 0.0, h)


def ylm_d(l, m, kx, ky, kz, hmati, dre, dim):
    """eesYlmOnD for l = 0, 1: dy = Ylm * d (times i for l = 1)."""
    rt_fpi = 1.0 / math.sqrt(4.0 * math.pi)
    rt_thrfpi = math.sqrt(3.0 / (4.0 * math.pi))
    rt_threpi = math.sqrt(1.5 / (4.0 * math.pi)) * math.sqrt(2.0)
    if l == 0:
        return dre * rt_fpi, dim * rt_fpi
    if l != 1:
        raise ValueError("only s and p channels")
    xk, yk, zk = gvec(kx, ky, kz, hmati)
    g = np.sqrt(xk * xk + yk * yk + zk * zk)
    nz = g != 0.0
    gsafe = np.where(nz, g, 1.0)
    if m == 0:
        y = rt_thrfpi * (zk / gsafe)
    else:
        gs = np.sqrt(xk * xk + yk * yk)
        gss = np.where(gs == 0.0, 1.0, gs)
        st = gs / gsafe
        if m == 1:
            ph = np.where(gs == 0.0, 1.0, xk / gss)
        else:
            ph = np.where(gs == 0.0, 0.0, yk / gss)
        y = rt_threpi * st * ph
    return np.where(nz, -dim * y, 0.0), np.where(nz, dre * y, 0.0)


def channel_dyp(ch, lay, hmati, nkf, spl, n_interp=N_INTERP):
    """dyp(G) of eesProjGchare for one channel (complex [npts])."""
    kx, ky, kz = lay.kx, lay.ky, lay.kz
    bre, bim = ees_weights(kx, ky, kz, nkf, n_interp)
    dr, di = ylm_d(ch["l"], ch["m"], kx, ky, kz, hmati, bre, bim)
    xk, yk, zk = gvec(kx, ky, kz, hmati)
    g = np.sqrt(xk * xk + yk * yk + zk * zk)
    ind, h = spline_lookup(g, spl["gmin"], spl["dg"], spl["nspl"])
    v = ch["vnl"]                     # [4][nspl]: v0..v3
    k = ind - 1
    vnow = ((v[3][k] * h + v[2][k]) * h + v[1][k]) * h + v[0][k]
    g0 = (kx == 0) & (ky == 0) & (kz == 0)
    if ch["l"] == 0:
        gz = ch["gzvps0"]
        dr = np.where(g0, dr * gz, dr * vnow)
        di = np.where(g0, 0.0, di * vnow)
    else:
        dr = np.where(g0, 0.0, dr * vnow)
        di = np.where(g0, 0.0, di * vnow)
    return dr + 1j * di


def atom_bsplines(pos, hmati, nkf, n_interp=N_INTERP):
    """eesAtmBsplineRgrp, separable factors per atom.

    Returns dict of arrays [natm][n_interp]: ia, ib, ic (0-based grid indices),
    mn_a/b/c and dmn_a/b/c, in the reference's interpolation order j = 1..n.
    """
    pos = np.asarray(pos, dtype=np.float64)
    h = hmati
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    s = [x * h[0] + y * h[3] + z * h[6], x * h[1] + y * h[4] + z * h[7],
         x * h[2] + y * h[5] + z * h[8]]
    out = {}
    grid = float(nkf)
    aj = np.arange(n_interp, dtype=np.float64)
    rn = np.arange(1, n_interp + 1, dtype=np.float64)
    rn1 = np.zeros(n_interp)
    rn1[1:] = 1.0 / np.arange(1, n_interp, dtype=np.float64)
    for d, name in enumerate("abc"):
        t = s[d]
        xm = t - 0.5
        nint = np.where(xm >= 0.0, np.trunc(xm + 0.5), np.trunc(xm - 0.5))  # SIMP_NINT
        t = t - nint
        t = np.where(t == 1.0, 0.0, t)
        t = t * grid
        it = t.astype(np.int64)
        frac = t - it
        u = frac[:, None] + aj[None, :]                        # ua[j] = frac + (j-1)
        idx = it[:, None] - (np.arange(1, n_interp + 1)[None, :] - 2)
        idx = np.where(idx > 0, idx, nkf + idx)
        idx = np.where(idx <= nkf, idx, idx - nkf)
        mn = np.zeros_like(u)
        mn[:, 0] = 1.0 - np.abs(u[:, 0] - 1.0)
        mn[:, 1] = 1.0 - np.abs(u[:, 1] - 1.0)
        dmn = np.zeros_like(u)
        for n in range(3, n_interp + 1):
            for j in range(n, 1, -1):
                mn[:, j - 1] = (u[:, j - 1] * mn[:, j - 1]
                                + (rn[n - 1] - u[:, j - 1]) * mn[:, j - 2]) * rn1[n - 1]
            mn[:, 0] = u[:, 0] * mn[:, 0] * rn1[n - 1]
            if n == n_interp - 1:
                dmn[:, 0] = mn[:, 0]
                dmn[:, 1:] = mn[:, 1:] - mn[:, :-1]
        out["i" + name] = (idx - 1).astype(np.int64)
        out["mn_" + name] = mn.copy()
        out["dmn_" + name] = dmn
    return out


def stencil(bs, i, hmati, nkf):
    """The 8x8x8 stencil of atom i: flat indices (c, b, a) and mn, dmn_x/y/z.

    Element order follows eesAtmBsplineRgrp IV (jc outer, jb, ja inner).
    """
    grid = float(nkf)
    h = hmati
    ia, ib, ic = bs["ia"][i], bs["ib"][i], bs["ic"][i]
    ma, mb, mc = bs["mn_a"][i], bs["mn_b"][i], bs["mn_c"][i]
    da, db, dc = bs["dmn_a"][i], bs["dmn_b"][i], bs["dmn_c"][i]
    C, B, A = np.meshgrid(np.arange(len(ic)), np.arange(len(ib)), np.arange(len(ia)),
                          indexing="ij")
    at = da[A] * mb[B] * mc[C] * grid
    bt = ma[A] * db[B] * mc[C] * grid
    ct = ma[A] * mb[B] * dc[C] * grid
    mn = ma[A] * mb[B] * mc[C]
    dx = at * h[0] + bt * h[1] + ct * h[2]
    dy = at * h[3] + bt * h[4] + ct * h[5]
    dz = at * h[6] + bt * h[7] + ct * h[8]
    return (ic[C], ib[B], ia[A]), mn, dx, dy, dz


class NLGrid:
    """The state's packed layout viewed on the NL grid (for the oracle FFTs)."""

    def __init__(self, lay, nkf):
        self.n = nkf
        self.npts = lay.npts
        self.kx, self.ky, self.kz = lay.kx, lay.ky, lay.kz
        self.runs = OL.runs_from_kvecs(lay.kx, lay.ky, lay.kz, nkf, nkf, nkf)
        self.nlines = len(self.runs) // 2

    line_tables = OL.Layout.line_tables


def nonlocal_ees(psi, lay, occ, vol, hmati, atoms, channels, spl, nkf=None,
                 n_interp=N_INTERP):
    """EES non-local for all states and channels.

    psi [S, npts] complex; atoms: dict pos [natm,3], typ [natm]; channels: list of
    dicts (type, l, m, vnl [4][nspl], gzvps0, vnorm); spl: gmin, dg, nspl.
    Returns (E_NL, fpsi [S, npts] to add to the force, fatm [natm, 3] to add).
    """
    if nkf is None:
        nkf = nl_grid_size(lay.kmax, EES_SCALE, n_interp)
    grid = NLGrid(lay, nkf)
    pos = np.asarray(atoms["pos"], dtype=np.float64)
    typ = np.asarray(atoms["typ"])
    natm = len(typ)
    bs = atom_bsplines(pos, hmati, nkf, n_interp)
    stens = [stencil(bs, i, hmati, nkf) for i in range(natm)]
    S = psi.shape[0]
    w = np.where(lay.kx == 0, 1.0, 2.0)
    g0 = np.nonzero((lay.kx == 0) & (lay.ky == 0) & (lay.kz == 0))[0]
    fpsi = np.zeros_like(psi)
    enl = 0.0
    fatm = np.zeros((natm, 3))
    for ch in channels:
        dyp = channel_dyp(ch, lay, hmati, nkf, spl, n_interp)
        members = np.nonzero(typ == ch["type"])[0]
        vn = ch["vnorm"] / vol
        d = dyp.copy()
        if len(g0):
            d[g0] = d[g0].real

        def chunk(s0, s1):
            """States s0..s1-1 of this channel: (E_NL, atom forces) partials; the
            psi force goes to fpsi.  An atom's 512 stencil points are distinct
            grid points, so its scatter needs no accumulation within itself."""
            proj = np.conj(dyp[None, :] * psi[s0:s1])
            pr = OF.state_g_to_r(proj, grid)              # [s, c, b, a]
            scr = np.zeros_like(pr)
            wn = np.asarray(occ[s0:s1], dtype=np.float64)
            e, fa = 0.0, np.zeros((natm, 3))
            for i in members:
                (c, b, a), mn, dx, dy, dz = stens[i]
                vals = pr[:, c, b, a].reshape(s1 - s0, -1)
                zr = vals @ mn.ravel()
                e += float(np.sum(zr * zr * vn * wn))
                zs = zr * 2.0 * vn * wn
                fa[i, 0] -= float(np.sum((vals @ dx.ravel()) * zs))
                fa[i, 1] -= float(np.sum((vals @ dy.ravel()) * zs))
                fa[i, 2] -= float(np.sum((vals @ dz.ravel()) * zs))
                scr[:, c, b, a] += zs[:, None, None, None] * mn[None]
            pg = OF.state_r_to_g(scr, grid)
            if len(g0):
                pg[:, g0] = pg[:, g0].real
            fpsi[s0:s1] += -w[None, :] * np.conj(d[None, :] * pg)
            return e, fa
        for e, fa in OF.state_map(chunk, S, 8):
            enl += e
            fatm += fa
    return enl, fpsi, fatm
