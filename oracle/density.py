"""Oracle: XC, Hartree + local pseudopotential + Ewald (reciprocal) in FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* PZ-LDA  CPXCFNCTS::CP_exc_calc  src_piny_physics_v1.0/abinito_physics/
  cp_xc_fnctl/cp_pz_lda.C:23-170.  rho is the scaled density (electrons/bohr^3);
  E_xc = (0.75 sum ex + sum ec) vol/N, v_xc = xfact + mufact.
  (rho <= 0 gives the reference NaN/inf; here those points contribute 0.)
* Hartree / local / Ewald  CPLOCAL::CP_hart_eext_calc  cp_local/cp_hart_ext.C:56-405,
  spline look-up CP_get_vpsnow :433-475.  Sums run over the density sphere
  |G|^2 <= 8 ecut_Ha (ecut4, :109) with weight 1 on Gx=0 and 2 elsewhere:
    vks(G)  = rho(G) 4 pi/(g^2 vol) + conj(vext(G)),  vext = sum_a e^{iG.R_a} vps_a(g)/vol
    E_H     = 1/2 sum w 4 pi |rho|^2/(g^2 vol)
    E_ext   = sum w Re(rho vext) + rho(0) sum_a gzvps_a/vol
    E_ewd   = 1/2 sum w 4 pi e^{-g^2/4alp^2}/(g^2 vol) |sum_a q_a e^{iG.R_a}|^2
  and the atom forces of :270-300.
* rho(G) = (vol/N) sum_r rho(r) e^{-iG.r} and V(r) = sum_G vks(G) e^{+iG.r} are the
  normalisations these sums need (E_H above is the Hartree energy only with them).
"""
import math

import numpy as np

PZ = dict(gamma=-0.14230, beta1=1.05290, beta2=0.33340, au=0.03110, bu=-0.0480,
          cu=0.00200, du=-0.01160)


def pz_lda(rho, vol):
    """(v_xc, E_xc, muxc) for rho [N^3] (cp_pz_lda.C:88-166)."""
    p = PZ
    r = np.asarray(rho, dtype=np.float64)
    pos = r > 0
    rr = np.where(pos, r, 1.0)
    rs = (3.0 / (4.0 * math.pi * rr)) ** (1.0 / 3.0)
    sq = np.sqrt(rs)
    xfact = -((3.0 * rr / math.pi) ** (1.0 / 3.0))
    rat1 = (7.0 / 6.0) * p["beta1"]
    rat2 = (4.0 / 3.0) * p["beta2"]
    cf1 = 1.0 + p["beta1"] * sq + p["beta2"] * rs
    cf2 = 1.0 + rat1 * sq + rat2 * rs
    c_hi = p["gamma"] / cf1
    m_hi = c_hi * (cf2 / cf1)
    lnrs = np.log(rs)
    c_lo = p["au"] * lnrs + p["bu"] + p["cu"] * rs * lnrs + p["du"] * rs
    third = 1.0 / 3.0
    m_lo = (p["au"] * lnrs + (p["bu"] - third * p["au"]) + 2.0 * third * p["cu"] * rs * lnrs
            + third * (2.0 * p["du"] - p["cu"]) * rs)
    hi = rs >= 1.0
    cfact = np.where(hi, c_hi, c_lo)
    mufact = np.where(hi, m_hi, m_lo)
    xfact = np.where(pos, xfact, 0.0)
    cfact = np.where(pos, cfact, 0.0)
    mufact = np.where(pos, mufact, 0.0)
    r0 = np.where(pos, r, 0.0)
    ex = np.sum(xfact * r0)
    ec = np.sum(cfact * r0)
    v = xfact + mufact
    vscale = vol / r.size
    return v, (0.75 * ex + ec) * vscale, np.sum(v * r0) * vscale


def spline_eval(tab, g):
    """CP_get_vpsnow (cp_hart_ext.C:459-471): cubic in h from the knot below g."""
    vps = np.asarray(tab["vps"])                    # [ntyp, 4, nspl] = vps0..vps3
    v0, v1, v2, v3 = vps[:, 0], vps[:, 1], vps[:, 2], vps[:, 3]
    gmin, dg, ns = tab["gmin"], tab["dg"], v0.shape[-1]
    iii = ((g - gmin) / dg + 1.0).astype(np.int64)
    iii = np.clip(iii, 1, ns)
    h = g - ((iii - 1) * dg + gmin)
    k = iii - 1
    return ((v3[:, k] * h + v2[:, k]) * h + v1[:, k]) * h + v0[:, k]


def hart_eext(rho_g, kx, ky, kz, box_len, ecut_ha, atoms, tab, alp_ewd):
    """CP_hart_eext_calc on packed density-sphere points.

    rho_g: complex [npts] in the reference convention rho(G) = (vol/N) sum rho e^{-iGr};
    atoms: dict(pos [natm,3], typ [natm] 0-based, q [ntyp]); tab: spline tables
    vps [ntyp, 4, nspl] (vps0..vps3), gmin, dg, gzvps [ntyp].
    Returns (vks [npts] complex, ehart, eext, ewd, force [natm, 3]).
    """
    from .fftpath import state_map
    vol = box_len ** 3
    tpi = 2.0 * math.pi / box_len
    kx, ky, kz = np.asarray(kx), np.asarray(ky), np.asarray(kz)
    gx_all, gy_all, gz_all = kx * tpi, ky * tpi, kz * tpi
    g2_all = gx_all * gx_all + gy_all * gy_all + gz_all * gz_all
    ecut4 = 8.0 * ecut_ha
    pos = np.asarray(atoms["pos"], dtype=np.float64)
    typ = np.asarray(atoms["typ"])
    q = np.asarray(atoms["q"], dtype=np.float64)[typ]
    natm = len(typ)
    vks = np.zeros(len(kx), dtype=np.complex128)

    def part(p0, p1):
        """Points p0..p1-1: vks there and the (ehart, ewd, eext, force) partials."""
        gx, gy, gz, g2 = gx_all[p0:p1], gy_all[p0:p1], gz_all[p0:p1], g2_all[p0:p1]
        rg = rho_g[p0:p1]
        sel = (g2 <= ecut4) & (g2 != 0)
        w = np.where(kx[p0:p1] == 0, 1.0, 2.0)
        g = np.sqrt(g2)
        vt = spline_eval(tab, g) / vol                     # [ntyp, n]
        vtemp = vt[typ]                                    # [natm, n]
        arg = np.outer(pos[:, 0], gx) + np.outer(pos[:, 1], gy) + np.outer(pos[:, 2], gz)
        h = np.exp(1j * arg)                               # e^{iG.R}  [natm, n]
        vext = np.sum(h * vtemp, axis=0)
        sewd = np.sum(h * q[:, None], axis=0)
        hart = np.where(sel, 4.0 * math.pi / np.where(sel, g2, 1.0) / vol, 0.0)
        vks[p0:p1] = np.where(sel, rg * hart + np.conj(vext), 0.0)
        eh = 0.5 * np.sum(np.where(sel, hart * np.abs(rg) ** 2 * w, 0.0))
        ewdf = np.where(sel, 4.0 * math.pi * np.exp(-g2 / (4.0 * alp_ewd ** 2))
                        / np.where(sel, g2, 1.0) / vol, 0.0)
        ew = 0.5 * np.sum(ewdf * np.abs(sewd) ** 2 * w)
        ee = np.sum(np.where(sel, (rg * vext).real * w, 0.0))
        # atom forces (cp_hart_ext.C:270-300)
        rr = np.where(sel, rg.real * w, 0.0)
        ri = np.where(sel, rg.imag * w, 0.0)
        sr = sewd.real * ewdf * w
        si = sewd.imag * ewdf * w
        tr = rr[None] * vtemp + sr[None] * q[:, None]
        ti = -ri[None] * vtemp + si[None] * q[:, None]
        t = tr * h.imag - ti * h.real                      # [natm, n]
        return eh, ew, ee, np.stack([t @ gx, t @ gy, t @ gz], axis=1)
    ehart = ewd = eext = 0.0
    force = np.zeros((natm, 3))
    for eh, ew, ee, fo in state_map(part, len(kx), 16384):
        ehart += eh
        ewd += ew
        eext += ee
        force += fo
    g2 = g2_all
    # G = 0 (:345-368)
    izero = np.nonzero(g2 == 0)[0]
    if len(izero):
        i0 = izero[0]
        v0 = np.sum(np.asarray(tab["gzvps"])[typ]) / vol
        vks[i0] = v0
        eext += v0 * rho_g[i0].real
    return vks, ehart, eext, ewd, force


def rho_to_g(rho_r, lay_d, vol):
    """rho(G) = (vol/N) sum_r rho(r) e^{-iG.r} on the packed density sphere."""
    from . import fftpath
    n = rho_r.shape[0]
    # state_r_to_g computes sum f e^{+iGr}; conj gives the e^{-iGr} sum for real f
    fg = fftpath.state_r_to_g(rho_r[None], lay_d)[0]
    return np.conj(fg) * (vol / n ** 3)


def vg_to_r(vks_g, lay_d):
    """V(r) = sum_G vks(G) e^{+iG.r} over the full sphere (Hermitian extension)."""
    from . import fftpath
    # state_g_to_r computes sum c e^{-iGr}; feed conj(vks) for the e^{+iGr} sum
    return fftpath.state_g_to_r(np.conj(vks_g)[None], lay_d)[0]


def density_layout(box_len, ecut_ry, n):
    """The density sphere (|G|^2/2 <= 4 ecut_Ha) in flip_data_set order, one chunk."""
    from . import layout as OL
    # loop bounds kmaxv = 2 kmax_cp (calc_cutoff, set_cp_ewald.C:205-207)
    kmax = OL.calc_kmax(box_len, ecut_ry)
    ka, kb, kc = OL.setkvec3d_sm(2.0 * ecut_ry, 2 * kmax, box_len)
    fx, fy, fz, _ = OL.flip_data_set(ka, kb, kc)
    lay = OL.Layout.__new__(OL.Layout)
    lay.box_len = float(box_len)
    lay.n = n
    lay.kx, lay.ky, lay.kz = fx, fy, fz
    lay.npts = len(fx)
    lay.runs = OL.runs_from_kvecs(fx, fy, fz, n, n, n)
    lay.nlines = len(lay.runs) // 2
    lay.nplane_x = int(fx.max()) + 1
    tpi = 2.0 * math.pi / box_len
    lay.g2 = (fx * tpi) ** 2 + (fy * tpi) ** 2 + (fz * tpi) ** 2
    lay.kx0 = fx == 0
    return lay
