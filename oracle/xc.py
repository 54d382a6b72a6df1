"""Oracle: BLYP gradient-corrected exchange-correlation in FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, for one Gamma-point spin-unpolarised density on the full grid:

* Becke 88 exchange gradient correction  CPXCFNCTS::becke_gcx_lda
  src_piny_physics_v1.0/abinito_physics/cp_xc_fnctl/cp_becke.C:20-77
  (spin densities rho/2, |grad rho|^2/4; beta = 0.0042, cp_grad_rho_ctrl.C:53);
* LYP correlation (local and gradient parts)  CPXCFNCTS::lyp_gcc
  cp_becke.C:91-173;
* the pointwise driver  CPXCFNCTS::CP_getGGAFunctional
  cp_grad_rho_ctrl.C:32-193: points with rho > rho_cut = 0.1 gga_cut, a
  smoothstep switch s(rho) with healing length 3.9 gga_cut, vks += df/drho,
  u = (grad rho / |grad rho|) df/d|grad rho|, E_GGA = (ex + ec) vol / N;
* the gradients and the White-Bird term of the density G space
  CP_Rho_GSpacePlane::divRhoVksGspace / acceptWhiteByrd
  (cp_density_ctrl/CP_Rho_GSpacePlane.C:278-400) and
  CP_Rho_RealSpacePlane::whiteByrdFFT / acceptWhiteByrd
  (CP_Rho_RealSpacePlane.C:1237-1340): grad rho and div u are spectral on the
  density sphere, and V_xc = v_LDA(x only) + df/drho - div u;
* with LYP on, CP_exc_calc keeps only Slater exchange (lyp_fact = 0,
  cp_pz_lda.C:62-63).

These are pinned to the reference's own routines compiled from their
sources under ``oracle/_ref`` (``ref_xc.cpp``), and the potential to finite
differences of the energy (tests/test_xc_oracle.py).
"""
import math

import numpy as np

BECKE_BETA = 0.0042          # cp_grad_rho_ctrl.C:53
GGA_CUT = 5.0e-5             # \gradient_cutoff default (set_sim_dict.C:556-559)
LYP = dict(a=0.049180, b=0.1320, c=0.25330, d=0.3490)   # cp_becke.C:114-117


def becke(rho, g2, beta=BECKE_BETA):
    """(f, df/drho, df/d|grad rho|) of becke_gcx_lda (cp_becke.C:44-73)."""
    rho = 0.5 * np.asarray(rho, dtype=np.float64)
    g2 = 0.25 * np.asarray(g2, dtype=np.float64)
    r43 = rho ** (4.0 / 3.0)
    r13 = rho ** (1.0 / 3.0)
    x = np.sqrt(g2) / r43
    root = np.sqrt(1.0 + x * x)
    asinch = np.log(x + root)
    bterm = 1.0 + 6.0 * beta * x * asinch
    bx = x * x / bterm
    bxx = x / bterm
    bpx = 2.0 * bxx - 6.0 * beta * bxx * bxx * (asinch + x / root)
    f = -2.0 * beta * r43 * bx
    dfdn = -beta * (4.0 / 3.0) * r13 * (bx - x * bpx)
    dfdg = -beta * bpx
    return f, dfdn, dfdg


def lyp(rho, g2):
    """(f, df/drho, df/d|grad rho|) of lyp_gcc (cp_becke.C:121-170)."""
    a, b, c, d = LYP["a"], LYP["b"], LYP["c"], LYP["d"]
    rho = np.asarray(rho, dtype=np.float64)
    g2 = np.asarray(g2, dtype=np.float64)
    cf = 0.30 * (3.0 * math.pi * math.pi) ** (2.0 / 3.0)
    drho = np.sqrt(g2)
    rm13 = rho ** (-1.0 / 3.0)
    rm113 = rho ** (-11.0 / 3.0)
    rm43 = rm13 / rho
    den = 1.0 + d * rm13
    den2 = den * den
    cexp = np.exp(-c * rm13)
    omega = cexp * rm113 / den
    br = (d * rm43 + den * (c * rm43 - 11.0 / rho)) / 3.0
    domega = omega * br / den
    delta = c * rm13 + d * rm13 / den
    br = (d * rm13 - den) * d * rm43 / den2
    ddelta = (-c * rm43 + br) / 3.0
    rho2 = rho * rho
    term1 = -a * rho / den
    br1 = ((5.0 - 7.0 / 6.0 * delta) / 3.0) * g2
    br2 = 4.0 * cf * rho ** (8.0 / 3.0) + br1
    br3 = (0.25 * br2 - 11.0 * g2 / 24.0) * rho2
    term2 = -a * b * omega * br3
    arho = 0.25 * br2 - 11.0 * g2 / 24.0
    darho = 0.25 * (32.0 * cf * rho ** (5.0 / 3.0) / 3.0 - 7.0 / 18.0 * ddelta * g2)
    dprho = 2.0 * arho * rho + darho * rho2
    dterm1 = -a * (1.0 + (4.0 / 3.0) * d * rm13) / den2
    dterm2 = -a * b * (domega * br3 + omega * dprho)
    f = term1 + term2
    dfdn = dterm1 + dterm2
    dfdg = -a * b * omega * (0.5 * ((5.0 - 7.0 / 6.0 * delta) / 3.0) - 11.0 / 12.0) * rho2 * drho
    return f, dfdn, dfdg


def gga_functional(rho, gx, gy, gz, vol, gga_cut=GGA_CUT, becke_on=True, lyp_on=True):
    """CP_getGGAFunctional (cp_grad_rho_ctrl.C:81-184) on flat arrays.

    Returns (df/drho to add to vks, ux, uy, uz, E_GGA).  Points with an exactly
    zero gradient (where the reference divides 0 by 0) get u = 0.
    """
    rho = np.asarray(rho, dtype=np.float64).ravel()
    gx, gy, gz = (np.asarray(v, dtype=np.float64).ravel() for v in (gx, gy, gz))
    n = rho.size
    rho_cut = 0.1 * gga_cut
    heali = 1.0 / (3.9 * gga_cut)
    on = rho > rho_cut
    r = np.where(on, rho, 1.0)
    g2 = gx * gx + gy * gy + gz * gz
    g2s = np.where(on, g2, 1.0)
    rsw = np.clip((r - rho_cut) * heali, 0.0, 1.0)
    srho = rsw * rsw * (3.0 - 2.0 * rsw)
    dsrho = 6.0 * rsw * (1.0 - rsw) * heali
    fx = dfx = dgx = np.zeros(n)
    if becke_on:
        fx, dfx, dgx = becke(r, g2s)
    fc = dfc = dgc = np.zeros(n)
    if lyp_on:
        fc, dfc, dgc = lyp(r, g2s)
    dfx = dfx * srho + fx * dsrho
    dfc = dfc * srho + fc * dsrho
    dg = (dgx + dgc) * srho
    fx = fx * srho
    fc = fc * srho
    dv = np.where(on, dfx + dfc, 0.0)
    e = np.sum(np.where(on, fx + fc, 0.0)) * vol / n
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(on & (g2 > 0.0), 1.0 / np.sqrt(np.where(g2 > 0.0, g2, 1.0)), 0.0)
    s = np.where(on, dg * inv, 0.0)
    return dv, gx * s, gy * s, gz * s, e


def _gvec(lay_d):
    tpi = 2.0 * math.pi / lay_d.box_len
    return lay_d.kx * tpi, lay_d.ky * tpi, lay_d.kz * tpi


def density_gradient(rho_r, lay_d, vol):
    """grad rho(r) from rho(G) on the density sphere (CP_Rho_GSpacePlane.C:278-320,
    the backward FFTs scaled 1/vol); cubic box."""
    from . import density as OD
    rg = OD.rho_to_g(rho_r, lay_d, vol)
    g = _gvec(lay_d)
    n = rho_r.shape[0]
    return [OD.vg_to_r(1j * gd * rg / vol, lay_d).reshape(n, n, n) for gd in g]


def white_byrd(ux, uy, uz, lay_d):
    """div u(r) on the density sphere: u scaled 1/N and transformed forward
    (whiteByrdFFT, CP_Rho_RealSpacePlane.C:1237-1260), i g.u(G) summed
    (acceptWhiteByrd, CP_Rho_GSpacePlane.C:374-392) and transformed back."""
    from . import density as OD
    n = ux.shape[0]
    g = _gvec(lay_d)
    w = 0.0
    for gd, u in zip(g, (ux, uy, uz)):
        # rho_to_g(f, vol = N) = sum_r f e^{-iG.r}: the forward transform / N * N
        ug = OD.rho_to_g(u, lay_d, float(n ** 3)) / n ** 3
        w = w + 1j * gd * ug
    return OD.vg_to_r(w, lay_d).reshape(n, n, n)


def blyp_vxc(rho_r, lay_d, vol, gga_cut=GGA_CUT):
    """(V_xc(r), E_xc, muxc) of BLYP: Slater exchange (CP_exc_calc with
    lyp = 1), the gradient correction, and the White-Bird divergence."""
    from . import density as OD
    v_lda, e_lda, mu = slater_lda(rho_r, vol)
    gx, gy, gz = density_gradient(rho_r, lay_d, vol)
    dv, ux, uy, uz, e_gga = gga_functional(rho_r, gx, gy, gz, vol, gga_cut)
    n = rho_r.shape[0]
    div = white_byrd(ux.reshape(n, n, n), uy.reshape(n, n, n), uz.reshape(n, n, n), lay_d)
    v = v_lda + dv.reshape(rho_r.shape) - div
    return v, e_lda + e_gga, mu, e_gga


def slater_lda(rho, vol):
    """CP_exc_calc with cp_lyp = 1 (cp_pz_lda.C:62-63, :117-150): exchange only."""
    r = np.asarray(rho, dtype=np.float64)
    pos = r > 0
    xfact = np.where(pos, -np.cbrt(3.0 * np.where(pos, r, 0.0) / math.pi), 0.0)
    r0 = np.where(pos, r, 0.0)
    vscale = vol / r.size
    return xfact, 0.75 * np.sum(xfact * r0) * vscale, np.sum(xfact * r0) * vscale
