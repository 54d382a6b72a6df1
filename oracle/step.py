"""Oracle: one CP electronic step in FP64 (the composition the GPU step runs).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

  rho (fftpath.density) -> V_KS = v_xc + Hartree/local (density.py)
  F = addForces(-2/N FFT^-1[V psi]) - kinetic term          (fftpath.py)
  lambda(i,j) = sum_p Re(conj psi_i F_j);  F_i <- F_i - wpt/2 sum_j psi_j lambda(j,i)
      (the orthonormality constraint: with S = 2 I it removes <psi_j|F_i>)
  velocity Verlet of CP_integrate_dyn / cp_evolve_vel / get_fictKE
      (cp_integrate/cp_dynamics.C:29-258) without the thermostat, Gx=0 and
      G=0 conventions of :165-200, redundant-half sync of
      CP_State_GSpacePlane.C:2862-3061
  S = pc_overlap(psi, psi); T = Schulz (S/2)^-1/2 (ortho.py); psi <- psi T
"""
import math

import numpy as np

from . import density as OD
from . import fftpath as OF
from . import ortho as OO


def point_classes(lay):
    kx, ky, kz = lay.kx, lay.ky, lay.kz
    cls = np.full(lay.npts, 3, dtype=np.int64)
    z = kx == 0
    cls[z & (ky == 0) & (kz == 0)] = 1
    cls[z & ((ky > 0) | ((ky == 0) & (kz > 0)))] = 2
    red = z & ((ky < 0) | ((ky == 0) & (kz < 0)))
    cls[red] = 0
    key = {(int(ky[i]), int(kz[i])): i for i in np.nonzero(z)[0]}
    ridx = np.nonzero(red)[0]
    rsrc = np.array([key[(-int(ky[i]), -int(kz[i]))] for i in ridx], dtype=np.int64)
    return cls, ridx, rsrc


def cp_mass(lay, tau_fs, cut_ry):
    """set_cpmass (set_cp_ewald.C:32-74)."""
    tau = tau_fs / 0.0241888
    m0 = 4.0 * tau * tau * 0.00050
    en = 0.5 * lay.g2
    m = np.where(en > 0.5 * cut_ry, m0 * en / (0.5 * cut_ry), m0)
    g0 = (lay.kx == 0) & (lay.ky == 0) & (lay.kz == 0)
    return np.where(g0, 0.5 * m0, m)


def integrate(F, psi, v, cmass, lay, dt, iteration):
    """Velocity Verlet without NHC; returns (psi, v, fictitious KE)."""
    cls, ridx, rsrc = point_classes(lay)
    live = cls != 0
    F = F.copy()
    v = v.copy()
    psi = psi.copy()
    g0 = cls == 1
    F[:, g0] = F[:, g0].real
    v[:, g0] = v[:, g0].real

    def kick(v):
        v = v.copy()
        v[:, live] += F[:, live] * (0.5 * dt / cmass[live])[None]
        v[:, g0] = v[:, g0].real
        return v
    if iteration > 1:
        v = kick(v)
    mfac = np.where(cls == 2, 2.0, 1.0) * cmass
    ke = 0.5 * np.sum(np.abs(v[:, live]) ** 2 * mfac[live][None])
    v = kick(v)
    psi[:, live] += v[:, live] * dt
    psi[:, ridx] = np.conj(psi[:, rsrc])
    v[:, ridx] = np.conj(v[:, rsrc])
    return psi, v, ke


def constrain(F, psi, lay):
    """F_i <- F_i - wpt/2 sum_j psi_j <psi_j|F_i> with <a|b> = sum_p Re(conj a b)."""
    lam = OO.real_view(psi) @ OO.real_view(F).T          # lam[j, i] = <psi_j|F_i>
    w = np.where(lay.kx == 0, 1.0, 2.0)
    return F - 0.5 * w[None] * (lam.T @ psi), lam


def forces(psi, occ, sysm, lay, dlay, chunk=16, nonlocal_on=False, nkf=None, xc="pz_lda",
           nonlocal_sf=False):
    """Energies, V_KS, constrained-force input F and atom forces (local + Ewald,
    plus the EES non-local pass when nonlocal_on: addForces adds its psi force,
    stateSlab.C:240-272).  xc = "blyp" takes the BLYP potential of oracle/xc.py."""
    vol = sysm.box_len ** 3
    rho = OF.density(psi, lay, occ, vol, chunk=chunk)
    if xc == "blyp":
        from . import xc as OX
        vxc, exc, muxc, _ = OX.blyp_vxc(rho, dlay, vol)
    else:
        vxc, exc, muxc = OD.pz_lda(rho, vol)
    rg = OD.rho_to_g(rho, dlay, vol)
    vg, eh, ee, ew, floc = OD.hart_eext(rg, dlay.kx, dlay.ky, dlay.kz, sysm.box_len,
                                       0.5 * sysm.ecut_ry, sysm.atoms_dict(), sysm.tab,
                                       sysm.alp_ewd)
    vks = vxc + OD.vg_to_r(vg, dlay)
    fv = OF.vpsi_force(psi, vks, lay, occ, chunk=chunk)
    enl, fnl, fatm = 0.0, None, None
    if nonlocal_on:
        from . import ees as OE
        enl, fnl, fatm = OE.nonlocal_ees(psi, lay, occ, vol, sysm.hmati(),
                                         dict(pos=sysm.pos, typ=sysm.typ), sysm.channels,
                                         sysm.tab, nkf)
        floc = floc + fatm
    if nonlocal_sf:  # the structure-factor path (oracle/sf.py)
        from . import sf as OSF
        enl, fatm, fnl = OSF.sf_pass(psi, occ, sysm)
        floc = floc + fatm
    F = OF.add_forces(fv, fnl, lay)
    F, eke = OF.eke(F, psi, lay, occ, sysm.ecut_ry)
    en = dict(EXC=exc, MUXC=muxc, EHART=eh, EEXT=ee, EWD=ew, EKE=float(np.sum(eke)), ENL=enl)
    en["ETOT"] = en["EKE"] + enl + eh + ee + exc
    return en, F, floc, rho, vks


def cp_step(psi, v, occ, sysm, lay, dlay, cmass, dt, iteration, nonlocal_on=False, nkf=None,
            xc="pz_lda", nonlocal_sf=False, nhc=None):
    """nhc = (params, per-state chain states, nres, nyosh) of oracle/isokin.py
    runs the thermostatted integrator (the chain states are updated)."""
    en, F, floc, rho, vks = forces(psi, occ, sysm, lay, dlay, nonlocal_on=nonlocal_on, nkf=nkf,
                                   xc=xc, nonlocal_sf=nonlocal_sf)
    Fc, lam = constrain(F, psi, lay)
    if nhc is None:
        psi2, v2, ke = integrate(Fc, psi, v, cmass, lay, dt, iteration)
    else:
        from . import isokin as OK
        cls, ridx, rsrc = point_classes(lay)
        psi2, v2, ke, en["NHC_KE"], en["NHC_POT"] = OK.integrate_nhc(
            Fc, psi, v, cmass, cls, ridx, rsrc, nhc[0], nhc[1], dt, iteration, nhc[2], nhc[3])
    en["FICT"] = ke
    S = OO.pc_overlap(psi2, psi2, lay.kx)
    T, it, _ = OO.schulz_tmat(S)
    psi3 = OO.back_multiply(psi2, T)
    return psi3, v2, en, floc, dict(S=S, T=T, lam=lam, iters=it)
