"""Oracle: one CP electronic step in FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Forces on the orthonormal coefficients psi_o (the same for both forms):
  rho (fftpath.density) -> V_KS = v_xc + Hartree/local (density.py)
  F = addForces(-2/N FFT^-1[V psi]) - kinetic term          (fftpath.py)
  lambda(j,i) = sum_p Re(conj psi_j F_i): the asymmetric PairCalculator,
      which runs without the double-pack factor (cpaimd.C:2527
      isDoublePackOn = 0 -> alpha = 1 in multiplyForward,
      ckPairCalculator.C:733-736); the 1/sqrt(2) and sqrt(2) scalings of psi
      and F on Gx=0 (CP_State_GSpacePlane.C:1933-1954) cancel in the product.

form "ortho_t" -- the reference's CP dynamics (cp_min_opt = 0), the default:
  gamma = orthoT . lambda                  Ortho::acceptSectionLambda, ortho.C:541-583
      (orthoT = T of the previous step's Ortho, ortho.C:358-365; the identity
      after a norb-tolerance reset, ortho.C:545-562)
  F_c = F . orthoT - W (psi_o . gamma)     bwMultiplyDynOrthoT (-F.T), ckPairCalculator.C:1444-1510,
                                           and the gamma GEMM of bwMultiplyHelper (:1372-1420);
                                           the sum negated by unpackLambda (CP_State_GSpacePlane.C:2197-2202)
                                           and scaled 1/sqrt(2) on Gx=0 by doLambda (:2253-2259),
                                           so W = 1/2 on Gx=0 and 1 elsewhere
  the non-orthogonal coefficients psi_no come back (doLambda :2262-2268) and
  are integrated (integrateModForce, :2582-2854): velocity Verlet of
  CP_integrate_dyn / cp_evolve_vel / get_fictKE (cp_dynamics.C:29-258),
  the second half kick skipped after a reset (halfStepEvolve = 0,
  cp_dynamics.C:58), redundant-half sync (:2862-3061)
  psi_no is saved (sendPsi :3090-3094); S = overlap(psi_no) (alpha = 2,
  Gx=0 scaled 1/sqrt(2)); max |S - 2I| >= cp_norb_tol (default 0.003,
  set_sim_dict.C:1161-1162) fails the check of Ortho::start_calc/maxCheck
  (ortho.C:255-262, :461-483, array_diag_max ortho.h:282-310): fatal on the
  first step, otherwise the finite-difference PsiV reset after the new psi
  (finiteDifferencePsiV, CP_State_GSpacePlane.C:3707-3770, order 0 as the
  default norb_fin_diff_order, set_sim_dict.C:1244-1247): psi_no <- psi_o(t+dt),
  v = (psi_o(t+dt) - psi_o(t)) / dt, orthoT <- I, next integrate without
  the second half kick
  T = Schulz (S/2)^-1/2 (ortho.py); psi_o = psi_no T  (bwMultiplyHelper 'N','N', :1314)

form "lowdin" -- the projection form kept as an option:
  F_i <- F_i - W sum_j psi_j lambda(j,i) (the constraint of minimisation,
  CP_State_GSpacePlane.C:2079-2088), Verlet on psi_o itself, S, T, psi <- psi T.
  At T = I both forms give the same first step.
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


def constrain_dyn(F, psi_o, T, lay):
    """The reference's dynamics constraint: gamma = T lambda and
    F_c = F.T - W (psi_o.gamma), states as rows: F_c[a] = sum_k T[k,a] F[k]
    - W sum_b gamma[b,a] psi_o[b].  Returns (F_c, lambda, gamma)."""
    lam = OO.real_view(psi_o) @ OO.real_view(F).T        # lam[j, i] = <psi_j|F_i>
    gam = T @ lam
    w = np.where(lay.kx == 0, 0.5, 1.0)
    return T.T @ F - w[None] * (gam.T @ psi_o), lam, gam


def norb_deviation(S):
    """max |S - 2I| over all elements (array_diag_max with diag = 2, spin-unpolarised)."""
    return float(np.max(np.abs(S - 2.0 * np.eye(S.shape[0]))))


def dyn_start(psi):
    """State of the reference form before its first step: the non-orthogonal
    coefficients are the given (orthonormal) ones and orthoT is the identity."""
    return dict(psi_no=np.array(psi, dtype=np.complex128), T=np.eye(psi.shape[0]),
                half_reset=False, resets=0, dev=0.0)


def forces(psi, occ, sysm, lay, dlay, chunk=16, nonlocal_on=False, nkf=None, xc="pz_lda",
           nonlocal_sf=False, eext_ees=None):
    """Energies, V_KS, constrained-force input F and atom forces (local + Ewald,
    plus the EES non-local pass when nonlocal_on: addForces adds its psi force,
    stateSlab.C:240-272).  xc = "blyp" takes the BLYP potential of oracle/xc.py.
    eext_ees = the EES grid size runs the local pass in its EES form
    (oracle/eext_ees.py, cp_eext_ees_opt)."""
    vol = sysm.box_len ** 3
    rho = OF.density(psi, lay, occ, vol, chunk=chunk)
    if xc == "blyp":
        from . import xc as OX
        vxc, exc, muxc, _ = OX.blyp_vxc(rho, dlay, vol)
    else:
        vxc, exc, muxc = OD.pz_lda(rho, vol)
    rg = OD.rho_to_g(rho, dlay, vol)
    if eext_ees:
        from . import eext_ees as OXE
        vg, eh, ee, ew, floc = OXE.hart_eext_ees(rg, dlay.kx, dlay.ky, dlay.kz, sysm.box_len,
                                                 0.5 * sysm.ecut_ry, sysm.atoms_dict(),
                                                 sysm.tab, sysm.alp_ewd, eext_ees)
    else:
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
            xc="pz_lda", nonlocal_sf=False, nhc=None, form="ortho_t", dyn=None, tol_norb=0.003,
            eext_ees=None):
    """One step on the orthonormal coefficients psi.  nhc = (params, per-state
    chain states, nres, nyosh) of oracle/isokin.py runs the thermostatted
    integrator (the chain states are updated).  form "ortho_t" carries the
    reference's dynamical state in ``dyn`` (dyn_start(psi) on iteration 1 when
    None; the updated dict is aux["dyn"]); form "lowdin" needs none.
    Returns (psi, v, energies, atom forces, aux)."""
    en, F, floc, rho, vks = forces(psi, occ, sysm, lay, dlay, nonlocal_on=nonlocal_on, nkf=nkf,
                                   xc=xc, nonlocal_sf=nonlocal_sf, eext_ees=eext_ees)
    if form == "lowdin":
        Fc, lam = constrain(F, psi, lay)
        x, it_eff, gam = psi, iteration, None
    elif form == "ortho_t":
        if dyn is None:
            if iteration != 1:
                raise ValueError("form ortho_t: iteration > 1 needs the state of the last step")
            dyn = dyn_start(psi)
        Fc, lam, gam = constrain_dyn(F, psi, dyn["T"], lay)
        x = dyn["psi_no"]
        it_eff = 1 if dyn["half_reset"] else iteration
    else:
        raise ValueError("form must be ortho_t or lowdin")
    if nhc is None:
        psi2, v2, ke = integrate(Fc, x, v, cmass, lay, dt, it_eff)
    else:
        from . import isokin as OK
        cls, ridx, rsrc = point_classes(lay)
        psi2, v2, ke, en["NHC_KE"], en["NHC_POT"] = OK.integrate_nhc(
            Fc, x, v, cmass, cls, ridx, rsrc, nhc[0], nhc[1], dt, it_eff, nhc[2], nhc[3])
    en["FICT"] = ke
    S = OO.pc_overlap(psi2, psi2, lay.kx)
    aux = dict(S=S, lam=lam, gamma=gam)
    if form == "ortho_t":
        dev = norb_deviation(S)
        fail = dev >= tol_norb
        if fail and iteration == 1:
            raise RuntimeError("S fails the norb tolerance on the first step: max|S-2I| = %g" % dev)
    T, it, _ = OO.schulz_tmat(S)
    psi3 = OO.back_multiply(psi2, T)
    aux.update(T=T, iters=it)
    if form == "ortho_t":
        nd = dict(psi_no=psi2, T=T, half_reset=False, resets=dyn["resets"], dev=dev)
        if fail:   # finiteDifferencePsiV, order 0
            v2 = (psi3 - psi) / dt
            nd.update(psi_no=psi3.copy(), T=np.eye(S.shape[0]), half_reset=True,
                      resets=dyn["resets"] + 1)
        aux["dyn"] = nd
    return psi3, v2, en, floc, aux
