"""Oracle: the CP velocity Verlet with isokinetic Nose-Hoover chains (ISOKIN_OPT = 1).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates for one chunk set of coefficients (one state here, as one G-space
chare holds it in the reference):

* CPINTEGRATE::initCPNHC  src_piny_physics_v1.0/abinito_physics/cp_integrate/
  cp_isokin.C:31-117: kT = te_ext/BOLTZ, tau = tau_fs/TIME_CONV, chain masses
  mNHC = (tau^2 kT degfree/nck, 2.5 tau^2 kT), double-well parameters v0, a2,
  a4 per chain, nck chunks of the non-redundant coefficients (div/rem split),
  degFreeSplt = 2 n (minus the G = 0 count on chunk 0);
* CPINTEGRATE::cp_isoNHC_update  cp_isokin.C:120-311: per chunk, Yoshida-Suzuki
  (nyosh weights, set_yosh :326-388) times RESPA (nresp) steps of the chains,
  the coefficient velocities scaled, the constraint re-imposed exactly;
* CPINTEGRATE::CP_integrate_dyn / cp_evolve_vel / get_fictKE  cp_dynamics.C:22-256:
  applyorder 2 (finish the previous step: kick, then thermostat) when
  iteration > 1, the fictitious KE, applyorder 1 (thermostat, then kick), the
  drift; during the velocity updates Gx=0 forces and masses are doubled and
  the G = 0 imaginary parts zeroed.

Pinned to the reference's own cp_isokin.C / cp_dynamics.C compiled from source
(oracle/ref_isokin.cpp, tests/test_isokin_oracle.py).
"""
import math

import numpy as np

BOLTZ = 315777.0       # piny_constants.h:52
TIME_CONV = 0.0241888  # piny_constants.h:58


def yosh(nyosh, dt):
    """set_yosh (cp_isokin.C:326-388): weights times dt, index 1..nyosh."""
    w = {1: [1.0]}
    t = 2.0 ** (1.0 / 3.0)
    w[3] = [1.0 / (2.0 - t), -t / (2.0 - t), 1.0 / (2.0 - t)]
    t4 = 4.0 ** (1.0 / 3.0)
    p2 = 1.0 / (4.0 - t4)
    w[5] = [p2, p2, 1.0 - 4.0 * p2, p2, p2]
    a, b, c = 0.784513610477560, 0.235573213359357, -1.17767998417887
    w[7] = [a, b, c, 1.0 - 2.0 * (a + b + c), c, b, a]
    q = [0.192, 0.554910818409783619692725006662999, 0.124659619941888644216504240951585,
         -0.843182063596933505315033808282941]
    w[9] = q + [1.0 - 2.0 * sum(q)] + q[::-1]
    return np.array(w[nyosh]) * dt


def init_nhc(ncoef, nzero, num, nck, te_ext, tau_fs):
    """initCPNHC (cp_isokin.C:31-117)."""
    kT = te_ext / BOLTZ
    tau = tau_fs / TIME_CONV
    degfree = float(2 * ncoef - nzero)
    pre = tau * tau * kT
    m = np.array([pre * degfree / nck, 2.5 * pre])
    r2 = float(num + 5)
    frac = np.array([(num + i + 5) / r2 for i in range(num)])
    v0 = 0.8 * kT * frac
    a2 = 1.6 * (0.8 * frac)
    a4 = a2 * a2
    div, rem = ncoef // nck, ncoef % nck
    istr, iend, dfs = [], [], []
    for k in range(nck):
        nstr = div * k + (rem if k >= rem else k)
        nnow = div + (1 if k < rem else 0)
        istr.append(nstr)
        iend.append(nstr + nnow)
        dfs.append(2.0 * nnow)
    dfs[0] -= nzero
    return dict(kT=kT, m=m, v0=v0, a2=a2, a4=a4, istr=istr, iend=iend, dfs=np.array(dfs),
                num=num, nck=nck)


def _hh(f, v, m, kT, w4):
    ffdot = (f[0] * f[0] * m[0] + f[1] * f[1] * m[1]) / kT
    pfdot = (f[0] * v[0] * m[0] + f[1] * v[1] * m[1]) / kT
    if ffdot * w4 * w4 > 1.0e-10:
        fr = math.sqrt(ffdot)
        arg = fr * w4
        ch, sh = math.cosh(arg), math.sinh(arg)
        h = (pfdot / ffdot) * (ch - 1.0) + (1.0 / fr) * sh
        hdot = (pfdot / fr) * sh + ch
    else:
        h = (((ffdot * pfdot / 24.0 * w4 + ffdot / 6.0) * w4 + 0.50 * pfdot) * w4 + 1.0) * w4
        hdot = ((ffdot * pfdot / 6.0 * w4 + ffdot / 2.0) * w4 + pfdot) * w4 + 1.0
    return h, hdot


def iso_update(v, m, p, st, dt, nresp, nyosh):
    """cp_isoNHC_update (cp_isokin.C:120-311) on the non-redundant velocities v
    (complex, with the doubled masses m); st = dict(x [nck,num,2], xp [nck,num,2],
    vn [nck,num,2]) updated in place; v scaled in place."""
    kT, mN = p["kT"], p["m"]
    w = yosh(nyosh, dt / nresp)
    for k in range(p["nck"]):
        sl = slice(p["istr"][k], p["iend"][k])
        gkt = p["dfs"][k] * kT
        ekin = float(np.sum(m[sl] * (v[sl].real ** 2 + v[sl].imag ** 2)))
        st["xp"][k, :, 0] = 0.0
        f = np.zeros((p["num"], 2))
        for i in range(p["num"]):
            f[i, 0] = (ekin - gkt) / mN[0]
            xp = st["xp"][k, i, 1]
            f[i, 1] = -(4.0 * p["v0"][i] / (p["a4"][i] * mN[1])) * (xp * (xp * xp - p["a2"][i]))
        scale = 1.0
        for _ in range(nresp):
            for iy in range(nyosh):
                w2, w4 = w[iy] * 0.5, w[iy] * 0.25
                vsum = 0.0
                for i in range(p["num"]):
                    h, hd = _hh(f[i], st["vn"][k, i], mN, kT, w4)
                    st["vn"][k, i, 0] = (st["vn"][k, i, 0] + f[i, 0] * h) / hd
                    st["vn"][k, i, 1] = (st["vn"][k, i, 1] + f[i, 1] * h) / hd
                    vsum += st["vn"][k, i, 0]
                aa = math.exp(-w4 * vsum)
                scale *= aa
                ekin *= aa * aa
                for i in range(p["num"]):
                    st["x"][k, i, 0] += kT * st["vn"][k, i, 0] * w2
                    st["x"][k, i, 1] += st["vn"][k, i, 0] * (ekin - gkt) * w2
                    st["xp"][k, i, 1] += st["vn"][k, i, 1] * w2
                scale *= aa
                ekin *= aa * aa
                for i in range(p["num"]):
                    f[i, 0] = (ekin - gkt) / mN[0]
                    xp = st["xp"][k, i, 1]
                    f[i, 1] = -(4.0 * p["v0"][i] / (p["a4"][i] * mN[1])) * (xp * (xp * xp - p["a2"][i]))
                for i in range(p["num"]):
                    h, hd = _hh(f[i], st["vn"][k, i], mN, kT, w4)
                    st["vn"][k, i, 0] = (st["vn"][k, i, 0] + f[i, 0] * h) / hd
                    st["vn"][k, i, 1] = (st["vn"][k, i, 1] + f[i, 1] * h) / hd
        v[sl] *= scale
        for i in range(p["num"]):
            en = mN[0] * st["vn"][k, i, 0] ** 2 + mN[1] * st["vn"][k, i, 1] ** 2
            st["vn"][k, i] *= math.sqrt(kT / en)


def default_state(p):
    """x = 0, v_NHC = (sqrt(kT/m0), 0): the isokinetic constraint holds."""
    nck, num = p["nck"], p["num"]
    vn = np.zeros((nck, num, 2))
    vn[:, :, 0] = math.sqrt(p["kT"] / p["m"][0])
    return dict(x=np.zeros((nck, num, 2)), xp=np.zeros((nck, num, 2)), vn=vn)


def sample_state(p, rng):
    """cpSamplNHC (cp_vel_sampl.C:118-196) with numpy normals in place of the
    reference's gaussran: v_j ~ N(0, kT/m_j), xp ~ N(0, a2), x = 0, each chain
    pair rescaled onto m0 v0^2 + m1 v1^2 = kT."""
    nck, num = p["nck"], p["num"]
    vn = rng.standard_normal((nck, num, 2)) * np.sqrt(p["kT"] / p["m"])[None, None, :]
    xp = rng.standard_normal((nck, num, 2)) * np.sqrt(p["a2"])[None, :, None]
    en = p["m"][0] * vn[..., 0] ** 2 + p["m"][1] * vn[..., 1] ** 2
    vn *= np.sqrt(p["kT"] / en)[..., None]
    return dict(x=np.zeros((nck, num, 2)), xp=xp, vn=vn)


def nhc_energies(p, st):
    """The NHC part of get_fictKE (cp_dynamics.C:231-240): (ekeNhc, potNHC)."""
    ek = 0.5 * float(np.sum(p["m"][None, None, :] * st["vn"] ** 2))
    return ek, float(np.sum(st["x"]))


def integrate_dyn_chare(psi, v, f, cmass, nzero, nuni, p, st, dt, iteration, nresp, nyosh):
    """CP_integrate_dyn (cp_dynamics.C:22-80) on one chare's non-redundant
    coefficients in the reference's order: G = 0 ([0, nzero)), the unique
    Gx = 0 points ([nzero, nuni)), the rest.  Returns (psi, v, fictitious KE,
    ekeNhc, potNHC) -- psi and v new arrays, st updated in place."""
    psi = np.array(psi, dtype=np.complex128)
    vv = np.array(v, dtype=np.complex128)
    ff = np.array(f, dtype=np.complex128)
    m = np.array(cmass, dtype=np.float64)
    g0 = slice(0, nzero)
    ux = slice(nzero, nuni)
    m2 = m.copy()
    m2[ux] *= 2.0

    def evolve(order):               # cp_evolve_vel (cp_dynamics.C:95-213)
        ff[g0] = ff[g0].real
        vv[g0] = vv[g0].real
        f2 = ff.copy()
        f2[ux] *= 2.0
        if order == 1:
            iso_update(vv, m2, p, st, dt, nresp, nyosh)
        vv[:] += f2 * (0.5 * dt / m2)
        if order == 2:
            iso_update(vv, m2, p, st, dt, nresp, nyosh)
        vv[g0] = vv[g0].real
    if iteration > 1:
        evolve(2)
    ke = 0.5 * float(np.sum(m2 * (vv.real ** 2 + vv.imag ** 2)))
    ekn, pot = nhc_energies(p, st)
    evolve(1)
    psi += vv * dt
    return psi, vv, ke, ekn, pot


def chare_order(cls):
    """Packed indices of one state's non-redundant points in the reference's
    chare order: G = 0 (class 1), the unique Gx = 0 points (class 2), the rest
    (class 3), each in packed order; and (nzero, nuni)."""
    cls = np.asarray(cls)
    o1, o2, o3 = (np.nonzero(cls == c)[0] for c in (1, 2, 3))
    return np.concatenate([o1, o2, o3]), len(o1), len(o1) + len(o2)


def integrate_nhc(F, psi, v, cmass, cls, ridx, rsrc, p, states, dt, iteration, nresp, nyosh):
    """The thermostatted Verlet step of every state (one chare per state, as
    the reference with one G-space chare per state): psi, v, F [S, npts];
    states a list of per-state chain dicts (updated).  Returns (psi, v,
    fictitious KE, ekeNhc, potNHC), the sums over states, after the redundant
    half is mirrored."""
    order, nzero, nuni = chare_order(cls)
    psi = np.array(psi, dtype=np.complex128)
    v = np.array(v, dtype=np.complex128)
    ke = ekn = pot = 0.0
    for s in range(psi.shape[0]):
        ps, vs, k, e1, e2 = integrate_dyn_chare(psi[s, order], v[s, order], F[s, order],
                                                np.asarray(cmass)[order], nzero, nuni, p,
                                                states[s], dt, iteration, nresp, nyosh)
        psi[s, order] = ps
        v[s, order] = vs
        ke += k
        ekn += e1
        pot += e2
    psi[:, ridx] = np.conj(psi[:, rsrc])
    v[:, ridx] = np.conj(v[:, rsrc])
    return psi, v, ke, ekn, pot
