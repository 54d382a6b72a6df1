"""Oracle: real-space ion-ion (Ewald) forces and the NVE atom integrator.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* CPRSPACEION::CP_getionforce  src_piny_physics_v1.0/abinito_physics/cp_ions/
  cp_rspace_ion.C:25-250 for a fully periodic cell (iperd = 3) without the
  Grimme term: every pair within half the shortest cell vector (minimum
  image through hmati / hmat, NINT rounding half away from zero) adds
  q_i q_j erfc(alp r) / r, with the reference's own erfc approximation (the
  9-term polynomial in tt = 1/(1 + p alp r) times e^{-(alp r)^2}, :40-48,
  :114-121), and its force; vself = -(sum q^2) alp/sqrt(pi) (1 - erfc(kcut /
  2 alp)) with kcut = sqrt(2 ecut), vbgr = -pi (sum q)^2 / (2 alp^2 vol)
  (:198-213).
* ATOMINTEGRATE::integrate_nve_2nd_half / integrate_nve_1st_half / computeEkin
  src_piny_physics_v1.0/classical_physics/integrate/integration_drivers.C:17-88,
  :337-355 (the NVE branch of ctrl_atom_integrate, control_integrate.C:22-200):
  v += dt/2 f/m (not on step 0), E_kin = 1/2 sum m v^2, then v += dt/2 f/m,
  x += dt v.
* ATOMINTEGRATE::integrate_nvt_2nd_half / _1st_half / applyNHC / computeENHC
  (integration_drivers.C:89-190, :358-565): the NVT branch with massive
  Nose-Hoover chains (one chain per atom and Cartesian component), pinned to
  the reference's integration_drivers.C compiled from source
  (oracle/ref_atomnhc.cpp).
"""
import math

import numpy as np

P = 0.3614
E = [0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
     0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
     0.06965131976970335]


def _poly(tt, c):
    acc = 0.0
    for e in reversed(c):
        acc = acc * tt + e
    return acc


def gerfc(x):
    """The reference's erfc(x) approximation (cp_rspace_ion.C:114-116)."""
    tt = 1.0 / (1.0 + P * x)
    return _poly(tt, E) * tt * np.exp(-x * x)


def _nint(x):
    return np.where(x >= 0.0, np.floor(x + 0.5), np.ceil(x - 0.5))


def ewald_rs(pos, q, hmat, hmati, vol, alp, ecut):
    """(pot_ewd_rs, vself, vbgr, forces [natm, 3]); hmat, hmati are 0-based
    column-major 3x3 (element (r, c) at [r + 3 c])."""
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    H = np.asarray(hmat, dtype=np.float64).reshape(3, 3).T     # H[r][c]
    Hi = np.asarray(hmati, dtype=np.float64).reshape(3, 3).T
    n = len(q)
    lens = np.sqrt(np.sum(H * H, axis=0))                      # cell vector lengths
    hmin = 0.5 * lens.min()
    de = [(k + 1) * e for k, e in enumerate(E)]
    f = np.zeros((n, 3))
    pot = 0.0
    for i in range(n - 1):
        d = pos[i] - pos[i + 1:]                               # [m, 3]
        s = d @ Hi.T
        s -= _nint(s)
        d = s @ H.T
        r2 = np.sum(d * d, axis=1)
        r = np.sqrt(r2)
        on = r <= hmin
        qij = q[i] * q[i + 1:]
        x = r * alp
        tt = 1.0 / (1.0 + P * x)
        eee = np.exp(-x * x)
        g = _poly(tt, E) * tt * eee
        dg = _poly(tt, de) * tt * tt * eee * P * alp + 2.0 * alp * alp * g * r
        vnow = np.where(on, qij * g / r, 0.0)
        dv = np.where(on, (g / r2 + dg / r) * qij / r, 0.0)
        pot += float(np.sum(vnow))
        fi = d * dv[:, None]
        f[i] += np.sum(fi, axis=0)
        f[i + 1:] -= fi
    vself = -(np.sum(q * q) * alp) / math.sqrt(math.pi)
    kcut = math.sqrt(2.0 * ecut)
    vself *= 1.0 - gerfc(kcut / (2.0 * alp))
    vbgr = -(0.5 * np.sum(q) ** 2 * math.pi) / (alp * alp * vol)
    return pot, vself, vbgr, f


def nve_step(itime, pos, vel, force, mass, dt):
    """(pos, vel, E_kin) after the NVE half steps of one MD step."""
    pos = np.array(pos, dtype=np.float64)
    vel = np.array(vel, dtype=np.float64)
    m = np.asarray(mass, dtype=np.float64)[:, None]
    f = np.asarray(force, dtype=np.float64)
    if itime > 0:
        vel += 0.5 * dt * f / m
    ekin = 0.5 * float(np.sum(m * vel * vel))
    vel += 0.5 * dt * f / m
    pos += dt * vel
    return pos, vel, ekin


def _yosh_w(nyosh, dt):
    from .isokin import yosh
    return yosh(nyosh, dt)


def apply_nhc(vel, mass, kT, mnhc, vn, pos_kt, dt, nres, nyosh):
    """ATOMINTEGRATE::applyNHC (integration_drivers.C:402-462) with massive
    chains: every Cartesian component of every atom has its own chain of
    length L = mnhc.shape[1]; vel [n, 3], vn [n, 3, L], pos_kt [n] updated
    in place.  kT [n], mnhc [n, L]."""
    n, L = mnhc.shape
    w = _yosh_w(nyosh, dt / nres)
    m = np.asarray(mass, dtype=np.float64)
    for i in range(n):
        mv2 = m[i] * vel[i] * vel[i]                       # [3]
        f = np.zeros((3, L))
        f[:, 0] = (mv2 - kT[i]) / mnhc[i, 0]
        for ic in range(1, L):
            f[:, ic] = (mnhc[i, ic - 1] * vn[i, :, ic - 1] ** 2 - kT[i]) / mnhc[i, ic]
        for _ in range(nres):
            for wy in w:
                w2, w4, w8 = wy * 0.5, wy * 0.25, wy * 0.125
                vn[i, :, L - 1] += f[:, L - 1] * w4
                for ic in range(L - 2, -1, -1):
                    aa = np.exp(-w8 * vn[i, :, ic + 1])
                    vn[i, :, ic] = vn[i, :, ic] * aa * aa + w4 * f[:, ic] * aa
                aa = np.exp(-w2 * vn[i, :, 0])
                vel[i] *= aa
                mv2 *= aa * aa
                pre = kT[i] * w2
                for ic in range(L):
                    pos_kt[i] += pre * (vn[i, 0, ic] + vn[i, 1, ic] + vn[i, 2, ic])
                f[:, 0] = (mv2 - kT[i]) / mnhc[i, 0]
                for ic in range(L - 1):
                    aa = np.exp(-w8 * vn[i, :, ic + 1])
                    vn[i, :, ic] = vn[i, :, ic] * aa * aa + w4 * f[:, ic] * aa
                    f[:, ic + 1] = (mnhc[i, ic] * vn[i, :, ic] ** 2 - kT[i]) / mnhc[i, ic + 1]
                vn[i, :, L - 1] += f[:, L - 1] * w4


def nvt_step(itime, pos, vel, force, mass, kT, mnhc, vn, pos_kt, dt, nres, nyosh):
    """integrate_nvt_2nd_half / computeEkin / computeENHC / integrate_nvt_1st_half
    (integration_drivers.C:89-190, :337-400): (pos, vel, E_kin, E_kin NHC,
    pot NHC); vn and pos_kt updated in place."""
    pos = np.array(pos, dtype=np.float64)
    vel = np.array(vel, dtype=np.float64)
    m = np.asarray(mass, dtype=np.float64)[:, None]
    f = np.asarray(force, dtype=np.float64)
    if itime > 0:
        vel += 0.5 * dt * f / m
        apply_nhc(vel, mass, kT, mnhc, vn, pos_kt, dt, nres, nyosh)
    ekin = 0.5 * float(np.sum(m * vel * vel))
    eknhc = 0.5 * float(np.sum(mnhc[:, None, :] * vn * vn))
    pot = float(np.sum(pos_kt))
    apply_nhc(vel, mass, kT, mnhc, vn, pos_kt, dt, nres, nyosh)
    vel += 0.5 * dt * f / m
    pos += dt * vel
    return pos, vel, ekin, eknhc, pot
