"""Oracle: the structure-factor (non-EES) nonlocal pseudopotential, l = 0.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, for one Gamma-point double-packed system, the reference's "N^3"
nonlocal path (selected when ees_nloc_on = 0):

* CPNONLOCAL::CP_calc_Struct_Fact  src_piny_physics_v1.0/abinito_physics/
  cp_nonlocal/cp_struct_fact.C:33-221: per nonlocal atom a (types with an l = 0
  channel; the reference hard-wires l = 0) and packed point G,
      S_a(G)   = conj( w(G) e^{iG.R_a} ) y00 v_0(|G|)      (w = 1 on kx = 0, else 2)
      S_a^d(G) = conj( i G_d w(G) e^{iG.R_a} ) y00 v_0(|G|)
  with v_0 the type's l = 0 radial spline (get_rad_proj :225-258: the knot
  below g, cubic in h; gzvps0 at G = 0), y00 = 1/sqrt(4 pi);
* CP_enl_matrix_calc  cp_nlmat.C:20-92 (double pack): z_a = sum over the
  real view of psi . S_a, and z_a^d likewise (the DGEMV into the real parts);
* CP_enl_atm_forc_calc  cp_nl_energy_forc.C:121-182: E_NL = occ sum_a
  vnorm_a/vol z_a^2; z'_a = 2 vnorm_a/vol z_a; F_a^d -= z'_a z_a^d (the atom
  forces and the psi force carry no occupation factor, as in the reference);
* CP_enl_force_calc  cp_nl_energy_forc.C:29-114 (double pack): the real view
  of the psi force -= sum_a z'_a S_a.
"""
import math

import numpy as np


def spline_l0(g, tab_t, gz0, nspl, gmin, dg):
    """get_rad_proj (cp_struct_fact.C:225-258) of one type's l = 0 spline rows
    tab_t = (v0, v1, v2, v3) at |G| = g (array)."""
    g = np.asarray(g, dtype=np.float64)
    iii = ((g - gmin) / dg).astype(np.int64) + 1
    iii = np.clip(iii, 1, nspl)
    h = g - ((iii - 1) * dg + gmin)
    v0, v1, v2, v3 = (np.asarray(t)[iii - 1] for t in tab_t)
    v = ((v3 * h + v2) * h + v1) * h + v0
    return np.where(g != 0.0, v, gz0)


def struct_fact(kx, ky, kz, box_len, frac, proj):
    """S [natm_nl, npts] and S^d [3, natm_nl, npts] (complex) for atoms at
    fractional positions frac [natm_nl, 3] with per-atom projectors
    proj [natm_nl, npts] (y00 v_0(|G|)); cubic box."""
    tpi = 2.0 * math.pi
    k = np.stack([kx, ky, kz]).astype(np.float64)              # [3, npts]
    g = k * (tpi / box_len)
    w = np.where(np.asarray(kx) == 0, 1.0, 2.0)
    phase = np.exp(1j * tpi * (np.asarray(frac) @ k))          # e^{iG.R}, [natm, npts]
    s = np.conj(w * phase) * proj
    sd = np.stack([np.conj(1j * g[d] * w * phase) * proj for d in range(3)])
    return s, sd


def real_view(c):
    return np.ascontiguousarray(c).view(np.float64)


def sf_nonlocal(psi, occ, vol, s, sd, vnorm):
    """(E_NL, atom forces [natm_nl, 3], psi force [S, npts]) of the l = 0
    structure-factor path for states psi [S, npts] (complex)."""
    pr = real_view(psi)                                        # [S, 2 npts]
    z = real_view(s) @ pr.T                                    # [natm, S]
    zd = np.stack([real_view(sd[d]) @ pr.T for d in range(3)])  # [3, natm, S]
    norm = np.asarray(vnorm, dtype=np.float64)[:, None] / vol
    enl = float(np.sum(np.asarray(occ)[None, :] * z * z * norm))
    zs = 2.0 * norm * z                                        # [natm, S]
    f = -np.stack([np.sum(zs * zd[d], axis=1) for d in range(3)], axis=1)
    fpsi_r = -(zs.T @ real_view(s))                            # [S, 2 npts]
    return enl, f, fpsi_r.view(np.complex128)


def system_tables(sysm):
    """(order, proj [natm_nl, npts], vnorm [natm_nl]) for a System's l = 0
    channels: the non-local atoms in type order (the reference's map_nl) with
    y00 v_0(|G|) of their type on the state layout."""
    lay = sysm.layout
    tab = sysm.tab
    ch0 = {c["type"]: c for c in sysm.channels if c["l"] == 0}
    order = np.array([i for i in np.argsort(sysm.typ, kind="stable") if sysm.typ[i] in ch0])
    tpi = 2.0 * math.pi / sysm.box_len
    g = np.sqrt((lay.kx * tpi) ** 2 + (lay.ky * tpi) ** 2 + (lay.kz * tpi) ** 2)
    y00 = 1.0 / math.sqrt(4.0 * math.pi)
    proj = np.stack([y00 * spline_l0(g, ch0[sysm.typ[i]]["vnl"], ch0[sysm.typ[i]]["gzvps0"],
                                     tab["nspl"], tab["gmin"], tab["dg"]) for i in order])
    vn0 = np.array([ch0[sysm.typ[i]]["vnorm"] for i in order])
    return order, proj, vn0


def sf_pass(psi, occ, sysm):
    """The whole pass for a System: (E_NL, atom forces [natm, 3] in atom order,
    psi force [S, npts])."""
    lay = sysm.layout
    order, proj, vn0 = system_tables(sysm)
    s, sd = struct_fact(lay.kx, lay.ky, lay.kz, sysm.box_len, sysm.pos[order] / sysm.box_len,
                        proj)
    enl, f, fpsi = sf_nonlocal(psi, occ, sysm.box_len ** 3, s, sd, vn0)
    fa = np.zeros((sysm.natm, 3))
    fa[order] = f
    return enl, fa, fpsi
