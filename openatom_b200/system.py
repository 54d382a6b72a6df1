"""Synthetic CP systems of the benchmark shapes (seeded, reproducible).

Coefficients: complex Gaussian x exp(-|G|^2/8) on the packed layout, with the
Gamma-point symmetry of the stored Gx=0 lower half (c(0,-ky,-kz) = conj
c(0,ky,kz), the relation flip_data_set builds, para_grp_parse.C:229-240) and a
real G=0 term, then Loewdin-orthonormalised to S = 2 I, the normalisation the
reference's Ortho expects (doc/orthoStoT.txt:9-20; cp_lowdin.C:197-199 halves S).
S_ij = sum_p wpt_p Re(conj c_i(p) c_j(p)), wpt = 1 on Gx=0 and 2 elsewhere, is
the overlap PairCalculator forms from the Gx=0-rescaled real view
(CP_State_GSpacePlane.C:3120-3123, ckPairCalculator.C:682-751).

The orthonormalisation runs in FP64 on the GPU with torch (input preparation,
not part of any measured path).
"""
import numpy as np
import torch


def kx0_partner(layout):
    """Index of the (0,-ky,-kz) partner of every Gx=0 point (-1 elsewhere)."""
    kx, ky, kz = layout.kx, layout.ky, layout.kz
    idx = np.full(layout.npts, -1, dtype=np.int64)
    sel = np.nonzero(kx == 0)[0]
    key = {(int(ky[i]), int(kz[i])): int(i) for i in sel}
    for i in sel:
        idx[i] = key[(-int(ky[i]), -int(kz[i]))]
    return idx


def overlap_weights(layout):
    return np.where(layout.kx == 0, 1.0, 2.0)


def make_psi(layout, nstates, seed=1234, device="cuda", orthonormalize=True):
    """[nstates, npts] complex128 coefficients on `device`."""
    rng = np.random.default_rng(seed)
    g2 = layout.g2()
    env = np.exp(-g2 / 8.0)
    re = rng.standard_normal((nstates, layout.npts))
    im = rng.standard_normal((nstates, layout.npts))
    c = (re + 1j * im) * env[None, :]
    part = kx0_partner(layout)
    sel = np.nonzero(part >= 0)[0]
    # make the Gx=0 plane Hermitian: keep the ky>0 or (ky=0,kz>=0) member, mirror it
    keep = sel[(layout.ky[sel] > 0) | ((layout.ky[sel] == 0) & (layout.kz[sel] >= 0))]
    c[:, part[keep]] = np.conj(c[:, keep])
    g0 = np.nonzero((layout.kx == 0) & (layout.ky == 0) & (layout.kz == 0))[0]
    c[:, g0] = c[:, g0].real
    psi = torch.from_numpy(c).to(device)
    if orthonormalize:
        psi = loewdin(psi, torch.from_numpy(overlap_weights(layout)).to(device))
    return psi


def overlap(psi, w):
    a = torch.view_as_real(psi)  # [S, npts, 2]
    aw = a * w[None, :, None].to(a.dtype)
    return torch.einsum("spc,tpc->st", aw, a)


def loewdin(psi, w):
    """psi <- (S/2)^(-1/2) psi so that the weighted overlap is 2 I (FP64)."""
    S = overlap(psi, w)
    evals, evecs = torch.linalg.eigh(S / 2.0)
    T = evecs @ torch.diag(evals.rsqrt()) @ evecs.T
    return (T.to(psi.dtype) @ psi).contiguous()


# ---------------------------------------------------------------------------
# atoms and local pseudopotentials

# Synthetic Gaussian pseudopotentials (Hartree atomic units):
#   v_loc(g) = -4 pi Z exp(-g^2 rc^2/4)/g^2 + c pi^1.5 b^3 exp(-g^2 b^2/4)
# i.e. the potential of a Gaussian ionic charge of width rc plus a short-range
# Gaussian c exp(-r^2/b^2).  The G=0 limit without the Coulomb term is
# gzvps = pi Z rc^2 + c pi^1.5 b^3.
SPECIES = {
    "O": dict(Z=6.0, rc=0.45, c=-2.5, b=0.55),
    "H": dict(Z=1.0, rc=0.25, c=-0.6, b=0.35),
}


def v_loc(sp, g):
    p = SPECIES[sp]
    g = np.asarray(g, dtype=np.float64)
    g2 = g * g
    with np.errstate(divide="ignore", invalid="ignore"):
        coul = np.where(g2 > 0, -4.0 * np.pi * p["Z"] * np.exp(-g2 * p["rc"] ** 2 / 4.0) / g2, 0.0)
    return coul + p["c"] * np.pi ** 1.5 * p["b"] ** 3 * np.exp(-g2 * p["b"] ** 2 / 4.0)


def gzvps(sp):
    p = SPECIES[sp]
    return np.pi * p["Z"] * p["rc"] ** 2 + p["c"] * np.pi ** 1.5 * p["b"] ** 3


def spline_tables(species, gmin, gmax, nspl=4000):
    """vps0..vps3 [ntyp, 4, nspl]: cubic coefficients of v_loc on g_i = gmin + i dg,
    the layout CP_get_vpsnow evaluates (cp_hart_ext.C:459-471)."""
    from scipy.interpolate import CubicSpline
    dg = (gmax - gmin) / (nspl - 1)
    g = gmin + dg * np.arange(nspl + 1)
    tab = np.zeros((len(species), 4, nspl))
    for t, sp in enumerate(species):
        cs = CubicSpline(g, v_loc(sp, g), bc_type="natural")
        # cs.c[k, i]: coefficient of (x - g_i)^(3-k) on interval i
        tab[t, 0] = cs.c[3, :nspl]
        tab[t, 1] = cs.c[2, :nspl]
        tab[t, 2] = cs.c[1, :nspl]
        tab[t, 3] = cs.c[0, :nspl]
    return dict(vps=tab, gmin=gmin, dg=dg, nspl=nspl,
                gzvps=np.array([gzvps(sp) for sp in species]),
                q=np.array([SPECIES[sp]["Z"] for sp in species]))


# Synthetic Kleinman-Bylander projectors, s and p, with Gaussian radials in g:
#   v_0(g) = A0 exp(-g^2 r0^2/4),   v_1(g) = A1 (g r1) exp(-g^2 r1^2/4)
# tabulated on the local tables' g grid; vnorm are the KB energies
# (cppseudo->vpsnorm) and gzvps0 = v_0(0), the G = 0 value of the s channel
# (eesProjGchare, cp_ees_nonlocal.C:663-673).
KB = {
    "O": dict(A0=6.0, r0=0.55, A1=3.0, r1=0.60, vn0=1.2, vn1=0.6),
    "H": dict(A0=1.5, r0=0.40, A1=0.6, r1=0.45, vn0=0.4, vn1=0.15),
}


def v_kb(sp, l, g):
    p = KB[sp]
    g = np.asarray(g, dtype=np.float64)
    if l == 0:
        return p["A0"] * np.exp(-g * g * p["r0"] ** 2 / 4.0)
    return p["A1"] * (g * p["r1"]) * np.exp(-g * g * p["r1"] ** 2 / 4.0)


def nonlocal_channels(species, gmin, dg, nspl):
    """EES channels (type, l, m) of every species, s then p (m = 0, 1, -1), each
    with its spline table [4][nspl] on g_i = gmin + i dg, vnorm and gzvps0."""
    from scipy.interpolate import CubicSpline
    g = gmin + dg * np.arange(nspl + 1)
    chans = []
    for t, sp in enumerate(species):
        for l, ms in ((0, (0,)), (1, (0, 1, -1))):
            cs = CubicSpline(g, v_kb(sp, l, g), bc_type="natural")
            tab = np.stack([cs.c[3, :nspl], cs.c[2, :nspl], cs.c[1, :nspl], cs.c[0, :nspl]])
            for m in ms:
                chans.append(dict(type=t, l=l, m=m, vnl=tab,
                                  gzvps0=float(v_kb(sp, 0, 0.0)) if l == 0 else 0.0,
                                  vnorm=KB[sp]["vn%d" % l]))
    return chans


def place_atoms(counts, box_len, seed=7, dmin=1.8, max_tries=200000):
    """Seeded uniform positions with a minimum (periodic) distance; returns
    (pos [natm, 3], typ [natm], species list)."""
    rng = np.random.default_rng(seed)
    species = list(counts.keys())
    pos, typ = [], []
    for t, sp in enumerate(species):
        for _ in range(counts[sp]):
            for _try in range(max_tries):
                x = rng.uniform(0.0, box_len, 3)
                ok = True
                for y in pos:
                    d = x - y
                    d -= box_len * np.round(d / box_len)
                    if d @ d < dmin * dmin:
                        ok = False
                        break
                if ok:
                    pos.append(x)
                    typ.append(t)
                    break
            else:
                raise RuntimeError("could not place atoms at the minimum distance")
    return np.array(pos), np.array(typ, dtype=np.int32), species


class System:
    """A synthetic water-like CP system of the benchmark shapes."""

    def __init__(self, box_len, ecut_ry, nstates, counts, nfft=None, seed=1234,
                 alp_ewd=3.5, nspl=4000):
        from .layout import StateLayout
        self.layout = StateLayout(box_len, ecut_ry, nfft=nfft)
        self.box_len = float(box_len)
        self.ecut_ry = float(ecut_ry)
        self.nstates = int(nstates)
        self.seed = seed
        self.pos, self.typ, self.species = place_atoms(counts, box_len, seed=seed + 1)
        self.natm = len(self.typ)
        tpi = 2.0 * np.pi / box_len
        gmax = np.sqrt(8.0 * 0.5 * ecut_ry) * 4.0 / 3.0 + tpi
        self.tab = spline_tables(self.species, 0.75 * tpi, gmax, nspl)
        self.alp_ewd = alp_ewd / box_len  # PINY divides the input alpha by the box side
        self.occ = np.ones(self.nstates)
        self.channels = nonlocal_channels(self.species, self.tab["gmin"], self.tab["dg"],
                                          self.tab["nspl"])

    def hmati(self):
        """Inverse cell matrix, column-major 3x3 flattened (cubic box)."""
        return (np.eye(3) / self.box_len).reshape(-1)

    def psi(self, device="cuda"):
        return make_psi(self.layout, self.nstates, seed=self.seed, device=device)

    def atoms_dict(self):
        return dict(pos=self.pos, typ=self.typ, q=self.tab["q"])
