"""The benchmark's synthetic CP systems, built with the oracle alone.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  The timed CPU
baseline (``bench.py --impl reference``) builds its inputs here so that it
neither imports the product package nor loads its library.  The definition
is the same as the product's input generator; tests/test_synth_oracle.py
checks that both produce the same system.

* G layout: oracle.layout.Layout (pinned bit-exact to the reference's own
  flip_data_set / get_chareG_line_prms / sort_commence).
* Coefficients: complex Gaussian x exp(-|G|^2/8) (numpy seeded generator),
  the stored Gx=0 lower half the conjugate of its partner
  (para_grp_parse.C:229-240), G=0 real, Loewdin-normalised to S = 2 I
  (doc/orthoStoT.txt:9-20) with the overlap weights 1 on Gx=0, 2 elsewhere.
* Atoms: seeded uniform positions at least 1.8 bohr apart (periodic).
* Local pseudopotentials: the Gaussian ionic charge of width rc plus a
  short-range Gaussian c exp(-r^2/b^2), tabulated as cubic splines on
  g_i = gmin + i dg in CP_get_vpsnow's layout (cp_hart_ext.C:459-471).
* Kleinman-Bylander s and p projectors with Gaussian radials, tabulated on the
  same grid, with their KB energies (vnorm) and the G=0 value of the s
  channel (eesProjGchare, cp_ees_nonlocal.C:663-673).
"""
import numpy as np

from . import layout as OL

SPECIES = {
    "O": dict(Z=6.0, rc=0.45, c=-2.5, b=0.55),
    "H": dict(Z=1.0, rc=0.25, c=-0.6, b=0.35),
}
KB = {
    "O": dict(A0=6.0, r0=0.55, A1=3.0, r1=0.60, vn0=1.2, vn1=0.6),
    "H": dict(A0=1.5, r0=0.40, A1=0.6, r1=0.45, vn0=0.4, vn1=0.15),
}


def v_loc(sp, g):
    p = SPECIES[sp]
    g2 = np.asarray(g, dtype=np.float64) ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        coul = np.where(g2 > 0, -4.0 * np.pi * p["Z"] * np.exp(-g2 * p["rc"] ** 2 / 4.0) / g2,
                        0.0)
    return coul + p["c"] * np.pi ** 1.5 * p["b"] ** 3 * np.exp(-g2 * p["b"] ** 2 / 4.0)


def v_kb(sp, l, g):
    p = KB[sp]
    g = np.asarray(g, dtype=np.float64)
    if l == 0:
        return p["A0"] * np.exp(-g * g * p["r0"] ** 2 / 4.0)
    return p["A1"] * (g * p["r1"]) * np.exp(-g * g * p["r1"] ** 2 / 4.0)


def _spline_rows(values_on_grid, nspl):
    """Cubic coefficients (v0, v1, v2, v3) per interval of a natural spline."""
    from scipy.interpolate import CubicSpline
    g, v = values_on_grid
    cs = CubicSpline(g, v, bc_type="natural")
    return np.stack([cs.c[3, :nspl], cs.c[2, :nspl], cs.c[1, :nspl], cs.c[0, :nspl]])


def place_atoms(counts, box_len, seed, dmin=1.8, max_tries=200000):
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


def make_psi(lay, nstates, seed):
    """[nstates, npts] complex128, S = 2 I with the Gx=0 weights (numpy FP64)."""
    rng = np.random.default_rng(seed)
    env = np.exp(-lay.g2 / 8.0)
    re = rng.standard_normal((nstates, lay.npts))
    im = rng.standard_normal((nstates, lay.npts))
    c = (re + 1j * im) * env[None, :]
    kx, ky, kz = lay.kx, lay.ky, lay.kz
    sel = np.nonzero(kx == 0)[0]
    key = {(int(ky[i]), int(kz[i])): int(i) for i in sel}
    keep = sel[(ky[sel] > 0) | ((ky[sel] == 0) & (kz[sel] >= 0))]
    part = np.array([key[(-int(ky[i]), -int(kz[i]))] for i in keep], dtype=np.int64)
    c[:, part] = np.conj(c[:, keep])
    g0 = np.nonzero((kx == 0) & (ky == 0) & (kz == 0))[0]
    c[:, g0] = c[:, g0].real
    w = np.where(kx == 0, 1.0, 2.0)
    a = np.stack([c.real, c.imag], axis=-1)
    S = np.einsum("spc,tpc->st", a * w[None, :, None], a)
    ev, V = np.linalg.eigh(S / 2.0)
    T = V @ np.diag(1.0 / np.sqrt(ev)) @ V.T
    return T @ c


class System:
    """The synthetic water-like CP system (same fields as the product's)."""

    def __init__(self, box_len, ecut_ry, nstates, counts, nfft=None, seed=1234, alp_ewd=3.5,
                 nspl=4000):
        self.layout = OL.Layout(box_len, ecut_ry, grid=nfft)
        self.box_len = float(box_len)
        self.ecut_ry = float(ecut_ry)
        self.nstates = int(nstates)
        self.seed = seed
        self.pos, self.typ, self.species = place_atoms(counts, box_len, seed=seed + 1)
        self.natm = len(self.typ)
        tpi = 2.0 * np.pi / box_len
        gmax = np.sqrt(8.0 * 0.5 * ecut_ry) * 4.0 / 3.0 + tpi
        gmin = 0.75 * tpi
        dg = (gmax - gmin) / (nspl - 1)
        g = gmin + dg * np.arange(nspl + 1)
        vps = np.stack([_spline_rows((g, v_loc(sp, g)), nspl) for sp in self.species])
        gz = [np.pi * SPECIES[sp]["Z"] * SPECIES[sp]["rc"] ** 2
              + SPECIES[sp]["c"] * np.pi ** 1.5 * SPECIES[sp]["b"] ** 3 for sp in self.species]
        self.tab = dict(vps=vps, gmin=gmin, dg=dg, nspl=nspl, gzvps=np.array(gz),
                        q=np.array([SPECIES[sp]["Z"] for sp in self.species]))
        self.alp_ewd = alp_ewd / box_len   # PINY divides the input alpha by the box side
        self.occ = np.ones(self.nstates)
        self.channels = []
        for t, sp in enumerate(self.species):
            for l, ms in ((0, (0,)), (1, (0, 1, -1))):
                tab = _spline_rows((g, v_kb(sp, l, g)), nspl)
                for m in ms:
                    self.channels.append(dict(type=t, l=l, m=m, vnl=tab,
                                              gzvps0=float(v_kb(sp, 0, 0.0)) if l == 0 else 0.0,
                                              vnorm=KB[sp]["vn%d" % l]))

    def hmati(self):
        """Inverse cell matrix, column-major 3x3 flattened (cubic box)."""
        return (np.eye(3) / self.box_len).reshape(-1)

    def psi(self):
        return make_psi(self.layout, self.nstates, self.seed)

    def atoms_dict(self):
        return dict(pos=self.pos, typ=self.typ, q=self.tab["q"])
