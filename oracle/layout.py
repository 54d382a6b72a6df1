"""Oracle: the reference's packed G-vector layout (Gamma point, double pack).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, step by step:

* ``calc_cutoff``            src_piny_physics_v1.0/interface/cp_ewald/set_cp_ewald.C:124-225
* ``radixme`` + fft table    set_cp_ewald.C:751-818, set_fftsizes set_cp_ewald.C:1505-1690
* ``setkvec3d_sm``           set_cp_ewald.C:523-680 (G=0 appended last, :674-677)
* ``flip_data_set``          src_charm_driver/utility/para_grp_parse.C:178-286
* ``processState``           src_charm_driver/utility/util.C:1331-1642
  (round-robin line deal :1433-1458, ``get_chareG_line_prms``
  para_grp_parse.C:21-170, per-chunk ``sort_kxky`` util.C:2223-2247)
* ``readStateIntoRuns``      util.C:861-1099 (two RunDescriptors per z-line)
* ``nkx0`` ranges            the Gx=0 points that ``CP_eke_calc`` (cp_eke.C:77-91)
  and ``GStateSlab::addForces`` (stateSlab.C:252-268) weight by 1 instead of 2.
"""
import math
import numpy as np

# set_fftsizes (set_cp_ewald.C:1505-1690): the allowed FFT sizes, in the order the
# reference lists them (note 112 twice and no 100, as in the reference table).
FFT_SIZES = [
    4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24, 28, 30, 32, 36, 40, 42, 44, 48, 56, 60,
    64, 66, 70, 72, 80, 84, 88, 90, 96, 112, 112, 120, 128, 128, 132, 140, 144, 154,
    160, 168, 176, 180, 192, 198, 210, 220, 224, 240, 252, 256, 264, 280, 288, 308,
    320, 330, 336, 352, 360, 384, 396, 420, 440, 448, 462, 480, 504, 512, 528, 560,
    576, 616, 630, 640, 660, 672, 704, 720, 768, 770, 792, 840, 880, 896, 924, 960,
    990, 1008, 1024]


def calc_kmax(box_len, ecut_ry):
    """kmax_cp of ``calc_cutoff`` (set_cp_ewald.C:190-215) for a cubic box.

    The reference halves the CP cutoff (Ry -> Ha, :171) and then uses
    temp = sqrt(ecut/2)/(pi*|hmati column|); a fractional part > 0.99 rounds up.
    """
    ecut_ha = 0.5 * ecut_ry
    tryv = 1.0 / box_len
    temp = math.sqrt(ecut_ha * 0.5) / (math.pi * tryv)
    it = int(temp)
    if temp - it > 0.99:
        it += 1
    return it


def radix_size(kmax):
    """``radixme`` (set_cp_ewald.C:751-818): smallest table size >= 2*(2*kmax+1)."""
    kk = 2 * (2 * kmax + 1)
    for k in FFT_SIZES:
        if k >= kk:
            return k
    raise ValueError("Bad Radix")


def setkvec3d_sm(ecut_ha, kmax, box_len):
    """Half-sphere k-vectors, ka>=0 then kb then kc ascending (set_cp_ewald.C:523-677).

    ``ecut_ha`` is the Hartree cutoff (|G|^2/2 <= ecut).  Returns int arrays of
    length nktot+1, G=(0,0,0) appended last as the reference does (:674-677).
    The cubic cell makes hmati diagonal (1/L); the loop bounds follow the
    reference's search for kbmin/kbmax/kcmin/kcmax.
    """
    h = 1.0 / box_len
    tpi = 2.0 * math.pi

    def e(a, b, c):
        x = a * h * tpi
        y = b * h * tpi
        z = c * h * tpi
        return (x * x + y * y + z * z) * 0.5

    ka_l, kb_l, kc_l = [], [], []
    i = 1
    while i <= kmax:
        if e(i, 0, 0) > ecut_ha:
            break
        i += 1
    kamax = i - 1
    for ka in range(0, kamax + 1):
        kbmin = 0 if ka == 0 else -kmax
        i = kbmin
        while i <= 0:
            if e(ka, i, 0) <= ecut_ha:
                break
            i += 1
        kbmin = i
        i = 1
        while i <= kmax:
            if e(ka, i, 0) > ecut_ha:
                break
            i += 1
        kbmax = i - 1
        for kb in range(kbmin, kbmax + 1):
            kcmin = 1 if (ka == 0 and kb == 0) else -kmax
            i = kcmin
            while i <= 0:
                if e(ka, kb, i) <= ecut_ha:
                    break
                i += 1
            kcmin = i
            i = 1
            while i <= kmax:
                if e(ka, kb, i) > ecut_ha:
                    break
                i += 1
            kcmax = i - 1
            for kc in range(kcmin, kcmax + 1):
                ka_l.append(ka)
                kb_l.append(kb)
                kc_l.append(kc)
    ka_l.append(0)
    kb_l.append(0)
    kc_l.append(0)
    return (np.array(ka_l, dtype=np.int32), np.array(kb_l, dtype=np.int32),
            np.array(kc_l, dtype=np.int32))


def flip_data_set(kx, ky, kz, data=None):
    """Mirror the Gx=0 half plane in front (para_grp_parse.C:178-286).

    Input is the PINY order (G=0 last).  Output length nktot+nplane0-1: the
    mirrored (0,-ky,-kz) points of the kx=0 half plane in reverse order, then
    G=0, then the original points.  ``data`` (complex) is conjugated for the
    mirrored points when given.
    """
    kx = np.asarray(kx)
    nktot = len(kx)
    nplane0 = int(np.count_nonzero(kx == 0))
    if kx[-1] != 0 or ky[-1] != 0 or kz[-1] != 0:
        raise ValueError("flip: last point is not G=0")
    if np.any(kx[:nplane0 - 1] != 0):
        raise ValueError("flip: kx=0 points are not first")
    head = np.arange(nplane0 - 2, -1, -1)
    okx = np.concatenate([kx[head], [0], kx[:nktot - 1]]).astype(np.int32)
    oky = np.concatenate([-np.asarray(ky)[head], [0], np.asarray(ky)[:nktot - 1]]).astype(np.int32)
    okz = np.concatenate([-np.asarray(kz)[head], [0], np.asarray(kz)[:nktot - 1]]).astype(np.int32)
    # reference check: ky non-decreasing over the mirrored head (:243-249)
    if np.any(np.diff(oky[:nplane0 - 1]) < 0):
        raise ValueError("flip: mirrored ky not ordered")
    od = None
    if data is not None:
        data = np.asarray(data)
        od = np.concatenate([np.conj(data[head]), data[-1:], data[:nktot - 1]])
    return okx, oky, okz, od


def get_chareG_line_prms(nktot, nchareG, npts):
    """Static load balance of z-lines into nchareG chunks (para_grp_parse.C:21-170).

    Returns (istrt_lgrp, iend_lgrp, npts_lgrp, nline_lgrp).
    """
    nline = len(npts)
    if nchareG > nline:
        raise ValueError("too many chunks")
    dev_min, nbal_min, ifirst = 0.0, 0, 0
    mmm = nktot // nchareG
    for ibal in range(0, mmm):
        nbal = ibal
        ntarg = nktot // nchareG
        if ntarg > nbal:
            ntarg -= nbal
        nmax, nmin, nnow, ic = 0, nktot, 0, 0
        for i in range(nline):
            nnow += int(npts[i])
            if nnow >= ntarg and ic < nchareG - 1:
                ic += 1
                nmin = min(nmin, nnow)
                nmax = max(nmax, nnow)
                nnow = 0
        nmin = min(nmin, nnow)
        nmax = max(nmax, nnow)
        dev = 100.0 * float(nmax - nmin) / float(max(nmin, 1))
        if ic == nchareG - 1:
            if dev < dev_min or ifirst == 0:
                ifirst, dev_min, nbal_min = 1, dev, nbal
    if ifirst == 0:
        raise ValueError("too many chunks")
    ntarg = nktot // nchareG
    if ntarg > nbal_min:
        ntarg = ntarg - nbal_min
    istrt = [0] * nchareG
    iend = [0] * nchareG
    nptsg = [0] * nchareG
    nlineg = [0] * nchareG
    ic = 0
    for i in range(nline):
        nptsg[ic] += int(npts[i])
        nlineg[ic] += 1
        if nptsg[ic] >= ntarg and ic < nchareG - 1:
            iend[ic] = i + 1
            ic += 1
            nptsg[ic] = 0
            nlineg[ic] = 0
            istrt[ic] = i + 1
    iend[nchareG - 1] = nline
    if min(nlineg) == 0 or min(nptsg) == 0:
        raise ValueError("too many chunks")
    return istrt, iend, nptsg, nlineg


def _line_starts(kx, ky):
    brk = np.nonzero((np.diff(kx) != 0) | (np.diff(ky) != 0))[0] + 1
    st = np.concatenate([[0], brk]).astype(np.int64)
    en = np.concatenate([brk, [len(kx)]]).astype(np.int64)
    return st, en


def process_state(kx, ky, kz, nchareG, data=None):
    """Reorder the flipped set into per-chunk, (kx,ky)-sorted lines (util.C:1331-1642).

    Lines are dealt round-robin to the nchareG chunks (:1433-1458), the chunk
    boundaries come from ``get_chareG_line_prms`` (:1506-1510) and every chunk's
    lines are sorted on kx then ky (``sort_kxky`` util.C:2223-2247; the (kx,ky)
    pairs are unique, so the order is the lexicographic one).
    """
    kx = np.asarray(kx)
    ky = np.asarray(ky)
    kz = np.asarray(kz)
    npk = len(kx)
    # the reference's checks (:1370-1399)
    if np.any(np.diff(kx) < 0):
        raise ValueError("Bad x-flip")
    st, en = _line_starts(kx, ky)
    nline = len(st)
    if nchareG > nline:
        raise ValueError("too many chunks")
    order_lines = [j for i in range(nchareG) for j in range(i, nline, nchareG)]
    perm = np.concatenate([np.arange(st[j], en[j]) for j in order_lines])
    kx1, ky1, kz1 = kx[perm], ky[perm], kz[perm]
    d1 = None if data is None else np.asarray(data)[perm]
    st1, en1 = _line_starts(kx1, ky1)
    npts_line = en1 - st1
    istrt, iend, nptsg, nlineg = get_chareG_line_prms(npk, nchareG, npts_line)
    perm2 = []
    loff = 0
    for i in range(nchareG):
        idx = list(range(loff, loff + nlineg[i]))
        idx.sort(key=lambda l: (int(kx1[st1[l]]), int(ky1[st1[l]])))
        for l in idx:
            perm2.append(np.arange(st1[l], en1[l]))
        loff += nlineg[i]
    perm2 = np.concatenate(perm2)
    out = (kx1[perm2].astype(np.int32), ky1[perm2].astype(np.int32),
           kz1[perm2].astype(np.int32))
    dec = dict(istrt_lgrp=istrt, iend_lgrp=iend, npts_lgrp=nptsg, nline_lgrp=nlineg)
    dout = None if d1 is None else d1[perm2]
    return out, dec, dout


def runs_from_kvecs(kx, ky, kz, nx, ny, nz):
    """RunDescriptors as built by ``readStateIntoRuns`` (util.C:933-1000).

    Returns an int32 array [nruns, 7] of (x, y, z, offset, length, inc, nz);
    every z-line gives a negative-kz run followed by a non-negative one.
    """
    kx = np.asarray(kx)
    ky = np.asarray(ky)
    kz = np.asarray(kz)
    n = len(kx)
    runs = []

    def wrap(v, m):
        return v + m if v < 0 else v
    cx, cy, cz = wrap(int(kx[0]), nx), wrap(int(ky[0]), ny), wrap(int(kz[0]), nz)
    tmpz = cz
    rsum, rlen = 0, 1
    if kz[0] >= 0:
        runs.append((cx, cy, cz, rsum, 0, 1, nz))
    for p in range(1, n):
        x, y, z = wrap(int(kx[p]), nx), wrap(int(ky[p]), ny), wrap(int(kz[p]), nz)
        if z == tmpz + 1 and x == cx and y == cy:
            rlen += 1
            tmpz += 1
        else:
            runs.append((cx, cy, cz, rsum, rlen, 1, nz))
            rsum += rlen
            if (cx != x or cy != y) and kz[p - 1] < 0:
                runs.append((cx, cy, 0, rsum, 0, 1, nz))
            if (cx != x or cy != y) and kz[p] >= 0:
                runs.append((x, y, 0, rsum, 0, 1, nz))
            cx, cy, cz, tmpz, rlen = x, y, z, z, 1
    runs.append((cx, cy, cz, rsum, rlen, 1, nz))
    rsum += rlen
    if kz[n - 1] < 0:
        runs.append((cx, cy, 0, rsum, 0, 1, nz))
    if rsum != n or len(runs) % 2 != 0:
        raise ValueError("broken run descriptors")
    return np.array(runs, dtype=np.int32)


class Layout:
    """The full Gamma-point state layout of one system (oracle side)."""

    def __init__(self, box_len, ecut_ry, nchareG=None, gexpand=1.0, grid=None):
        self.box_len = float(box_len)
        self.ecut_ry = float(ecut_ry)
        self.kmax = calc_kmax(box_len, ecut_ry)
        n = radix_size(self.kmax) if grid is None else int(grid)
        if n < 2 * (2 * self.kmax + 1):
            raise ValueError("grid too small for the cutoff")
        self.n = n
        ka, kb, kc = setkvec3d_sm(0.5 * ecut_ry, self.kmax, box_len)
        self.nktot = len(ka) - 1  # half sphere without G=0
        fx, fy, fz, _ = flip_data_set(ka, kb, kc)
        self.nplane_x = int(fx.max()) + 1
        if nchareG is None:
            nchareG = int(gexpand * self.nplane_x)
        self.nchareG = nchareG
        (kx, ky, kz), self.decomp, _ = process_state(fx, fy, fz, nchareG)
        self.kx, self.ky, self.kz = kx, ky, kz
        self.npts = len(kx)
        self.runs = runs_from_kvecs(kx, ky, kz, n, n, n)
        self.nlines = len(self.runs) // 2
        tpi = 2.0 * math.pi / self.box_len
        self.g2 = ((kx * tpi) ** 2 + (ky * tpi) ** 2 + (kz * tpi) ** 2).astype(np.float64)
        # per-point double-pack weight: 1 on the Gx=0 plane, 2 elsewhere
        self.wpt = np.where(kx == 0, 1.0, 2.0)
        self.kx0 = (kx == 0)

    # per-line tables ------------------------------------------------------
    def line_tables(self):
        """Per z-line: x, y (wrapped), packed offset, lengths and start z of both runs.

        ``zneg`` is where ``expandGSpace`` puts the first negative-kz point
        (runs[r].z + nfftz - runs[0].nz, fftCache.C:481-486) and ``zpos`` the first
        non-negative one (runs[r+1].z, :490-494).
        """
        r = self.runs
        neg, pos = r[0::2], r[1::2]
        nsub = self.n - int(r[0, 6])
        return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(),
                    off=neg[:, 3].copy(), nneg=neg[:, 4].copy(),
                    npos=pos[:, 4].copy(), zneg=(neg[:, 2] + nsub).astype(np.int32),
                    zpos=pos[:, 2].copy())
