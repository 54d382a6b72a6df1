"""Oracle (test infrastructure only): the reference's state-file writer and
reader restated in Python.

write_bytes follows writeStateFile (src_charm_driver/utility/util.C:1955-2180)
with sort_psi_output (:2180-2220): the points sorted by
(kz - kzmin) + (ky - kymin) nz + (kx - kxmin) nz ny; the ones after G=0 in
that order, then G=0; text lines "%g %g %d %d %d \\n" (:1987-1996), binary
records double, double, int, int, int after four int header words
(:2042-2064).  read_records follows readState (util.C:1143-1170, :1280-1296):
records up to and including G=0.  pack follows flip_data_set
(para_grp_parse.C:178-286): the redundant Gx=0 half is the conjugate of its
partner.
"""
import struct

import numpy as np


def _order(kx, ky, kz):
    kx, ky, kz = (np.asarray(k, dtype=np.int64) for k in (kx, ky, kz))
    nyr = ky.max() - ky.min() + 1
    nzr = kz.max() - kz.min() + 1
    key = (kz - kz.min()) + (ky - ky.min()) * nzr + (kx - kx.min()) * nzr * nyr
    idx = np.argsort(key, kind="stable")
    g0 = np.nonzero((kx[idx] == 0) & (ky[idx] == 0) & (kz[idx] == 0))[0]
    return idx, int(g0[0])


def write_bytes(coef, kx, ky, kz, grid, binary):
    idx, istrt = _order(kx, ky, kz)
    seq = list(idx[istrt + 1:]) + [idx[istrt]]
    n = len(kx) - istrt
    if not binary:
        out = ["%d %d %d %d\n" % (n, grid[0], grid[1], grid[2])]
        for p in seq:
            out.append("%g %g %d %d %d \n" % (coef[p].real, coef[p].imag, kx[p], ky[p], kz[p]))
        return "".join(out).encode()
    out = [struct.pack("<4i", n, *grid)]
    for p in seq:
        out.append(struct.pack("<ddiii", coef[p].real, coef[p].imag, int(kx[p]), int(ky[p]),
                               int(kz[p])))
    return b"".join(out)


def read_records(data, binary):
    recs = {}
    if not binary:
        lines = data.decode().splitlines()
        n, nx, ny, nz = (int(v) for v in lines[0].split())
        for ln in lines[1:n + 1]:
            t = ln.split()
            re, im, x, y, z = float(t[0]), float(t[1]), int(t[2]), int(t[3]), int(t[4])
            recs[(x, y, z)] = complex(re, im)
            if x == 0 and y == 0 and z == 0:
                break
        return recs, (nx, ny, nz)
    n, nx, ny, nz = struct.unpack_from("<4i", data, 0)
    off = 16
    for _ in range(n):
        re, im, x, y, z = struct.unpack_from("<ddiii", data, off)
        off += 28
        recs[(x, y, z)] = complex(re, im)
        if x == 0 and y == 0 and z == 0:
            break
    return recs, (nx, ny, nz)


def pack(recs, kx, ky, kz):
    out = np.zeros(len(kx), dtype=np.complex128)
    for p, (x, y, z) in enumerate(zip(kx, ky, kz)):
        if x == 0 and (y < 0 or (y == 0 and z < 0)):
            out[p] = np.conj(recs[(0, -int(y), -int(z))])
        else:
            out[p] = recs[(int(x), int(y), int(z))]
    return out
