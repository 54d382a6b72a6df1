"""Oracle: state FFTs, density and V_KS.psi in FP64, following the reference steps.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

FFTW-2 sign conventions (``fftCache.C:252-255`` plans): FFTW_FORWARD is
exp(-2 pi i jk/n), FFTW_BACKWARD exp(+2 pi i jk/n), both unnormalised;
``rfftwnd`` COMPLEX_TO_REAL uses the +i sign and REAL_TO_COMPLEX the -i sign.

* expand / pack            fftCache.C:460-553
* G->R, G-chare (z)        doStpFFTGtoR_Gchare fftCache.C:1133-1159
* transpose                CP_State_GSpacePlane.C:1473-1498 + CP_State_RealSpacePlane.C:248-268
                           (line (x,y) goes to x + y*(nx/2+1) of plane z)
* G->R, R-chare (y, x)     doStpFFTGtoR_Rchare fftCache.C:1167-1243 (imag flip :1209-1213)
* density                  CP_State_RealSpacePlane.C:349-355 (occ*wkpt*psi^2),
                           CP_Rho_RealSpacePlane.C:630-650 (x 1/vol)
* V.psi                    CP_State_RealSpacePlane.C:580-587
* R->G, R-chare (x, y)     doStpFFTRtoG_Rchare fftCache.C:1252-1319 (imag flip :1272-1274)
* R->G, G-chare (z), pack  doStpFFTRtoG_Gchare fftCache.C:1099-1123
* force scale              CP_State_GSpacePlane.C:1605-1612 (-2/(nx ny nz))
* addForces                stateSlab.C:240-272 (x2 off the Gx=0 plane)
* kinetic energy           CP_eke_calc cp_eke.C:30-140
"""
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft

_WORKERS = 1
_POOL = None
_TLS = threading.local()


def _w():
    """pocketfft threads for a call: 1 inside a state_map chunk (the chunks
    already run concurrently), all of them otherwise."""
    return 1 if getattr(_TLS, "inner", False) else _WORKERS


def set_workers(n):
    """Host threads the oracle may use: state chunks run concurrently on a
    thread pool (numpy and pocketfft release the GIL in the array work)."""
    global _WORKERS, _POOL
    _WORKERS = max(1, int(n))
    if _POOL is not None:
        _POOL.shutdown()
    _POOL = ThreadPoolExecutor(_WORKERS) if _WORKERS > 1 else None


def state_map(fn, n, chunk):
    """[fn(s0, s1) for the chunks of range(n)] in chunk order, concurrently when
    set_workers gave more than one thread (results do not depend on it)."""
    spans = [(s0, min(n, s0 + chunk)) for s0 in range(0, n, chunk)]
    if _POOL is None or len(spans) == 1 or getattr(_TLS, "inner", False):
        return [fn(a, b) for a, b in spans]

    def run(ab):
        _TLS.inner = True
        try:
            return fn(*ab)
        finally:
            _TLS.inner = False
    return list(_POOL.map(run, spans))


def _line_index(lay):
    """Flat [nlines * n] position of every packed point (the layout of the
    line loops of expandGSpace / packGSpace), cached on the layout."""
    idx = getattr(lay, "_line_idx", None)
    if idx is None:
        t = lay.line_tables()
        n = lay.n
        idx = np.empty(lay.npts, dtype=np.int64)
        for l in range(lay.nlines):
            o, nn, npo = int(t['off'][l]), int(t['nneg'][l]), int(t['npos'][l])
            zn, zp = int(t['zneg'][l]), int(t['zpos'][l])
            idx[o:o + nn] = l * n + zn + np.arange(nn)
            idx[o + nn:o + nn + npo] = l * n + zp + np.arange(npo)
        lay._line_idx = idx
    return idx


def expand(psi, lay):
    """[S, npts] complex -> [S, nlines, n] complex z-lines (expandGSpace)."""
    S = psi.shape[0]
    out = np.zeros((S, lay.nlines * lay.n), dtype=np.complex128)
    out[:, _line_index(lay)] = psi
    return out.reshape(S, lay.nlines, lay.n)


def pack(lines, lay):
    """[S, nlines, n] -> [S, npts] (packGSpace)."""
    S = lines.shape[0]
    return lines.reshape(S, -1)[:, _line_index(lay)]


def state_g_to_r(psi, lay):
    """Packed psi(G) [S, npts] -> real psi(r) [S, nz, ny, nx] (FP64)."""
    n = lay.n
    t = lay.line_tables()
    z = sfft.fft(expand(psi, lay), axis=2, workers=_w())               # FFTW_FORWARD along z
    S = psi.shape[0]
    plane = np.zeros((S, n, n, n // 2 + 1), dtype=np.complex128)   # [s, z, y, x]
    plane[:, :, t['y'], t['x']] = np.transpose(z, (0, 2, 1))
    plane = sfft.fft(plane, axis=2, workers=_w())      # FFTW_FORWARD along y
    plane = np.conj(plane)                                 # imag flip
    return sfft.irfft(plane, n=n, axis=3, workers=_w()) * n  # rfftw C2R (+i, unnormalised)


def state_r_to_g(f, lay):
    """Real f(r) [S, nz, ny, nx] -> packed F(G) [S, npts], unscaled (FP64)."""
    n = lay.n
    t = lay.line_tables()
    X = np.conj(sfft.rfft(f, axis=3, workers=_w()))    # rfftw R2C (-i), imag flip
    X = sfft.ifft(X, axis=2, workers=_w()) * n         # FFTW_BACKWARD along y
    lines = np.transpose(X[:, :, t['y'], t['x']], (0, 2, 1))   # [s, line, z]
    lines = sfft.ifft(lines, axis=2, workers=_w()) * n  # FFTW_BACKWARD along z
    return pack(lines, lay)


def density(psi, lay, occ, vol, chunk=16):
    """rho(r) = sum_s occ_s psi_s(r)^2 / vol, [nz, ny, nx] FP64 (chunk partials
    summed in chunk order)."""
    n = lay.n

    def part(s0, s1):
        pr = state_g_to_r(psi[s0:s1], lay)
        return np.einsum('s,szyx->zyx', occ[s0:s1], pr * pr)
    rho = np.zeros((n, n, n))
    for p in state_map(part, psi.shape[0], chunk):
        rho += p
    return rho / vol


def vpsi_force(psi, vks, lay, occ, chunk=16):
    """F(G) = -2/N * FFT^-1[occ * V_KS * psi(r)]  (before addForces)."""
    n = lay.n
    out = np.zeros(psi.shape, dtype=np.complex128)

    def part(s0, s1):
        pr = state_g_to_r(psi[s0:s1], lay)
        f = pr * vks[None] * occ[s0:s1, None, None, None]
        out[s0:s1] = state_r_to_g(f, lay) * (-2.0 / float(n * n * n))
    state_map(part, psi.shape[0], chunk)
    return out


def add_forces(force_vks, force_nl, lay):
    """GStateSlab::addForces: x2 off the Gx=0 plane, then + non-local force."""
    w = np.where(lay.kx == 0, 1.0, 2.0)
    out = force_vks * w[None]
    if force_nl is not None:
        out = out + force_nl
    return out


def eke(force, psi, lay, occ, ecut_ry):
    """CP_eke_calc: F -= w g^2 psi, E_kin = sum w g^2 |psi|^2 / 2 (cp_eke.C:77-125)."""
    g2 = lay.g2
    w = np.where(lay.kx == 0, 1.0, 2.0)
    inside = g2 <= ecut_ry
    wt = occ[:, None] * (w * g2)[None]
    f = np.where(inside[None], force - psi * wt, 0.0)
    e = 0.5 * np.sum(np.where(inside[None], wt * np.abs(psi) ** 2, 0.0), axis=1)
    return f, e
