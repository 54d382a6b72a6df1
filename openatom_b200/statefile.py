"""State files in the reference's format (host side, through libcpstep).

One state per file, as ``writeStateFile`` / ``readState``
(src_charm_driver/utility/util.C:1955-2180, :1107-1330) write and read them:
header ``npts nx ny nz``, then the stored half sphere sorted by (kx, ky, kz)
with G=0 last.  ``fmt`` is "text" (``%g``, as lossy as the reference's),
"binary", "text.gz" or "binary.gz" (zlib, ``.gz`` appended to the name).
"""
import ctypes

import numpy as np

from . import _lib

FORMATS = {"text": 0, "binary": 1, "text.gz": 2, "binary.gz": 3}


def _ip(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def write_state(path, coef, layout, fmt="binary", grid=None):
    """Write one state's packed coefficients (complex128 [npts], the layout's order)."""
    c = np.ascontiguousarray(coef, dtype=np.complex128)
    if c.shape != (layout.npts,):
        raise ValueError("coef must be [npts] complex")
    kx, ky, kz = (np.ascontiguousarray(k, dtype=np.int32) for k in (layout.kx, layout.ky, layout.kz))
    n = grid if grid is not None else (layout.n, layout.n, layout.n)
    _lib.call("cpstep_state_write", str(path).encode(), FORMATS[fmt], layout.npts,
              _ip(c.view(np.float64)), _ip(kx), _ip(ky), _ip(kz), int(n[0]), int(n[1]), int(n[2]))


def read_state(path, layout, fmt="binary"):
    """Read one state into the layout's packed order; returns (coef, (nx, ny, nz))."""
    kx, ky, kz = (np.ascontiguousarray(k, dtype=np.int32) for k in (layout.kx, layout.ky, layout.kz))
    out = np.zeros(layout.npts, dtype=np.complex128)
    nx, ny, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _lib.call("cpstep_state_read", str(path).encode(), FORMATS[fmt], layout.npts, _ip(kx),
              _ip(ky), _ip(kz), _ip(out.view(np.float64)), ctypes.byref(nx), ctypes.byref(ny),
              ctypes.byref(nz))
    return out, (nx.value, ny.value, nz.value)


def write_states(pattern, psi, layout, fmt="binary", grid=None):
    """psi [S, npts]: one file per state, ``pattern % (s + 1)`` (states counted from 1)."""
    for s in range(psi.shape[0]):
        write_state(pattern % (s + 1), psi[s], layout, fmt, grid)


def read_states(pattern, nstates, layout, fmt="binary"):
    return np.stack([read_state(pattern % (s + 1), layout, fmt)[0] for s in range(nstates)])
