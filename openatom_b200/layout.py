"""Host mirror of the reference's state G-vector layout, built by libcpstep.

``StateLayout`` holds what OpenAtom's state chares hold after start-up: the
packed (kx, ky, kz) order of one state and its RunDescriptors
(src_charm_driver/utility/util.C:861-1099, :1331-1642), computed by
``cpstep_layout_build`` in the C++ library.
"""
import ctypes
import math

import numpy as np

from . import _lib


class StateLayout:
    def __init__(self, box_len, ecut_ry, nfft=None, nchareG=0):
        L = _lib.lib()
        kmax, n, nk, npts = (ctypes.c_int() for _ in range(4))
        _lib.check("cpstep_layout_sizes",
                   L.cpstep_layout_sizes(float(box_len), float(ecut_ry), ctypes.byref(kmax),
                                         ctypes.byref(n), ctypes.byref(nk), ctypes.byref(npts)))
        self.box_len = float(box_len)
        self.ecut_ry = float(ecut_ry)
        self.kmax = kmax.value
        self.n_radix = n.value
        self.n = int(nfft) if nfft else n.value
        self.nktot = nk.value
        cap = npts.value
        kx = np.zeros(cap, np.int32)
        ky = np.zeros(cap, np.int32)
        kz = np.zeros(cap, np.int32)
        runs_cap = 2 * cap + 2
        runs = np.zeros((runs_cap, 7), np.int32)
        np_out, nr_out = ctypes.c_int(), ctypes.c_int()
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        _lib.check("cpstep_layout_build",
                   L.cpstep_layout_build(self.box_len, self.ecut_ry, int(nchareG), self.n, cap,
                                         ip(kx), ip(ky), ip(kz), ctypes.byref(np_out), runs_cap,
                                         ip(runs), ctypes.byref(nr_out)))
        self.npts = np_out.value
        self.kx, self.ky, self.kz = kx[:self.npts], ky[:self.npts], kz[:self.npts]
        self.runs = runs[:nr_out.value].copy()
        self.nlines = len(self.runs) // 2
        self.nplane_x = int(self.kx.max()) + 1

    @property
    def hmat(self):
        """Cubic cell matrix, column-major 3x3 (bohr)."""
        return np.diag([self.box_len] * 3).astype(np.float64).reshape(-1, order="F")

    @property
    def vol(self):
        return self.box_len ** 3

    def gvectors(self):
        tpi = 2.0 * math.pi / self.box_len
        return np.stack([self.kx * tpi, self.ky * tpi, self.kz * tpi], axis=1)

    def g2(self):
        g = self.gvectors()
        return np.sum(g * g, axis=1)
