"""ctypes binding of libcpstep.so (the C ABI declared in include/cpstep.h).

The library is built in-tree (``python -m openatom_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcpstep.so")

CPSTEP_OK = 0
CPSTEP_ERR_ARG = 1
CPSTEP_ERR_CUDA = 2
CPSTEP_ERR_LAYOUT = 3
CPSTEP_ERR_NOCONV = 4
CPSTEP_ERR_STATE = 5
CPSTEP_ERR_NORB = 6
CONSTRAINT_ORTHO_T = 0
CONSTRAINT_LOWDIN = 1
PREC_FP64 = 0
PREC_MIXED = 1

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every exported entry point of include/cpstep.h
SIGNATURES = {
    "cpstep_version": (ctypes.c_int, []),
    "cpstep_last_error": (ctypes.c_char_p, []),
    "cpstep_launch_count": (ctypes.c_ulonglong, []),
    "cpstep_ctx_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "cpstep_phase_times": (ctypes.c_int, [_vp, _c_dbl_p, _c_int_p]),
    "cpstep_layout_sizes": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, _c_int_p, _c_int_p,
                                           _c_int_p, _c_int_p]),
    "cpstep_layout_build": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p,
                                           _c_int_p, _c_int_p, ctypes.c_int, _c_int_p,
                                           _c_int_p]),
    "cpstep_ctx_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, ctypes.c_int,
                                         _c_int_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _c_dbl_p, ctypes.c_double]),
    "cpstep_ctx_destroy": (ctypes.c_int, [_vp]),
    "cpstep_ctx_set_stream": (ctypes.c_int, [_vp, _vp]),
    "cpstep_ctx_info": (ctypes.c_int, [_vp, _c_int_p, _c_int_p]),
    "cpstep_ctx_sync": (ctypes.c_int, [_vp]),
    "cpstep_expand_gspace": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "cpstep_pack_gspace": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "cpstep_stp_fft_gtor": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "cpstep_stp_fft_rtog": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "cpstep_density": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "cpstep_vks_psi": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "cpstep_eke": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cpstep_pc_overlap": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int]),
    "cpstep_pc_backmultiply": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                              ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "cpstep_dgemm": (ctypes.c_int, [_vp, ctypes.c_char, ctypes.c_char, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp,
                                    ctypes.c_int, _vp, ctypes.c_int, ctypes.c_double, _vp,
                                    ctypes.c_int]),
    "cpstep_ortho_tmat": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, _c_int_p, _c_dbl_p]),
    "cpstep_set_atoms": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_int_p, _c_dbl_p,
                                        _c_dbl_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        _c_dbl_p, _c_dbl_p, ctypes.c_double]),
    "cpstep_rho_layout": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p,
                                         _c_int_p]),
    "cpstep_exc_calc": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "cpstep_rho_fft_r2g": (ctypes.c_int, [_vp, _vp, _vp]),
    "cpstep_hart_eext": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cpstep_vks_fft_g2r": (ctypes.c_int, [_vp, _vp, _vp]),
    "cpstep_vks_from_rho": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cpstep_set_xc": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "cpstep_gga_functional": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cpstep_nl_grid_size": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "cpstep_eext_grid_size": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "cpstep_set_local_ees": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "cpstep_set_nonlocal": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           _c_int_p, _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p,
                                           _c_dbl_p]),
    "cpstep_ees_nonlocal": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "cpstep_set_nonlocal_sf": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p,
                                              _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "cpstep_sf_nonlocal": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "cpstep_ion_forces": (ctypes.c_int, [_vp, _vp, _vp]),
    "cpstep_atoms_integrate": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                              ctypes.c_double, _vp]),
    "cpstep_set_cp_mass": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    "cpstep_set_cp_thermostat": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int]),
    "cpstep_cp_thermostat_state": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "cpstep_set_atom_thermostat": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  _vp, _vp]),
    "cpstep_atom_thermostat_state": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "cpstep_cp_integrate": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int,
                                           _vp]),
    "cpstep_cp_step": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int, _vp,
                                      _vp]),
    "cpstep_step_status": (ctypes.c_int, [_vp, _c_int_p, _c_int_p]),
    "cpstep_set_constraint": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "cpstep_dyn_state": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _c_int_p]),
    "cpstep_dyn_status": (ctypes.c_int, [_vp, _c_dbl_p, _c_int_p]),
    "cpstep_set_gemm_path": (ctypes.c_int, [_vp, ctypes.c_int]),
    "cpstep_state_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _vp,
                                          _vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int]),
    "cpstep_state_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                         _vp, _vp, _c_int_p, _c_int_p, _c_int_p]),
    "cpstep_ctx_set_graph": (ctypes.c_int, [_vp, ctypes.c_int]),
    "cpstep_tune_get": (ctypes.c_int, [_vp, _c_int_p, ctypes.c_int]),
    "cpstep_tune_set": (ctypes.c_int, [_vp, _c_int_p, ctypes.c_int]),
    "cpstep_autotune": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double)]),
    "cpstep_batch_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)]),
    "cpstep_batch_destroy": (ctypes.c_int, [_vp]),
    "cpstep_batch_set_stream": (ctypes.c_int, [_vp, _vp]),
    "cpstep_batch_set_graph": (ctypes.c_int, [_vp, ctypes.c_int]),
    "cpstep_batch_status": (ctypes.c_int, [_vp, _c_int_p, _c_int_p,
                                           ctypes.POINTER(ctypes.c_ulonglong)]),
    "cpstep_batch_step": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                         ctypes.POINTER(_vp), ctypes.c_double, ctypes.c_int,
                                         ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "cpstep_ctx_graph_status": (ctypes.c_int, [_vp, _c_int_p, _c_int_p,
                                               ctypes.POINTER(ctypes.c_ulonglong)]),
    "cpstep_device_errors": (ctypes.c_int, [_vp, _c_int_p]),
    "cpstep_set_positions": (ctypes.c_int, [_vp, _vp]),
    "cpstep_pc_overlap_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, _vp, ctypes.c_double,
                                                 ctypes.c_double, _vp, ctypes.c_int, _vp]),
    "cpstep_cp_step_host": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int,
                                           _vp, _vp, _vp]),
}
NENERGY = 14
(E_EXC, E_MUXC, E_HART, E_EXT, E_EWD, E_EXT_G0, E_KE, E_NL, E_TOT, E_FICT, E_EXC_GGA, E_EWD_RS,
 E_NHC_KE, E_NHC_POT) = range(14)


class CpstepError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__("%s failed (code %d): %s" % (fn, code, msg))
        self.code = code


_lib = None


def lib():
    """Load libcpstep.so once; raise if it is absent (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcpstep.so is not built (run `python -m openatom_b200.build`); "
                              "openatom_b200 has no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(name, code):
    if code != CPSTEP_OK:
        msg = lib().cpstep_last_error()
        raise CpstepError(name, code, msg.decode() if msg else "")


def call(name, *args):
    check(name, getattr(lib(), name)(*args))


def ptr(t):
    """Device pointer of a torch tensor as c_void_p (None for None)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def int_array(a):
    import numpy as np
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_c_int_p)
