"""openatom_b200: the OpenAtom Car-Parrinello electronic step on one B200.

The compute path is libcpstep.so (hand-written sm_100a CUDA behind the C ABI
in include/cpstep.h); this package is the Python host mirror of the
reference's operator interface.  Importing it does not need a GPU; calling a
compute entry point needs the built library and a CUDA device.
"""
from ._lib import lib, CpstepError, PREC_FP64, PREC_MIXED  # noqa: F401

__all__ = ["lib", "CpstepError", "PREC_FP64", "PREC_MIXED"]
