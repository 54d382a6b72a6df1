"""Independent systems stepped together: one ``StepContext`` per system, one
electronic step of all of them per ``StepBatch.step``, replayed as a single
CUDA graph with a branch per system (``cpstep_batch_*``)."""
import ctypes

from . import _lib


class StepBatch:
    def __init__(self, contexts):
        self.contexts = list(contexts)
        n = len(self.contexts)
        arr = (ctypes.c_void_p * n)(*[c._h for c in self.contexts])
        h = ctypes.c_void_p()
        _lib.call("cpstep_batch_create", ctypes.byref(h), n, arr)
        self._h = h

    def close(self):
        if self._h:
            _lib.call("cpstep_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_graph(self, enable):
        _lib.call("cpstep_batch_set_graph", self._h, 1 if enable else 0)

    def status(self):
        en, cap, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_ulonglong()
        _lib.call("cpstep_batch_status", self._h, ctypes.byref(en), ctypes.byref(cap),
                  ctypes.byref(k))
        return bool(en.value), bool(cap.value), int(k.value)

    def step(self, psis, vpsis, occs, dt, iteration, energies, forces=None):
        """One step of every system (device tensors, one per context)."""
        n = len(self.contexts)
        P = lambda ts: (ctypes.c_void_p * n)(*[None if t is None else t.data_ptr() for t in ts])
        import torch
        s = torch.cuda.current_stream().cuda_stream  # the graph runs after torch's work
        _lib.call("cpstep_batch_set_stream", self._h, ctypes.c_void_p(s))
        _lib.call("cpstep_batch_step", self._h, P(psis), P(vpsis), P(occs), float(dt),
                  int(iteration), P(energies), P(forces) if forces is not None else None)
