"""Batched H|psi> over independent, uneven cells in one CUDA graph."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, lib


class CellBatch:
    """Applies H to every cell's orbital block with one graph launch."""

    def __init__(self, hams):
        self.hams = list(hams)
        arr = (ctypes.c_void_p * len(self.hams))(*[h._h.value for h in self.hams])
        out = ctypes.c_void_p()
        call("inqb_batch_create", arr, len(self.hams), ctypes.byref(out))
        self._b = out

    def autotune(self, Ms):
        """Pick each cell's launch schedule for its orbital count (inqb_autotune) and
        start a fresh batch, so the next apply captures the graph with them."""
        scheds = [h.autotune(int(M)) for h, M in zip(self.hams, Ms)]
        self.close()
        arr = (ctypes.c_void_p * len(self.hams))(*[h._h.value for h in self.hams])
        out = ctypes.c_void_p()
        call("inqb_batch_create", arr, len(self.hams), ctypes.byref(out))
        self._b = out
        return scheds

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            lib().inqb_batch_destroy(self._b)
        self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, psis, outs):
        n = len(self.hams)
        for h, x, y in zip(self.hams, psis, outs):
            h._check(x), h._check(y)
        P = (ctypes.c_void_p * n)(*[x.data_ptr() for x in psis])
        Q = (ctypes.c_void_p * n)(*[y.data_ptr() for y in outs])
        Ms = np.ascontiguousarray([x.shape[1] for x in psis], np.int32)
        lds = np.ascontiguousarray([x.stride(0) for x in psis], np.int32)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        call("inqb_batch_apply_h", self._b, P, Q, Ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
             lds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), stream)
        return outs
