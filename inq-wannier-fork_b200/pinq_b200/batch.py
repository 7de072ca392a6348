"""Batched H|psi> over independent, uneven cells: one persistent launch over work
items (cell, pass, tile) where the cells allow it, else one CUDA graph."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, lib


MODES = {"auto": 0, "graph": 1, "persistent": 2}


class CellBatch:
    """Applies H to every cell's orbital block with one launch: a persistent kernel
    over a device work queue (mode "persistent"), a CUDA graph with one branch per
    cell ("graph"), or the one autotune_form measured faster ("auto", the graph until
    then)."""

    def __init__(self, hams, mode: str = "auto"):
        self.hams = list(hams)
        self.mode = mode
        self._create()

    def _create(self):
        arr = (ctypes.c_void_p * len(self.hams))(*[h._h.value for h in self.hams])
        out = ctypes.c_void_p()
        call("inqb_batch_create", arr, len(self.hams), ctypes.byref(out))
        self._b = out
        call("inqb_batch_set_mode", self._b, MODES[self.mode])

    def autotune_form(self, psis, outs):
        """Time the graph and the persistent form on these blocks and make the faster the
        one mode "auto" runs; returns (form, ms per apply of each: {"graph": .., "persistent":
        .. or None where the cells do not fit the persistent kernel})."""
        n = len(self.hams)
        P = (ctypes.c_void_p * n)(*[x.data_ptr() for x in psis])
        Q = (ctypes.c_void_p * n)(*[y.data_ptr() for y in outs])
        Ms = np.ascontiguousarray([x.shape[1] for x in psis], np.int32)
        lds = np.ascontiguousarray([x.stride(0) for x in psis], np.int32)
        form = ctypes.c_int()
        ms = (ctypes.c_double * 2)()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        call("inqb_batch_autotune", self._b, P, Q, Ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
             lds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), stream, ctypes.byref(form), ms)
        return ({1: "graph", 2: "persistent"}[form.value],
                {"graph": ms[0], "persistent": ms[1] if ms[1] > 0 else None})

    def set_mode(self, mode: str):
        self.mode = mode
        call("inqb_batch_set_mode", self._b, MODES[mode])

    def info(self) -> dict:
        """The form the last apply set up and, for the persistent form, its work items
        and CTAs."""
        f, n, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("inqb_batch_info", self._b, ctypes.byref(f), ctypes.byref(n), ctypes.byref(c))
        form = {0: None, 1: "graph", 2: "persistent"}[f.value]
        return {"form": form, "items": n.value, "ctas": c.value}

    def status(self):
        """Synchronise; raises InqbError (INQB_ERR_TIMEOUT) when a device-side wait of a
        persistent launch gave up since the last call."""
        call("inqb_batch_status", self._b, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))

    def set_wait_limit(self, seconds: float):
        call("inqb_batch_set_wait_limit", self._b, float(seconds))

    def test_unreachable_wait(self, on: bool):
        call("inqb_batch_test_unreachable_wait", self._b, 1 if on else 0)

    def autotune(self, Ms):
        """Pick each cell's launch schedule for its orbital count (inqb_autotune) and
        start a fresh batch, so the next apply captures the graph with them."""
        scheds = [h.autotune(int(M)) for h, M in zip(self.hams, Ms)]
        self.close()
        self._create()
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
