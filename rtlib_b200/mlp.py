"""Host-side handle of the learned directional guide (rtpg_mlp_* over the C ABI)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr, stream_ptr

N_PARAMS = 16384
LOBES = 8


class MLPGuide:
    def __init__(self, aabb_min, aabb_max, seed=1, learning_rate=1e-3, record_capacity=1 << 18):
        mn = (C.c_float * 3)(*[float(v) for v in aabb_min])
        mx = (C.c_float * 3)(*[float(v) for v in aabb_max])
        h = C.c_void_p()
        call("rtpg_mlp_create", mn, mx, int(seed), float(learning_rate), int(record_capacity), C.byref(h))
        self.h = h
        self.aabb_min, self.aabb_max = tuple(aabb_min), tuple(aabb_max)
        self.capacity = int(record_capacity)

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_mlp_destroy", self.h)
            self.h = None

    def params(self):
        w = np.empty(N_PARAMS, np.float32)
        call("rtpg_mlp_params", self.h, w.ctypes.data, None, None)
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, np.float32)
        call("rtpg_mlp_params", self.h, None, w.ctypes.data, None)

    def eval(self, pos, nrm, wo, raw=True, stream=None):
        import torch
        n = pos.shape[0]
        out = torch.empty((n, 48 if raw else 40), dtype=torch.float32, device=pos.device)
        call("rtpg_mlp_eval", self.h, n, ptr(pos), ptr(nrm), ptr(wo), ptr(out) if raw else None,
             None if raw else ptr(out), stream_ptr(stream))
        return out

    def loss_grad(self, pos, nrm, wo, wi, w, stream=None):
        """(loss, gradient (16384,) float32 device tensor) over the given records."""
        import torch
        g = torch.zeros(N_PARAMS, dtype=torch.float32, device=pos.device)
        loss = C.c_float()
        call("rtpg_mlp_loss_grad", self.h, pos.shape[0], ptr(pos), ptr(nrm), ptr(wo), ptr(wi), ptr(w), ptr(g),
             C.byref(loss), stream_ptr(stream))
        return loss.value, g

    def train(self, records=None, batch=1 << 14, epochs=1, stream=None):
        """Adam steps on the given (pos, nrm, wo, wi, w) device tensors or on the record buffer."""
        loss = C.c_float()
        if records is None:
            call("rtpg_mlp_train", self.h, 0, None, None, None, None, None, int(batch), int(epochs), C.byref(loss),
                 stream_ptr(stream))
        else:
            pos, nrm, wo, wi, w = records
            call("rtpg_mlp_train", self.h, pos.shape[0], ptr(pos), ptr(nrm), ptr(wo), ptr(wi), ptr(w), int(batch),
                 int(epochs), C.byref(loss), stream_ptr(stream))
        return loss.value

    def records(self, clear=False, stream=None):
        c = C.c_uint32()
        call("rtpg_mlp_records", self.h, C.byref(c), int(bool(clear)), stream_ptr(stream))
        return c.value

    def status(self, clear=False, stream=None):
        s = C.c_uint32()
        call("rtpg_mlp_status", self.h, C.byref(s), int(bool(clear)), stream_ptr(stream))
        return s.value

    def set_wait_test(self, skip_mma, poll_limit=0):
        """Test mode of the bounded tensor-core waits: skip_mma=True issues no MMA, so every
        wait runs out after poll_limit polls and the kernels report RTPG_STATUS_TIMEOUT."""
        call("rtpg_mlp_set_wait_test", self.h, int(bool(skip_mma)), int(poll_limit))

    def record_views(self, n=None):
        """The first n records (default: all written, up to the capacity) as torch tensors that
        view the guide's record buffer: pos, nrm, wo, wi (n x 3), w and pdf (n), where pdf is the
        density the tracer sampled the record's direction with."""
        import torch
        n = min(self.records(), self.capacity) if n is None else int(n)
        ptrs = [C.c_void_p() for _ in range(6)]
        call("rtpg_mlp_record_arrays", self.h, *[C.byref(p) for p in ptrs[:5]])
        call("rtpg_mlp_record_pdfs", self.h, C.byref(ptrs[5]))

        class _View:
            def __init__(self, ptr, shape):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False),
                                                 "version": 3, "strides": None}

        out = []
        for p, k in zip(ptrs, (3, 3, 3, 3, 1, 1)):
            shape = (n, 3) if k == 3 else (n,)
            out.append(torch.as_tensor(_View(p.value, shape), device="cuda") if n > 0 else
                       torch.empty(shape, dtype=torch.float32, device="cuda"))
        return tuple(out)
