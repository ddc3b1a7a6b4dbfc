"""Host-side mirrors of RTLib's hash grid and Morton quadtree over the C ABI.

``HashGrid`` stands for DoubleBufferedHashGrid3Buffer (RTLibExtOPX7Test.h:1472-1570) with the
device routines DoubleBufferedHashGrid3T::FindFromCur / FindFromPrv batched;
``MortonQuadTrees`` for RTMortonQuadTreeWrapperT (OPX7UtilsMorton.h:590-764) with
MortonQuadTreeWrapperT::Record / SampleAndPdf / Pdf batched and the pyramid build;
``MortonQuadTreeController`` for RTMortonQuadTreeControllerT (OPX7UtilsMorton.h:766-993).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr, stream_ptr

KEY_REFERENCE, KEY_MORTON = 0, 1


class HashGrid:
    def __init__(self, aabb_min, aabb_max, bounds, num_slots, keying=KEY_REFERENCE, max_batch=0):
        mn = (C.c_float * 3)(*[float(v) for v in aabb_min])
        mx = (C.c_float * 3)(*[float(v) for v in aabb_max])
        b = (C.c_uint32 * 3)(*[int(v) for v in bounds])
        h = C.c_void_p()
        call("rtpg_hashgrid_create", mn, mx, b, int(num_slots), int(keying), int(max_batch), C.byref(h))
        self.h = h
        self.num_slots = int(num_slots)

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_hashgrid_destroy", self.h)
            self.h = None

    def clear(self, stream=None):
        call("rtpg_hashgrid_clear", self.h, stream_ptr(stream))

    def swap(self, stream=None):
        call("rtpg_hashgrid_swap", self.h, stream_ptr(stream))

    def insert(self, pos, out_slot, out_key=None, stream=None):
        call("rtpg_hashgrid_insert", self.h, int(pos.shape[0]), ptr(pos), ptr(out_slot), ptr(out_key),
             stream_ptr(stream))

    def lookup(self, pos, out_slot, stream=None):
        call("rtpg_hashgrid_lookup", self.h, int(pos.shape[0]), ptr(pos), ptr(out_slot), stream_ptr(stream))

    def cells(self, pos, out_cell=None, out_key=None, stream=None):
        call("rtpg_hashgrid_cells", self.h, int(pos.shape[0]), ptr(pos), ptr(out_cell), ptr(out_key),
             stream_ptr(stream))

    def export(self, previous=False, stream=None):
        t = np.empty(self.num_slots, np.uint64)
        call("rtpg_hashgrid_export", self.h, int(previous), t.ctypes.data, stream_ptr(stream))
        return t

    def status(self, clear=False, stream=None):
        s = C.c_uint32()
        call("rtpg_hashgrid_status", self.h, C.byref(s), int(clear), stream_ptr(stream))
        return s.value


NOALLOC_MAX_POINTS = 1 << 16


def insert_noalloc(aabb_min, aabb_max, bounds, table, pos, out_slot, keying=KEY_REFERENCE, status=None, stream=None):
    """Batch insert without any device allocation (rtpg_hashgrid_insert_noalloc).

    For callers that cannot allocate device memory -- an application that owns every
    allocation under a fixed budget, work enqueued while the stream is being captured into a
    CUDA graph, or a real-time loop that must not block in the allocator.  `table` is the
    caller's current table (uint64 keys, num_slots entries, zero = empty), updated in place.
    At most NOALLOC_MAX_POINTS points per call.  Calls share one fixed scratch array on the
    device, so overlapping calls must be ordered by the caller."""
    mn = (C.c_float * 3)(*[float(v) for v in aabb_min])
    mx = (C.c_float * 3)(*[float(v) for v in aabb_max])
    b = (C.c_uint32 * 3)(*[int(v) for v in bounds])
    call("rtpg_hashgrid_insert_noalloc", mn, mx, b, int(table.shape[0]), int(keying), ptr(table), ptr(status),
         int(pos.shape[0]), ptr(pos), ptr(out_slot), stream_ptr(stream))


class MortonQuadTrees:
    def __init__(self, num_cells, level=6, fraction=0.3, fixed_point_bits=0):
        h = C.c_void_p()
        call("rtpg_mqt_create", int(num_cells), int(level), float(fraction), int(fixed_point_bits), C.byref(h))
        self.h = h
        self.num_cells, self.level = int(num_cells), int(level)

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_mqt_destroy", self.h)
            self.h = None

    @property
    def per_cell(self):
        return ((1 << (2 * (self.level + 1))) - 1) // 3

    def clear(self, stream=None):
        call("rtpg_mqt_clear", self.h, stream_ptr(stream))

    def record(self, cell, dir, value, canonical=None, stream=None):
        if canonical is None:
            canonical = dir.shape[-1] == 2
        call("rtpg_mqt_record", self.h, int(cell.shape[0]), ptr(cell), ptr(dir), int(bool(canonical)), ptr(value),
             stream_ptr(stream))

    def update(self, stream=None):
        call("rtpg_mqt_update", self.h, stream_ptr(stream))

    def sample_pdf(self, cell, seeds=None, seed_base=0, out_uv=None, out_pdf=None, out_dir=None, out_pdf_tree=None,
                   stream=None):
        call("rtpg_mqt_sample_pdf", self.h, int(cell.shape[0]), ptr(cell), ptr(seeds), int(seed_base), ptr(out_uv),
             ptr(out_pdf), ptr(out_dir), ptr(out_pdf_tree), stream_ptr(stream))

    def pdf(self, cell, dir, out, canonical=None, tree_level=False, stream=None):
        if canonical is None:
            canonical = dir.shape[-1] == 2
        call("rtpg_mqt_pdf", self.h, int(cell.shape[0]), ptr(cell), ptr(dir), int(bool(canonical)), ptr(out),
             int(bool(tree_level)), stream_ptr(stream))

    def export(self, stream=None):
        leaves = np.empty(self.num_cells << (2 * self.level), np.int64)
        pyr = np.empty(self.num_cells * self.per_cell, np.float32)
        call("rtpg_mqt_export", self.h, leaves.ctypes.data, pyr.ctypes.data, stream_ptr(stream))
        return leaves, pyr

    def status(self, clear=False, stream=None):
        s = C.c_uint32()
        call("rtpg_mqt_status", self.h, C.byref(s), int(clear), stream_ptr(stream))
        return s.value


TRACE_RECORD, TRACE_RECORD_AND_SAMPLE, TRACE_SAMPLE, TRACE_LOCATE = 0, 1, 2, 3


class MortonQuadTreeController:
    """The doubling pass schedule of the hash-grid guide, with the LOCATE phase."""

    def __init__(self, trees, sample_for_budget, iteration_for_built=3, iteration_for_locate=0,
                 ratio_for_budget=0.3, samples_per_launch=1):
        h = C.c_void_p()
        call("rtpg_mqt_controller_create", trees.h, int(sample_for_budget), int(iteration_for_built),
             int(iteration_for_locate), float(ratio_for_budget), int(samples_per_launch), C.byref(h))
        self.h = h
        self.trees = trees

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_mqt_controller_destroy", self.h)
            self.h = None

    def start(self):
        call("rtpg_mqt_controller_start", self.h)

    def begin(self, stream=None):
        call("rtpg_mqt_controller_begin", self.h, stream_ptr(stream))

    def end(self, stream=None):
        call("rtpg_mqt_controller_end", self.h, stream_ptr(stream))

    def get(self):
        st, it, tmp, ex = C.c_int32(), C.c_uint32(), C.c_uint32(), C.c_int32()
        call("rtpg_mqt_controller_get", self.h, C.byref(st), C.byref(it), C.byref(tmp), C.byref(ex))
        return {"state": st.value, "iteration": it.value, "samples_in_pass": tmp.value, "executing": bool(ex.value)}
