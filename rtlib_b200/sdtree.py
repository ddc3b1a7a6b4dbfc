"""Host-side mirror of RTLib's SD-tree API over the C ABI.

``SDTree`` plays the part of RTSTreeWrapperT (OPX7UtilsPathGuiding.h:1333-1767) and
``SDTreeController`` that of RTSTreeControllerT (:1769-1920); the batch calls stand in for
the device routines the reference's OptiX programs call per hit (Record, Sample, Pdf).
Arrays are CUDA tensors (float32 / uint32 / uint8, contiguous); every call is asynchronous
on the current torch stream unless a stream is passed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr, stream_ptr

TRACE_RECORD, TRACE_RECORD_AND_SAMPLE, TRACE_SAMPLE = 0, 1, 2


class _Caps(C.Structure):
    _fields_ = [("max_stree_nodes", C.c_uint32), ("max_dtrees", C.c_uint32),
                ("max_dtree_nodes_total", C.c_uint32), ("fixed_point_bits", C.c_int32)]


class Export:
    """Canonical pre-order streams of a tree (see rtpg_sdtree_export)."""

    def __init__(self, smask, scalars, counts, dmask, dsums):
        self.smask, self.scalars, self.counts, self.dmask, self.dsums = smask, scalars, counts, dmask, dsums

    @property
    def topology(self):
        return (self.smask.tobytes(), self.counts.tobytes(), self.dmask.tobytes())


class SDTree:
    """RTSTreeWrapperT(ctx, aabbMin, aabbMax, maxDTreeDepth=20, fraction=0.3)."""

    def __init__(self, aabb_min, aabb_max, max_dtree_depth=20, fraction=0.3, max_stree_nodes=0, max_dtrees=0,
                 max_dtree_nodes_total=0, fixed_point_bits=0):
        caps = _Caps(max_stree_nodes, max_dtrees, max_dtree_nodes_total, fixed_point_bits)
        mn = (C.c_float * 3)(*[float(v) for v in aabb_min])
        mx = (C.c_float * 3)(*[float(v) for v in aabb_max])
        h = C.c_void_p()
        call("rtpg_sdtree_create", mn, mx, int(max_dtree_depth), float(fraction), C.byref(caps), C.byref(h))
        self.h = h
        self.fraction = fraction

    def close(self):
        if getattr(self, "h", None):
            call("rtpg_sdtree_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- RTSTreeWrapperT::Clear / Reset / Build
    def clear(self, stream=None):
        call("rtpg_sdtree_clear", self.h, stream_ptr(stream))

    def reset(self, iteration, samples_per_pass, stream=None):
        call("rtpg_sdtree_reset", self.h, int(iteration), int(samples_per_pass), stream_ptr(stream))

    def refine(self, spatial_threshold, max_mb=2000, dtree_subdiv_th=0.01, stream=None):
        call("rtpg_sdtree_refine", self.h, int(spatial_threshold), int(max_mb), float(dtree_subdiv_th),
             stream_ptr(stream))

    def build(self, stream=None):
        call("rtpg_sdtree_build", self.h, stream_ptr(stream))

    # --- device routines, batched
    def record(self, pos, dir, radiance, wo_pdf=None, stat_weight=None, is_delta=None, canonical=None, stream=None):
        n = pos.shape[0]
        if canonical is None:
            canonical = dir.shape[-1] == 2
        call("rtpg_sdtree_record", self.h, int(n), ptr(pos), ptr(dir), int(bool(canonical)), ptr(radiance),
             ptr(wo_pdf), ptr(stat_weight), ptr(is_delta), stream_ptr(stream))

    def sample_pdf(self, pos, seeds=None, seed_base=0, out_uv=None, out_pdf_uv=None, out_dir=None, out_pdf_dir=None,
                   stream=None):
        call("rtpg_sdtree_sample_pdf", self.h, int(pos.shape[0]), ptr(pos), ptr(seeds), int(seed_base), ptr(out_uv),
             ptr(out_pdf_uv), ptr(out_dir), ptr(out_pdf_dir), stream_ptr(stream))

    def pdf(self, pos, dir, out, canonical=None, stream=None):
        if canonical is None:
            canonical = dir.shape[-1] == 2
        call("rtpg_sdtree_pdf", self.h, int(pos.shape[0]), ptr(pos), ptr(dir), int(bool(canonical)), ptr(out),
             stream_ptr(stream))

    # --- inspection
    def stats(self, stream=None):
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        call("rtpg_sdtree_stats", self.h, C.byref(a), C.byref(b), C.byref(c), stream_ptr(stream))
        return {"stree_nodes": a.value, "dtrees": b.value, "dtree_nodes": c.value}

    def status(self, clear=False, stream=None):
        s = C.c_uint32()
        call("rtpg_sdtree_status", self.h, C.byref(s), int(clear), stream_ptr(stream))
        return s.value

    def memory_footprint(self):
        b = C.c_uint64()
        call("rtpg_sdtree_memory_footprint", self.h, C.byref(b))
        return b.value

    def export(self, sampling=True, stream=None):
        sizes = np.zeros(3, np.int64)
        call("rtpg_sdtree_export", self.h, int(sampling), sizes.ctypes.data, None, None, None, None, None,
             stream_ptr(stream))
        e = Export(np.empty(sizes[0], np.uint8), np.empty(sizes[1] * 4, np.float32), np.empty(sizes[1], np.int64),
                   np.empty(sizes[2], np.uint8), np.empty(sizes[2] * 4, np.float32))
        call("rtpg_sdtree_export", self.h, int(sampling), sizes.ctypes.data, e.smask.ctypes.data,
             e.scalars.ctypes.data, e.counts.ctypes.data, e.dmask.ctypes.data, e.dsums.ctypes.data,
             stream_ptr(stream))
        return e

    def import_(self, building: Export, sampling: Export, stream=None):
        """Replace the tree with the one two exports (building, sampling) describe."""
        b, s = building, sampling
        if b.smask.tobytes() != s.smask.tobytes() or b.counts.shape != s.counts.shape:
            raise ValueError("building and sampling exports describe different spatial trees")
        a = lambda x, t: np.ascontiguousarray(x, t)
        smask, scal = a(s.smask, np.uint8), a(s.scalars, np.float32)
        bc, bm, bs = a(b.counts, np.int64), a(b.dmask, np.uint8), a(b.dsums, np.float32)
        sc, sm, ss = a(s.counts, np.int64), a(s.dmask, np.uint8), a(s.dsums, np.float32)
        call("rtpg_sdtree_import", self.h, int(smask.shape[0]), int(sc.shape[0]), smask.ctypes.data, scal.ctypes.data,
             int(bm.shape[0]), bc.ctypes.data, bm.ctypes.data, bs.ctypes.data, int(sm.shape[0]), sc.ctypes.data,
             sm.ctypes.data, ss.ctypes.data, stream_ptr(stream))


class SDTreeController:
    """RTSTreeControllerT(tree, sampleForBudget, iterationForBuilt=0, ratioForBudget=0.5,
    samplePerLaunch=1): Start / BegTrace / EndTrace / GetState / GetIteration."""

    def __init__(self, tree: SDTree, sample_for_budget, iteration_for_built=0, ratio_for_budget=0.5,
                 samples_per_launch=1):
        self.tree = tree
        h = C.c_void_p()
        call("rtpg_controller_create", tree.h, int(sample_for_budget), int(iteration_for_built),
             float(ratio_for_budget), int(samples_per_launch), C.byref(h))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_controller_destroy", self.h)
            self.h = None

    def start(self):
        call("rtpg_controller_start", self.h)

    def begin(self, stream=None):
        call("rtpg_controller_begin", self.h, stream_ptr(stream))

    def end(self, stream=None):
        call("rtpg_controller_end", self.h, stream_ptr(stream))

    def get(self):
        st, it, sp, ex = C.c_int32(), C.c_uint32(), C.c_uint32(), C.c_int32()
        call("rtpg_controller_get", self.h, C.byref(st), C.byref(it), C.byref(sp), C.byref(ex))
        return {"state": st.value, "iteration": it.value, "samples_in_pass": sp.value, "executing": bool(ex.value)}
