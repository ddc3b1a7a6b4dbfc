"""ctypes bindings to the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``    -- oracle/_build/liboracle.so, this project's C restatement (rtpg_oracle.c);
* ``Reference`` -- oracle/_ref/libref_rtlib.so, RTLib's own guiding code built on the host
                   (oracle/ref), available where the reference tree was present at build
                   time or where the prebuilt library travelled with the repository.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may import this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_rtlib.so")

_f = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64 = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
P = C.c_void_p


def build_oracle() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


def reference_tree() -> str:
    """Location of the RTLib source tree: $RTLIB_REFERENCE, else a checkout named
    ``reference`` beside this repository."""
    return os.environ.get("RTLIB_REFERENCE",
                          os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))


def build_reference() -> bool:
    """Build oracle/_ref from the reference tree when it is present.  Returns whether the
    library exists afterwards."""
    ref = reference_tree()
    if os.path.isdir(ref):
        subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={ref}"],
                              stdout=subprocess.DEVNULL)
    return os.path.exists(REF_SO)


def _opt(a, dtype):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=dtype).ctypes.data_as(P)


class _Export:
    def __init__(self, smask, scalars, counts, dmask, dsums):
        self.smask, self.scalars, self.counts, self.dmask, self.dsums = smask, scalars, counts, dmask, dsums

    @property
    def topology(self):
        return (self.smask.tobytes(), self.counts.tobytes(), self.dmask.tobytes())


class Oracle:
    """SD-tree / hash grid / Morton quadtree restated in C (rtpg_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = self.L = C.CDLL(ORACLE_SO)
        L.or_sdtree_new.restype = P
        L.or_sdtree_new.argtypes = [_f, _f, C.c_int, C.c_float, C.c_int, C.c_uint32]
        L.or_sdtree_free.argtypes = [P]
        L.or_sdtree_status.argtypes = [P]
        L.or_sdtree_status.restype = C.c_uint32
        L.or_sdtree_record.argtypes = [P, C.c_int64, _f, _f, _f, P, P, P]
        L.or_sdtree_build.argtypes = [P]
        L.or_sdtree_refine.argtypes = [P, C.c_uint64, C.c_int]
        L.or_sdtree_export.argtypes = [P, C.c_int, _i64]
        L.or_sdtree_export_copy.argtypes = [_u8, _f, _i64, _u8, _f]
        L.or_sdtree_sample_pdf.argtypes = [P, C.c_int64, _f, _u32, P, P, P, P]
        L.or_sdtree_pdf.argtypes = [P, C.c_int64, _f, _f, _f]
        L.or_sdtree_num_stree_nodes.argtypes = [P]
        L.or_sdtree_num_stree_nodes.restype = C.c_uint32
        L.or_sdtree_num_dtrees.argtypes = [P]
        L.or_sdtree_num_dtrees.restype = C.c_uint32
        L.or_pcg1d.argtypes = [C.c_uint32]
        L.or_pcg1d.restype = C.c_uint32
        L.or_dir_to_canonical.argtypes = [C.c_int64, _f, _f]
        L.or_hashgrid_insert.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u32, _u32]
        L.or_hashgrid_lookup.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u32, _u32]
        L.or_mhash_insert.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u64, _u32, P]
        L.or_mhash_lookup.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u64, _u32]
        L.or_morton3.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.or_morton3.restype = C.c_uint64
        L.or_morton2.argtypes = [C.c_uint32, C.c_uint32]
        L.or_morton2.restype = C.c_uint32
        L.or_mqt_record.argtypes = [C.c_int64, C.c_uint32, C.c_int, _i64, _u32, _f, _f, P]
        L.or_mqt_build.argtypes = [C.c_uint32, C.c_uint32, C.c_int, _i64, _f]
        L.or_mqt_sample_pdf.argtypes = [C.c_int64, C.c_uint32, _f, _u32, _u32, _f, _f, P]

    # ---- SD-tree
    def sdtree(self, aabb_min, aabb_max, max_dtree_depth=20, subdiv_th=0.01, frac_bits=24, node_cap=65535):
        return OracleSDTree(self, aabb_min, aabb_max, max_dtree_depth, subdiv_th, frac_bits, node_cap)

    def dir_to_canonical(self, d):
        d = np.ascontiguousarray(d, dtype=np.float32)
        out = np.empty((d.shape[0], 2), np.float32)
        self.L.or_dir_to_canonical(d.shape[0], d, out)
        return out

    # ---- hash grid (reference keying)
    def hashgrid_insert(self, pos, off, size, bounds, nslots, cur):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        self.L.or_hashgrid_insert(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                                  np.asarray(bounds, np.uint32), nslots, cur, out)
        return out

    def hashgrid_lookup(self, pos, off, size, bounds, nslots, prv):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        self.L.or_hashgrid_lookup(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                                  np.asarray(bounds, np.uint32), nslots, prv, out)
        return out

    # ---- hit queries
    def intersect(self, tri_v, org, dir, tmin=0.0, tmax=1e20, any_hit=False):
        """Brute-force closest (or any) hit of each ray over every triangle, in scene order:
        (t, prim), t = -1 and prim = 0xffffffff for a miss."""
        tri_v = np.ascontiguousarray(tri_v, np.float32)
        org, dir = np.ascontiguousarray(org, np.float32), np.ascontiguousarray(dir, np.float32)
        n = org.shape[0]
        t, prim = np.empty(n, np.float32), np.empty(n, np.uint32)
        self.L.or_intersect.argtypes = [_f, C.c_uint32, C.c_int64, _f, _f, C.c_float, C.c_float, C.c_int, _f, _u32]
        self.L.or_intersect(tri_v, tri_v.reshape(-1, 9).shape[0], n, org, dir, tmin, tmax, int(any_hit), t, prim)
        return t, prim

    def mhash_insert(self, pos, off, size, bounds, nslots, cur):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        keys = np.empty(pos.shape[0], np.uint64)
        self.L.or_mhash_insert(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                               np.asarray(bounds, np.uint32), nslots, cur, out, keys.ctypes.data_as(P))
        return out, keys

    def mhash_lookup(self, pos, off, size, bounds, nslots, prv):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        self.L.or_mhash_lookup(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                               np.asarray(bounds, np.uint32), nslots, prv, out)
        return out

    # ---- Morton quadtree
    def mqt_record(self, level, frac_bits, leaves, cell, uv, value):
        st = np.zeros(1, np.uint32)
        self.L.or_mqt_record(cell.shape[0], level, frac_bits, leaves, np.ascontiguousarray(cell, np.uint32),
                             np.ascontiguousarray(uv, np.float32), np.ascontiguousarray(value, np.float32),
                             st.ctypes.data_as(P))
        return int(st[0])

    def mqt_build(self, ncells, level, frac_bits, leaves):
        per = ((1 << (2 * (level + 1))) - 1) // 3
        pyr = np.empty(ncells * per, np.float32)
        self.L.or_mqt_build(ncells, level, frac_bits, leaves, pyr)
        return pyr

    def mqt_sample_pdf(self, level, pyramid, cell, seeds):
        n = cell.shape[0]
        uv = np.empty((n, 2), np.float32)
        pdf = np.empty(n, np.float32)
        pe = np.empty(n, np.float32)
        self.L.or_mqt_sample_pdf(n, level, pyramid, np.ascontiguousarray(cell, np.uint32),
                                 np.ascontiguousarray(seeds, np.uint32), uv, pdf, pe.ctypes.data_as(P))
        return uv, pdf, pe


class OracleSDTree:
    def __init__(self, o, mn, mx, max_depth, th, bits, cap):
        self.o, self.L = o, o.L
        self.h = self.L.or_sdtree_new(np.asarray(mn, np.float32), np.asarray(mx, np.float32), max_depth, th, bits, cap)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_sdtree_free(self.h)
            self.h = None

    def record(self, pos, uv, radiance, wo_pdf=None, stat_w=None, is_delta=None):
        pos = np.ascontiguousarray(pos, np.float32)
        self.L.or_sdtree_record(self.h, pos.shape[0], pos, np.ascontiguousarray(uv, np.float32),
                                np.ascontiguousarray(radiance, np.float32), _opt(wo_pdf, np.float32),
                                _opt(stat_w, np.float32), _opt(is_delta, np.uint8))

    def build(self):
        self.L.or_sdtree_build(self.h)

    def refine(self, spatial_th, max_mb=2000):
        self.L.or_sdtree_refine(self.h, int(spatial_th), int(max_mb))

    @property
    def status(self):
        return int(self.L.or_sdtree_status(self.h))

    def num_stree_nodes(self):
        return int(self.L.or_sdtree_num_stree_nodes(self.h))

    def num_dtrees(self):
        return int(self.L.or_sdtree_num_dtrees(self.h))

    def export(self, sampling=True):
        sz = np.zeros(5, np.int64)
        self.L.or_sdtree_export(self.h, int(sampling), sz)
        e = _Export(np.empty(sz[0], np.uint8), np.empty(sz[1] * 4, np.float32), np.empty(sz[1], np.int64),
                    np.empty(sz[2], np.uint8), np.empty(sz[2] * 4, np.float32))
        self.L.or_sdtree_export_copy(e.smask, e.scalars, e.counts, e.dmask, e.dsums)
        return e

    def sample_pdf(self, pos, seeds, with_dir=False):
        pos = np.ascontiguousarray(pos, np.float32)
        n = pos.shape[0]
        uv = np.empty((n, 2), np.float32)
        pdf = np.empty(n, np.float32)
        d = np.empty((n, 3), np.float32) if with_dir else None
        pd = np.empty(n, np.float32) if with_dir else None
        self.L.or_sdtree_sample_pdf(self.h, n, pos, np.ascontiguousarray(seeds, np.uint32), uv.ctypes.data_as(P),
                                    pdf.ctypes.data_as(P), _opt(d, np.float32) if with_dir else None,
                                    pd.ctypes.data_as(P) if with_dir else None)
        if with_dir:
            # _opt copies; use the buffers directly instead
            d2 = np.empty((n, 3), np.float32)
            pd2 = np.empty(n, np.float32)
            self.L.or_sdtree_sample_pdf(self.h, n, pos, np.ascontiguousarray(seeds, np.uint32), None, None,
                                        d2.ctypes.data_as(P), pd2.ctypes.data_as(P))
            return uv, pdf, d2, pd2
        return uv, pdf

    def pdf(self, pos, uv):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.float32)
        self.L.or_sdtree_pdf(self.h, pos.shape[0], pos, np.ascontiguousarray(uv, np.float32), out)
        return out


class Reference:
    """RTLib's own guiding code (oracle/_ref/libref_rtlib.so)."""

    def __init__(self):
        if not os.path.exists(REF_SO) and not build_reference():
            raise FileNotFoundError(REF_SO)
        L = self.L = C.CDLL(REF_SO)
        L.ref_sdtree_new.restype = P
        L.ref_sdtree_new.argtypes = [_f, _f]
        L.ref_sdtree_free.argtypes = [P]
        L.ref_sdtree_record.argtypes = [P, C.c_int64, _f, P, P, _f, P, P, P]
        L.ref_sdtree_build.argtypes = [P]
        L.ref_sdtree_refine.argtypes = [P, C.c_uint64, C.c_int, C.c_int, C.c_float]
        L.ref_sdtree_threshold.argtypes = [C.c_int, C.c_int]
        L.ref_sdtree_threshold.restype = C.c_uint64
        L.ref_sdtree_num_stree_nodes.argtypes = [P]
        L.ref_sdtree_num_stree_nodes.restype = C.c_int64
        L.ref_sdtree_export.argtypes = [P, C.c_int, _i64]
        L.ref_sdtree_export_copy.argtypes = [_u8, _f, _i64, _u8, _f]
        L.ref_sdtree_sample_pdf.argtypes = [P, C.c_int64, _f, _u32, P, P, P, P, C.c_int]
        L.ref_sdtree_pdf.argtypes = [P, C.c_int64, _f, _f, _f]
        L.ref_pcg1d.argtypes = [C.c_uint32]
        L.ref_pcg1d.restype = C.c_uint32
        L.ref_xxhash.argtypes = [C.c_uint32]
        L.ref_xxhash.restype = C.c_uint32
        L.ref_xorshift32_floats.argtypes = [C.c_uint32, C.c_int, _f, _u32]
        L.ref_dir_to_canonical.argtypes = [C.c_int64, _f, _f]
        L.ref_canonical_to_dir.argtypes = [C.c_int64, _f, _f]
        L.ref_hashgrid_insert.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u32, _u32]
        L.ref_hashgrid_lookup.argtypes = [C.c_int64, _f, _f, _f, _u32, C.c_uint32, _u32, _u32]
        L.ref_mqt_record.argtypes = [C.c_int64, C.c_uint32, C.c_uint32, _f, _u32, _f, _f]
        L.ref_mqt_build.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _f]
        L.ref_mqt_sample_pdf.argtypes = [C.c_int64, C.c_uint32, C.c_uint32, _f, _u32, _u32, _f, _f, P]
        L.ref_morton2_code.argtypes = [C.c_uint32, C.c_uint32]
        L.ref_morton2_code.restype = C.c_uint32

    def sdtree(self, mn, mx):
        return RefSDTree(self, mn, mx)

    def xorshift32_floats(self, seed, n):
        out = np.empty(n, np.float32)
        st = np.zeros(1, np.uint32)
        self.L.ref_xorshift32_floats(seed, n, out, st)
        return out, int(st[0])

    def dir_to_canonical(self, d):
        d = np.ascontiguousarray(d, dtype=np.float32)
        out = np.empty((d.shape[0], 2), np.float32)
        self.L.ref_dir_to_canonical(d.shape[0], d, out)
        return out

    def hashgrid_insert(self, pos, off, size, bounds, nslots, cur):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        self.L.ref_hashgrid_insert(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                                   np.asarray(bounds, np.uint32), nslots, cur, out)
        return out

    def hashgrid_lookup(self, pos, off, size, bounds, nslots, prv):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.uint32)
        self.L.ref_hashgrid_lookup(pos.shape[0], pos, np.asarray(off, np.float32), np.asarray(size, np.float32),
                                   np.asarray(bounds, np.uint32), nslots, prv, out)
        return out

    def mqt_record(self, level, weights, cell, uv, value):
        per = ((1 << (2 * (6 + 1))) - 1) // 3
        self.L.ref_mqt_record(cell.shape[0], level, per, weights, np.ascontiguousarray(cell, np.uint32),
                              np.ascontiguousarray(uv, np.float32), np.ascontiguousarray(value, np.float32))

    def mqt_build(self, ncells, level, weights):
        per = ((1 << (2 * (6 + 1))) - 1) // 3
        self.L.ref_mqt_build(ncells, level, per, weights)

    def mqt_sample_pdf(self, level, weights, cell, seeds):
        per = ((1 << (2 * (6 + 1))) - 1) // 3
        n = cell.shape[0]
        uv = np.empty((n, 2), np.float32)
        pdf = np.empty(n, np.float32)
        pe = np.empty(n, np.float32)
        self.L.ref_mqt_sample_pdf(n, level, per, weights, np.ascontiguousarray(cell, np.uint32),
                                  np.ascontiguousarray(seeds, np.uint32), uv, pdf, pe.ctypes.data_as(P))
        return uv, pdf, pe


class RefSDTree:
    def __init__(self, r, mn, mx):
        self.L = r.L
        self.h = self.L.ref_sdtree_new(np.asarray(mn, np.float32), np.asarray(mx, np.float32))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_sdtree_free(self.h)
            self.h = None

    def record(self, pos, uv=None, radiance=None, wo_pdf=None, stat_w=None, is_delta=None, dir_xyz=None):
        pos = np.ascontiguousarray(pos, np.float32)
        uvp = np.ascontiguousarray(uv, np.float32) if uv is not None else None
        dp = np.ascontiguousarray(dir_xyz, np.float32) if dir_xyz is not None else None
        wo = np.ascontiguousarray(wo_pdf, np.float32) if wo_pdf is not None else None
        sw = np.ascontiguousarray(stat_w, np.float32) if stat_w is not None else None
        dl = np.ascontiguousarray(is_delta, np.uint8) if is_delta is not None else None
        self.L.ref_sdtree_record(self.h, pos.shape[0], pos,
                                 uvp.ctypes.data_as(P) if uvp is not None else None,
                                 dp.ctypes.data_as(P) if dp is not None else None,
                                 np.ascontiguousarray(radiance, np.float32),
                                 wo.ctypes.data_as(P) if wo is not None else None,
                                 sw.ctypes.data_as(P) if sw is not None else None,
                                 dl.ctypes.data_as(P) if dl is not None else None)

    def build(self):
        self.L.ref_sdtree_build(self.h)

    def refine(self, spatial_th, max_mb=2000, max_dtree_depth=20, subdiv_th=0.01):
        self.L.ref_sdtree_refine(self.h, int(spatial_th), int(max_mb), int(max_dtree_depth), float(subdiv_th))

    def num_stree_nodes(self):
        return int(self.L.ref_sdtree_num_stree_nodes(self.h))

    def export(self, sampling=True):
        sz = np.zeros(5, np.int64)
        self.L.ref_sdtree_export(self.h, int(sampling), sz)
        e = _Export(np.empty(sz[0], np.uint8), np.empty(sz[1] * 4, np.float32), np.empty(sz[1], np.int64),
                    np.empty(sz[2], np.uint8), np.empty(sz[2] * 4, np.float32))
        self.L.ref_sdtree_export_copy(e.smask, e.scalars, e.counts, e.dmask, e.dsums)
        return e

    def sample_pdf(self, pos, seeds, threads=1, with_dir=False):
        pos = np.ascontiguousarray(pos, np.float32)
        n = pos.shape[0]
        uv = np.empty((n, 2), np.float32)
        pdf = np.empty(n, np.float32)
        d = np.empty((n, 3), np.float32)
        pd = np.empty(n, np.float32)
        self.L.ref_sdtree_sample_pdf(self.h, n, pos, np.ascontiguousarray(seeds, np.uint32), uv.ctypes.data_as(P),
                                     pdf.ctypes.data_as(P), d.ctypes.data_as(P) if with_dir else None,
                                     pd.ctypes.data_as(P) if with_dir else None, int(threads))
        if with_dir:
            return uv, pdf, d, pd
        return uv, pdf

    def pdf(self, pos, uv):
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty(pos.shape[0], np.float32)
        self.L.ref_sdtree_pdf(self.h, pos.shape[0], pos, np.ascontiguousarray(uv, np.float32), out)
        return out


# ------------------------------------------------------------------ integrator oracle
class _OMat(C.Structure):
    _fields_ = [("diffuse", C.c_float * 3), ("tex", C.c_int32), ("specular", C.c_float * 3), ("shininess", C.c_float),
                ("emission", C.c_float * 3), ("ref_index", C.c_float), ("type", C.c_int32), ("pad", C.c_int32 * 3)]


class _OScene(C.Structure):
    _fields_ = [("tri_v", P), ("tri_mat", P), ("tri_uv", P), ("ntris", C.c_uint32), ("mats", P), ("light_tris", P),
                ("light_first", P), ("light_count", P), ("light_emit", P), ("nlights", C.c_uint32), ("tex", P),
                ("tex_w", C.c_uint32), ("tex_h", C.c_uint32), ("eye", C.c_float * 3), ("cu", C.c_float * 3),
                ("cv", C.c_float * 3), ("cw", C.c_float * 3), ("bg", C.c_float * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("max_depth", C.c_uint32), ("num_candidates", C.c_uint32),
                ("fraction", C.c_float), ("tri_xf", P)]


def tracer_seeds(width, height, seed):
    """The per-pixel Xorshift32 seeds rtpg_tracer_clear derives: pcg1d(pcg1d(p) ^ seed*0x9E3779B9) | 1."""
    def pcg(x):
        state = (x * np.uint64(747796405) + np.uint64(2891336453)) & np.uint64(0xFFFFFFFF)
        word = (((state >> ((state >> np.uint64(28)) + np.uint64(4))) ^ state) * np.uint64(277803737)) & np.uint64(0xFFFFFFFF)
        return ((word >> np.uint64(22)) ^ word) & np.uint64(0xFFFFFFFF)
    p = np.arange(width * height, dtype=np.uint64)
    s = np.uint64((seed * 0x9E3779B9) & 0xFFFFFFFF)
    return (pcg(pcg(p) ^ s) | np.uint64(1)).astype(np.uint32)


class OracleRenderer:
    """CPU restatement of the guided integrator (rtpg_oracle.c, or_render) for small scenes."""

    def __init__(self, oracle, scene, max_depth=8, num_candidates=32, seed=1, fraction=0.3, width=None, height=None,
                 texture=None, background=(0.0, 0.0, 0.0)):
        L = self.L = oracle.L
        L.or_render.argtypes = [P, C.c_uint32, P, P, C.c_uint32, C.c_uint32, _u32, np.ctypeslib.ndpointer(np.float64)]
        L.or_render.restype = C.c_int64
        s = scene
        self.keep = {k: np.ascontiguousarray(s[k]) for k in ("tri_v", "tri_mat", "tri_uv", "light_tris", "light_first",
                                                             "light_count", "light_emission")}
        mats = (_OMat * len(s["materials"]))()
        for i, m in enumerate(s["materials"]):
            mats[i].diffuse[:] = m["diffuse"]
            mats[i].specular[:] = m["specular"]
            mats[i].emission[:] = m["emission"]
            mats[i].shininess = m["shininess"]
            mats[i].ref_index = m["ref_index"]
            mats[i].type = m["type"]
            mats[i].tex = m["texture"]
        self.mats = mats
        o = self.sc = _OScene()
        k = self.keep
        o.tri_v, o.tri_mat, o.tri_uv = k["tri_v"].ctypes.data, k["tri_mat"].ctypes.data, k["tri_uv"].ctypes.data
        o.ntris = k["tri_v"].shape[0]
        # the triangles' world -> triangle-frame rows the hit test uses (or_tri_transforms)
        L.or_tri_transforms.argtypes = [P, C.c_uint32, P]
        xf = self.keep["tri_xf"] = np.empty((max(o.ntris, 1), 12), np.float32)
        L.or_tri_transforms(o.tri_v, o.ntris, xf.ctypes.data)
        o.tri_xf = xf.ctypes.data
        o.mats = C.cast(mats, P)
        o.light_tris, o.light_first = k["light_tris"].ctypes.data, k["light_first"].ctypes.data
        o.light_count, o.light_emit = k["light_count"].ctypes.data, k["light_emission"].ctypes.data
        o.nlights = k["light_first"].shape[0]
        if texture is not None:
            self.tex = np.ascontiguousarray(texture, np.float32)
            o.tex, o.tex_h, o.tex_w = self.tex.ctypes.data, self.tex.shape[0], self.tex.shape[1]
        cam = s["camera"]
        o.eye[:], o.cu[:], o.cv[:], o.cw[:] = (list(map(float, cam[x])) for x in ("eye", "u", "v", "w"))
        o.bg[:] = list(background)
        o.width, o.height = int(width or s["width"]), int(height or s["height"])
        o.max_depth, o.num_candidates, o.fraction = max_depth, num_candidates, fraction
        self.width, self.height = o.width, o.height
        self.seeds = tracer_seeds(o.width, o.height, seed)
        self.accum = np.zeros(3 * o.width * o.height, np.float64)
        self.samples = 0

    def render(self, spp, flags, tree=None, grid=None, threads=1):
        """spp samples per pixel.  threads > 1 splits every frame into bands of pixels rendered
        on that many host threads; an SD-tree then receives each band's records in a private
        shadow that is merged into it exactly after the frame (grid guides stay single-threaded)."""
        npx = self.width * self.height
        if threads <= 1 or grid is not None:
            for _ in range(spp):
                self.L.or_render(C.byref(self.sc), int(flags), tree.h if tree is not None else None,
                                 C.byref(grid.g) if grid is not None else None, 0, npx, self.seeds, self.accum)
            self.samples += spp
            return
        import concurrent.futures as cf
        L = self.L
        L.or_sdtree_shadow_new.argtypes = [P]
        L.or_sdtree_shadow_new.restype = P
        L.or_sdtree_shadow_merge.argtypes = [P, P]
        bands = [(npx * k // threads, npx * (k + 1) // threads) for k in range(threads)]
        with cf.ThreadPoolExecutor(threads) as ex:
            for _ in range(spp):
                shadows = [L.or_sdtree_shadow_new(tree.h) if tree is not None else None for _ in bands]

                def one(k):
                    a, b = bands[k]
                    L.or_render(C.byref(self.sc), int(flags), shadows[k], None, a, b, self.seeds, self.accum)

                list(ex.map(one, range(threads)))
                if tree is not None:
                    for sh in shadows:
                        L.or_sdtree_shadow_merge(tree.h, sh)
        self.samples += spp

    def image(self):
        return (self.accum / max(self.samples, 1)).reshape(self.height, self.width, 3).astype(np.float32)

    def restart(self, seed=1):
        """Zero the accumulation and restart the per-pixel streams (rtpg_tracer_clear)."""
        self.seeds = tracer_seeds(self.width, self.height, seed)
        self.accum[:] = 0
        self.samples = 0

    def set_light_emission(self, rgb, light_material_first):
        """Emitter radiances for NEE and the emissive materials light i = material first + i."""
        rgb = np.asarray(rgb, np.float32).reshape(-1, 3)
        self.keep["light_emission"][:] = rgb.reshape(-1)
        for i, c in enumerate(rgb):
            self.mats[light_material_first + i].emission[:] = [float(x) for x in c]

    def render_guided(self, tree, budget, ratio_for_budget=1.0, iteration_for_built=0, base_flags=1, threads=1):
        """RTSTreeControllerT::BegTrace / EndTrace (OPX7UtilsPathGuiding.h:1808-1887) with one
        sample per launch, flags by state as the application sets them."""
        remain, pas, per_all, per_tmp, it = budget, 0, 0, 0, 0
        while True:
            if per_tmp == 0:
                remain -= pas
                pas = min(remain, 1 << it)
                if remain - pas < 2 * pas or per_all >= ratio_for_budget * budget:
                    pas = remain
                if remain > pas and it > 0:
                    tree.refine(int(np.sqrt(2.0 ** it * pas / 4.0) * 4000), 2000)
            flags = (base_flags & 3) | 8
            if it > iteration_for_built:
                flags |= 16 if remain > pas else 16 | 32
            self.render(1, flags, tree, threads=threads)
            per_all += 1
            per_tmp += 1
            if per_tmp >= pas:
                tree.build()
                it += 1
                per_tmp = 0
            if per_all > budget:
                break

    def render_grid_guided(self, grid, budget, iteration_for_built=3, iteration_for_locate=0, ratio_for_budget=0.3,
                           base_flags=1, max_launches=1 << 30):
        """RTMortonQuadTreeControllerT::BegTrace / EndTrace (OPX7UtilsMorton.h:818-922) with one
        sample per launch, flags by state and the hash grid's current -> previous copy after
        every finished pass, as TracePipeline does for the HT tracers
        (RTLibExtOPX7TestApplication.cpp:2174-2222)."""
        grid.clear_trees()
        remain = ((budget - 1 + 1) // 1) * 1
        pas, per_all, per_tmp, it = 0, 0, 0, 0
        for _ in range(max_launches):
            if per_tmp == 0:
                remain -= pas
                pas = min(remain, 1 << it)
                if remain - pas < 2 * pas or per_all >= ratio_for_budget * budget:
                    pas = remain
            flags = (base_flags & 3) | 4
            if it > iteration_for_built:
                flags |= 16 if remain > pas else 16 | 32
            elif not it > iteration_for_locate:
                flags |= 64
            self.render(1, flags, grid=grid)
            per_all += 1
            per_tmp += 1
            if per_tmp >= pas:
                it += 1
                if it > iteration_for_built:
                    grid.update()
                per_tmp = 0
            if per_tmp == 0:
                grid.swap()
            if per_all > budget:
                break


class _OGrid(C.Structure):
    _fields_ = [("off", C.c_float * 3), ("size", C.c_float * 3), ("bounds", C.c_uint32 * 3), ("nslots", C.c_uint32),
                ("keying", C.c_int32), ("cur", P), ("prv", P), ("level", C.c_uint32), ("bits", C.c_int32),
                ("leaves", P), ("pyramid", P), ("fraction", C.c_float), ("status", C.c_uint32)]


class OracleGrid:
    """Hash grid (current / previous tables of 64-bit keys) with one Morton quadtree per slot,
    the state of the HT tracers (DoubleBufferedHashGrid3Buffer + RTMortonQuadTreeWrapperT)."""

    def __init__(self, oracle, aabb_min, aabb_max, bounds, nslots, keying=0, level=4, fraction=0.3, frac_bits=24):
        self.o = oracle
        self.nslots, self.level, self.bits = int(nslots), int(level), int(frac_bits)
        self.cur = np.zeros(self.nslots, np.uint64)
        self.prv = np.zeros(self.nslots, np.uint64)
        self.per = ((1 << (2 * (self.level + 1))) - 1) // 3
        self.leaves = np.zeros(self.nslots << (2 * self.level), np.int64)
        self.pyramid = np.zeros(self.nslots * self.per, np.float32)
        g = self.g = _OGrid()
        g.off[:] = [float(v) for v in aabb_min]
        g.size[:] = [float(np.float32(b) - np.float32(a)) for a, b in zip(aabb_min, aabb_max)]
        g.bounds[:] = [int(b) for b in bounds]
        g.nslots, g.keying = self.nslots, int(keying)
        g.cur, g.prv = self.cur.ctypes.data, self.prv.ctypes.data
        g.level, g.bits = self.level, self.bits
        g.leaves, g.pyramid = self.leaves.ctypes.data, self.pyramid.ctypes.data
        g.fraction = float(fraction)

    def clear(self):
        self.cur[:] = 0
        self.prv[:] = 0

    def clear_trees(self):
        self.leaves[:] = 0
        self.pyramid[:] = 0

    def swap(self):
        self.prv[:] = self.cur

    def update(self):
        self.pyramid[:] = self.o.mqt_build(self.nslots, self.level, self.bits, self.leaves)
        self.leaves[:] = 0

    @property
    def status(self):
        return self.g.status


# ------------------------------------------------------------------ integrator known answers
class IntegratorKAT:
    """The integrator's building blocks one call at a time, on the C restatement (``Oracle``)
    or on RTLib's own code run on the host (``Reference``): cosine and Phong lobe sampling,
    random_in_unit_triangle, Reservoir::Update, MeshLightList::Sample and the whole
    closest-hit shading of a vertex.  Xorshift32 seeds go in, end states come out."""

    def __init__(self, checker, scene, max_depth=8, num_candidates=32, fraction=0.5):
        self.ref = isinstance(checker, Reference)
        self.L = L = checker.L
        self.max_depth, self.num_candidates, self.fraction = max_depth, num_candidates, fraction
        pre = "ref_kat_" if self.ref else "or_kat_"
        self.fn = {k: getattr(L, pre + k) for k in ("cosine", "phong", "triangle", "reservoir", "light", "shade")}
        for k in ("cosine", "triangle"):
            self.fn[k].argtypes = [C.c_int64, _f, _u32, _f]
        self.fn["phong"].argtypes = [C.c_int64, _f, _f, _u32, _f]
        self.fn["reservoir"].argtypes = [C.c_int64, C.c_int32, _f, _f, np.ctypeslib.ndpointer(np.int32), _f, _u32]
        case = [C.c_int64, _f, _f, _f, _u32, _f, _u32, _u32, _u32, _f, _u32]
        if self.ref:
            self.fn["light"].argtypes = [C.c_int64, _f, _u32, _f]
            self.fn["shade"].argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, P, C.c_float] + case
            mats = scene["materials"]
            mf = np.array([[*m["diffuse"], *m["specular"], *m["emission"], m["shininess"], m["ref_index"]]
                           for m in mats], np.float32)
            mt = np.array([m["type"] for m in mats], np.int32)
            L.ref_kat_set_scene.argtypes = [_f, C.c_uint32, _u32, _f, np.ctypeslib.ndpointer(np.int32), C.c_uint32,
                                            _u32, _u32, _u32, _f, C.c_uint32]
            tv = np.ascontiguousarray(scene["tri_v"], np.float32)
            L.ref_kat_set_scene(tv, tv.shape[0], np.ascontiguousarray(scene["tri_mat"], np.uint32), mf, mt, len(mats),
                                np.ascontiguousarray(scene["light_tris"], np.uint32),
                                np.ascontiguousarray(scene["light_first"], np.uint32),
                                np.ascontiguousarray(scene["light_count"], np.uint32),
                                np.ascontiguousarray(scene["light_emission"], np.float32), len(scene["light_first"]))
        else:
            self.fn["light"].argtypes = [P, C.c_int64, _f, _u32, _f]
            self.fn["shade"].argtypes = [P, C.c_uint32, P] + case
            self.r = OracleRenderer(checker, scene, max_depth=max_depth, num_candidates=num_candidates,
                                    fraction=fraction, width=1, height=1)

    @staticmethod
    def _a(x, t):
        return np.ascontiguousarray(x, t)

    def cosine(self, normal, seeds):
        st = self._a(seeds, np.uint32).copy()
        out = np.empty((st.shape[0], 3), np.float32)
        self.fn["cosine"](st.shape[0], self._a(normal, np.float32), st, out)
        return out, st

    def phong(self, refl, shininess, seeds):
        st = self._a(seeds, np.uint32).copy()
        out = np.empty((st.shape[0], 3), np.float32)
        self.fn["phong"](st.shape[0], self._a(refl, np.float32), self._a(shininess, np.float32), st, out)
        return out, st

    def triangle(self, verts, seeds):
        st = self._a(seeds, np.uint32).copy()
        out = np.empty((st.shape[0], 3), np.float32)
        self.fn["triangle"](st.shape[0], self._a(verts, np.float32), st, out)
        return out, st

    def reservoir(self, w, rnd):
        w, rnd = self._a(w, np.float32), self._a(rnd, np.float32)
        k = w.shape[0]
        sel, ws, m = np.empty(k, np.int32), np.empty(k, np.float32), np.empty(k, np.uint32)
        self.fn["reservoir"](k, w.shape[1], w, rnd, sel, ws, m)
        return sel, ws, m

    def light(self, p_in, seeds):
        st = self._a(seeds, np.uint32).copy()
        out = np.empty((st.shape[0], 14), np.float32)
        if self.ref:
            self.fn["light"](st.shape[0], self._a(p_in, np.float32), st, out)
        else:
            self.fn["light"](C.byref(self.r.sc), st.shape[0], self._a(p_in, np.float32), st, out)
        return out, st

    def shade(self, flags, cases, tree=None):
        """cases: org, dir (n x 3), t, prim, thr (n x 3), pflags, depth, seeds.  Returns the 17
        floats per case (position, direction, throughput after, BSDF value, radiance added,
        cosine, woPdf), the hit flags and the end states.  tree: a matching RefSDTree or
        OracleSDTree for USE_TREE."""
        c = cases
        st = self._a(c["seeds"], np.uint32).copy()
        n = st.shape[0]
        out, fl = np.empty((n, 17), np.float32), np.empty(n, np.uint32)
        args = (n, self._a(c["org"], np.float32), self._a(c["dir"], np.float32), self._a(c["t"], np.float32),
                self._a(c["prim"], np.uint32), self._a(c["thr"], np.float32), self._a(c["pflags"], np.uint32),
                self._a(c["depth"], np.uint32), st, out, fl)
        th = tree.h if tree is not None else None
        if self.ref:
            self.fn["shade"](int(flags), self.max_depth, self.num_candidates, th, self.fraction, *args)
        else:
            self.fn["shade"](C.byref(self.r.sc), int(flags), th, *args)
        return out, fl, st
