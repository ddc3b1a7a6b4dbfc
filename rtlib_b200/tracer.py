"""Host-side mirror of the integrator over the C ABI (rtpg_scene_*, rtpg_tracer_*).

``Scene`` owns the BVH of a triangle soup; ``Tracer`` plays the part of RTLib's test
application for one scene (RTLibExtOPX7TestApplication: Params, TracePipeline, accumulation);
``render`` is one launch with explicit PARAM_FLAG_* flags, ``render_guided`` the controller-
driven loop of the PG tracers; ``render_grid`` / ``render_grid_guided`` the same for the HT
tracers (hash grid + Morton quadtrees, SimpleGuide2.cu).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, ptr, stream_ptr

FLAG_NEE, FLAG_RIS, FLAG_USE_GRID, FLAG_USE_TREE, FLAG_BUILD, FLAG_FINAL, FLAG_LOCATE = 1, 2, 4, 8, 16, 32, 64
FLAG_USE_MLP = 128


class _Material(C.Structure):
    _fields_ = [("diffuse", C.c_float * 3), ("specular", C.c_float * 3), ("emission", C.c_float * 3),
                ("shininess", C.c_float), ("ref_index", C.c_float), ("type", C.c_int32), ("diffuse_texture", C.c_int32)]


class _Camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("u", C.c_float * 3), ("v", C.c_float * 3), ("w", C.c_float * 3)]


class _Desc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("max_depth", C.c_uint32),
                ("num_candidates", C.c_uint32), ("background", C.c_float * 3), ("seed", C.c_uint32),
                ("light_emission", C.POINTER(C.c_float))]


class Scene:
    """BVH over a triangle soup tri_v (nt, 9) float32 CUDA tensor."""

    def __init__(self, tri_v, stream=None):
        import torch
        self.tri_v = tri_v.contiguous()
        nt = self.tri_v.shape[0]
        self.indices = torch.arange(3 * nt, dtype=torch.int32, device=tri_v.device).view(nt, 3)
        h = C.c_void_p()
        call("rtpg_scene_create", ptr(self.tri_v), 3 * nt, ptr(self.indices), nt, stream_ptr(stream), C.byref(h))
        self.h = h
        self.ntris = nt

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_scene_destroy", self.h)
            self.h = None

    def intersect(self, org, dir, tmin=None, tmax=None, any_hit=False, out_t=None, out_prim=None, out_uv=None,
                  stream=None):
        call("rtpg_scene_intersect", self.h, int(org.shape[0]), ptr(org), ptr(dir), ptr(tmin), ptr(tmax),
             int(bool(any_hit)), ptr(out_t), ptr(out_prim), ptr(out_uv), stream_ptr(stream))


class Tracer:
    def __init__(self, scene_dict, device, max_depth=8, num_candidates=32, seed=1, background=(0.0, 0.0, 0.0),
                 width=None, height=None, textures=None):
        import torch
        s = scene_dict
        self.device = device
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.tri_v = T(s["tri_v"])
        self.tri_mat = T(s["tri_mat"].view(np.int32))
        self.tri_uv = T(s["tri_uv"])
        self.light_tris = T(s["light_tris"].view(np.int32))
        self.scene = Scene(self.tri_v)
        mats = (_Material * len(s["materials"]))()
        for i, m in enumerate(s["materials"]):
            mats[i].diffuse[:] = m["diffuse"]
            mats[i].specular[:] = m["specular"]
            mats[i].emission[:] = m["emission"]
            mats[i].shininess = m["shininess"]
            mats[i].ref_index = m["ref_index"]
            mats[i].type = m["type"]
            mats[i].diffuse_texture = m["texture"]
        cam = _Camera()
        for k in ("eye", "u", "v", "w"):
            getattr(cam, k)[:] = [float(x) for x in s["camera"][k]]
        self.width = int(width or s["width"])
        self.height = int(height or s["height"])
        emis = np.ascontiguousarray(s["light_emission"], np.float32)
        self._emis = emis
        desc = _Desc(self.width, self.height, int(max_depth), int(num_candidates),
                     (C.c_float * 3)(*background), int(seed), emis.ctypes.data_as(C.POINTER(C.c_float)))
        first = np.ascontiguousarray(s["light_first"], np.uint32)
        count = np.ascontiguousarray(s["light_count"], np.uint32)
        h = C.c_void_p()
        call("rtpg_tracer_create", self.scene.h, ptr(self.tri_v), ptr(self.tri_mat), ptr(self.tri_uv), mats,
             len(s["materials"]), ptr(self.light_tris), first.ctypes.data, count.ctypes.data, len(first),
             C.byref(cam), C.byref(desc), C.byref(h))
        self.h = h
        self.textures = {}
        for i, t in (textures or {}).items():
            self.set_texture(i, t)

    def __del__(self):
        if getattr(self, "h", None):
            call("rtpg_tracer_destroy", self.h)
            self.h = None

    def set_texture(self, index, rgb):
        """rgb: (h, w, 3) float32 CUDA tensor, kept referenced."""
        self.textures[index] = rgb
        call("rtpg_tracer_set_texture", self.h, int(index), int(rgb.shape[1]), int(rgb.shape[0]), ptr(rgb))

    def set_seed(self, seed):
        call("rtpg_tracer_set_seed", self.h, int(seed))

    def clear(self, stream=None):
        call("rtpg_tracer_clear", self.h, stream_ptr(stream))

    def render(self, spp, flags=FLAG_NEE, tree=None, stream=None):
        call("rtpg_tracer_render", self.h, int(spp), int(flags), tree.h if tree is not None else None,
             stream_ptr(stream))

    def render_guided(self, tree, controller, base_flags=FLAG_NEE, samples_per_launch=1, max_launches=1 << 30,
                      stream=None):
        call("rtpg_tracer_render_guided", self.h, tree.h, controller.h, int(base_flags), int(samples_per_launch),
             int(max_launches), stream_ptr(stream))

    def render_grid(self, spp, flags, grid, mqt, stream=None):
        call("rtpg_tracer_render_grid", self.h, int(spp), int(flags), grid.h, mqt.h, stream_ptr(stream))

    def render_grid_guided(self, grid, mqt, controller, base_flags=FLAG_NEE, samples_per_launch=1,
                           max_launches=1 << 30, stream=None):
        call("rtpg_tracer_render_grid_guided", self.h, grid.h, mqt.h, controller.h, int(base_flags),
             int(samples_per_launch), int(max_launches), stream_ptr(stream))

    def render_mlp(self, spp, flags, mlp, fraction=0.5, record_keep=1.0, fallback=None, mlp_share=0.5, stream=None):
        call("rtpg_tracer_render_mlp", self.h, int(spp), int(flags) | FLAG_USE_MLP, mlp.h,
             fallback.h if fallback is not None else None, float(fraction), float(mlp_share), float(record_keep),
             stream_ptr(stream))

    def set_light_emission(self, rgb):
        """rgb: (num_lights, 3) host array; NEE radiance and material emission of every light."""
        a = np.ascontiguousarray(rgb, np.float32).reshape(-1)
        call("rtpg_tracer_set_light_emission", self.h, a.ctypes.data, a.size // 3)

    def render_adjoint(self, spp, d_image, flags=FLAG_NEE, texture_index=-1, grad_texture=None, grad_light=None,
                       stream=None):
        """Adds d(loss)/d(texture texels) and d(loss)/d(light radiances) for a loss with gradient
        d_image w.r.t. the mean image of the spp samples rtpg_tracer_render would draw next."""
        call("rtpg_tracer_render_adjoint", self.h, int(spp), int(flags), ptr(d_image), int(texture_index),
             ptr(grad_texture), ptr(grad_light), stream_ptr(stream))

    def image(self, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty((self.height, self.width, 3), dtype=torch.float32, device=self.device)
        call("rtpg_tracer_image", self.h, ptr(out), stream_ptr(stream))
        return out

    def image64(self, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty((self.height, self.width, 3), dtype=torch.float64, device=self.device)
        call("rtpg_tracer_image_f64", self.h, ptr(out), stream_ptr(stream))
        return out

    def accumulation(self):
        """(device pointer of the FP64 accumulation, samples so far)."""
        p, s = C.c_void_p(), C.c_uint64()
        call("rtpg_tracer_accumulation", self.h, C.byref(p), C.byref(s))
        return p.value, s.value

    def counters(self, stream=None):
        a, b = C.c_uint64(), C.c_uint64()
        call("rtpg_tracer_counters", self.h, C.byref(a), C.byref(b), stream_ptr(stream))
        return {"path_bounces": a.value, "shadow_rays": b.value}

    def path_depths(self, stream=None):
        import torch
        out = torch.empty((self.height, self.width), dtype=torch.int32, device=self.device)
        call("rtpg_tracer_path_depths", self.h, ptr(out), stream_ptr(stream))
        return out

    def set_timing(self, enable):
        call("rtpg_tracer_set_timing", self.h, int(bool(enable)))

    def timings(self):
        """Summed device ms and launch counts of raygen / bounce / finish."""
        ms = np.zeros(3, np.float64)
        n = np.zeros(3, np.uint64)
        call("rtpg_tracer_timings", self.h, ms.ctypes.data, n.ctypes.data)
        return dict(zip(("raygen", "bounce", "finish"), zip(ms.tolist(), n.tolist())))

    def stats(self):
        a, b = C.c_uint64(), C.c_uint64()
        call("rtpg_tracer_stats", self.h, C.byref(a), C.byref(b))
        return {"samples": a.value, "paths": b.value}
