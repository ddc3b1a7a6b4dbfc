"""Loader of the native library (rtlib_b200/librtpg.so) and ctypes signatures of the C ABI
declared in include/rtpg.h.  There is no fallback: if the library is missing or fails to
load, every entry point raises."""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtpg.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "rtpg.h")

P = C.c_void_p
I32, U32, I64, U64, F32 = C.c_int32, C.c_uint32, C.c_int64, C.c_uint64, C.c_float

_lib = None


class RtpgError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


# name -> argtypes (all return int status unless listed in _RESTYPE)
_SIGS = {
    "rtpg_last_error": [],
    "rtpg_version": [],
    "rtpg_query_limits": [P, P, P],
    "rtpg_sdtree_create": [P, P, U32, F32, P, P],
    "rtpg_sdtree_destroy": [P],
    "rtpg_sdtree_clear": [P, P],
    "rtpg_sdtree_record": [P, I64, P, P, C.c_int, P, P, P, P, P],
    "rtpg_sdtree_build": [P, P],
    "rtpg_sdtree_refine": [P, U64, I32, F32, P],
    "rtpg_sdtree_reset": [P, I32, I32, P],
    "rtpg_sdtree_sample_pdf": [P, I64, P, P, U32, P, P, P, P, P],
    "rtpg_sdtree_pdf": [P, I64, P, P, C.c_int, P, P],
    "rtpg_sdtree_stats": [P, P, P, P, P],
    "rtpg_sdtree_memory_footprint": [P, P],
    "rtpg_sdtree_status": [P, P, C.c_int, P],
    "rtpg_sdtree_export": [P, C.c_int, P, P, P, P, P, P, P],
    "rtpg_sdtree_import": [P, I64, I64, P, P, I64, P, P, P, I64, P, P, P, P],
    "rtpg_controller_create": [P, U32, U32, F32, U32, P],
    "rtpg_controller_destroy": [P],
    "rtpg_controller_start": [P],
    "rtpg_controller_begin": [P, P],
    "rtpg_controller_end": [P, P],
    "rtpg_controller_get": [P, P, P, P, P],
    "rtpg_hashgrid_create": [P, P, P, U32, I32, U32, P],
    "rtpg_hashgrid_destroy": [P],
    "rtpg_hashgrid_clear": [P, P],
    "rtpg_hashgrid_swap": [P, P],
    "rtpg_hashgrid_insert": [P, I64, P, P, P, P],
    "rtpg_hashgrid_lookup": [P, I64, P, P, P],
    "rtpg_hashgrid_cells": [P, I64, P, P, P, P],
    "rtpg_hashgrid_export": [P, C.c_int, P, P],
    "rtpg_hashgrid_status": [P, P, C.c_int, P],
    "rtpg_hashgrid_device_view": [P, P, P],
    "rtpg_hashgrid_insert_noalloc": [P, P, P, U32, I32, P, P, I64, P, P, P],
    "rtpg_mqt_create": [U32, U32, F32, I32, P],
    "rtpg_mqt_destroy": [P],
    "rtpg_mqt_clear": [P, P],
    "rtpg_mqt_record": [P, I64, P, P, C.c_int, P, P],
    "rtpg_mqt_update": [P, P],
    "rtpg_mqt_sample_pdf": [P, I64, P, P, U32, P, P, P, P, P],
    "rtpg_mqt_pdf": [P, I64, P, P, C.c_int, P, C.c_int, P],
    "rtpg_mqt_export": [P, P, P, P],
    "rtpg_mqt_status": [P, P, C.c_int, P],
    "rtpg_mqt_controller_create": [P, U32, U32, U32, F32, U32, P],
    "rtpg_mqt_controller_destroy": [P],
    "rtpg_mqt_controller_start": [P],
    "rtpg_mqt_controller_begin": [P, P],
    "rtpg_mqt_controller_end": [P, P],
    "rtpg_mqt_controller_get": [P, P, P, P, P],
    "rtpg_scene_create": [P, U32, P, U32, P, P],
    "rtpg_scene_destroy": [P],
    "rtpg_scene_intersect": [P, I64, P, P, P, P, C.c_int, P, P, P, P],
    "rtpg_tracer_create": [P, P, P, P, P, U32, P, P, P, U32, P, P, P],
    "rtpg_tracer_destroy": [P],
    "rtpg_tracer_set_texture": [P, U32, U32, U32, P],
    "rtpg_tracer_set_seed": [P, U32],
    "rtpg_tracer_clear": [P, P],
    "rtpg_tracer_render": [P, U32, U32, P, P],
    "rtpg_tracer_render_guided": [P, P, P, U32, U32, U32, P],
    "rtpg_tracer_render_grid": [P, U32, U32, P, P, P],
    "rtpg_mlp_create": [P, P, U32, F32, U32, P],
    "rtpg_mlp_destroy": [P],
    "rtpg_mlp_params": [P, P, P, P],
    "rtpg_mlp_eval": [P, I64, P, P, P, P, P, P],
    "rtpg_mlp_loss_grad": [P, I64, P, P, P, P, P, P, P, P],
    "rtpg_mlp_train": [P, I64, P, P, P, P, P, U32, U32, P, P],
    "rtpg_mlp_records": [P, P, C.c_int, P],
    "rtpg_mlp_record_arrays": [P, P, P, P, P, P],
    "rtpg_mlp_record_pdfs": [P, P],
    "rtpg_mlp_status": [P, P, C.c_int, P],
    "rtpg_mlp_set_wait_test": [P, C.c_int, U32],
    "rtpg_tracer_set_light_emission": [P, P, U32],
    "rtpg_tracer_image_f64": [P, P, P],
    "rtpg_tracer_render_mlp": [P, U32, U32, P, P, F32, F32, F32, P],
    "rtpg_tracer_render_adjoint": [P, U32, U32, P, I32, P, P, P],
    "rtpg_tracer_render_grid_guided": [P, P, P, P, U32, U32, U32, P],
    "rtpg_tracer_image": [P, P, P],
    "rtpg_tracer_accumulation": [P, P, P],
    "rtpg_tracer_stats": [P, P, P],
    "rtpg_tracer_set_timing": [P, C.c_int],
    "rtpg_tracer_counters": [P, P, P, P],
    "rtpg_tracer_path_depths": [P, P, P],
    "rtpg_tracer_timings": [P, P, P],
}
_RESTYPE = {"rtpg_last_error": C.c_char_p}


def declared_symbols():
    """Function names declared in include/rtpg.h."""
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rtpg_[a-z0-9_]+)\s*\(", text)))


def register(name, argtypes, restype=C.c_int):
    _SIGS[name] = argtypes
    if restype is not C.c_int:
        _RESTYPE[name] = restype
    if _lib is not None:
        fn = getattr(_lib, name)
        fn.argtypes = argtypes
        fn.restype = restype


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"rtlib_b200 native library not built: {LIB_PATH} is missing "
                               "(run __graft_entry__.build() or python rtlib_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name, argtypes in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def call(name, *args):
    r = getattr(lib(), name)(*args)
    if r != 0:
        msg = lib().rtpg_last_error()
        raise RtpgError(name, r, msg.decode() if msg else "")
    return r


def ptr(x):
    """Device/host pointer of a torch tensor, a numpy array, an int, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take a pointer of {type(x)}")


def stream_ptr(stream=None):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream
