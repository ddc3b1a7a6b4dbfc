"""The application's trace configuration (TraceConfigData, RTLib/Src/Core/Include/RTLib/Core/
Scene.h:10-86: the "Config" object of a scene.json) and its tracers, run on this library.

``TraceConfig.from_json`` reads the same keys (Width, Height, Samples, SamplesPerSave,
MaxSamples, MaxTimes, MaxDepth, EnableVis, DefTracer, Custom, Tracers); ``run`` renders one of
the application's tracers by name with the Custom options it reads and their defaults
(RTLibExtOPX7TestApplication.cpp:303-376: SdTree.Fraction / RatioForBudget /
IterationForBuilt, MortonTree.Fraction / RatioForBudget / IterationForBuilt, HashGrid.CellSize
/ GridSize, Ris.NumCandidates, MissData.BgColor):

    DEF, NEE, RIS           unguided (flags 0, NEE, NEE | RIS)
    PGDEF, PGNEE, PGRIS     SD-tree guided under RTSTreeControllerT's schedule
    HTDEF, HTNEE, HTRIS     hash grid + Morton quadtrees under RTMortonQuadTreeControllerT's
                            schedule, the grid's current table copied to the previous one after
                            every pass
Scenes are the procedural builders of rtlib_b200.scenes (OBJ loading is not part of this
library); the world AABB is the scene's, padded by 0.005 as InitSdTree / InitGrids pad it."""
from __future__ import annotations

import json
import time
from dataclasses import dataclass, field

import numpy as np

TRACERS = ("DEF", "NEE", "RIS", "PGDEF", "PGNEE", "PGRIS", "HTDEF", "HTNEE", "HTRIS")


@dataclass
class TraceConfig:
    width: int
    height: int
    samples: int
    samples_per_save: int
    max_samples: int
    max_depth: int
    max_times: float = float("inf")
    enable_vis: bool = False
    def_tracer: str = "NONE"
    image_path: str = ""
    custom: dict = field(default_factory=dict)
    tracers: dict = field(default_factory=dict)

    @staticmethod
    def from_json(obj):
        """obj: the Config object (a dict), a scene.json dict holding "Config", or a path."""
        if isinstance(obj, str):
            with open(obj) as f:
                obj = json.load(f)
        if "Config" in obj:
            obj = obj["Config"]
        return TraceConfig(width=int(obj["Width"]), height=int(obj["Height"]), samples=int(obj["Samples"]),
                           samples_per_save=int(obj["SamplesPerSave"]), max_samples=int(obj["MaxSamples"]),
                           max_depth=int(obj["MaxDepth"]), max_times=float(obj.get("MaxTimes", float("inf"))),
                           enable_vis=bool(obj.get("EnableVis", False)), def_tracer=obj.get("DefTracer", "NONE"),
                           image_path=obj.get("ImagePath", ""), custom=dict(obj.get("Custom", {})),
                           tracers=dict(obj.get("Tracers", {})))

    def get(self, key, default):
        return self.custom.get(key, default)


def _aabb(scene, pad=0.005):
    v = np.asarray(scene["tri_v"], np.float32).reshape(-1, 3)
    return tuple(float(x) - pad for x in v.min(0)), tuple(float(x) + pad for x in v.max(0))


def run(cfg, scene, device, tracer=None, stream=None):
    """Render `tracer` (default cfg.def_tracer) over cfg.max_samples samples (or cfg.max_times
    seconds for the unguided tracers).  Returns (tracer object, mean image (h, w, 3) float32
    host array, samples, seconds)."""
    import torch

    from .hashgrid import KEY_REFERENCE, HashGrid, MortonQuadTreeController, MortonQuadTrees
    from .sdtree import SDTree, SDTreeController
    from .tracer import FLAG_NEE, FLAG_RIS, Tracer

    name = (tracer or cfg.def_tracer).upper()
    if name not in TRACERS:
        raise ValueError(f"unknown tracer {name!r}; one of {TRACERS}")
    base = name[-3:] if name[:2] in ("PG", "HT") else name
    flags = {"DEF": 0, "NEE": FLAG_NEE, "RIS": FLAG_NEE | FLAG_RIS}[base]
    bg = tuple(cfg.get("MissData.BgColor", (0.0, 0.0, 0.0)))
    tr = Tracer(scene, device, max_depth=cfg.max_depth, num_candidates=int(cfg.get("Ris.NumCandidates", 32)),
                width=cfg.width, height=cfg.height, background=bg)
    spl = max(1, cfg.samples)
    mn, mx = _aabb(scene)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if name.startswith("PG"):
        tree = SDTree(mn, mx, fraction=float(cfg.get("SdTree.Fraction", 0.3)))
        ctrl = SDTreeController(tree, cfg.max_samples, int(cfg.get("SdTree.IterationForBuilt", 0)),
                                float(cfg.get("SdTree.RatioForBudget", 0.3)), spl)
        ctrl.start()
        tr.render_guided(tree, ctrl, flags, samples_per_launch=spl, stream=stream)
        tr._keep = (tree, ctrl)
    elif name.startswith("HT"):
        size = int(cfg.get("HashGrid.CellSize", 128 * 128 * 4))
        bounds = tuple(int(b) for b in cfg.get("HashGrid.GridSize", (128, 64, 128)))
        grid = HashGrid(mn, mx, bounds, size, keying=KEY_REFERENCE)
        trees = MortonQuadTrees(size, level=int(cfg.get("MortonTree.Level", 6)),
                                fraction=float(cfg.get("MortonTree.Fraction", 0.3)))
        ctrl = MortonQuadTreeController(trees, cfg.max_samples, int(cfg.get("MortonTree.IterationForBuilt", 3)), 0,
                                        float(cfg.get("MortonTree.RatioForBudget", 0.3)), spl)
        grid.clear(stream)
        ctrl.start()
        tr.render_grid_guided(grid, trees, ctrl, flags, samples_per_launch=spl, stream=stream)
        tr._keep = (grid, trees, ctrl)
    else:
        done = 0
        while done < cfg.max_samples and time.perf_counter() - t0 < cfg.max_times:
            tr.render(spl, flags, stream=stream)
            done += spl
            if cfg.max_times != float("inf"):
                torch.cuda.synchronize()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    img = tr.image(stream=stream).cpu().numpy()
    return tr, img, tr.stats()["samples"], dt
