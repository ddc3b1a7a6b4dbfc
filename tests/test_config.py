"""Trace configuration (TraceConfigData of a scene.json) parsing, CPU."""
from rtlib_b200.config import TRACERS, TraceConfig


def test_parse_config_and_defaults():
    cfg = TraceConfig.from_json({"Config": {"ImagePath": "out", "Width": 64, "Height": 32, "Samples": 1,
                                            "SamplesPerSave": 16, "MaxSamples": 31, "MaxDepth": 8,
                                            "DefTracer": "PGNEE", "Custom": {"SdTree.Fraction": 0.5}}})
    assert (cfg.width, cfg.height, cfg.samples, cfg.max_samples, cfg.max_depth) == (64, 32, 1, 31, 8)
    assert cfg.def_tracer == "PGNEE" and cfg.max_times == float("inf") and not cfg.enable_vis
    assert cfg.get("SdTree.Fraction", 0.3) == 0.5 and cfg.get("MortonTree.Fraction", 0.3) == 0.3
    assert set(TRACERS) >= {"DEF", "NEE", "RIS", "PGNEE", "PGRIS", "HTNEE", "HTRIS"}
