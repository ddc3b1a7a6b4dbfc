"""CPU-side pieces of the benchmark: the hash-grid workload's inputs and its CPU baseline, which
times RTLib's own per-point routines (the reference build)."""
import numpy as np

import bench
from rtlib_b200 import workloads as W


def test_hashgrid_inputs_shapes_and_determinism():
    a = W.hashgrid_inputs(1 << 10, 1 << 12, 0)
    b = W.hashgrid_inputs(1 << 10, 1 << 12, 0)
    assert a["points"].shape == (1 << 10, 3) and a["queries"].shape == (1 << 12, 3)
    assert a["uv"].shape == (1 << 12, 2) and a["value"].shape == (1 << 12,) and a["seeds"].dtype == np.uint32
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert (a["uv"] >= 0).all() and (a["uv"] <= 1).all() and (a["value"] > 0).all() and (a["seeds"] != 0).all()
    lo, hi = np.array(bench.HG_AABB[0]), np.array(bench.HG_AABB[1])
    assert ((a["points"] >= lo) & (a["points"] <= hi)).all()


def test_hashgrid_cpu_baseline_runs():
    cb = bench.cpu_baseline_hashgrid(seconds=0.0, scale_log2=8)
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["value"] > 0
    assert cb["unit"] == "Mops/s" and "RTLib" in cb["sample"]
