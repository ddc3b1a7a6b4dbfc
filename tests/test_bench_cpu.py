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


def test_threaded_shared_tree_render_matches_one_thread():
    """The Cornell CPU baseline renders each frame in pixel bands on several threads into one
    shared SD-tree (thread-private fixed-point sums merged after the frame): image, tree
    topology and sums are identical to a single-threaded render."""
    from oracle.oracle import Oracle, OracleRenderer
    from rtlib_b200 import scenes
    o = Oracle()
    sc = scenes.cornell_box(40, 40)
    out = []
    for threads in (1, 4):
        t = o.sdtree(*bench.C_AABB)
        r = OracleRenderer(o, sc, max_depth=8, fraction=0.5, width=40, height=40)
        r.render_guided(t, 15, ratio_for_budget=1.0, threads=threads)
        out.append((r.image(), t.export(True), t.export(False)))
    (ia, sa, ba), (ib, sb, bb) = out
    np.testing.assert_array_equal(ia, ib)
    assert sa.topology == sb.topology and ba.topology == bb.topology
    np.testing.assert_array_equal(sa.dsums, sb.dsums)
    np.testing.assert_array_equal(ba.dsums, bb.dsums)
    np.testing.assert_array_equal(sa.scalars, sb.scalars)
