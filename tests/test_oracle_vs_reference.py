"""Pins the CPU oracle (oracle/rtpg_oracle.c) to RTLib's own code.

* golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from the
  reference built on the host) -- always run;
* the live reference library (oracle/_ref) on the full 2^20-record workload -- when built.

Topology, hash slots, Morton codes and RNG streams are bit-exact.  Sums: RTLib accumulates in
float (order-dependent), the oracle in int64 fixed point; they agree within the float
accumulation error, and the oracle agrees with a float64 sum of the same records.
"""
import os

import numpy as np
import pytest

from rtlib_b200 import workloads as W

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(G, name))


def _xs32(seed, n):
    s = int(seed)
    out = []
    for _ in range(n):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        b = (s >> 9) | (0x7F << 23)
        out.append(np.array([b], np.uint32).view(np.float32)[0] - np.float32(1))
    return np.array(out, np.float32), s


def test_kat_rng_hash_canonical(oracle):
    k = _load("kat_math.npz")
    got = np.array([oracle.L.or_pcg1d(int(x)) for x in k["xs"]], np.uint32)
    np.testing.assert_array_equal(got, k["pcg1d"])
    for s, f, st in zip(k["seeds"], k["xs32_floats"], k["xs32_state"]):
        mine, state = _xs32(s, 16)
        np.testing.assert_array_equal(mine, f)
        assert state == st
    uv = oracle.dir_to_canonical(k["dirs"])
    np.testing.assert_allclose(uv, k["canon"], rtol=0, atol=2e-7)
    m = np.array([[oracle.L.or_morton2(int(x), int(y)) for y in range(64)] for x in range(64)], np.uint32)
    np.testing.assert_array_equal(m, k["morton2"])


def test_golden_sdtree_topology_and_sums(oracle):
    g = _load("sdtree_small.npz")
    o = oracle.sdtree((0, 0, 0), (1, 1, 1))
    for it, th in zip((1, 2), g["th"]):
        o.record(g["pos"], g["uv"], g["radiance"])
        o.build()
        e = o.export(True)
        assert e.smask.tobytes() == g[f"p{it}_smask"].tobytes()
        assert e.counts.tobytes() == g[f"p{it}_counts"].tobytes()
        assert e.dmask.tobytes() == g[f"p{it}_dmask"].tobytes()
        np.testing.assert_allclose(e.dsums, g[f"p{it}_dsums"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(e.scalars, g[f"p{it}_scalars"], rtol=1e-5, atol=1e-6)
        o.refine(int(th))
        e = o.export(False)
        assert e.smask.tobytes() == g[f"r{it}_smask"].tobytes()
        assert e.counts.tobytes() == g[f"r{it}_counts"].tobytes()
        assert e.dmask.tobytes() == g[f"r{it}_dmask"].tobytes()
    o.record(g["pos"], g["uv"], g["radiance"])
    o.build()
    e = o.export(True)
    assert e.topology == (g["p3_smask"].tobytes(), g["p3_counts"].tobytes(), g["p3_dmask"].tobytes())
    np.testing.assert_allclose(e.dsums, g["p3_dsums"], rtol=1e-5, atol=1e-6)
    uv, pdf = o.sample_pdf(g["qpos"], g["qseeds"])
    same = np.all(uv == g["sample_uv"], axis=1)
    assert same.mean() >= 0.999
    np.testing.assert_allclose(pdf[same], g["sample_pdf"][same], rtol=1e-5)


def test_golden_hashgrid_slots(oracle):
    g = _load("hashgrid_small.npz")
    cur = np.zeros(int(g["nslots"][0]), np.uint32)
    slots = oracle.hashgrid_insert(g["pos"], g["off"], g["size"], g["bounds"], int(g["nslots"][0]), cur)
    np.testing.assert_array_equal(slots, g["slots"])
    np.testing.assert_array_equal(cur, g["table"])
    assert (slots == 0xFFFFFFFF).any(), "fixture should exercise a full bucket"
    look = oracle.hashgrid_lookup(g["qpos"], g["off"], g["size"], g["bounds"], int(g["nslots"][0]), cur)
    np.testing.assert_array_equal(look, g["lookup"])


def test_golden_morton_quadtree(oracle):
    g = _load("mqt_small.npz")
    level, ncells, bits = int(g["level"][0]), int(g["ncells"][0]), 24
    per_ref = ((1 << 14) - 1) // 3
    leaves = np.zeros(ncells << (2 * level), np.int64)
    oracle.mqt_record(level, bits, leaves, g["cell"], g["uv"], g["value"])
    ref_leaves = g["leaves"].reshape(ncells, per_ref)[:, (4**level - 1) // 3:(4**level - 1) // 3 + 4**level]
    np.testing.assert_allclose(np.ldexp(leaves.astype(np.float64), -bits).reshape(ncells, -1), ref_leaves,
                               rtol=1e-5, atol=1e-5)
    pyr = oracle.mqt_build(ncells, level, bits, leaves)
    per = ((1 << (2 * (level + 1))) - 1) // 3
    np.testing.assert_allclose(pyr.reshape(ncells, per), g["pyramid"].reshape(ncells, per_ref)[:, :per],
                               rtol=1e-5, atol=1e-4)
    uv, pdf, pe = oracle.mqt_sample_pdf(level, pyr, g["qcell"], g["qseeds"])
    same = np.all(uv == g["sample_uv"], axis=1)
    assert same.mean() >= 0.999
    np.testing.assert_allclose(pdf[same], g["sample_pdf"][same], rtol=1e-4)
    np.testing.assert_allclose(pe[same], g["pdf_eval"][same], rtol=1e-4)


def test_live_reference_config1(oracle, reference):
    """Full SD-tree standalone workload against the live reference build."""
    rec = W.sdtree_records(1 << 20, 0)
    o = oracle.sdtree((0, 0, 0), (1, 1, 1))
    r = reference.sdtree((0, 0, 0), (1, 1, 1))
    for it in (1, 2):
        o.record(rec["pos"], rec["uv"], rec["radiance"])
        r.record(rec["pos"], rec["uv"], rec["radiance"])
        o.build()
        r.build()
        eo, er = o.export(True), r.export(True)
        assert eo.topology == er.topology
        # the reference's sequential float sums carry ~1e-5 relative rounding at 2^18 records
        # per quadrant; the oracle's fixed-point sums match a float64 sum far more tightly
        np.testing.assert_allclose(eo.dsums, er.dsums, rtol=5e-5, atol=1e-3)
        th = W.spatial_threshold(it)
        o.refine(th)
        r.refine(th)
        assert o.export(False).topology == r.export(False).topology
    # exactness of the first-pass root sum of one leaf against float64
    o2 = oracle.sdtree((0, 0, 0), (1, 1, 1))
    o2.record(rec["pos"], rec["uv"], rec["radiance"])
    o2.build()
    e = o2.export(True)
    exact = np.float64(rec["radiance"]).sum()
    assert abs(e.scalars[1] - exact) / exact < 1e-6
    q = W.sdtree_queries(1 << 16, 1)
    uo, po = o.sample_pdf(q["pos"], q["seeds"])
    ur, pr = r.sample_pdf(q["pos"], q["seeds"])
    same = np.all(uo == ur, axis=1)
    assert same.mean() > 0.999
    np.testing.assert_allclose(po[same], pr[same], rtol=1e-5)


def test_live_reference_hashgrid_random(oracle, reference):
    rng = np.random.default_rng(99)
    off, size, bounds, nslots = np.zeros(3, np.float32), np.ones(3, np.float32), np.array([64, 64, 64], np.uint32), 2048
    pos = rng.random((30000, 3), dtype=np.float32)
    a, b = np.zeros(nslots, np.uint32), np.zeros(nslots, np.uint32)
    np.testing.assert_array_equal(oracle.hashgrid_insert(pos, off, size, bounds, nslots, a),
                                  reference.hashgrid_insert(pos, off, size, bounds, nslots, b))
    np.testing.assert_array_equal(a, b)
