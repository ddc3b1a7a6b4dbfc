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


def test_live_reference_exact_sums_sample_identically(oracle, reference):
    """Why a few queries in 1000 differ above: RTLib sums radiance in float in record order,
    the restatement exactly, so a quadrant sum can differ by an ulp and a sample that falls
    within that ulp of a boundary takes the other quadrant.  With radiance in multiples of
    1/64 and few enough records, every float sum of RTLib is exact too: then the trees,
    their sums and every sample and pdf agree bit for bit."""
    rec = W.sdtree_records(1 << 16, 5)
    rad = (np.maximum(np.round(rec["radiance"] * 64.0), 1.0) / 64.0).astype(np.float32)
    assert float(rad.astype(np.float64).sum()) * 64 < 2 ** 24
    o = oracle.sdtree((0, 0, 0), (1, 1, 1))
    r = reference.sdtree((0, 0, 0), (1, 1, 1))
    for th in (4000, 2000):
        for t in (o, r):
            t.record(rec["pos"], rec["uv"], rad)
            t.build()
        eo, er = o.export(True), r.export(True)
        assert eo.topology == er.topology
        np.testing.assert_array_equal(eo.dsums, er.dsums)
        np.testing.assert_array_equal(eo.scalars, er.scalars)
        o.refine(th)
        r.refine(th)
    q = W.sdtree_queries(1 << 16, 6)
    uo, po = o.sample_pdf(q["pos"], q["seeds"])
    ur, pr = r.sample_pdf(q["pos"], q["seeds"])
    np.testing.assert_array_equal(uo, ur)
    np.testing.assert_array_equal(po, pr)


def test_live_reference_hashgrid_random(oracle, reference):
    rng = np.random.default_rng(99)
    off, size, bounds, nslots = np.zeros(3, np.float32), np.ones(3, np.float32), np.array([64, 64, 64], np.uint32), 2048
    pos = rng.random((30000, 3), dtype=np.float32)
    a, b = np.zeros(nslots, np.uint32), np.zeros(nslots, np.uint32)
    np.testing.assert_array_equal(oracle.hashgrid_insert(pos, off, size, bounds, nslots, a),
                                  reference.hashgrid_insert(pos, off, size, bounds, nslots, b))
    np.testing.assert_array_equal(a, b)


# ---------------------------------------------------------------- integrator (A-6)
# RTLib's shading code run on the host (oracle/ref stages SimpleKernel.h:26-143 and
# SimpleGuide.cu:28-47, 287-496) against the C restatement.  Random numbers: the same
# draws in the same order (end states equal).  Floats: bit-exact except where sin / cos
# enter (the restatement forms cos(2 pi x) as cospi(2x), as the CUDA path does), within
# 5e-4 of max(|value|, 1e-3).
SHADE_RTOL = 5e-4


def _kat_scene():
    import kat_integrator as K
    return K, K.scene()


def _check_shade(mine, ref):
    (o, f, s), (ro, rf, rs) = mine, ref
    np.testing.assert_array_equal(f, rf)
    np.testing.assert_array_equal(s, rs)
    err = np.abs(o - ro) / np.maximum(np.abs(ro), 1e-3)
    assert err.max() <= SHADE_RTOL, err.max()
    assert (o == ro).all(1).mean() > 0.6  # the rest carry the sin / cos ulps


def test_golden_integrator_building_blocks(oracle):
    from oracle.oracle import IntegratorKAT
    g = _load("kat_integrator.npz")
    K, sc = _kat_scene()
    k = IntegratorKAT(oracle, sc, fraction=0.5)
    d, st = k.cosine(g["normal"], g["seeds"])
    np.testing.assert_array_equal(st, g["cos_state"])
    np.testing.assert_allclose(d, g["cos_dir"], rtol=0, atol=1e-6)
    for got, want in zip(k.phong(g["normal"], g["shininess"], g["seeds"]), (g["phong_dir"], g["phong_state"])):
        np.testing.assert_array_equal(got, want)
    for got, want in zip(k.triangle(g["tri"], g["seeds"]), (g["tri_point"], g["tri_state"])):
        np.testing.assert_array_equal(got, want)
    for got, want in zip(k.light(g["p_in"], g["seeds"]), (g["light"], g["light_state"])):
        np.testing.assert_array_equal(got, want)
    for got, want in zip(k.reservoir(g["res_w"], g["res_rnd"]), (g["res_sel"], g["res_wsum"], g["res_m"])):
        np.testing.assert_array_equal(got, want)
    assert (g["res_sel"] == -1).any() and (g["res_sel"] >= 0).any()


def test_golden_integrator_shading(oracle):
    """Closest-hit shading of 1024 vertices on Phong (Lambertian and glossy), glass and
    emitter triangles, front and back faces, under DEF, NEE, NEE+RIS, SD-tree recording and
    SD-tree guiding with NEE and with RIS, against RTLib's own __closesthit__radiance."""
    from oracle.oracle import IntegratorKAT
    g = _load("kat_integrator.npz")
    K, sc = _kat_scene()
    k = IntegratorKAT(oracle, sc, fraction=0.5)
    tree = K.build_tree(oracle, K.tree_records())
    cases = {key[5:]: g[key] for key in g.files if key.startswith("case_")}
    for fl in g["flag_sets"]:
        fl = int(fl)
        _check_shade(k.shade(fl, cases, tree if fl & 8 else None),
                     (g[f"shade{fl}_out"], g[f"shade{fl}_flags"], g[f"shade{fl}_state"]))
    # the fixture covers every branch: glass (delta flag), Phong with NEE, emitters (finish)
    f = g["shade25_flags"]
    assert (f & 2).any() and (f & 16).any() and ((f & 8) == 0).any()


def test_live_reference_integrator(oracle, reference):
    from oracle.oracle import IntegratorKAT
    K, sc = _kat_scene()
    mine, ref = IntegratorKAT(oracle, sc, fraction=0.5), IntegratorKAT(reference, sc, fraction=0.5)
    rng = np.random.default_rng(99)
    n = 20000
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    seeds = rng.integers(1, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    shin = rng.uniform(0.0, 300.0, n).astype(np.float32)
    for a, b in ((mine.phong(nrm, shin, seeds), ref.phong(nrm, shin, seeds)),
                 (mine.light(nrm * 0.3 + 0.5, seeds), ref.light(nrm * 0.3 + 0.5, seeds))):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    (d, s), (rd, rs) = mine.cosine(nrm, seeds), ref.cosine(nrm, seeds)
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_allclose(d, rd, rtol=0, atol=1e-6)
    rec = K.tree_records()
    to, tr = K.build_tree(oracle, rec), K.build_tree(reference, rec)
    assert to.export(True).topology == tr.export(True).topology
    cases = K.shade_cases(sc, n, 7)
    for fl in K.FLAG_SETS:
        _check_shade(mine.shade(fl, cases, to if fl & 8 else None), ref.shade(fl, cases, tr if fl & 8 else None))
