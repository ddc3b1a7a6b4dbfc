"""SD-tree parity: CUDA path (through the C ABI) vs the CPU oracle on identical seeded inputs.

Bit-exact: topology, fixed-point sums converted to float, stat-weights, sampled canonical
points and their pdfs.  Directions (canonical_to_dir uses sincosf/sqrtf on the device and
libm on the host) within 2e-6 absolute.
"""
import numpy as np
import pytest

from rtlib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _same_export(eg, eo):
    assert eg.topology == eo.topology
    np.testing.assert_array_equal(eg.scalars, eo.scalars)
    np.testing.assert_array_equal(eg.dsums, eo.dsums)


def _pair(oracle, mn=(0, 0, 0), mx=(1, 1, 1), **kw):
    from rtlib_b200.sdtree import SDTree
    return SDTree(mn, mx, **kw), oracle.sdtree(mn, mx)


def _queries(g, o, q, dev, with_dir=True):
    import torch
    n = q["pos"].shape[0]
    pos, seeds = _t(q["pos"], dev), _t(q["seeds"], dev)
    uv = torch.empty((n, 2), dtype=torch.float32, device=dev)
    pdf = torch.empty(n, dtype=torch.float32, device=dev)
    d = torch.empty((n, 3), dtype=torch.float32, device=dev)
    pd = torch.empty(n, dtype=torch.float32, device=dev)
    g.sample_pdf(pos, seeds, out_uv=uv, out_pdf_uv=pdf, out_dir=d if with_dir else None,
                 out_pdf_dir=pd if with_dir else None)
    torch.cuda.synchronize()
    ou, op, od, opd = o.sample_pdf(q["pos"], q["seeds"], with_dir=True)
    np.testing.assert_array_equal(uv.cpu().numpy(), ou)
    np.testing.assert_array_equal(pdf.cpu().numpy(), op)
    if with_dir:
        np.testing.assert_allclose(d.cpu().numpy(), od, atol=2e-6, rtol=0)
        pdg = pd.cpu().numpy()
        close = np.isclose(pdg, opd, rtol=1e-5, atol=0)
        assert close.mean() > 0.999, close.mean()


def test_config1_single_pass(cuda, oracle):
    """2^20 records, build, refine at 12000*sqrt(2), then 2^18 sample+pdf queries."""
    rec = W.sdtree_records(1 << 20, 0)
    g, o = _pair(oracle)
    g.record(_t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda))
    o.record(rec["pos"], rec["uv"], rec["radiance"])
    _same_export(g.export(sampling=False), o.export(sampling=False))
    g.build()
    o.build()
    _same_export(g.export(sampling=True), o.export(sampling=True))
    th = W.spatial_threshold(1)
    g.refine(th)
    o.refine(th)
    eg, eo = g.export(sampling=False), o.export(sampling=False)
    _same_export(eg, eo)
    assert len(eg.smask) == 127 and len(eg.counts) == 64
    _same_export(g.export(sampling=True), o.export(sampling=True))
    _queries(g, o, W.sdtree_queries(1 << 18, 1), cuda)
    assert g.status() == 0


def test_two_pass_realistic_depth(cuda, oracle):
    """Record into the refined topology a second time: sample/pdf descend deep quadtrees."""
    rec = W.sdtree_records(1 << 20, 0)
    g, o = _pair(oracle)
    P, U, R = _t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda)
    for it in (1, 2):
        g.record(P, U, R)
        o.record(rec["pos"], rec["uv"], rec["radiance"])
        g.build()
        o.build()
        _same_export(g.export(sampling=True), o.export(sampling=True))
        th = W.spatial_threshold(it)
        g.refine(th)
        o.refine(th)
        _same_export(g.export(sampling=False), o.export(sampling=False))
    _queries(g, o, W.sdtree_queries(1 << 18, 7), cuda)
    st = g.stats()
    assert st["dtree_nodes"] > 1000


def test_record_direction_vectors(cuda, oracle):
    """dir given as unit vectors: the device computes the canonical map with atan2f; the
    topology after refine and the sums agree with the oracle fed host-side canonicals up to
    records within an ulp of a quadrant boundary."""
    rec = W.sdtree_records(1 << 18, 3)
    g, o = _pair(oracle)
    g.record(_t(rec["pos"], cuda), _t(rec["dir"], cuda), _t(rec["radiance"], cuda), canonical=False)
    o.record(rec["pos"], oracle.dir_to_canonical(rec["dir"]), rec["radiance"])
    g.build()
    o.build()
    eg, eo = g.export(), o.export()
    assert eg.topology == eo.topology
    np.testing.assert_allclose(eg.dsums, eo.dsums, rtol=1e-4, atol=1e-3)


def test_edge_records(cuda, oracle):
    """Empty batch, delta vertices, zero / negative / NaN / inf values, positions on and
    outside the box, woPdf 0: the same records are skipped on both sides."""
    rng = np.random.default_rng(5)
    n = 4096
    pos = rng.random((n, 3), dtype=np.float32)
    pos[:8] = [[1, 1, 1], [0, 0, 0], [1, 0, 1], [-0.5, 0.2, 0.3], [1.7, 0.1, 0.1], [0.5, 0.5, 0.5],
               [0.999999, 0.5, 1.0], [0, 1, 0]]
    uv = rng.random((n, 2), dtype=np.float32)
    uv[:6] = [[0, 0], [1, 1], [0.5, 0.5], [1, 0], [0, 1], [0.25, 0.75]]
    rad = rng.lognormal(0, 1, n).astype(np.float32)
    rad[10:14] = [0, -1, np.nan, np.inf]
    wo = np.ones(n, np.float32)
    wo[20:24] = [0, -1, np.inf, 1e-30]
    sw = np.ones(n, np.float32)
    sw[30:34] = [0, -2, np.nan, 0.5]
    dl = np.zeros(n, np.uint8)
    dl[40:48] = 1
    g, o = _pair(oracle, (-1, -2, -1), (2, 1, 3))
    g.record(_t(pos[:0], cuda), _t(uv[:0], cuda), _t(rad[:0], cuda))
    for _ in range(2):
        g.record(_t(pos, cuda), _t(uv, cuda), _t(rad, cuda), _t(wo, cuda), _t(sw, cuda), _t(dl, cuda))
        o.record(pos, uv, rad, wo, sw, dl)
        g.build()
        o.build()
        _same_export(g.export(), o.export())
        g.refine(1500)
        o.refine(1500)
        _same_export(g.export(sampling=False), o.export(sampling=False))
    q = {"pos": pos, "seeds": rng.integers(1, 2**32, n, dtype=np.uint64).astype(np.uint32)}
    _queries(g, o, q, cuda, with_dir=False)


def test_clear_and_empty_tree_queries(cuda, oracle):
    """A cleared tree samples uniformly with pdf 1/(4 pi) (GetMean() <= 0, PG.h:478-490)."""
    g, o = _pair(oracle)
    rec = W.sdtree_records(1 << 12, 9)
    g.record(_t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda))
    g.build()
    g.clear()
    q = W.sdtree_queries(1 << 12, 11)
    _queries(g, o, q, cuda)
    assert g.stats() == {"stree_nodes": 1, "dtrees": 1, "dtree_nodes": 1}


def test_memory_guard_and_capacity(cuda, oracle):
    """max_mb = 0 skips the spatial refine (footprint / 1e6 >= 0); a tiny STree capacity
    sets RTPG_STATUS_STREE_CAPACITY instead of overflowing."""
    from rtlib_b200.sdtree import SDTree
    rec = W.sdtree_records(1 << 16, 2)
    g, o = _pair(oracle)
    g.record(_t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda))
    o.record(rec["pos"], rec["uv"], rec["radiance"])
    g.build(); o.build()
    g.refine(100, max_mb=0); o.refine(100, max_mb=0)
    _same_export(g.export(sampling=False), o.export(sampling=False))
    assert g.stats()["stree_nodes"] == 1
    # 16 STree nodes allow three levels of splits (2^(k+1) <= 16); the cut is reported
    small = SDTree((0, 0, 0), (1, 1, 1), max_stree_nodes=16)
    small.record(_t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda))
    small.build()
    small.refine(100)
    assert small.status() & 0x4
    assert small.stats()["stree_nodes"] == 15
    # a second refine that would need more nodes than remain is skipped as a whole
    small.record(_t(rec["pos"], cuda), _t(rec["uv"], cuda), _t(rec["radiance"], cuda))
    small.build()
    small.status(clear=True)
    small.refine(100)
    assert small.status() & 0x4
    assert small.stats()["stree_nodes"] == 15


def _schedule(budget, built, ratio, spl):
    """RTSTreeControllerT::BegTrace/EndTrace (PG.h:1808-1887) restated: (state, iteration,
    reset?, build?) per launch."""
    out = []
    remain = ((budget - 1 + spl) // spl) * spl
    pas = 0
    per_all = per_tmp = it = 0
    executing = True
    while executing:
        reset = False
        if per_tmp == 0:
            remain -= pas
            pas = min(remain, (1 << it) * spl)
            if remain - pas < 2 * pas or per_all >= ratio * float(budget):
                pas = remain
            reset = remain > pas and it > 0
        state = (1 if remain > pas else 2) if it > built else 0
        per_all += spl
        per_tmp += spl
        build = per_tmp >= pas
        out.append((state, it, reset, build))
        if build:
            it += 1
            per_tmp = 0
        if per_all > budget:
            executing = False
    return out


def test_controller_schedule(cuda):
    from rtlib_b200.sdtree import SDTree, SDTreeController
    t = SDTree((0, 0, 0), (1, 1, 1))
    c = SDTreeController(t, sample_for_budget=100, iteration_for_built=0, ratio_for_budget=0.5, samples_per_launch=1)
    c.start()
    got = []
    while True:
        c.begin()
        s = c.get()
        if not s["executing"]:
            break
        c.end()
        got.append((s["state"], s["iteration"]))
    want = [(a, b) for a, b, _, _ in _schedule(100, 0, 0.5, 1)]
    assert got == want
    assert {g[1] for g in got} == set(range(max(g[1] for g in got) + 1))


def _two_pass(g, o, rec, dev, n_refines=2):
    P, U, R = _t(rec["pos"], dev), _t(rec["uv"], dev), _t(rec["radiance"], dev)
    for it in range(1, n_refines + 1):
        if g is not None:
            g.record(P, U, R)
            g.build()
            g.refine(W.spatial_threshold(it) // 16)
        if o is not None:
            o.record(rec["pos"], rec["uv"], rec["radiance"])
            o.build()
            o.refine(W.spatial_threshold(it) // 16)
    if g is not None:
        g.record(P, U, R)
    if o is not None:
        o.record(rec["pos"], rec["uv"], rec["radiance"])


def test_import_round_trip(cuda):
    """export -> import into a fresh handle -> export gives identical building and sampling
    streams, and the imported tree samples exactly as the original."""
    import torch
    from rtlib_b200.sdtree import SDTree
    rec = W.sdtree_records(1 << 16, 21)
    g = SDTree((0, 0, 0), (1, 1, 1))
    _two_pass(g, None, rec, cuda)
    g.build()  # sampling trees from the last records; building trees keep their sums
    eb, es = g.export(sampling=False), g.export(sampling=True)
    assert len(eb.counts) > 8 and eb.dmask.shape[0] > len(eb.counts)
    h = SDTree((0, 0, 0), (1, 1, 1))
    h.import_(eb, es)
    _same_export(h.export(sampling=False), eb)
    _same_export(h.export(sampling=True), es)
    assert h.stats() == g.stats()
    q = W.sdtree_queries(1 << 14, 22)
    outs = []
    for t in (g, h):
        uv = torch.empty((q["pos"].shape[0], 2), dtype=torch.float32, device=cuda)
        pdf = torch.empty(q["pos"].shape[0], dtype=torch.float32, device=cuda)
        t.sample_pdf(_t(q["pos"], cuda), _t(q["seeds"], cuda), out_uv=uv, out_pdf_uv=pdf)
        outs.append((uv.cpu().numpy(), pdf.cpu().numpy()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    assert h.status() == 0


def test_import_oracle_tree_then_continue(cuda, oracle):
    """A tree built by the CPU oracle, imported to the GPU, samples bit-identically; recording
    into it, building and refining then stays bit-identical to the oracle continuing alone."""
    from rtlib_b200.sdtree import SDTree
    rec = W.sdtree_records(1 << 16, 31)
    o = oracle.sdtree((0, 0, 0), (1, 1, 1))
    _two_pass(None, o, rec, cuda)
    o.build()
    g = SDTree((0, 0, 0), (1, 1, 1))
    g.import_(o.export(sampling=False), o.export(sampling=True))
    _same_export(g.export(sampling=True), o.export(sampling=True))
    _queries(g, o, W.sdtree_queries(1 << 14, 32), cuda)
    # continue: refine, record a new batch, build
    th = W.spatial_threshold(3) // 16
    g.refine(th)
    o.refine(th)
    rec2 = W.sdtree_records(1 << 16, 33)
    g.record(_t(rec2["pos"], cuda), _t(rec2["uv"], cuda), _t(rec2["radiance"], cuda))
    o.record(rec2["pos"], rec2["uv"], rec2["radiance"])
    g.build()
    o.build()
    _same_export(g.export(sampling=True), o.export(sampling=True))
    _queries(g, o, W.sdtree_queries(1 << 14, 34), cuda)
    assert g.status() == 0


def test_import_rejects_inconsistent_streams(cuda):
    from rtlib_b200._lib import RtpgError
    from rtlib_b200.sdtree import SDTree
    rec = W.sdtree_records(1 << 14, 41)
    g = SDTree((0, 0, 0), (1, 1, 1))
    _two_pass(g, None, rec, cuda, n_refines=1)
    g.build()
    eb, es = g.export(sampling=False), g.export(sampling=True)
    h = SDTree((0, 0, 0), (1, 1, 1))
    bad = type(eb)(eb.smask, eb.scalars, eb.counts.copy(), eb.dmask, eb.dsums)
    bad.counts[0] += 1  # node counts no longer add up to the stream
    with pytest.raises(RtpgError):
        h.import_(bad, es)
    small = SDTree((0, 0, 0), (1, 1, 1), max_dtrees=4)
    with pytest.raises(RtpgError):
        small.import_(eb, es)
    # the failed imports left the handles usable
    h.import_(eb, es)
    _same_export(h.export(sampling=True), es)
