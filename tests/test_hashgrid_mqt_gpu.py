"""Hash grid and Morton quadtree parity: CUDA path (C ABI) vs the CPU oracle and the golden
fixtures from RTLib's own code.  Slots, keys, Morton codes, fixed-point leaves, pyramids,
samples and pdfs are bit-exact against the oracle."""
import os

import numpy as np
import pytest

from rtlib_b200 import workloads as W

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _insert(hg, pos, dev):
    import torch
    out = torch.empty(pos.shape[0], dtype=torch.int32, device=dev)
    hg.insert(_t(pos, dev), out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


def _lookup(hg, pos, dev):
    import torch
    out = torch.empty(pos.shape[0], dtype=torch.int32, device=dev)
    hg.lookup(_t(pos, dev), out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("max_batch", [0, 777])
def test_hashgrid_golden(cuda, max_batch):
    """Sequential-insertion slots of RTLib's FindFromCur, including full buckets; chunked
    inserts (max_batch) keep the same slots."""
    from rtlib_b200.hashgrid import HashGrid
    g = np.load(os.path.join(G, "hashgrid_small.npz"))
    mn, sz = g["off"], g["size"]
    hg = HashGrid(mn, mn + sz, g["bounds"], int(g["nslots"][0]), max_batch=max_batch)
    slots = _insert(hg, g["pos"], cuda)
    np.testing.assert_array_equal(slots, g["slots"])
    np.testing.assert_array_equal(hg.export().astype(np.uint32), g["table"])
    assert hg.status() & 0x10
    assert _lookup(hg, g["qpos"], cuda).tolist() == [0xFFFFFFFF] * len(g["qpos"])  # prv still empty
    hg.swap()
    np.testing.assert_array_equal(_lookup(hg, g["qpos"], cuda), g["lookup"])


def test_hashgrid_reference_keying_vs_oracle(cuda, oracle):
    from rtlib_b200.hashgrid import HashGrid
    rng = np.random.default_rng(21)
    mn, mx, bounds, nslots = np.array([-2, -1, -3], np.float32), np.array([2, 3, 1], np.float32), [256, 128, 256], 1 << 16
    hg = HashGrid(mn, mx, bounds, nslots)
    cur = np.zeros(nslots, np.uint32)
    for batch in range(3):
        pos = (rng.random((1 << 18, 3), dtype=np.float32) * (mx - mn) + mn).astype(np.float32)
        pos[: 1 << 16] = pos[: 1 << 16] * np.float32(0.05)  # dense cluster: repeated cells
        want = oracle.hashgrid_insert(pos, mn, mx - mn, bounds, nslots, cur)
        np.testing.assert_array_equal(_insert(hg, pos, cuda), want)
    np.testing.assert_array_equal(hg.export().astype(np.uint32), cur)
    hg.swap()
    q = (rng.random((1 << 16, 3), dtype=np.float32) * (mx - mn) + mn).astype(np.float32)
    np.testing.assert_array_equal(_lookup(hg, q, cuda), oracle.hashgrid_lookup(q, mn, mx - mn, bounds, nslots, cur))


def test_hashgrid_morton_keying(cuda, oracle):
    """63-bit Morton keys at 2^21 cells per axis (21 bits per axis), 2^20 slots."""
    import torch
    from rtlib_b200.hashgrid import KEY_MORTON, HashGrid
    rng = np.random.default_rng(3)
    mn, mx, bounds, nslots = np.zeros(3, np.float32), np.full(3, 10, np.float32), [1 << 21] * 3, 1 << 20
    hg = HashGrid(mn, mx, bounds, nslots, keying=KEY_MORTON)
    pos = (rng.random((1 << 19, 3), dtype=np.float32) * 10).astype(np.float32)
    pos[: 1 << 17] = pos[: 1 << 10][rng.integers(0, 1 << 10, 1 << 17)]  # repeats
    cur = np.zeros(nslots, np.uint64)
    want, keys = oracle.mhash_insert(pos, mn, mx - mn, bounds, nslots, cur)
    out = torch.empty(pos.shape[0], dtype=torch.int32, device=cuda)
    k = torch.empty(pos.shape[0], dtype=torch.int64, device=cuda)
    hg.insert(_t(pos, cuda), out, k)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
    np.testing.assert_array_equal(k.cpu().numpy().view(np.uint64), keys)
    np.testing.assert_array_equal(hg.export(), cur)
    cells = torch.empty((16, 3), dtype=torch.int32, device=cuda)
    hg.cells(_t(pos[:16], cuda), cells)
    c = cells.cpu().numpy().view(np.uint32)
    for i in range(16):
        assert oracle.L.or_morton3(int(c[i, 0]), int(c[i, 1]), int(c[i, 2])) + 1 == keys[i]


@pytest.mark.parametrize("level", [1, 2, 3, 4, 5, 6, 7])
def test_mqt_vs_oracle(cuda, oracle, level):
    """Record, pyramid build (each level has its own build kernel shape), sample and pdf bit
    for bit against the oracle."""
    import torch
    from rtlib_b200.hashgrid import MortonQuadTrees
    ncells, bits = 1024, 24
    rng = np.random.default_rng(8)
    n = 1 << 18
    rec = W.sdtree_records(n, 4)
    cell = rng.integers(0, ncells, n).astype(np.uint32)
    cell[:100] = 0xFFFFFFFF
    uv = rec["uv"]
    uv[100:104] = [[1, 1], [0, 1], [1, 0], [0.5, 0.5]]
    val = rec["radiance"]
    val[200:204] = [0, -1, np.nan, np.inf]
    t = MortonQuadTrees(ncells, level)
    leaves = np.zeros(ncells << (2 * level), np.int64)
    for _ in range(2):
        t.record(_t(cell, cuda), _t(uv, cuda), _t(val, cuda))
        oracle.mqt_record(level, bits, leaves, cell, uv, val)
    gl, _ = t.export()
    np.testing.assert_array_equal(gl, leaves)
    t.update()
    pyr = oracle.mqt_build(ncells, level, bits, leaves)
    gl, gp = t.export()
    assert not gl.any()
    np.testing.assert_array_equal(gp, pyr)
    qn = 1 << 16
    qcell = rng.integers(0, ncells, qn).astype(np.uint32)
    seeds = rng.integers(1, 2**32, qn, dtype=np.uint64).astype(np.uint32)
    ouv, opdf, ope = oracle.mqt_sample_pdf(level, pyr, qcell, seeds)
    guv = torch.empty((qn, 2), dtype=torch.float32, device=cuda)
    gpt = torch.empty(qn, dtype=torch.float32, device=cuda)
    gpw = torch.empty(qn, dtype=torch.float32, device=cuda)
    t.sample_pdf(_t(qcell, cuda), _t(seeds, cuda), out_uv=guv, out_pdf=gpw, out_pdf_tree=gpt)
    pe = torch.empty(qn, dtype=torch.float32, device=cuda)
    t.pdf(_t(qcell, cuda), guv, pe, tree_level=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(guv.cpu().numpy(), ouv)
    np.testing.assert_array_equal(gpt.cpu().numpy(), opdf)
    np.testing.assert_array_equal(pe.cpu().numpy(), ope)
    np.testing.assert_array_equal(gpw.cpu().numpy(), (opdf.astype(np.float64) * (0.25 / np.pi)).astype(np.float32))


def test_mqt_golden(cuda):
    """Against RTLib's float-accumulated Morton trees (golden fixture)."""
    import torch
    from rtlib_b200.hashgrid import MortonQuadTrees
    g = np.load(os.path.join(G, "mqt_small.npz"))
    level, ncells = int(g["level"][0]), int(g["ncells"][0])
    t = MortonQuadTrees(ncells, level)
    t.record(_t(g["cell"], cuda), _t(g["uv"], cuda), _t(g["value"], cuda))
    t.update()
    _, pyr = t.export()
    per_ref = ((1 << 14) - 1) // 3
    per = ((1 << (2 * (level + 1))) - 1) // 3
    np.testing.assert_allclose(pyr.reshape(ncells, per), g["pyramid"].reshape(ncells, per_ref)[:, :per],
                               rtol=1e-5, atol=1e-4)
    qn = g["qcell"].shape[0]
    guv = torch.empty((qn, 2), dtype=torch.float32, device=cuda)
    gpt = torch.empty(qn, dtype=torch.float32, device=cuda)
    t.sample_pdf(_t(g["qcell"], cuda), _t(g["qseeds"], cuda), out_uv=guv, out_pdf_tree=gpt)
    torch.cuda.synchronize()
    uv = guv.cpu().numpy()
    same = np.all(uv == g["sample_uv"], axis=1)
    assert same.mean() >= 0.999
    np.testing.assert_allclose(gpt.cpu().numpy()[same], g["sample_pdf"][same], rtol=1e-4)
