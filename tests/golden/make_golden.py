"""Generate the golden fixtures of tests/golden/ from RTLib's own code.

Runs the reference oracle (oracle/_ref/libref_rtlib.so, RTLib's guiding headers compiled on
the host by oracle/ref) on small seeded inputs and stores inputs and outputs as .npz files,
so the parity tests can check the CPU oracle (and the CUDA path) against the reference on
machines where the reference tree is absent.

    python tests/golden/make_golden.py [kat sdtree hashgrid mqt integrator]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from rtlib_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def kat(r):
    xs = np.array([0, 1, 2, 3, 17, 255, 65535, 123456789, 0xDEADBEEF, 0xFFFFFFFF], np.uint32)
    pcg = np.array([r.L.ref_pcg1d(int(x)) for x in xs], np.uint32)
    xxh = np.array([r.L.ref_xxhash(int(x)) for x in xs], np.uint32)
    seeds = np.array([1, 2, 12345, 0x9E3779B9, 0xFFFFFFFF], np.uint32)
    floats, states = [], []
    for s in seeds:
        f, st = r.xorshift32_floats(int(s), 16)
        floats.append(f)
        states.append(st)
    rng = np.random.default_rng(3)
    d = rng.normal(size=(256, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:6] = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0]]
    uv = r.dir_to_canonical(d)
    mx = np.arange(64, dtype=np.uint32)
    m2 = np.array([[r.L.ref_morton2_code(int(x), int(y)) for y in mx] for x in mx], np.uint32)
    np.savez_compressed(os.path.join(OUT, "kat_math.npz"), xs=xs, pcg1d=pcg, xxhash=xxh, seeds=seeds,
                        xs32_floats=np.array(floats), xs32_state=np.array(states, np.uint32), dirs=d, canon=uv,
                        morton2=m2)


def sdtree(r):
    """Two passes of record -> build -> refine on 2^14 records (thresholds scaled to the
    record count), then 4096 sample+pdf queries."""
    rec = W.sdtree_records(1 << 14, 42)
    q = W.sdtree_queries(4096, 43)
    t = r.sdtree((0, 0, 0), (1, 1, 1))
    out = {}
    for it, th in ((1, 400), (2, 300)):
        t.record(rec["pos"], rec["uv"], rec["radiance"])
        t.build()
        e = t.export(True)
        out.update({f"p{it}_smask": e.smask, f"p{it}_scalars": e.scalars, f"p{it}_counts": e.counts,
                    f"p{it}_dmask": e.dmask, f"p{it}_dsums": e.dsums})
        t.refine(th)
        e = t.export(False)
        out.update({f"r{it}_smask": e.smask, f"r{it}_counts": e.counts, f"r{it}_dmask": e.dmask})
    t.record(rec["pos"], rec["uv"], rec["radiance"])
    t.build()
    e = t.export(True)
    out.update({"p3_smask": e.smask, "p3_counts": e.counts, "p3_dmask": e.dmask, "p3_dsums": e.dsums,
                "p3_scalars": e.scalars})
    uv, pdf = t.sample_pdf(q["pos"], q["seeds"])
    np.savez_compressed(os.path.join(OUT, "sdtree_small.npz"), pos=rec["pos"], uv=rec["uv"], radiance=rec["radiance"],
                        qpos=q["pos"], qseeds=q["seeds"], sample_uv=uv, sample_pdf=pdf, th=np.array([400, 300]),
                        **out)


def hashgrid(r):
    """Sequential inserts into a 128x64x128 grid with 4096 slots (128 buckets of 32), then
    lookups of other points in the filled table."""
    rng = np.random.default_rng(7)
    off = np.array([-1.0, -0.5, -1.0], np.float32)
    size = np.array([2.0, 1.0, 2.0], np.float32)
    bounds = np.array([128, 64, 128], np.uint32)
    nslots = 4096
    # clustered points so that buckets repeat and some fill up
    centers = rng.random((300, 3)).astype(np.float32) * size + off
    pos = (centers[rng.integers(0, 300, 20000)] + rng.normal(0, 0.02, (20000, 3))).astype(np.float32)
    pos = np.clip(pos, off, off + size).astype(np.float32)
    # corners and a point beyond the far corner (clamped to bounds - 1).  Points below the
    # near corner are left out: RTLib converts the negative float to unsigned, which is
    # undefined on the host (the device conversion saturates to 0, as the oracle does).
    pos[:4] = [[-1, -0.5, -1], [1, 0.5, 1], [5, 5, 5], [0.999, 0.499, 0.999]]
    cur = np.zeros(nslots, np.uint32)
    slots = r.hashgrid_insert(pos, off, size, bounds, nslots, cur)
    qpos = (centers[rng.integers(0, 300, 5000)] + rng.normal(0, 0.05, (5000, 3))).astype(np.float32)
    qpos = np.clip(qpos, off, off + size).astype(np.float32)
    look = r.hashgrid_lookup(qpos, off, size, bounds, nslots, cur.copy())
    np.savez_compressed(os.path.join(OUT, "hashgrid_small.npz"), off=off, size=size, bounds=bounds,
                        nslots=np.array([nslots]), pos=pos, slots=slots, table=cur, qpos=qpos, lookup=look)


def mqt(r):
    """Morton quadtree (MaxLevel 6): leaf records into 16 cells, the pyramid build, then
    SampleAndPdf / Pdf."""
    rng = np.random.default_rng(11)
    level, ncells = 6, 16
    per = ((1 << (2 * (6 + 1))) - 1) // 3
    n = 20000
    cell = rng.integers(0, ncells, n).astype(np.uint32)
    cell[:10] = 0xFFFFFFFF
    rec = W.sdtree_records(n, 12)
    uv = rec["uv"]
    uv[0] = [0.0, 0.0]
    val = rec["radiance"]
    w = np.zeros(ncells * per, np.float32)
    r.mqt_record(level, w, cell, uv, val)
    leaves = w.copy()
    r.mqt_build(ncells, level, w)
    q = 8192
    qcell = rng.integers(0, ncells, q).astype(np.uint32)
    seeds = rng.integers(1, 2**32, q, dtype=np.uint64).astype(np.uint32)
    suv, spdf, pe = r.mqt_sample_pdf(level, w, qcell, seeds)
    np.savez_compressed(os.path.join(OUT, "mqt_small.npz"), level=np.array([level]), ncells=np.array([ncells]),
                        cell=cell, uv=uv, value=val, leaves=leaves, pyramid=w, qcell=qcell, qseeds=seeds,
                        sample_uv=suv, sample_pdf=spdf, pdf_eval=pe)


def integrator(r):
    """The integrator's building blocks from RTLib's own code (SimpleKernel.h, SimpleGuide.cu,
    Random.h, VectorFunction.h, staged by oracle/ref): cosine and Phong lobe samples, points
    in triangles, reservoir sequences, light samples of the glass / Phong Cornell box (2 x 2
    light meshes), and whole closest-hit shadings of 1024 random vertices under each flag set,
    the SD-tree ones in the tree both sides build from tests/kat_integrator.py's records."""
    sys.path.insert(0, os.path.dirname(OUT))
    import kat_integrator as K
    from oracle.oracle import IntegratorKAT
    sc = K.scene()
    kat_ = IntegratorKAT(r, sc, fraction=0.5)
    rng = np.random.default_rng(17)
    n = 2048
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    seeds = rng.integers(1, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    shin = rng.choice(np.array([1.0, 10.0, 40.0, 200.0], np.float32), n)
    tri = rng.uniform(-1, 1, (n, 9)).astype(np.float32)
    pin = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    w = rng.lognormal(0.0, 1.0, (256, 32)).astype(np.float32)
    w[::5, ::3] = 0.0
    w[7] = 0.0
    rnd = rng.random((256, 32)).astype(np.float32)
    cos_d, cos_s = kat_.cosine(nrm, seeds)
    ph_d, ph_s = kat_.phong(nrm, shin, seeds)
    tr_p, tr_s = kat_.triangle(tri, seeds)
    lt_o, lt_s = kat_.light(pin, seeds)
    sel, wsum, m = kat_.reservoir(w, rnd)
    out = dict(normal=nrm, seeds=seeds, shininess=shin, tri=tri, p_in=pin, res_w=w, res_rnd=rnd, cos_dir=cos_d,
               cos_state=cos_s, phong_dir=ph_d, phong_state=ph_s, tri_point=tr_p, tri_state=tr_s, light=lt_o,
               light_state=lt_s, res_sel=sel, res_wsum=wsum, res_m=m)
    cases = K.shade_cases(sc, 1024, 23)
    out.update({"case_" + k: v for k, v in cases.items()})
    tree = K.build_tree(r, K.tree_records())
    for fl in K.FLAG_SETS:
        o, f, st = kat_.shade(fl, cases, tree if fl & 8 else None)
        out.update({f"shade{fl}_out": o, f"shade{fl}_flags": f, f"shade{fl}_state": st})
    np.savez_compressed(os.path.join(OUT, "kat_integrator.npz"), flag_sets=np.array(K.FLAG_SETS), **out)


if __name__ == "__main__":
    r = Reference()
    which = sys.argv[1:] or ["kat", "sdtree", "hashgrid", "mqt", "integrator"]
    for name in which:
        globals()[name](r)
    print("golden fixtures", which, "written to", OUT)
