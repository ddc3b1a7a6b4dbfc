"""Inputs of the integrator's known-answer tests (not a test module): random shading
vertices on every material of the glass / Phong Cornell box and SD-trees that the C
restatement and RTLib's own code build identically."""
import numpy as np

from rtlib_b200 import scenes
from rtlib_b200 import workloads as W

AABB = ((-0.005,) * 3, (1.005,) * 3)
# RTLib's PARAM_FLAG_* combinations the shading is checked under: unguided without NEE, NEE,
# NEE + RIS, SD-tree recording, SD-tree guided (BUILD) with NEE and with RIS
FLAG_SETS = (0, 1, 3, 8, 8 | 16 | 1, 8 | 16 | 3)


def scene():
    return scenes.cornell_box(8, 8, light_grid=2, materials="glass_phong")


def shade_cases(sc, n, seed):
    """n hits spread over all triangles: a uniform point of the triangle reached from a
    random direction (three in four from the front side) over a distance in [0.05, 1.2],
    with a random throughput, previous hit flags (none, COUNT_EMITTED, COUNT_EMITTED|DELTA),
    depth 0..7 and Xorshift32 seed."""
    rng = np.random.default_rng(seed)
    tv = sc["tri_v"].astype(np.float64).reshape(-1, 3, 3)
    prim = rng.integers(0, tv.shape[0], n).astype(np.uint32)
    u, v = rng.random(n), rng.random(n)
    flip = u + v > 1
    u[flip], v[flip] = 1 - u[flip], 1 - v[flip]
    v0, e1, e2 = tv[prim, 0], tv[prim, 1] - tv[prim, 0], tv[prim, 2] - tv[prim, 0]
    point = v0 + u[:, None] * e1 + v[:, None] * e2
    fn = np.cross(e1, e2)
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    front = rng.random(n) < 0.75
    s = np.sign((d * fn).sum(1))
    d *= np.where(front, -s, s)[:, None]
    t = rng.uniform(0.05, 1.2, n)
    d32 = d.astype(np.float32)
    org = (point - t[:, None] * d32.astype(np.float64)).astype(np.float32)
    return {"org": org, "dir": d32, "t": t.astype(np.float32), "prim": prim,
            "thr": rng.uniform(0.05, 1.0, (n, 3)).astype(np.float32),
            "pflags": rng.choice(np.array([0, 8, 10], np.uint32), n, p=[0.5, 0.35, 0.15]).astype(np.uint32),
            "depth": rng.integers(0, 8, n).astype(np.uint32),
            "seeds": (rng.integers(1, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) | np.uint32(1))}


def tree_records(seed=5, n=4096):
    """Records whose radiance is a multiple of 1/64: every float sum of RTLib's tree is then
    exact and equal to the fixed-point sums of the restatement, so both build the same tree."""
    rec = W.sdtree_records(n, seed)
    rad = np.maximum(np.round(rec["radiance"] * 64.0), 1.0) / 64.0
    return rec["pos"], rec["uv"], rad.astype(np.float32)


def build_tree(checker, records, th=1000):
    """record -> build -> refine -> record -> build, on an Oracle or a Reference."""
    pos, uv, rad = records
    t = checker.sdtree(*AABB)
    t.record(pos, uv, rad)
    t.build()
    t.refine(th)
    t.record(pos, uv, rad)
    t.build()
    return t
