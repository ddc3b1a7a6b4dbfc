"""Seeded synthetic inputs for the guiding hot path (numpy, host side).

The SD-tree standalone workload: radiance records with positions uniform in the unit cube,
directions from a 4-lobe von Mises-Fisher mixture (kappa 50, lobe axes uniform on the
sphere, equal weights), FP32 lognormal(0, 1) radiance, woPdf 1 and statistical weight 1;
then sample+pdf queries at uniform positions, each with its own Xorshift32 seed.  The same
arrays feed the CUDA path, the CPU oracle and the reference build, so every implementation
sees identical bits.
"""
from __future__ import annotations

import numpy as np

INV_2PI_F = np.float32(0.15915494309189533576888376337251436203445964574046)
TWO_PI_F = np.float32(6.283185307179586476925286766559)


def dir_to_canonical(d: np.ndarray) -> np.ndarray:
    """Equal-area cylindrical map of unit directions to [0,1]^2, in float32.

    Same formula as RTLib's dir_to_canonical (VectorFunction.h:5706-5720):
    u = (clamp(z) + 1) / 2, v = atan2(y, x) / (2 pi) with phi wrapped into [0, 2 pi).
    """
    d = np.asarray(d, dtype=np.float32)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    ok = np.isfinite(x) & np.isfinite(y) & np.isfinite(z)
    z = np.clip(z, np.float32(-1), np.float32(1))
    phi = np.arctan2(y, x).astype(np.float32)
    phi = np.where(phi < 0, phi + TWO_PI_F, phi).astype(np.float32)
    u = ((z + np.float32(1)) / np.float32(2)).astype(np.float32)
    v = (phi * INV_2PI_F).astype(np.float32)
    out = np.stack([u, v], axis=1).astype(np.float32)
    out[~ok] = 0
    return np.ascontiguousarray(out)


def sample_vmf(mu: np.ndarray, kappa: float, rng: np.random.Generator) -> np.ndarray:
    """Wood's method on S^2: w = 1 + log(u + (1-u) e^{-2k}) / k, uniform azimuth."""
    n = mu.shape[0]
    u = rng.random(n)
    w = 1.0 + np.log(u + (1.0 - u) * np.exp(-2.0 * kappa)) / kappa
    phi = 2.0 * np.pi * rng.random(n)
    # orthonormal frame around mu
    a = np.where(np.abs(mu[:, :1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(mu, a)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(mu, t)
    s = np.sqrt(np.clip(1.0 - w * w, 0.0, None))
    d = w[:, None] * mu + s[:, None] * (np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * b)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def sdtree_records(n: int, seed: int = 0, lobes: int = 4, kappa: float = 50.0):
    """Records of the SD-tree standalone workload.  Returns a dict of contiguous arrays:
    pos (n,3) f32, dir (n,3) f32, uv (n,2) f32 canonical, radiance (n,) f32."""
    rng = np.random.Generator(np.random.PCG64(seed))
    axes = rng.normal(size=(lobes, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    pos = rng.random((n, 3), dtype=np.float32)
    lobe = rng.integers(0, lobes, n)
    d = sample_vmf(axes[lobe], kappa, rng).astype(np.float32)
    radiance = rng.lognormal(0.0, 1.0, n).astype(np.float32)
    return {
        "pos": np.ascontiguousarray(pos),
        "dir": np.ascontiguousarray(d),
        "uv": dir_to_canonical(d),
        "radiance": np.ascontiguousarray(radiance),
    }


def sdtree_queries(n: int, seed: int = 1):
    """Sample+pdf queries: uniform positions and one nonzero Xorshift32 seed each."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.random((n, 3), dtype=np.float32)
    seeds = rng.integers(1, 2**32, n, dtype=np.uint64).astype(np.uint32)
    return {"pos": np.ascontiguousarray(pos), "seeds": np.ascontiguousarray(seeds)}


def spatial_threshold(iteration: int) -> int:
    """Spatial split threshold of the standalone workload: 12000 * sqrt(2^iter), as an
    integer sample count (RTLib compares the stat-weight with a size_t threshold)."""
    return int(12000.0 * np.sqrt(2.0 ** iteration))


def surface_points(tri_v: np.ndarray, n: int, seed: int) -> np.ndarray:
    """n points uniform by area on the triangles tri_v (nt, 9), float32 (n, 3)."""
    tv = np.asarray(tri_v, np.float64).reshape(-1, 3, 3)
    area = 0.5 * np.linalg.norm(np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0]), axis=1)
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = rng.choice(tv.shape[0], size=n, p=area / area.sum())
    a, b = rng.random(n), rng.random(n)
    m = a + b > 1.0
    a[m], b[m] = 1.0 - a[m], 1.0 - b[m]
    p = tv[idx, 0] + a[:, None] * (tv[idx, 1] - tv[idx, 0]) + b[:, None] * (tv[idx, 2] - tv[idx, 0])
    return np.ascontiguousarray(p.astype(np.float32))


def hashgrid_inputs(n_points: int, n_queries: int, seed: int = 0):
    """The hash-grid guide workload on the occluded-light scene: n_points surface points to
    insert (seed), n_queries surface points to look up (seed + 1), and for every query a
    record direction from a 4-lobe vMF mixture (kappa 50) as canonical (u, v), a lognormal(0, 1)
    record value and a nonzero Xorshift32 seed for sample+pdf."""
    from .scenes import occluded_rooms
    sc = occluded_rooms(64, 36)
    geom = sc["tri_v"][: sc["geometry_triangles"]]
    pts = surface_points(geom, n_points, seed)
    qpos = surface_points(geom, n_queries, seed + 1)
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    axes = rng.normal(size=(4, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    d = sample_vmf(axes[rng.integers(0, 4, n_queries)], 50.0, rng).astype(np.float32)
    value = rng.lognormal(0.0, 1.0, n_queries).astype(np.float32)
    seeds = rng.integers(1, 2**32, n_queries, dtype=np.uint64).astype(np.uint32)
    return {"points": pts, "queries": qpos, "uv": dir_to_canonical(d), "value": np.ascontiguousarray(value),
            "seeds": np.ascontiguousarray(seeds)}
