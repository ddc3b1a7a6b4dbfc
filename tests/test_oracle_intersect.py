"""The oracle's hit test (coordinate transformation, the arithmetic the device's tri_hit uses)
against an independent float64 Moller-Trumbore brute force: the same closest triangle and the
same distance to float precision on random triangle soups, the Cornell box and grazing rays.
The device is held to the oracle bit for bit by tests/test_tracer_gpu.py."""
import numpy as np

from oracle.oracle import Oracle
from rtlib_b200 import scenes


def _mt64(tri_v, o, d, tmin, tmax):
    v = tri_v.reshape(-1, 3, 3).astype(np.float64)
    v0, e1, e2 = v[:, 0], v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
    best_t = np.full(o.shape[0], np.inf)
    best_p = np.full(o.shape[0], 0xFFFFFFFF, np.uint32)
    for i in range(o.shape[0]):
        di = d[i].astype(np.float64)
        p = np.cross(di, e2)
        det = np.einsum("ij,ij->i", e1, p)
        with np.errstate(all="ignore"):
            inv = 1.0 / det
            s = o[i].astype(np.float64) - v0
            u = np.einsum("ij,ij->i", s, p) * inv
            q = np.cross(s, e1)
            w = (q @ di) * inv
            t = np.einsum("ij,ij->i", e2, q) * inv
        ok = (np.abs(det) > 0) & (u >= 0) & (w >= 0) & (u + w <= 1) & (t > tmin) & (t < tmax)
        if ok.any():
            k = int(np.argmin(np.where(ok, t, np.inf)))
            best_t[i], best_p[i] = t[k], k
    return best_t, best_p


def _check(tri, o, d, agree=0.999):
    t, p = Oracle().intersect(tri, o, d, 1e-4, 1e20)
    bt, bp = _mt64(tri, o, d, 1e-4, 1e20)
    assert (p == bp).mean() >= agree, (p == bp).mean()
    hit = (p == bp) & (bp != 0xFFFFFFFF)
    np.testing.assert_allclose(t[hit], bt[hit], rtol=2e-5, atol=1e-6)
    return hit.mean()


def test_random_soup():
    rng = np.random.default_rng(3)
    c = rng.random((400, 3)) * 4
    tri = (c[:, None, :] + rng.normal(0, 0.2, (400, 3, 3))).astype(np.float32).reshape(-1, 9)
    o = (rng.random((1500, 3)) * 5 - 0.5).astype(np.float32)
    d = rng.normal(size=(1500, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    assert _check(tri, o, d) > 0.2


def test_cornell_box_and_any_hit():
    tri = np.ascontiguousarray(scenes.cornell_box(8, 8)["tri_v"], np.float32)
    rng = np.random.default_rng(4)
    o = rng.uniform(0.02, 0.98, (3000, 3)).astype(np.float32)
    d = rng.normal(size=(3000, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    assert _check(tri, o, d) > 0.5
    # any hit within 0.3: hit exactly where the closest hit lies within 0.3
    t, p = Oracle().intersect(tri, o, d, 1e-4, 0.3, any_hit=True)
    tc, pc = Oracle().intersect(tri, o, d, 1e-4, 1e20)
    assert np.array_equal(p != 0xFFFFFFFF, (pc != 0xFFFFFFFF) & (tc < 0.3))


def test_grazing_and_parallel_rays():
    # a unit square in z = 0; rays parallel to it never hit, rays at grazing angles do
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0], [1, 0, 0, 1, 1, 0, 0, 1, 0]], np.float32)
    n = 500
    rng = np.random.default_rng(5)
    o = np.column_stack([rng.uniform(0.05, 0.95, n), rng.uniform(0.05, 0.95, n), np.full(n, 0.5)]).astype(np.float32)
    par = np.column_stack([rng.normal(size=n), rng.normal(size=n), np.zeros(n)]).astype(np.float32)
    t, p = Oracle().intersect(tri, o, par, 1e-4, 1e20)
    assert (p == 0xFFFFFFFF).all()
    # 1-6 degrees above the plane, from 1 cm over it: hits 0.1-0.6 away, some beyond the square
    phi = rng.uniform(0, 2 * np.pi, n)
    el = np.radians(rng.uniform(1.0, 6.0, n))
    graze = np.column_stack([np.cos(phi) * np.cos(el), np.sin(phi) * np.cos(el), -np.sin(el)]).astype(np.float32)
    low = o.copy()
    low[:, 2] = 0.01
    assert _check(tri, low, graze, agree=1.0) > 0.3


def test_transform_rows_map_the_vertices():
    """Rows of or_tri_transforms: v0 -> (u, v) = (0, 0), v1 -> (1, 0), v2 -> (0, 1), every vertex at
    normal offset 0, and v0 + n at offset 1 (n = e1 x e2)."""
    import ctypes as C
    rng = np.random.default_rng(6)
    tri = rng.normal(size=(64, 3, 3)).astype(np.float32)
    o = Oracle()
    xf = np.empty((64, 12), np.float32)
    o.L.or_tri_transforms.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    o.L.or_tri_transforms(tri.ctypes.data, 64, xf.ctypes.data)
    r = xf.reshape(64, 3, 4).astype(np.float64)

    def coords(x):
        return np.einsum("tkj,tj->tk", r[:, :, :3], x) + r[:, :, 3]

    v0, v1, v2 = (tri[:, k].astype(np.float64) for k in range(3))
    n = np.cross(v1 - v0, v2 - v0)
    np.testing.assert_allclose(coords(v0), np.zeros((64, 3)), atol=1e-5)
    np.testing.assert_allclose(coords(v1), np.tile([1.0, 0.0, 0.0], (64, 1)), atol=1e-5)
    np.testing.assert_allclose(coords(v2), np.tile([0.0, 1.0, 0.0], (64, 1)), atol=1e-5)
    np.testing.assert_allclose(coords(v0 + n), np.tile([0.0, 0.0, 1.0], (64, 1)), atol=1e-5)
