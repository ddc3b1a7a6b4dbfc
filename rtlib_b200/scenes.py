"""Procedural scenes of the integrator workloads (numpy, host side).

Each builder returns a dict of contiguous arrays describing a triangle soup:
  tri_v     (nt, 9) float32   v0, v1, v2 of every triangle; the face normal
                              cross(v1 - v0, v2 - v0) points to the lit side
  tri_mat   (nt,)   uint32    material index
  tri_uv    (nt, 6) float32   texture coordinates of v0, v1, v2
  materials list of dicts     diffuse, specular, emission, shininess, ref_index, type, texture
  light_tris, light_first, light_count, light_emission   NEE light meshes (MeshLightList)
  camera    dict eye/u/v/w    (RayGenData)
"""
from __future__ import annotations

import numpy as np

PHONG, GLASS, NEE_LIGHT, DEF_LIGHT = 0, 1, 2, 3


def _mat(diffuse=(0, 0, 0), specular=(0, 0, 0), emission=(0, 0, 0), shininess=0.0, ref_index=1.0, type=PHONG,
         texture=-1):
    return {"diffuse": tuple(map(float, diffuse)), "specular": tuple(map(float, specular)),
            "emission": tuple(map(float, emission)), "shininess": float(shininess), "ref_index": float(ref_index),
            "type": int(type), "texture": int(texture)}


class _Builder:
    def __init__(self):
        self.tris, self.mats, self.uvs = [], [], []

    def quad(self, p, e1, e2, mat, uv=((0, 0), (1, 0), (1, 1), (0, 1))):
        p, e1, e2 = (np.asarray(x, np.float64) for x in (p, e1, e2))
        a, b, c, d = p, p + e1, p + e1 + e2, p + e2
        self.tris += [np.concatenate([a, b, c]), np.concatenate([a, c, d])]
        self.mats += [mat, mat]
        (ua, ub, uc, ud) = uv
        self.uvs += [np.array([*ua, *ub, *uc], np.float64), np.array([*ua, *uc, *ud], np.float64)]
        return len(self.tris) - 2

    def box(self, center, size, yaw_deg, mat):
        """Axis-aligned box rotated about +y, outward normals (12 triangles)."""
        c = np.asarray(center, np.float64)
        h = np.asarray(size, np.float64) / 2
        t = np.radians(yaw_deg)
        R = np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])
        ex, ey, ez = R @ np.array([2 * h[0], 0, 0]), R @ np.array([0, 2 * h[1], 0]), R @ np.array([0, 0, 2 * h[2]])
        o = c - (ex + ey + ez) / 2
        self.quad(o, ex, ez, mat)             # bottom  (-y)
        self.quad(o + ey, ez, ex, mat)        # top     (+y)
        self.quad(o, ey, ex, mat)             # front   (-z)
        self.quad(o + ez, ex, ey, mat)        # back    (+z)
        self.quad(o, ez, ey, mat)             # left    (-x)
        self.quad(o + ex, ey, ez, mat)        # right   (+x)

    def mesh(self, verts, faces, mat):
        for f in faces:
            self.tris.append(np.concatenate([verts[f[0]], verts[f[1]], verts[f[2]]]))
            self.mats.append(mat)
            self.uvs.append(np.zeros(6))

    def arrays(self):
        return (np.ascontiguousarray(np.array(self.tris, np.float32)),
                np.ascontiguousarray(np.array(self.mats, np.uint32)),
                np.ascontiguousarray(np.array(self.uvs, np.float32)))


def _camera(eye, look, up, vfov_deg, aspect):
    eye, look, up = (np.asarray(x, np.float64) for x in (eye, look, up))
    w = look - eye
    w /= np.linalg.norm(w)
    u = np.cross(w, up)
    u /= np.linalg.norm(u)
    v = np.cross(u, w)
    th = np.tan(np.radians(vfov_deg) / 2)
    return {"eye": eye.astype(np.float32), "u": (u * th * aspect).astype(np.float32),
            "v": (v * th).astype(np.float32), "w": w.astype(np.float32)}


def cornell_box(width=512, height=512, light_grid=1, back_texture=False, materials="lambert"):
    """Cornell-style box in [0,1]^3: five wall quads, two boxes rotated -18 / +18 degrees
    (34 triangles), and a 0.25 x 0.25 emissive quad under the ceiling, radiance (17,12,4),
    split into light_grid x light_grid quads (each its own NEE light mesh).  Albedos 0.73
    (white), (0.65,0.05,0.05) (red, left), (0.12,0.45,0.15) (green, right).  back_texture
    gives the back wall material diffuse texture 0 (albedo 1 times the texture).

    materials="glass_phong" exercises RTLib's other two shading branches: the tall box is a
    dielectric (index 1.5, specular (0.98, 0.98, 0.98); SimpleGuide.cu:424-491), the back wall a
    Phong surface (diffuse 0.45, specular 0.25, shininess 40) and the short box a glossy one
    (diffuse 0.2, specular 0.6, shininess 200), so the Phong lobe and its selection
    probability (SimpleGuide.cu:331-377) and delta vertices enter every path."""
    b = _Builder()
    if materials not in ("lambert", "glass_phong"):
        raise ValueError(f"unknown material set {materials!r}")
    gp = materials == "glass_phong"
    back = (_mat(diffuse=(1.0, 1.0, 1.0) if back_texture else (0.73, 0.73, 0.73), texture=0 if back_texture else -1)
            if not gp else _mat(diffuse=(0.45, 0.45, 0.45), specular=(0.25, 0.25, 0.25), shininess=40.0))
    mats = [_mat(diffuse=(0.73, 0.73, 0.73)), _mat(diffuse=(0.65, 0.05, 0.05)), _mat(diffuse=(0.12, 0.45, 0.15)), back]
    W, R, G, BK = 0, 1, 2, 3
    short_box, tall_box = W, W
    if gp:
        mats.append(_mat(diffuse=(0.2, 0.2, 0.2), specular=(0.6, 0.6, 0.6), shininess=200.0))
        short_box = len(mats) - 1
        mats.append(_mat(specular=(0.98, 0.98, 0.98), ref_index=1.5, type=GLASS))
        tall_box = len(mats) - 1
    b.quad((0, 0, 0), (0, 0, 1), (1, 0, 0), W)      # floor, normal +y
    b.quad((0, 1, 0), (1, 0, 0), (0, 0, 1), W)      # ceiling, normal -y
    b.quad((0, 0, 0), (1, 0, 0), (0, 1, 0), BK)     # back wall z=0, normal +z
    b.quad((0, 0, 0), (0, 1, 0), (0, 0, 1), R)      # left wall x=0, normal +x
    b.quad((1, 0, 0), (0, 0, 1), (0, 1, 0), G)      # right wall x=1, normal -x
    # the boxes stand 1 mm above the floor: a bottom face coplanar with the floor would make
    # the closest hit a tie between two triangles with opposite normals
    b.box((0.33, 0.151, 0.62), (0.3, 0.3, 0.3), -18.0, short_box)
    b.box((0.66, 0.301, 0.36), (0.3, 0.6, 0.3), 18.0, tall_box)
    n_geom = len(b.tris)
    light_first, light_count, light_emit = [], [], []
    s = 0.25 / light_grid
    lmat0 = len(mats)
    for j in range(light_grid):
        for i in range(light_grid):
            mats.append(_mat(emission=(17.0, 12.0, 4.0), type=NEE_LIGHT))
            t0 = b.quad((0.375 + i * s, 0.999, 0.375 + j * s), (s, 0, 0), (0, 0, s), len(mats) - 1)
            light_first.append(t0 - n_geom)
            light_count.append(2)
            light_emit.append((17.0, 12.0, 4.0))
    tri_v, tri_mat, tri_uv = b.arrays()
    light_tris = np.arange(n_geom, len(b.tris), dtype=np.uint32)
    return {"tri_v": tri_v, "tri_mat": tri_mat, "tri_uv": tri_uv, "materials": mats, "light_tris": light_tris,
            "light_first": np.array(light_first, np.uint32), "light_count": np.array(light_count, np.uint32),
            "light_emission": np.array(light_emit, np.float32).reshape(-1), "light_material_first": lmat0,
            "camera": _camera((0.5, 0.5, 1.95), (0.5, 0.5, 0.0), (0, 1, 0), 40.0, width / height),
            "width": width, "height": height, "geometry_triangles": n_geom}


def _icosphere(level):
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]

        nf = []
        for a, b_, c in f:
            ab, bc, ca = mid(a, b_), mid(b_, c), mid(c, a)
            nf += [(a, ab, ca), (b_, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v), np.array(f)


def occluded_rooms(width=1280, height=720, n_objects=2048, n_lights=4096, seed=3, sphere_level=3, light_margin=0.25):
    """The occluded-light scene: a 10 x 4 x 10 room filled with n_objects random icospheres and
    boxes (radii U[0.05, 0.4]); light enters only through a 1 x 2 doorway in the x = 10 wall
    from a neighbouring 4 x 4 x 10 room whose far wall (x = 14, facing the doorway) holds
    n_lights emissive triangles, each its own NEE light with radiance lognormal(0, 1.5) (grey).  With level-3 icospheres (1280
    triangles) for 807 of the objects and boxes for the rest the scene has about 2^20
    triangles.

    The emitter panel keeps a margin of `light_margin` metres from the light room's floor,
    ceiling and side walls.  An emitter whose edge touches another surface makes the NEE
    estimator at that surface's points next to the edge unbounded (cos * cos / d^2 with d -> 0)
    and of infinite variance, so an image error would then be dominated by a few fireflies;
    with the margin the geometry term of a light-room surface is at most 1 / margin^2."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    mats = [_mat(diffuse=(0.7, 0.7, 0.7)), _mat(diffuse=(0.6, 0.55, 0.5)), _mat(diffuse=(0.5, 0.6, 0.7))]
    # main room walls (normals inward), open towards nothing: closed box except the doorway
    b.quad((0, 0, 0), (0, 0, 10), (10, 0, 0), 0)          # floor
    b.quad((0, 4, 0), (10, 0, 0), (0, 0, 10), 0)          # ceiling
    b.quad((0, 0, 0), (10, 0, 0), (0, 4, 0), 0)           # z = 0
    b.quad((0, 0, 10), (0, 4, 0), (10, 0, 0), 0)          # z = 10
    b.quad((0, 0, 0), (0, 4, 0), (0, 0, 10), 0)           # x = 0
    # x = 10 wall with a doorway z in [4.5, 5.5], y in [0, 2]; both faces
    for (z0, z1, y0, y1) in ((0, 4.5, 0, 4), (5.5, 10, 0, 4), (4.5, 5.5, 2, 4)):
        b.quad((10, y0, z0), (0, 0, z1 - z0), (0, y1 - y0, 0), 0)   # facing -x (main room)
        b.quad((10, y0, z0), (0, y1 - y0, 0), (0, 0, z1 - z0), 0)   # facing +x (light room)
    # light room x in [10, 14]
    b.quad((10, 0, 0), (0, 0, 10), (4, 0, 0), 1)          # floor
    b.quad((10, 0, 0), (4, 0, 0), (0, 4, 0), 1)           # z = 0
    b.quad((10, 0, 10), (0, 4, 0), (4, 0, 0), 1)          # z = 10
    b.quad((14, 0, 0), (0, 0, 10), (0, 4, 0), 1)          # x = 14
    b.quad((10, 4, 0), (4, 0, 0), (0, 0, 10), 1)          # ceiling behind the lights
    # objects
    sv, sf = _icosphere(sphere_level)
    n_sph = min(n_objects, 807)
    kinds = np.array([1] * n_sph + [0] * (n_objects - n_sph))
    rng.shuffle(kinds)
    eye = np.array([7.5, 1.6, 3.6])
    for k in kinds:
        r = rng.uniform(0.05, 0.4)
        # nothing within 1.5 m of the camera (its view would start inside an object)
        while True:
            c = np.array([rng.uniform(r, 10 - r), rng.uniform(r, 4 - r), rng.uniform(r, 10 - r)])
            if np.linalg.norm(c - eye) > r * 1.8 + 1.5:
                break
        m = int(rng.integers(0, 3))
        if k:
            b.mesh(sv * r + c, sf, m)
        else:
            b.box(c, (2 * r, 2 * r, 2 * r), rng.uniform(0, 90), m)
    n_geom = len(b.tris)
    # emissive triangles tiling the light room's far wall (x = 14) just in front of it, facing
    # the doorway (-x): gz x gy quads of two triangles
    nq = n_lights // 2
    gz = 1 << int(np.floor(np.log2(max(1.0, np.sqrt(nq * 2.5)))))
    gy = max(1, nq // gz)
    rad = rng.lognormal(0.0, 1.5, 2 * gy * gz).astype(np.float32)
    light_emit, light_first = [], []
    k = 0
    ly, lz = 4.0 - 2 * light_margin, 10.0 - 2 * light_margin
    for i in range(gy):
        for j in range(gz):
            p = (13.99, light_margin + ly * i / gy, light_margin + lz * j / gz)
            e1, e2 = (0, 0, lz / gz), (0, ly / gy, 0)
            # quad(p, e1, e2): normal e1 x e2 = -x
            for tri in range(2):
                mats.append(_mat(emission=(rad[k],) * 3, type=NEE_LIGHT))
                k += 1
            i0 = b.quad(p, e1, e2, len(mats) - 2)
            b.mats[i0 + 1] = len(mats) - 1
            light_first += [i0 - n_geom, i0 + 1 - n_geom]
            light_emit += [(rad[k - 2],) * 3, (rad[k - 1],) * 3]
    tri_v, tri_mat, tri_uv = b.arrays()
    light_tris = np.arange(n_geom, len(b.tris), dtype=np.uint32)
    return {"tri_v": tri_v, "tri_mat": tri_mat, "tri_uv": tri_uv, "materials": mats, "light_tris": light_tris,
            "light_first": np.array(light_first, np.uint32), "light_count": np.ones(len(light_first), np.uint32),
            "light_emission": np.array(light_emit, np.float32).reshape(-1),
            "camera": _camera(tuple(eye), (10.0, 1.0, 5.0), (0, 1, 0), 60.0, width / height),
            "width": width, "height": height, "geometry_triangles": n_geom}
