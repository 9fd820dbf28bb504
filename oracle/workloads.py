"""The benchmark workloads as plain arrays, for processes that drive only the
reference's own code (bench.py --impl reference) and must not load this
project's library. Test infrastructure, like everything under oracle/.

Each generator restates the seeded generator of the same name in
rayon_b200/scenes.py draw for draw (same numpy PCG64 streams, same order of
draws, same arrays); tests/test_workloads.py checks that both produce
identical materials, geometry arrays, cameras and settings. Materials are
refbind.RefMaterial structures (the rb_material_desc layout), and cameras
take their frame from the reference's own CameraBase (refbind.camera_frame).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .refbind import RefMaterial, as_ref_material

KIND_SPHERE, KIND_RECT, KIND_TRI, KIND_SDF = 0, 1, 2, 3
# Scene::MaterialType / SDFType numbering (scene_description.hpp:29-43, 296-309)
LAMBERTIAN, METAL, GLASS, LIGHT, ANISOTROPIC_METAL = 0, 1, 4, 6, 10
SDF_TORUS, SDF_CAPSULE, SDF_ROUND_BOX = 2, 3, 32


def lambertian(c) -> RefMaterial:
    return as_ref_material(dict(type=LAMBERTIAN, albedo=c))


def metal(c, fuzz) -> RefMaterial:
    return as_ref_material(dict(type=METAL, albedo=c, roughness=fuzz, metallic=1.0))


def glass(ior) -> RefMaterial:
    return as_ref_material(dict(type=GLASS, albedo=(1, 1, 1), refractive_index=ior, transmission=1.0))


def light(e) -> RefMaterial:
    return as_ref_material(dict(type=LIGHT, albedo=(1, 1, 1), emission=e))


def ggx_from_f0(roughness, f0) -> RefMaterial:
    s = np.sqrt(f0)
    eta = (1 + s) / (1 - s)
    return as_ref_material(dict(type=ANISOTROPIC_METAL, albedo=(1, 1, 1), roughness=roughness, anisotropy=0.0,
                                metallic=1.0, eta=(eta, eta, eta), k=(0.0, 0.0, 0.0)))


@dataclass
class Camera:
    look_from: tuple
    look_at: tuple
    vup: tuple = (0.0, 1.0, 0.0)
    vfov: float = 40.0

    def frame(self, width: int, height: int) -> np.ndarray:
        from .refbind import camera_frame
        return camera_frame(self, width, height)


@dataclass
class Workload:
    name: str
    materials: list
    kinds: np.ndarray
    params: np.ndarray
    mats: np.ndarray
    camera: Camera
    width: int
    height: int
    spp: int
    depth: int
    background: float = 1.0
    dof: tuple | None = None
    sdf_blend: float = 0.0
    sdf_steps: int = 256
    sdf_eps: float = 1e-4
    views: list = field(default_factory=list)

    @property
    def n(self) -> int:
        return int(self.kinds.shape[0])


class _Arrays:
    def __init__(self):
        self.materials, self.rows, self.kinds, self.mats = [], [], [], []

    def mat(self, m) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def add(self, kind, values, m):
        p = np.zeros(18)
        p[:len(values)] = values
        self.kinds.append(kind)
        self.rows.append(p)
        self.mats.append(m)

    def arrays(self):
        return (np.asarray(self.kinds, np.uint8), np.asarray(self.rows, np.float64).reshape(-1, 18),
                np.asarray(self.mats, np.int32))


def one_weekend(seed: int = 42, width: int = 400, height: int = 225, spp: int = 32, depth: int = 10) -> Workload:
    """400x225, 32 spp, depth 10: ground r=1000, three r=1 spheres, 22x22 grid of
    r=0.2 spheres; per cell: choose, u, v, then Lambert albedo U3*U3 / metal
    U[0.5,1]^3 + fuzz U[0,0.5] / glass 1.5 at 80/15/5 %."""
    rng = np.random.default_rng(seed)
    A = _Arrays()
    A.add(KIND_SPHERE, [0, -1000, 0, 1000], A.mat(lambertian((0.5, 0.5, 0.5))))
    A.add(KIND_SPHERE, [0, 1, 0, 1.0], A.mat(glass(1.5)))
    A.add(KIND_SPHERE, [-4, 1, 0, 1.0], A.mat(lambertian((0.4, 0.2, 0.1))))
    A.add(KIND_SPHERE, [4, 1, 0, 1.0], A.mat(metal((0.7, 0.6, 0.5), 0.0)))
    for a in range(-11, 11):
        for b in range(-11, 11):
            choose, u, v = rng.random(3)
            if choose < 0.8:
                m = A.mat(lambertian(rng.random(3) * rng.random(3)))
            elif choose < 0.95:
                alb = rng.uniform(0.5, 1.0, 3)
                m = A.mat(metal(alb, rng.uniform(0.0, 0.5)))
            else:
                m = A.mat(glass(1.5))
            A.add(KIND_SPHERE, [a + 0.9 * u, 0.2, b + 0.9 * v, 0.2], m)
    k, p, m = A.arrays()
    return Workload("one_weekend", A.materials, k, p, m, Camera((13, 2, 3), (0, 0, 0), (0, 1, 0), 20.0), width, height,
                    spp, depth, background=1.0, dof=(0.1, 10.0))


def _box(lo, hi, angle_deg, offset):
    """12 triangles of the box [lo, hi] rotated about +y by angle_deg, then moved by offset."""
    th = np.deg2rad(angle_deg)
    ct, st = np.cos(th), np.sin(th)
    corners = [np.array([x, y, z], float) for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])]
    v = [np.array([ct * q[0] + st * q[2], q[1], -st * q[0] + ct * q[2]]) + np.asarray(offset, float) for q in corners]
    out = []
    for f in [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]:
        out.append(np.concatenate([v[f[0]], v[f[1]], v[f[2]]]))
        out.append(np.concatenate([v[f[0]], v[f[2]], v[f[3]]]))
    return out


def cornell(width: int = 512, height: int = 512, spp: int = 256, depth: int = 16) -> Workload:
    """555^3 box of five quads, a 130x105 ceiling light (emission 15), two white
    boxes (165x330x165 at +15 deg, 165^3 at -18 deg) as 24 triangles; background 0."""
    A = _Arrays()
    red, white = A.mat(lambertian((0.65, 0.05, 0.05))), A.mat(lambertian((0.73, 0.73, 0.73)))
    green, lt = A.mat(lambertian((0.12, 0.45, 0.15))), A.mat(light((15.0, 15.0, 15.0)))
    for q, m in [((555, 0, 0, 0, 555, 0, 0, 0, 555), green), ((0, 0, 0, 0, 555, 0, 0, 0, 555), red),
                 ((343, 554, 332, -130, 0, 0, 0, 0, -105), lt), ((0, 0, 0, 555, 0, 0, 0, 0, 555), white),
                 ((555, 555, 555, -555, 0, 0, 0, 0, -555), white), ((0, 0, 555, 555, 0, 0, 0, 555, 0), white)]:
        A.add(KIND_RECT, q, m)
    for t in _box((0, 0, 0), (165, 330, 165), 15.0, (265, 0, 295)) + _box((0, 0, 0), (165, 165, 165), -18.0,
                                                                          (130, 0, 65)):
        A.add(KIND_TRI, t, white)
    k, p, m = A.arrays()
    return Workload("cornell", A.materials, k, p, m, Camera((278, 278, -800), (278, 278, 0), (0, 1, 0), 40.0), width,
                    height, spp, depth, background=0.0)


def unit_icosphere(level: int) -> np.ndarray:
    """Triangles (20 * 4^level, 3, 3) of the unit icosahedron subdivided at edge
    midpoints (each pushed back to the sphere) level times."""
    g = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, g, 0], [1, g, 0], [-1, -g, 0], [1, -g, 0], [0, -1, g], [0, 1, g], [0, -1, -g], [0, 1, -g],
                  [g, 0, -1], [g, 0, 1], [-g, 0, -1], [-g, 0, 1]], float)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                  [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    t = v[f]
    for _ in range(level):
        a, b, c = t[:, 0], t[:, 1], t[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        t = np.stack([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                      np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3, 3)
    return t


def icospheres(seed: int = 7, count: int = 64, level: int = 6, width: int = 1920, height: int = 1080, spp: int = 64,
               depth: int = 8) -> Workload:
    """64 level-6 icospheres: per sphere centre U[-50,50]^3, radius U[1,4],
    roughness U[0.05,0.8], F0 U[0.02,0.95] (GGX conductor); Lambert ground quad."""
    rng = np.random.default_rng(seed)
    unit = unit_icosphere(level).reshape(-1, 9)
    materials = [lambertian((0.5, 0.5, 0.5))]
    tris, tm = [], []
    for _ in range(count):
        c = rng.uniform(-50, 50, 3)
        r = rng.uniform(1, 4)
        rough = rng.uniform(0.05, 0.8)
        f0 = rng.uniform(0.02, 0.95)
        materials.append(ggx_from_f0(rough, f0))
        tris.append(unit * r + np.tile(c, 3))
        tm.append(np.full(unit.shape[0], len(materials) - 1, np.int32))
    tri = np.concatenate(tris)
    n = tri.shape[0]
    kinds = np.full(n + 1, KIND_TRI, np.uint8)
    kinds[0] = KIND_RECT
    params = np.zeros((n + 1, 18))
    params[0, :9] = [-200, -56, -200, 400, 0, 0, 0, 0, 400]
    params[1:, :9] = tri
    mats = np.concatenate([[0], np.concatenate(tm)]).astype(np.int32)
    return Workload("icospheres", materials, kinds, params, mats, Camera((0, 40, 170), (0, 0, 0), (0, 1, 0), 45.0),
                    width, height, spp, depth, background=1.0)


def sdf_field(seed: int = 11, count: int = 256, width: int = 1280, height: int = 720, spp: int = 128, depth: int = 8,
              views: int = 16) -> Workload:
    """256 SDF primitives (rounded box / torus / capsule by a uniform draw),
    position U[-20,20]^3, size U[0.5,3], rotation U[0,2pi)^3, Lambert / GGX /
    glass at 0.5 / 0.3 / 0.2; smooth union k = 0.2; 16 orbit views at radius 60."""
    rng = np.random.default_rng(seed)
    A = _Arrays()
    A.add(KIND_RECT, [-400, -25, -400, 800, 0, 0, 0, 0, 800], A.mat(lambertian((0.5, 0.5, 0.5))))
    for _ in range(count):
        kind = int(rng.integers(0, 3))
        pos = rng.uniform(-20, 20, 3)
        size = rng.uniform(0.5, 3.0)
        rot = rng.uniform(0, 2 * np.pi, 3)
        mk = rng.random()
        col = rng.uniform(0.2, 0.9, 3)
        if mk < 0.5:
            m = A.mat(lambertian(col))
        elif mk < 0.8:
            m = A.mat(ggx_from_f0(rng.uniform(0.05, 0.8), rng.uniform(0.02, 0.95)))
        else:
            m = A.mat(glass(1.5))
        t, prm = ((SDF_ROUND_BOX, (size, size * 0.8, size * 0.6)) if kind == 0 else
                  (SDF_TORUS, (size, size * 0.3, 0)) if kind == 1 else (SDF_CAPSULE, (size * 0.4, size, 0)))
        A.add(KIND_SDF, [t, *pos, *prm, *rot], m)
    k, p, m = A.arrays()
    vs = [Camera((60 * np.cos(2 * np.pi * v / views), 15, 60 * np.sin(2 * np.pi * v / views)), (0, 0, 0), (0, 1, 0),
                 45.0) for v in range(views)]
    return Workload("sdf_field", A.materials, k, p, m, vs[0], width, height, spp, depth, background=1.0,
                    sdf_blend=0.2, sdf_steps=256, sdf_eps=1e-4, views=vs)


WORKLOADS = {"one_weekend": one_weekend, "cornell": cornell, "icospheres": icospheres, "sdf_field": sdf_field}
