"""Seeded synthetic workloads.

Each generator returns a SceneSpec: materials plus geometry in insertion order,
the camera and the render settings. The spec is plain arrays, so the same
scene can be fed to this library, to the FP64 oracle and to the reference's
own SceneDescription through its builder calls (addSphere / addRectangle /
addTriangle), never through YAML (which caps at 1000 geometries and has no
SDF primitives, yaml_scene_loader.cc:411, 436-490).

Configurations (parameters as specified for the benchmark suite):
  one_weekend   400x225, 32 spp, depth 10, ~488 spheres, DOF aperture 0.1, seed 42
  cornell       512x512, 256 spp, depth 16, 6 quads + 24 triangles, background 0
  icospheres    1920x1080, 64 spp, depth 8, 64 level-6 icospheres (5,242,880 tris) + ground
  sdf_field     1280x720, 128 spp, depth 8, 256 SDF primitives, smooth union k = 0.2, 16 views
Draw order of every generator is documented inline; numpy's PCG64 (default_rng)
with the stated seed drives all draws.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import scene as S

KIND_SPHERE, KIND_RECT, KIND_TRI, KIND_SDF = 0, 1, 2, 3


@dataclass
class Camera:
    look_from: tuple
    look_at: tuple
    vup: tuple = (0.0, 1.0, 0.0)
    vfov: float = 40.0

    def frame(self, width: int, height: int) -> np.ndarray:
        return S.camera_frame(self.look_from, self.look_at, self.vup, self.vfov, width, height)


@dataclass
class SceneSpec:
    name: str
    materials: list
    kinds: np.ndarray            # (n,) uint8, KIND_*
    params: np.ndarray           # (n, 18) float64: sphere c,r | rect corner,u,v | tri v0,v1,v2 | sdf
    mats: np.ndarray             # (n,) int32
    camera: Camera
    width: int
    height: int
    spp: int
    depth: int
    background: float = 1.0
    dof: tuple | None = None     # (aperture radius, focus distance)
    sdf_blend: float = 0.0
    sdf_steps: int = 256
    sdf_eps: float = 1e-4
    views: list = field(default_factory=list)

    @property
    def n(self) -> int:
        return int(self.kinds.shape[0])

    def to_scene(self) -> S.SceneDescription:
        sc = S.SceneDescription()
        for m in self.materials:
            sc.add_material(m)
        i = 0
        n = self.n
        while i < n:
            j = i
            while j < n and self.kinds[j] == self.kinds[i]:
                j += 1
            k = int(self.kinds[i])
            p, m = self.params[i:j], self.mats[i:j]
            if k == KIND_SPHERE:
                sc.add_spheres(p[:, :4], mat_ids=m)
            elif k == KIND_TRI:
                sc.add_triangles(p[:, :9], mat_ids=m)
            elif k == KIND_RECT:
                for q, mm in zip(p, m):
                    sc.add_rectangle(q[0:3], q[3:6], q[6:9], int(mm))
            elif k == KIND_SDF:
                for q, mm in zip(p, m):
                    sc.add_sdf(int(q[0]), q[1:4], q[4:7], int(mm), rotation=q[7:10])
            i = j
        if self.sdf_blend > 0 or (self.kinds == KIND_SDF).any():
            sc.set_sdf_blend(self.sdf_blend, self.sdf_steps, self.sdf_eps)
        return sc


class _Builder:
    def __init__(self):
        self.materials, self.kinds, self.params, self.mats = [], [], [], []

    def mat(self, m) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def sphere(self, c, r, m):
        p = np.zeros(18)
        p[0:3], p[3] = c, r
        self.kinds.append(KIND_SPHERE); self.params.append(p); self.mats.append(m)

    def rect(self, corner, u, v, m):
        p = np.zeros(18)
        p[0:3], p[3:6], p[6:9] = corner, u, v
        self.kinds.append(KIND_RECT); self.params.append(p); self.mats.append(m)

    def tri(self, v0, v1, v2, m):
        p = np.zeros(18)
        p[0:3], p[3:6], p[6:9] = v0, v1, v2
        self.kinds.append(KIND_TRI); self.params.append(p); self.mats.append(m)

    def sdf(self, t, pos, prm, rot, m):
        p = np.zeros(18)
        p[0], p[1:4], p[4:7], p[7:10] = t, pos, prm, rot
        self.kinds.append(KIND_SDF); self.params.append(p); self.mats.append(m)

    def arrays(self):
        return (np.asarray(self.kinds, np.uint8), np.asarray(self.params, np.float64).reshape(-1, 18),
                np.asarray(self.mats, np.int32))


def one_weekend(seed: int = 42, width: int = 400, height: int = 225, spp: int = 32, depth: int = 10) -> SceneSpec:
    """One-Weekend final scene. Draw order per grid cell (a, b) in row-major order
    a, b in [-11, 11): choose, u, v, then the material's draws: Lambert albedo =
    U3 * U3 (six draws), metal albedo U[0.5,1]^3 then fuzz U[0,0.5], glass none."""
    rng = np.random.default_rng(seed)
    B = _Builder()
    B.sphere((0, -1000, 0), 1000, B.mat(S.lambertian((0.5, 0.5, 0.5))))
    B.sphere((0, 1, 0), 1.0, B.mat(S.glass(1.5)))
    B.sphere((-4, 1, 0), 1.0, B.mat(S.lambertian((0.4, 0.2, 0.1))))
    B.sphere((4, 1, 0), 1.0, B.mat(S.metal((0.7, 0.6, 0.5), 0.0)))
    for a in range(-11, 11):
        for b in range(-11, 11):
            choose, u, v = rng.random(3)
            c = (a + 0.9 * u, 0.2, b + 0.9 * v)
            if choose < 0.8:
                alb = rng.random(3) * rng.random(3)
                m = B.mat(S.lambertian(alb))
            elif choose < 0.95:
                alb = rng.uniform(0.5, 1.0, 3)
                fuzz = rng.uniform(0.0, 0.5)
                m = B.mat(S.metal(alb, fuzz))
            else:
                m = B.mat(S.glass(1.5))
            B.sphere(c, 0.2, m)
    k, p, m = B.arrays()
    return SceneSpec("one_weekend", B.materials, k, p, m, Camera((13, 2, 3), (0, 0, 0), (0, 1, 0), 20.0),
                     width, height, spp, depth, background=1.0, dof=(0.1, 10.0))


def _box_tris(lo, hi, angle_deg, offset):
    """12 triangles of an axis-aligned box rotated about +y then translated."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    c = [np.array([x, y, z]) for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])]
    th = np.deg2rad(angle_deg)
    ct, st = np.cos(th), np.sin(th)

    def tf(p):
        return np.array([ct * p[0] + st * p[2], p[1], -st * p[0] + ct * p[2]]) + np.asarray(offset, float)

    v = [tf(p) for p in c]  # index = 4*ix + 2*iy + iz
    faces = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    tris = []
    for f in faces:
        tris.append((v[f[0]], v[f[1]], v[f[2]]))
        tris.append((v[f[0]], v[f[2]], v[f[3]]))
    return tris


def cornell(width: int = 512, height: int = 512, spp: int = 256, depth: int = 16) -> SceneSpec:
    """Cornell box: 555^3, five walls and a 130x105 ceiling light (emission 15) as
    quads, two white boxes (165^3 at -18 deg, 165x330x165 at +15 deg) as 24 triangles."""
    B = _Builder()
    red = B.mat(S.lambertian((0.65, 0.05, 0.05)))
    white = B.mat(S.lambertian((0.73, 0.73, 0.73)))
    green = B.mat(S.lambertian((0.12, 0.45, 0.15)))
    lightm = B.mat(S.light((15.0, 15.0, 15.0)))
    B.rect((555, 0, 0), (0, 555, 0), (0, 0, 555), green)
    B.rect((0, 0, 0), (0, 555, 0), (0, 0, 555), red)
    B.rect((343, 554, 332), (-130, 0, 0), (0, 0, -105), lightm)
    B.rect((0, 0, 0), (555, 0, 0), (0, 0, 555), white)
    B.rect((555, 555, 555), (-555, 0, 0), (0, 0, -555), white)
    B.rect((0, 0, 555), (555, 0, 0), (0, 555, 0), white)
    for t in _box_tris((0, 0, 0), (165, 330, 165), 15.0, (265, 0, 295)):
        B.tri(*t, white)
    for t in _box_tris((0, 0, 0), (165, 165, 165), -18.0, (130, 0, 65)):
        B.tri(*t, white)
    k, p, m = B.arrays()
    return SceneSpec("cornell", B.materials, k, p, m, Camera((278, 278, -800), (278, 278, 0), (0, 1, 0), 40.0),
                     width, height, spp, depth, background=0.0)


def icosphere(level: int) -> np.ndarray:
    """Unit icosphere triangles (20 * 4^level, 3, 3) by midpoint subdivision."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
                      [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                      [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                      [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    tris = verts[faces]
    for _ in range(level):
        a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tris = np.stack([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                         np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3, 3)
    return tris


def icospheres(seed: int = 7, count: int = 64, level: int = 6, width: int = 1920, height: int = 1080, spp: int = 64,
               depth: int = 8) -> SceneSpec:
    """64 level-6 icospheres (81,920 tris each): per sphere draw centre U[-50,50]^3,
    radius U[1,4], roughness U[0.05,0.8], F0 U[0.02,0.95] (GGX conductor, k = 0,
    eta from F0); a Lambert ground quad at y = -56 spanning 400 x 400."""
    rng = np.random.default_rng(seed)
    unit = icosphere(level).reshape(-1, 9)
    mats = []
    ground = S.lambertian((0.5, 0.5, 0.5))
    mats.append(ground)
    tris, tmat = [], []
    for i in range(count):
        c = rng.uniform(-50, 50, 3)
        r = rng.uniform(1, 4)
        rough = rng.uniform(0.05, 0.8)
        f0 = rng.uniform(0.02, 0.95)
        mats.append(S.ggx_from_f0(rough, f0))
        tris.append(unit * r + np.tile(c, 3))
        tmat.append(np.full(unit.shape[0], len(mats) - 1, np.int32))
    tri = np.concatenate(tris)
    n = tri.shape[0]
    kinds = np.full(n + 1, KIND_TRI, np.uint8)
    params = np.zeros((n + 1, 18))
    params[1:, :9] = tri
    kinds[0] = KIND_RECT
    params[0, :9] = [-200, -56, -200, 400, 0, 0, 0, 0, 400]
    m = np.concatenate([[0], np.concatenate(tmat)]).astype(np.int32)
    return SceneSpec("icospheres", mats, kinds, params, m, Camera((0, 40, 170), (0, 0, 0), (0, 1, 0), 45.0),
                     width, height, spp, depth, background=1.0)


def sdf_field(seed: int = 11, count: int = 256, width: int = 1280, height: int = 720, spp: int = 128, depth: int = 8,
              views: int = 16) -> SceneSpec:
    """256 SDF primitives (rounded box, torus, capsule in turn by a uniform draw),
    position U[-20,20]^3, size U[0.5,3], rotation U[0,2pi)^3, materials drawn
    Lambert / GGX / dielectric with probabilities 0.5 / 0.3 / 0.2; smooth union
    k = 0.2, 256 steps, epsilon 1e-4; 16 orbit views at radius 60."""
    rng = np.random.default_rng(seed)
    B = _Builder()
    B.rect((-400, -25, -400), (800, 0, 0), (0, 0, 800), B.mat(S.lambertian((0.5, 0.5, 0.5))))
    for i in range(count):
        kind = int(rng.integers(0, 3))
        pos = rng.uniform(-20, 20, 3)
        size = rng.uniform(0.5, 3.0)
        rot = rng.uniform(0, 2 * np.pi, 3)
        mk = rng.random()
        col = rng.uniform(0.2, 0.9, 3)
        if mk < 0.5:
            m = B.mat(S.lambertian(col))
        elif mk < 0.8:
            m = B.mat(S.ggx_from_f0(rng.uniform(0.05, 0.8), rng.uniform(0.02, 0.95)))
        else:
            m = B.mat(S.glass(1.5))
        if kind == 0:
            B.sdf(S.SDF_ROUND_BOX, pos, (size, size * 0.8, size * 0.6), rot, m)
        elif kind == 1:
            B.sdf(S.SDF_TORUS, pos, (size, size * 0.3, 0), rot, m)
        else:
            B.sdf(S.SDF_CAPSULE, pos, (size * 0.4, size, 0), rot, m)
    k, p, m = B.arrays()
    vs = []
    for v in range(views):
        a = 2 * np.pi * v / views
        vs.append(Camera((60 * np.cos(a), 15, 60 * np.sin(a)), (0, 0, 0), (0, 1, 0), 45.0))
    return SceneSpec("sdf_field", B.materials, k, p, m, vs[0], width, height, spp, depth, background=1.0,
                     sdf_blend=0.2, sdf_steps=256, sdf_eps=1e-4, views=vs)


CONFIGS = {"one_weekend": one_weekend, "cornell": cornell, "icospheres": icospheres, "sdf_field": sdf_field}


def orbit(camera: Camera, angle: float) -> Camera:
    """The camera rotated about the vertical axis through its target by `angle` radians."""
    lf = np.array(camera.look_from, float)
    la = np.array(camera.look_at, float)
    d = lf - la
    r = float(np.hypot(d[0], d[2]))
    a0 = float(np.arctan2(d[2], d[0])) + angle
    return Camera((la[0] + r * np.cos(a0), lf[1], la[2] + r * np.sin(a0)), camera.look_at, camera.vup, camera.vfov)


SERVING_RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]


def serving_mix(n: int, rate: float = 50.0, n_scenes: int = 4, seed: int = 4, spp_range=(16, 1024)) -> list:
    """The serving stream: Poisson arrivals at `rate` jobs/s; per job draw the
    inter-arrival time, a resolution uniformly from SERVING_RESOLUTIONS, spp
    log-uniform over spp_range, a scene index uniformly over n_scenes and an
    orbit angle U[0, 2pi). Returns dicts (scene, width, height, spp, angle, t)."""
    rng = np.random.default_rng(seed)
    jobs = []
    t = 0.0
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        w, h = SERVING_RESOLUTIONS[int(rng.integers(0, len(SERVING_RESOLUTIONS)))]
        spp = int(np.exp(rng.uniform(np.log(spp_range[0]), np.log(spp_range[1]))))
        si = int(rng.integers(0, n_scenes))
        ang = float(rng.uniform(0, 2 * np.pi))
        jobs.append(dict(scene=si, width=w, height=h, spp=spp, angle=ang, t=t))
    return jobs
