"""Seeded scene cases shared by the golden-fixture generator and the tests."""
from __future__ import annotations

import numpy as np

from rayon_b200 import scene as S
from rayon_b200 import scenes


def grid_soup(n: int = 3000, seed: int = 5) -> scenes.SceneSpec:
    """Triangles with vertices on an integer grid: many equal centroid keys (sort ties)."""
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 20, size=(n, 9)).astype(float)
    k = np.full(n, scenes.KIND_TRI, np.uint8)
    p = np.zeros((n, 18))
    p[:, :9] = v
    m = np.zeros(n, np.int32)
    return scenes.SceneSpec("grid_soup", [S.lambertian((0.6, 0.6, 0.6))], k, p, m,
                            scenes.Camera((10, 10, -30), (10, 10, 10), (0, 1, 0), 50.0), 96, 96, 4, 4)


def small_icospheres() -> scenes.SceneSpec:
    return scenes.icospheres(seed=3, count=8, level=3, width=160, height=90, spp=8, depth=6)


def mixed_materials() -> scenes.SceneSpec:
    """Every legacy material kind once, on spheres in a lit box."""
    B = scenes._Builder()
    mats = [S.lambertian((0.7, 0.3, 0.2)), S.mirror((0.9, 0.9, 0.9)), S.metal((0.8, 0.7, 0.3), 0.0),
            S.metal((0.6, 0.6, 0.9), 0.4), S.glass(1.5), S.constant((0.2, 0.9, 0.3)),
            S.material(S.SHOW_NORMALS), S.anisotropic_metal(0.3, 0.6, (0.18, 0.42, 1.37), (3.42, 2.35, 1.77)),
            S.anisotropic_metal(0.0, 0.0, (1.35, 0.97, 0.53), (7.47, 6.40, 5.28)),
            S.thin_film(420.0, 1.33, 1.0), S.clear_coat((0.1, 0.3, 0.8), 0.05, 1.5),
            S.material(S.LAMBERTIAN, albedo=(0.9, 0.9, 0.9), pattern=1, pattern_color=(0.1, 0.1, 0.1),
                       pattern_param1=12, pattern_param2=0.33)]
    ids = [B.mat(m) for m in mats]
    floor = B.mat(S.lambertian((0.5, 0.5, 0.5)))
    lightm = B.mat(S.light((8.0, 8.0, 8.0)))
    for i, mid in enumerate(ids):
        x = (i % 4) * 2.5 - 3.75
        z = (i // 4) * 2.5 - 2.5
        B.sphere((x, 1.0, z), 1.0, mid)
    B.rect((-10, 0, -10), (20, 0, 0), (0, 0, 20), floor)
    B.rect((-2, 8, -2), (4, 0, 0), (0, 0, 4), lightm)
    k, p, m = B.arrays()
    return scenes.SceneSpec("mixed_materials", B.materials, k, p, m,
                            scenes.Camera((0, 6, 12), (0, 1, 0), (0, 1, 0), 45.0), 96, 72, 16, 8, background=0.3)


def icospheres8() -> scenes.SceneSpec:
    """A reduced icosphere configuration: 8 level-5 icospheres (163,840 GGX
    triangles) from the icosphere generator's seed, 320x180, depth 8."""
    return scenes.icospheres(seed=7, count=8, level=5, width=320, height=180, spp=64, depth=8)


def sdf_pin(seed: int = 21) -> scenes.SceneSpec:
    """SDF primitives of the four kinds the reference's CPU path and this
    project both implement (sphere, box, torus, capsule), rotated, hard union."""
    rng = np.random.default_rng(seed)
    B = scenes._Builder()
    for i in range(24):
        t = i % 4
        pos = rng.uniform(-6, 6, 3)
        s = rng.uniform(0.6, 2.0)
        rot = rng.uniform(0, 2 * np.pi, 3)
        prm = {0: (s, 0, 0), 1: (s, 0.8 * s, 0.6 * s), 2: (s, 0.3 * s, 0), 3: (0.4 * s, s, 0)}[t]
        B.sdf(t, pos, prm, rot, B.mat(S.lambertian(rng.uniform(0.2, 0.9, 3))))
    k, p, m = B.arrays()
    return scenes.SceneSpec("sdf_pin", B.materials, k, p, m, scenes.Camera((3, 7, 18), (0, 0, 0), (0, 1, 0), 45.0),
                            160, 120, 4, 4, background=1.0, sdf_blend=0.0, sdf_steps=128, sdf_eps=1e-4)


BVH_CASES = {
    "one_weekend": lambda: scenes.one_weekend(),
    "cornell": lambda: scenes.cornell(),
    "grid_soup": lambda: grid_soup(),
    "small_icospheres": small_icospheres,
    "mixed_materials": mixed_materials,
}

# (case, width, height) for primary-hit goldens from the reference's CUDA hit test
HIT_CASES = {
    "one_weekend": (lambda: scenes.one_weekend(), 400, 225),
    "cornell": (lambda: scenes.cornell(), 256, 256),
    "grid_soup": (lambda: grid_soup(), 96, 96),
    "small_icospheres": (small_icospheres, 320, 180),
    "mixed_materials": (mixed_materials, 192, 144),
}

# (case, width, height, spp, depth) of the reference CUDA renders kept for
# converged-image RMSE checks
REFIMG_CASES = {
    "cornell": (lambda: scenes.cornell(), 64, 64, 4096, 16),
    "mixed_materials": (mixed_materials, 48, 36, 4096, 8),
    "one_weekend": (lambda: scenes.one_weekend(), 400, 225, 4096, 10),
    "icospheres8": (icospheres8, 320, 180, 2048, 8),
}

# Per-configuration FP64 oracle ground truth on a seeded pixel subset of the
# full frame: (case, pixels, spp). The benchmark workloads at their own sizes.
ORACLE_PX_CASES = {
    "one_weekend": (lambda: scenes.one_weekend(), 1024, 32768),
    "cornell": (lambda: scenes.cornell(), 1024, 32768),
    "icospheres": (lambda: scenes.icospheres(), 1024, 16384),
    "sdf_field": (lambda: scenes.sdf_field(), 1024, 16384),
}
