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
