"""The seeded synthetic workloads against the benchmark configurations they stand
in for (counts, sizes, value ranges, cameras and render settings), and the
serving request stream against its stated distributions. CPU only: these check
the inputs every GPU test and the benchmark render."""
import numpy as np
import pytest

from rayon_b200 import scene as S
from rayon_b200 import scenes


def _types(spec):
    return np.array([spec.materials[int(m)].type for m in spec.mats])


def test_one_weekend_configuration():
    sp = scenes.one_weekend()
    assert (sp.width, sp.height, sp.spp, sp.depth) == (400, 225, 32, 10)
    assert sp.camera.look_from == (13, 2, 3) and tuple(sp.camera.look_at) == (0, 0, 0) and sp.camera.vfov == 20.0
    assert sp.dof == (0.1, 10.0)
    assert sp.n == 4 + 22 * 22 and (sp.kinds == scenes.KIND_SPHERE).all()
    c, r = sp.params[:, :3], sp.params[:, 3]
    np.testing.assert_array_equal(c[0], [0, -1000, 0])
    assert r[0] == 1000
    np.testing.assert_array_equal(c[1:4], [[0, 1, 0], [-4, 1, 0], [4, 1, 0]])
    np.testing.assert_array_equal(r[1:4], 1.0)
    mt = _types(sp)
    assert list(mt[1:4]) == [S.GLASS, S.LAMBERTIAN, S.METAL]
    assert sp.materials[int(sp.mats[1])].refractive_index == pytest.approx(1.5)
    np.testing.assert_allclose(list(sp.materials[int(sp.mats[2])].albedo), [0.4, 0.2, 0.1])
    m3 = sp.materials[int(sp.mats[3])]
    np.testing.assert_allclose(list(m3.albedo), [0.7, 0.6, 0.5])
    assert m3.roughness == 0.0
    # the 22 x 22 grid: one sphere of radius 0.2 per cell, at (a + 0.9u, 0.2, b + 0.9v)
    small = c[4:]
    np.testing.assert_array_equal(r[4:], 0.2)
    np.testing.assert_array_equal(small[:, 1], 0.2)
    cells = np.stack([np.floor(small[:, 0]), np.floor(small[:, 2])], 1)
    assert len({tuple(x) for x in cells}) == 484
    assert cells.min() == -11 and cells.max() == 10
    assert ((small[:, 0] - cells[:, 0]) <= 0.9).all() and ((small[:, 2] - cells[:, 1]) <= 0.9).all()
    # materials drawn 80 / 15 / 5 % with their stated ranges
    t = mt[4:]
    for kind, p in ((S.LAMBERTIAN, 0.80), (S.METAL, 0.15), (S.GLASS, 0.05)):
        assert abs((t == kind).mean() - p) < 0.08
    for i in np.flatnonzero(t == S.METAL) + 4:
        m = sp.materials[int(sp.mats[i])]
        assert all(0.5 <= a <= 1.0 for a in m.albedo) and 0.0 <= m.roughness <= 0.5
    for i in np.flatnonzero(t == S.LAMBERTIAN) + 4:
        assert all(0.0 <= a < 1.0 for a in sp.materials[int(sp.mats[i])].albedo)
    # seeded: the same scene every time
    np.testing.assert_array_equal(scenes.one_weekend().params, sp.params)


def test_cornell_configuration():
    sp = scenes.cornell()
    assert (sp.width, sp.height, sp.spp, sp.depth, sp.background) == (512, 512, 256, 16, 0.0)
    assert (sp.kinds == scenes.KIND_RECT).sum() == 6 and (sp.kinds == scenes.KIND_TRI).sum() == 24 and sp.n == 30
    p = sp.params
    q4 = p[sp.kinds == scenes.KIND_RECT]
    corners = np.concatenate([q4[:, 0:3], q4[:, 0:3] + q4[:, 3:6], q4[:, 0:3] + q4[:, 6:9],
                              q4[:, 0:3] + q4[:, 3:6] + q4[:, 6:9]])
    assert corners.min() >= 0 and corners.max() <= 555
    lights = [i for i in range(sp.n) if sp.materials[int(sp.mats[i])].type == S.LIGHT]
    assert len(lights) == 1
    q = p[lights[0]]
    assert sorted([np.linalg.norm(q[3:6]), np.linalg.norm(q[6:9])]) == [105.0, 130.0]
    assert q[1] == 554
    np.testing.assert_array_equal(list(sp.materials[int(sp.mats[lights[0]])].emission), [15, 15, 15])
    albedos = {tuple(np.round(list(sp.materials[int(m)].albedo), 2)) for m in sp.mats[sp.kinds == scenes.KIND_RECT]}
    assert {(0.73, 0.73, 0.73), (0.65, 0.05, 0.05), (0.12, 0.45, 0.15)} <= albedos
    # two white boxes of 12 triangles: 165 x 330 x 165 and 165^3, standing on the floor
    tris = p[sp.kinds == scenes.KIND_TRI, :9].reshape(2, 12, 3, 3)
    heights = sorted(float(b[..., 1].max() - b[..., 1].min()) for b in tris)
    assert heights == pytest.approx([165.0, 330.0])
    assert all(b[..., 1].min() == pytest.approx(0.0) for b in tris)
    for b in tris:  # rotation about +y keeps the horizontal edge lengths at 165
        e = b[:, 1, [0, 2]] - b[:, 0, [0, 2]]
        lens = np.linalg.norm(e, axis=1)
        assert np.isclose(lens, 165.0).any() and lens.max() <= 165.0 * np.sqrt(2) + 1e-9


def test_icosphere_level_six():
    tri = scenes.icosphere(6)
    assert tri.shape == (20 * 4 ** 6, 3, 3) == (81920, 3, 3)
    np.testing.assert_allclose(np.linalg.norm(tri, axis=2), 1.0, rtol=1e-12)
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    assert area.sum() == pytest.approx(4 * np.pi, rel=2e-3)  # inscribed polyhedron, just under the sphere
    assert area.sum() < 4 * np.pi


def test_icospheres_configuration():
    sp = scenes.icospheres()
    assert (sp.width, sp.height, sp.spp, sp.depth) == (1920, 1080, 64, 8)
    assert sp.n == 1 + 5_242_880 and sp.kinds[0] == scenes.KIND_RECT
    assert (sp.kinds[1:] == scenes.KIND_TRI).all()
    tri = sp.params[1:, :9].reshape(64, 81920, 3, 3)
    mats = sp.mats[1:].reshape(64, 81920)
    assert (mats == mats[:, :1]).all() and len(set(mats[:, 0])) == 64
    for s in range(64):
        v = tri[s].reshape(-1, 3)
        c = (v.max(0) + v.min(0)) / 2
        r = np.linalg.norm(v - c, axis=1)
        assert (np.abs(c) <= 50).all()
        assert 1.0 <= r.mean() <= 4.0 and np.ptp(r) < 1e-9 * r.mean() + 1e-3 * r.mean()
        m = sp.materials[int(mats[s, 0])]
        assert m.type == S.ANISOTROPIC_METAL and 0.05 <= m.roughness <= 0.8 and m.anisotropy == 0.0
        eta = m.eta[0]
        f0 = ((eta - 1) / (eta + 1)) ** 2
        assert 0.02 <= f0 <= 0.95 and list(m.k) == [0.0, 0.0, 0.0]
    assert sp.materials[int(sp.mats[0])].type == S.LAMBERTIAN


def test_sdf_field_configuration():
    sp = scenes.sdf_field()
    assert (sp.width, sp.height, sp.spp, sp.depth) == (1280, 720, 128, 8)
    assert (sp.sdf_blend, sp.sdf_steps, sp.sdf_eps) == (0.2, 256, 1e-4)
    assert len(sp.views) == 16
    for cam in sp.views:
        lf = np.array(cam.look_from)
        assert np.hypot(lf[0], lf[2]) == pytest.approx(60.0) and tuple(cam.look_at) == (0, 0, 0)
    sdf = sp.kinds == scenes.KIND_SDF
    assert sdf.sum() == 256 and sp.n == 257
    p = sp.params[sdf]
    kinds = p[:, 0].astype(int)
    assert set(kinds) == {S.SDF_ROUND_BOX, S.SDF_TORUS, S.SDF_CAPSULE}
    assert (np.abs(p[:, 1:4]) <= 20).all()
    size = np.where(kinds == S.SDF_CAPSULE, p[:, 5], p[:, 4])
    assert (size >= 0.5).all() and (size <= 3.0).all()
    t = _types(sp)[sdf]
    for kind, frac in ((S.LAMBERTIAN, 0.5), (S.ANISOTROPIC_METAL, 0.3), (S.GLASS, 0.2)):
        assert abs((t == kind).mean() - frac) < 0.125


def test_serving_stream_distributions():
    mix = scenes.serving_mix(2000, rate=50.0)
    assert mix == scenes.serving_mix(2000, rate=50.0)  # seeded
    t = np.array([j["t"] for j in mix])
    assert (np.diff(t) > 0).all()
    assert np.diff(t, prepend=0.0).mean() == pytest.approx(1 / 50.0, rel=0.1)
    res = {(j["width"], j["height"]) for j in mix}
    assert res == set(scenes.SERVING_RESOLUTIONS)
    spp = np.array([j["spp"] for j in mix])
    assert spp.min() >= 16 and spp.max() <= 1024
    assert np.log(spp + 0.5).mean() == pytest.approx((np.log(16) + np.log(1024)) / 2, abs=0.12)
    ang = np.array([j["angle"] for j in mix])
    assert ang.min() >= 0 and ang.max() < 2 * np.pi
    assert {j["scene"] for j in mix} == {0, 1, 2, 3}


def test_orbit_keeps_radius_and_height():
    cam = scenes.cornell().camera
    assert scenes.orbit(cam, 0.0).look_from == pytest.approx(cam.look_from)
    assert scenes.orbit(cam, 2 * np.pi).look_from == pytest.approx(cam.look_from, abs=1e-9)
    for a in (0.3, 1.7, 4.0):
        o = scenes.orbit(cam, a)
        d0 = np.subtract(cam.look_from, cam.look_at)
        d1 = np.subtract(o.look_from, o.look_at)
        assert np.hypot(d1[0], d1[2]) == pytest.approx(np.hypot(d0[0], d0[2]))
        assert d1[1] == pytest.approx(d0[1])
        assert np.arctan2(d1[2], d1[0]) % (2 * np.pi) == pytest.approx((np.arctan2(d0[2], d0[0]) + a) % (2 * np.pi))


@pytest.mark.parametrize("name,kw", [("one_weekend", {}), ("cornell", {}), ("icospheres", dict(count=5, level=2)),
                                     ("sdf_field", {})])
def test_reference_arm_generators_equal_the_workloads(name, kw):
    """oracle/workloads.py (used by the process that drives only the reference)
    builds the same scenes as rayon_b200/scenes.py, bit for bit."""
    from oracle import workloads
    a = getattr(scenes, name)(**kw)
    b = getattr(workloads, name)(**kw)
    np.testing.assert_array_equal(a.kinds, b.kinds)
    np.testing.assert_array_equal(a.params, b.params)
    np.testing.assert_array_equal(a.mats, b.mats)
    assert len(a.materials) == len(b.materials)
    for ma, mb in zip(a.materials, b.materials):
        assert bytes(ma) == bytes(mb)
    for f in ("width", "height", "spp", "depth", "background", "dof", "sdf_blend", "sdf_steps", "sdf_eps"):
        assert getattr(a, f) == getattr(b, f), f
    cams_a = [a.camera] + list(a.views)
    cams_b = [b.camera] + list(b.views)
    assert len(cams_a) == len(cams_b)
    for ca, cb in zip(cams_a, cams_b):
        for f in ("look_from", "look_at", "vup", "vfov"):
            np.testing.assert_array_equal(np.asarray(getattr(ca, f), float), np.asarray(getattr(cb, f), float))


def test_material_struct_layouts_agree():
    """The oracle's mirror of rb_material_desc has the library's layout."""
    import ctypes as C

    from oracle.refbind import RefMaterial
    from rayon_b200._native import MaterialDesc
    assert C.sizeof(RefMaterial) == C.sizeof(MaterialDesc)
    for (n1, _), (n2, _) in zip(RefMaterial._fields_, MaterialDesc._fields_):
        assert n1 == n2 and getattr(RefMaterial, n1).offset == getattr(MaterialDesc, n2).offset
