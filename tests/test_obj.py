"""OBJ ingest (rb_scene_load_obj) against the reference's own OBJLoader::loadOBJ
(src/rayon/scenes/obj_loader.hpp:34-140), compiled from its sources: the same
triangles, normals and materials, bit for bit, on files that exercise its
parsing rules."""
import numpy as np
import pytest

from oracle import refbind
from rayon_b200 import scene as S

needs_ref = pytest.mark.skipif(not refbind.host_available(), reason="reference drivers (oracle/_ref) not built")

QUIRKS = "\r\n".join([
    "# comment",
    "",
    "   # indented comment",
    "mtllib scene.mtl",
    "o thing",
    "v 0 0 0",
    "v 1 0 0",
    "v 1 1 0",
    "v 0 1 0   ",
    "  v 0.5 0.5 1.5e0",
    "v +2 .5 5.",
    "v 1e 2 3",            # '1e' is not a number: line skipped
    "v 1.2.3 4",           # reads 1.2, then .3, then 4
    "v 7 8",               # too few numbers: skipped
    "vn 0 0 1",
    "vn 0 1 0",
    "vn 1 0 0",
    "vt 0.5 0.5",
    "usemtl red",
    "s 1",
    "f 1 2 3",
    "f 1/1 2/1 3/1",
    "f 1/1/1 2/1/2 3/1/3",
    "f 1//1 2//2 3//3 4//1",        # quad with normals: fan of two
    "f 1 2 3 4 5",                  # pentagon: fan of three
    "f -1 -2 -3",                   # relative indices
    "f -1//-1 -2//-2 -3//-3",
    "f 0 1 2",                      # index 0 stays 0
    "f 1 2 99",                     # out of range: skipped
    "f 1 2",                        # degenerate face: nothing
    "f 1//9 2//1 3//1",             # normal index out of range: no normals
    "f 1/2 2/3 3/4 ",
    "f 5abc 6 7",                   # stoi reads the leading digits
    "g group",
    "f 2 3 4",
    "v 3 3 3",
    "f -1 1 2",
])


def _ours(path, mat, pos=(0, 0, 0), scale=(1, 1, 1)):
    sc = S.SceneDescription()
    sc.add_material(S.lambertian((0.5, 0.5, 0.5)))
    n = sc.load_obj(path, mat, pos, scale)
    g = sc.export_geometry()
    return n, g


@needs_ref
@pytest.mark.parametrize("pos,scale", [((0, 0, 0), (1, 1, 1)), ((1.5, -2.0, 0.25), (2.0, 0.5, -3.0))])
def test_obj_matches_reference_loader(tmp_path, pos, scale):
    p = tmp_path / "quirks.obj"
    p.write_bytes(QUIRKS.encode())
    n, g = _ours(p, 0, pos, scale)
    rn, r = refbind.reference_obj_triangles(p, 0, pos, scale)
    assert n == rn and g.shape[0] == r.shape[0] == n
    assert (g[:, 0] == 4).all()  # RB_GEOM_TRIANGLE
    np.testing.assert_array_equal(g[:, 4:13], r[:, 0:9])          # vertices, bit for bit
    np.testing.assert_array_equal(g[:, 3], r[:, 18])              # has_normals
    hn = r[:, 18] == 1
    np.testing.assert_array_equal(g[hn, 13:22], r[hn, 9:18])      # normals where present
    np.testing.assert_array_equal(g[:, 1], r[:, 19])              # material


@needs_ref
def test_obj_random_mesh_matches_reference(tmp_path):
    rng = np.random.default_rng(3)
    lines = []
    for _ in range(500):
        x, y, z = rng.normal(size=3) * 10
        lines.append(f"v {x:.9g} {y:.6e} {z!r}")
    for _ in range(200):
        lines.append("vn %.7f %.7f %.7f" % tuple(rng.normal(size=3)))
    for _ in range(1500):
        k = int(rng.integers(3, 6))
        idx = rng.integers(1, 501, size=k)
        nrm = rng.integers(1, 201, size=k)
        form = int(rng.integers(0, 3))
        toks = [str(a) if form == 0 else f"{a}//{b}" if form == 1 else f"{a}/1/{b}" for a, b in zip(idx, nrm)]
        lines.append("f " + " ".join(toks))
    p = tmp_path / "mesh.obj"
    p.write_text("\n".join(lines) + "\n")
    n, g = _ours(p, 0)
    rn, r = refbind.reference_obj_triangles(p, 0)
    assert n == rn
    np.testing.assert_array_equal(g[:, 4:13], r[:, 0:9])
    np.testing.assert_array_equal(g[:, 3], r[:, 18])
    hn = r[:, 18] == 1
    np.testing.assert_array_equal(g[hn, 13:22], r[hn, 9:18])


def test_obj_errors(tmp_path):
    sc = S.SceneDescription()
    sc.add_material(S.lambertian((0.5, 0.5, 0.5)))
    with pytest.raises(RuntimeError, match="cannot open"):
        sc.load_obj(tmp_path / "missing.obj", 0)
    p = tmp_path / "bad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nf a b c\n")
    with pytest.raises(RuntimeError, match="malformed face index"):
        sc.load_obj(p, 0)
    assert sc.num_geometries == 1  # the face before the malformed one stays
