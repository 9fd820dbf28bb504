"""The 4-wide copy of the BVH that the render kernels traverse, checked on the
host (no GPU): every leaf of the binary tree is reached exactly once, every
wide node is reached once, refs stay in range and every child node's boxes lie
inside the box of the slot that leads to it. Scenes from a leaf root to a tree
large enough for the parallel build of subtrees (more than 256 pending
children after the breadth-first top)."""
import pytest

from rayon_b200 import scenes


@pytest.mark.parametrize("name", ["cornell", "one_weekend", "ico_small", "ico_large", "single"])
def test_wide_tree_reaches_every_leaf_once(name):
    if name == "ico_small":
        spec = scenes.icospheres(count=8, level=3)
    elif name == "ico_large":
        spec = scenes.icospheres(count=24, level=4)   # 122,880 triangles: thousands of wide nodes
    elif name == "single":
        spec = scenes.cornell()
    else:
        spec = getattr(scenes, name)()
    sc = spec.to_scene()
    if name == "single":                          # a tree whose root is a leaf
        from rayon_b200 import scene as S
        sc = S.SceneDescription()
        m = sc.add_material(S.lambertian((0.5, 0.5, 0.5)))
        sc.add_sphere((0, 0, 0), 1.0, m)
    sc.build_bvh()
    info = sc.check_wide()
    assert info["leaves_reached"] == info["binary_leaves"] > 0
    if name == "single":
        assert info["wide_nodes"] == 0
    else:
        assert info["wide_nodes"] > 0
    if name == "ico_large":
        assert info["wide_nodes"] > 2000
        # each wide node replaces up to three binary interior nodes
        assert info["wide_nodes"] * 3 >= info["binary_leaves"] - 1
