"""The oracle's smooth SDF field against a plain sphere tracer of the whole
smooth union, restated here in numpy.

The oracle (and both GPU engines) fold only the primitives whose k-inflated
bounding spheres hold the current point, clamp each step to the next such
window's entry, and jump over a window once a lone convex primitive's
distance is seen growing (the convex skip). The plain tracer folds every
primitive in index order at every step, as RayON's CPU SDF shapes march the
smooth union (cpu_renderers/cpu_shapes/sdf.hpp:410-416 polynomial smooth
minimum, 510-560 sphere tracing). Both must find the same surface at the same
distance for primary rays."""
import numpy as np

from oracle.oracle import OracleScene
from rayon_b200 import scenes

GEOM_RECTANGLE, GEOM_SDF = 1, 6
SPHERE, BOX, TORUS, CAPSULE, ROUND_BOX = 0, 1, 2, 3, 32


def _sdf_prims(geoms):
    """(type, pos, a, b, c, round, world->local matrix) per SDF row, in the
    oracle's conventions (rounding radius 0.2 x the smallest half extent,
    rotation Rz Ry Rx from the three angles)."""
    out = []
    for r in geoms:
        if int(r[0]) != GEOM_SDF:
            continue
        p = r[4:22]
        t = int(p[0])
        a, b, c = p[4], p[5], p[6]
        rnd = 0.2 * min(a, b, c) if t == ROUND_BOX else 0.0
        cx, sx, cy, sy, cz, sz = np.cos(p[7]), np.sin(p[7]), np.cos(p[8]), np.sin(p[8]), np.cos(p[9]), np.sin(p[9])
        R = np.array([[cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx],
                      [sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx],
                      [-sy, cy * sx, cy * cx]])
        out.append((t, np.array(p[1:4]), a, b, c, rnd, R))
    return out


def _dist(prim, P):
    t, pos, a, b, c, rnd, R = prim
    q = (P - pos) @ R  # R^T (p - pos) for each row
    if t == SPHERE:
        return np.linalg.norm(q, axis=1) - a
    if t in (BOX, ROUND_BOX):
        qq = np.abs(q) - (np.array([a, b, c]) - rnd)
        out = np.linalg.norm(np.maximum(qq, 0.0), axis=1)
        return out + np.minimum(qq.max(axis=1), 0.0) - rnd
    if t == TORUS:
        qx = np.hypot(q[:, 0], q[:, 2]) - a
        return np.hypot(qx, q[:, 1]) - b
    if t == CAPSULE:
        y = np.clip(q[:, 1], -0.5 * b, 0.5 * b)
        return np.linalg.norm(np.stack([q[:, 0], q[:, 1] - y, q[:, 2]], axis=1), axis=1) - a
    return np.full(len(P), 1e30)


def _union(prims, P, k):
    F = _dist(prims[0], P)
    for pr in prims[1:]:
        d = _dist(pr, P)
        h = np.clip(0.5 + 0.5 * (d - F) / k, 0.0, 1.0)
        F = d * (1.0 - h) + F * h - k * h * (1.0 - h)
    return F


def _rect_hits(geoms, o, d, tmin):
    best = np.full(len(d), np.inf)
    for r in geoms:
        if int(r[0]) != GEOM_RECTANGLE:
            continue
        q, u, v = r[4:7], r[7:10], r[10:13]
        n = np.cross(u, v)
        den = d @ n
        with np.errstate(divide="ignore", invalid="ignore"):
            t = ((q - o) @ n) / den
        p = o + t[:, None] * d - q
        al, be = p @ u / (u @ u), p @ v / (v @ v)
        ok = (np.abs(den) > 1e-12) & (t >= tmin) & (al >= 0) & (al <= 1) & (be >= 0) & (be <= 1)
        best = np.where(ok & (t < best), t, best)
    return best


def test_windowed_field_matches_plain_sphere_tracing():
    spec = scenes.sdf_field(count=48, width=64, height=36)
    sc = spec.to_scene()
    sc.build_bvh()
    w, h = 64, 36
    fr = spec.camera.frame(w, h)
    o_ids, o_t, _ = OracleScene(sc, sdf=(spec.sdf_blend, spec.sdf_steps, spec.sdf_eps)).primary(fr, w, h)
    geoms = sc.export_geometry()
    prims = _sdf_prims(geoms)
    assert len(prims) == 48
    # pixel-centre rays as the oracle's primary pass builds them
    center, p00, du, dv = fr[0:3], fr[3:6], fr[6:9], fr[9:12]
    ys, xs = np.mgrid[0:h, 0:w]
    d = (p00 + xs.reshape(-1, 1) * du + ys.reshape(-1, 1) * dv) - center
    o = np.broadcast_to(center, d.shape)
    tmin = 0.001
    tmax = _rect_hits(geoms, center, d, tmin)
    il = 1.0 / np.linalg.norm(d, axis=1)
    t = np.full(len(d), tmin)
    hit = np.full(len(d), -1.0)
    live = np.ones(len(d), bool)
    for _ in range(spec.sdf_steps):
        idx = np.nonzero(live)[0]
        if idx.size == 0:
            break
        F = _union(prims, o[idx] + t[idx, None] * d[idx], spec.sdf_blend)
        done = F < spec.sdf_eps
        hit[idx[done]] = t[idx[done]]
        live[idx[done]] = False
        t[idx[~done]] += F[~done] * il[idx[~done]]
        live[idx[~done & (t[idx] > tmax[idx])]] = False
    plain_field = (hit >= 0) & (hit <= tmax)
    oracle_field = o_ids.reshape(-1) == -2
    assert plain_field.sum() > 0.05 * len(d)  # the view sees the field
    agree = (plain_field == oracle_field).mean()
    assert agree >= 0.98, agree
    both = plain_field & oracle_field
    dt = np.abs(o_t.reshape(-1)[both] - hit[both]) / il[both]  # distance along the ray
    assert np.mean(dt < 2e-3) >= 0.98, np.sort(dt)[-10:]


def _pin_case():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from cases import sdf_pin
    return sdf_pin()


def _ray_lengths(fr, w, h):
    ys, xs = np.mgrid[0:h, 0:w]
    d = fr[3:6][None, None] + xs[..., None] * fr[6:9] + ys[..., None] * fr[9:12] - fr[0:3]
    return np.linalg.norm(d, axis=-1)


def _check_against_reference(ids, t, oids, ot, fr, w, h):
    """Same object on every pixel; distances within the march epsilon (both
    stop at the first point closer than 1e-4 to the surface, approaching it
    from different starting points)."""
    np.testing.assert_array_equal(oids, ids)
    hit = ids >= 0
    assert 0.15 < hit.mean() < 0.9
    dist = ot * _ray_lengths(fr, w, h)   # the oracle's t is in units of the unnormalised ray
    assert np.abs(dist - t)[hit].max() < 2e-4


def test_oracle_sdf_primitives_match_reference_cpu_hits():
    """The oracle's hard-union SDF primitives (sphere, box, torus, capsule,
    rotated) against the reference's own CPU path: SDFShape::hit marching
    each shape with SDF::rayMarch (cpu_shapes/sdf_shape.hpp:307-330,
    sdf.hpp:114-160, 518-566) at its defaults (128 steps, epsilon 1e-4), on
    the committed fixture of its pixel-centre hits (tests/golden/sdf_hits_ref.npz,
    made by make_golden.py --sdf)."""
    from pathlib import Path
    spec = _pin_case()
    g = np.load(Path(__file__).resolve().parent / "golden" / "sdf_hits_ref.npz")
    w, h, fr = int(g["width"]), int(g["height"]), g["frame"]
    np.testing.assert_array_equal(fr, spec.camera.frame(w, h))
    sc = spec.to_scene()   # no BVH: geometry stays in insertion order, as the reference's object list
    o = OracleScene(sc, use_bvh=False, sdf=(0.0, spec.sdf_steps, spec.sdf_eps))
    oids, ot, _ = o.primary(fr, w, h)
    _check_against_reference(g["ids"], g["t"], oids, ot, fr, w, h)


def test_oracle_sdf_primitives_match_reference_live():
    """As above, with the reference's CPU path run live (oracle/_ref)."""
    import pytest

    from oracle import refbind
    if not refbind.host_available():
        pytest.skip("reference drivers (oracle/_ref) not built")
    spec = _pin_case()
    w, h = spec.width, spec.height
    fr = refbind.camera_frame(spec.camera, w, h)
    ids, t, _ = refbind.RefScene(spec).cpu_primary(fr, w, h)
    o = OracleScene.from_arrays(spec, sdf=(0.0, spec.sdf_steps, spec.sdf_eps))
    oids, ot, _ = o.primary(fr, w, h)
    _check_against_reference(ids, t, oids, ot, fr, w, h)
