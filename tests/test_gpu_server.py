"""Batched multi-job engine and serving loop: each job's result is the same
alone and in a mix, agrees with the per-frame kernel on the same sample
streams, admission respects the HBM budget, FP64 accumulation, progressive
frames and trace latencies."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import mixed_materials  # noqa: E402

from rayon_b200 import render, scenes, serving  # noqa: E402

pytestmark = pytest.mark.gpu

# alone vs mixed: only the grouping of samples into Kahan-compensated FP32
# partial sums differs (each iteration's share of samples depends on the mix)
RTOL, ATOL_PER_SPP = 2e-5, 2e-5


def _scenes():
    out = []
    for spec in (scenes.cornell(), scenes.one_weekend(), mixed_materials()):
        sc = spec.to_scene()
        sc.build_bvh()
        out.append((spec, sc, sc.upload()))
    return out


def _jobs(server_ids, specs):
    reqs = []
    dims = [(64, 64, 64), (80, 45, 48), (48, 36, 32), (96, 96, 16), (40, 30, 100)]
    for k, (w, h, spp) in enumerate(dims):
        si = k % len(specs)
        spec = specs[si][0]
        reqs.append((serving.job(server_ids[si], spec.camera.frame(w, h), w, h, spp, spec.depth,
                                 background=spec.background, dof=spec.dof, nee=(k == 4), seed=1000 + k), w, h, spp))
    return reqs


# per_frame_classes: 0 = every class on the batched kernel; 6 = diffuse and
# classic jobs on the per-frame kernel (one launch per job and iteration)
@pytest.mark.parametrize("pfc", [0, 6])
def test_same_alone_and_in_mix(cuda, pfc):
    S = _scenes()
    mix = serving.Server(paths_per_iteration=200_000, max_spp_per_iteration=16, per_frame_classes=pfc)
    ids = [mix.add_scene(ds) for _, _, ds in S]
    reqs = _jobs(ids, S)
    jids = [mix.submit(r) for r, *_ in reqs]
    mix.drain()
    for (r, w, h, spp), jid in zip(reqs, jids):
        st = mix.status(jid)
        assert st.state == 2 and st.spp_done == spp
        got = mix.fetch(jid, w, h)
        alone = serving.Server(paths_per_iteration=1 << 26, max_spp_per_iteration=64, per_frame_classes=pfc)
        aid = [alone.add_scene(ds) for _, _, ds in S]
        r.scene = aid[r.scene]
        a = alone.submit(r)
        alone.drain()
        ref = alone.fetch(a, w, h)
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL_PER_SPP * spp)
        alone.close()
    mix.close()


def test_shared_and_per_job_scene_kernels_agree(cuda):
    """A class whose jobs share one scene and one setting runs the batched
    kernel with the scene as a launch parameter; jobs of two scenes (or two
    settings) in one class read it from the job table. Both give each job the
    result it gets alone."""
    spec = scenes.cornell(width=48, height=48)
    sc = spec.to_scene()
    sc.build_bvh()
    ds_a, ds_b = sc.upload(), sc.upload()
    fr = spec.camera.frame(48, 48)
    mix = serving.Server(paths_per_iteration=1 << 26, max_spp_per_iteration=16)
    ia, ib = mix.add_scene(ds_a), mix.add_scene(ds_b)
    reqs = [serving.job(ia, fr, 48, 48, 32, spec.depth, background=0.0, seed=7),
            serving.job(ib, fr, 48, 48, 32, spec.depth, background=0.0, seed=8),      # second scene: per-job records
            serving.job(ia, fr, 48, 48, 32, spec.depth, background=0.0, light=2.0, seed=9)]  # other setting
    jids = [mix.submit(r) for r in reqs]
    mix.drain()
    for r, jid, sid in zip(reqs, jids, (0, 1, 0)):
        got = mix.fetch(jid, 48, 48)
        alone = serving.Server(paths_per_iteration=1 << 26, max_spp_per_iteration=16)
        aid = alone.add_scene(ds_a if sid == 0 else ds_b)
        r.scene = aid
        a = alone.submit(r)
        alone.drain()
        np.testing.assert_allclose(got, alone.fetch(a, 48, 48), rtol=RTOL, atol=ATOL_PER_SPP * 32)
        alone.close()
    mix.close()
    ds_a.free()
    ds_b.free()


@pytest.mark.parametrize("pfc", [0, 6])
def test_server_matches_per_frame_kernel(cuda, pfc):
    spec = scenes.cornell(width=64, height=64)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    srv = serving.Server(paths_per_iteration=64 * 64 * 8, per_frame_classes=pfc)
    sid = srv.add_scene(ds)
    fr = spec.camera.frame(64, 64)
    j = srv.submit(serving.job(sid, fr, 64, 64, 32, spec.depth, background=0.0, seed=0))
    srv.drain()
    got = srv.fetch(j, 64, 64)
    ref = render.render_accumulate(ds, fr, 64, 64, 32, spec.depth, background=0.0)  # same streams (salt 0)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-4 * 32)
    srv.close()


def test_admission_budget_and_rejection(cuda):
    S = _scenes()
    # room for two 64x64 jobs (32 B per pixel each) but not three
    srv = serving.Server(budget_bytes=2 * 64 * 64 * 32 + 100, paths_per_iteration=64 * 64 * 4)
    sid = srv.add_scene(S[0][2])
    spec = S[0][0]
    fr = spec.camera.frame(64, 64)
    jids = [srv.submit(serving.job(sid, fr, 64, 64, 16, 8, background=0.0, seed=k)) for k in range(5)]
    big = srv.submit(serving.job(sid, spec.camera.frame(512, 512), 512, 512, 4, 8, background=0.0))
    peak_active = 0
    while True:
        left = srv.step()
        active = sum(srv.status(j).state == 1 for j in jids)
        peak_active = max(peak_active, active)
        for j in jids:
            if srv.status(j).state == 2:
                srv.release(j) if srv.status(j).device_bytes else None
        if left == 0:
            break
    assert peak_active <= 2
    assert all(srv.status(j).state == 2 for j in jids)
    assert srv.status(big).state == -1  # can never fit the budget
    st = srv.stats()
    assert st.peak_device_bytes <= 2 * 64 * 64 * 32 + 100
    assert st.jobs_rejected == 1
    srv.close()


def test_fp64_accumulation_and_frames(cuda):
    spec = scenes.cornell(width=48, height=48)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    srv = serving.Server(paths_per_iteration=48 * 48 * 8, frames_every=1)
    sid = srv.add_scene(ds)
    fr = spec.camera.frame(48, 48)
    a = srv.submit(serving.job(sid, fr, 48, 48, 40, spec.depth, background=0.0, seed=7))
    b = srv.submit(serving.job(sid, fr, 48, 48, 40, spec.depth, background=0.0, seed=7, fp64=True))
    srv.drain()
    ra, fa = srv.fetch(a, 48, 48, frame=True)
    rb, fb = srv.fetch(b, 48, 48, frame=True)
    np.testing.assert_allclose(ra, rb, rtol=1e-5, atol=1e-4)
    expect = (256 * np.minimum(np.sqrt(np.maximum(ra / 40, 0)), 0.999)).astype(np.uint8)
    assert np.abs(fa[..., :3].astype(int) - expect).max() <= 1
    assert (fa[..., 3] == 255).all()
    assert srv.stats().frames >= 2
    srv.close()


def test_trace_latencies(cuda):
    S = _scenes()
    srv = serving.Server(paths_per_iteration=1 << 20)
    ids = [srv.add_scene(ds) for _, _, ds in S]
    reqs = []
    rng = np.random.default_rng(0)
    t = 0.0
    for k in range(30):
        t += rng.exponential(1 / 200.0)
        si = k % 3
        spec = S[si][0]
        reqs.append(serving.job(ids[si], spec.camera.frame(64, 48), 64, 48, int(rng.integers(4, 32)), spec.depth,
                                background=spec.background, dof=spec.dof, seed=k, arrival=t))
    lat = srv.run_trace(reqs, realtime=True)
    assert (lat > 0).all()
    st = srv.stats()
    assert st.jobs_done == 30 and st.p99_latency >= st.p50_latency > 0
    assert st.paths == sum(r.width * r.height * r.spp for r in reqs)
    srv.close()


def test_sdf_field_jobs_on_the_wavefront_engine(cuda):
    # jobs of a smooth-SDF scene run on the wavefront engine (FP64
    # accumulation); the same job through the batched kernel and the
    # per-frame kernel (salt 0 = the job's seed 0) draws the same streams
    spec = scenes.sdf_field(count=48, width=48, height=32)
    w, h, spp = 48, 32, 16
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    out = {}
    for wf in (True, False):
        srv = serving.Server(paths_per_iteration=w * h * 8, max_spp_per_iteration=8, wavefront_field=wf)
        sid = srv.add_scene(ds)
        j = srv.submit(serving.job(sid, fr, w, h, spp, spec.depth, background=spec.background, seed=0))
        srv.drain()
        st = srv.status(j)
        assert st.state == 2 and st.spp_done == spp
        out[wf] = srv.fetch(j, w, h)
        assert srv.stats().paths == w * h * spp
        srv.close()
    ref = render.render_accumulate(ds, fr, w, h, spp, spec.depth, background=spec.background)
    for got in out.values():
        bad = (np.abs(got - ref) > 2e-3 * (1 + np.abs(ref)) * spp).any(axis=2)
        assert bad.mean() < 0.04, bad.mean()
        np.testing.assert_allclose(got.mean((0, 1)), ref.mean((0, 1)), rtol=2e-2, atol=1e-3)
    ds.free()


def test_wavefront_jobs_beside_class_kernels(cuda):
    # an iteration with smooth-SDF jobs runs them on the wavefront engine's
    # stream while the class kernels run; every job still gets its alone result
    sdf = scenes.sdf_field(count=48, width=48, height=32)
    box = scenes.cornell(width=64, height=64)
    dss = []
    for spec in (sdf, box):
        sc = spec.to_scene()
        sc.build_bvh()
        dss.append(sc.upload())
    reqs = [(0, 48, 32, 16), (1, 64, 64, 32), (0, 40, 24, 8), (1, 48, 48, 16)]
    specs = (sdf, box)

    def job(ids, k, si, w, h, spp):
        sp = specs[si]
        return serving.job(ids[si], sp.camera.frame(w, h), w, h, spp, sp.depth, background=sp.background,
                           seed=50 + k)

    mix = serving.Server(paths_per_iteration=1 << 16, max_spp_per_iteration=8)
    ids = [mix.add_scene(ds) for ds in dss]
    jids = [mix.submit(job(ids, k, *r)) for k, r in enumerate(reqs)]
    mix.drain()
    for k, (r, jid) in enumerate(zip(reqs, jids)):
        si, w, h, spp = r
        assert mix.status(jid).spp_done == spp
        got = mix.fetch(jid, w, h)
        alone = serving.Server(paths_per_iteration=1 << 26, max_spp_per_iteration=64)
        aid = [alone.add_scene(ds) for ds in dss]
        a = alone.submit(job(aid, k, *r))
        alone.drain()
        np.testing.assert_allclose(got, alone.fetch(a, w, h), rtol=RTOL, atol=ATOL_PER_SPP * spp)
        alone.close()
    mix.close()
    for ds in dss:
        ds.free()


def test_latency_target_controller(cuda):
    # the path quantum follows clamp(target / measured, 0.5, 2) per full
    # iteration: from a 64 M-path quantum it settles where an iteration takes
    # about the target time
    spec = scenes.cornell()
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    target = 4.0
    srv = serving.Server(paths_per_iteration=64 << 20, max_spp_per_iteration=1024, target_iteration_ms=target)
    sid = srv.add_scene(ds)
    fr = spec.camera.frame(512, 512)
    ms = []
    for k in range(6):
        srv.submit(serving.job(sid, fr, 512, 512, 1024, spec.depth, background=0.0, seed=k))
    while srv.step() > 0:
        ms.append(srv.stats().last_iteration_ms)
    st = srv.stats()
    assert st.quantum_paths < 64 << 20
    tail = ms[len(ms) // 2:-2]  # settled iterations (the last ones drain the queue)
    assert tail and 0.4 * target < float(np.median(tail)) < 2.5 * target, ms
    srv.close()
    ds.free()


def test_per_job_convergence(cuda):
    # a job with a convergence test completes before its spp once its pixels
    # stop changing; its image agrees with the full-spp render (per sample)
    spec = scenes.cornell(width=48, height=48)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(48, 48)
    srv = serving.Server(paths_per_iteration=48 * 48 * 64, max_spp_per_iteration=64)
    sid = srv.add_scene(ds)
    early = srv.submit(serving.job(sid, fr, 48, 48, 16384, spec.depth, background=0.0, seed=1,
                                   converge=(0.01, 128, 0.95)))
    full = srv.submit(serving.job(sid, fr, 48, 48, 4096, spec.depth, background=0.0, seed=2))
    srv.drain()
    se, sf = srv.status(early), srv.status(full)
    assert se.state == 2 and sf.state == 2
    assert 128 <= se.spp_done < 16384 and sf.spp_done == 4096
    a = srv.fetch(early, 48, 48) / se.spp_done
    b = srv.fetch(full, 48, 48) / sf.spp_done
    np.testing.assert_allclose(a.mean(), b.mean(), rtol=0.05)
    srv.close()
    ds.free()
