"""GPU parity of the batched multi-scene trace (tim_rt_batch_*): one persistent
launch over jobs on scenes of uneven size must give, for every job, exactly the
outputs of tracing that job alone (tim_rt_trace on the same scene, rays and
mode), whatever the launch configuration and ray-sort key; the plain form is
also checked against the oracle directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (triangles, rays, mode) per job; scene 1 is used by two jobs
JOBS = [(2000, 3000, 2), (300, 1000, 0), (300, 700, 1), (40, 257, 2), (20000, 9000, 0), (1, 64, 2),
        (6000, 4096, 1), (0, 0, 0)]


@pytest.fixture(scope="module")
def mctx(native):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def world(mctx, native):
    """Uploads the distinct scenes and makes each job's rays (host and device copies)."""
    import torch
    from tim_raytracing_b200 import scenes
    built, sids = {}, {}
    jobs = []
    for j, (ntri, nray, mode) in enumerate(JOBS):
        key = max(ntri, 1)
        if key not in sids:
            s = scenes.random_triangles(1000 + key, key)
            img = native.build_bvh(s)
            built[key] = (s, img)
            sids[key] = mctx.upload(img, s, quant8=True)
        rays = scenes.random_rays(77 + j, nray)
        d_rays = torch.from_numpy(rays).cuda() if nray else torch.empty((1, 8), device="cuda")
        jobs.append(dict(sid=sids[key], key=key, mode=mode, rays=rays, d_rays=d_rays))
    yield built, jobs
    for sid in sids.values():
        mctx.free_scene(sid)


def _outputs(jobs):
    import torch
    for J in jobs:
        n = max(len(J["rays"]), 1)
        J["d_hit"] = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
        J["d_nid"] = torch.zeros(n, dtype=torch.int32, device="cuda")
        J["d_bary"] = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    return [(J["sid"], J["mode"], len(J["rays"]), J["d_rays"], J["d_hit"], J["d_nid"], J["d_bary"]) for J in jobs]


def _check_against_alone(ctx, native, jobs, wide):
    for J in jobs:
        n = len(J["rays"])
        if n == 0:
            continue
        mode = J["mode"] | (native.TRACE_WIDE if wide else 0)
        h, nid, b, _ = ctx.trace(J["sid"], J["rays"], mode)
        gh = J["d_hit"].cpu().numpy().view(np.uint32)[:n]
        gn = J["d_nid"].cpu().numpy().view(np.uint32)[:n]
        gb = J["d_bary"].cpu().numpy()[:n]
        assert np.array_equal(gh, h), (J["key"], J["mode"])
        assert np.array_equal(gn, nid)
        assert np.array_equal(gb.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("wide", [False, True])
@pytest.mark.parametrize("ray_sort", [0, 1, 2])
def test_batch_matches_alone(mctx, native, world, wide, ray_sort):
    import torch
    built, jobs = world
    b = mctx.batch_create(_outputs(jobs), wide=wide)
    try:
        rays, _ = mctx.batch_info(b)
        assert rays == sum(len(J["rays"]) for J in jobs)
        mctx.set_launch_config(block=128, refill_min=16, ray_sort=ray_sort)
        mctx.batch_launch(b)
        torch.cuda.synchronize()
        _check_against_alone(mctx, native, jobs, wide)
    finally:
        mctx.set_launch_config()
        mctx.batch_destroy(b)


def test_batch_plain_matches_oracle(mctx, native, oracle_mod, world):
    import torch
    built, jobs = world
    b = mctx.batch_create(_outputs(jobs))
    try:
        mctx.set_launch_config(block=64, refill_min=8)
        mctx.batch_launch(b)
        torch.cuda.synchronize()
        for J in jobs:
            n = len(J["rays"])
            if n == 0:
                continue
            s, img = built[J["key"]]
            sc = oracle_mod.Scene(img, s.positions, s.normals)
            oh, on, ob, _ = oracle_mod.trace(sc, J["rays"], J["mode"])
            assert np.array_equal(J["d_hit"].cpu().numpy().view(np.uint32)[:n], oh)
            assert np.array_equal(J["d_nid"].cpu().numpy().view(np.uint32)[:n], on)
            assert np.array_equal(J["d_bary"].cpu().numpy()[:n].view(np.uint32), ob.view(np.uint32))
    finally:
        mctx.set_launch_config()
        mctx.batch_destroy(b)


def test_batch_graph_replay(mctx, native, world):
    """The launch is captured once in a CUDA graph; replays after the rays were
    rewritten in place trace the new rays."""
    import torch
    from tim_raytracing_b200 import scenes
    built, jobs = world
    b = mctx.batch_create(_outputs(jobs), wide=True)
    try:
        mctx.set_launch_config(block=128, refill_min=16, ray_sort=2)
        mctx.batch_launch(b)              # sizes the sort scratch before capture
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            mctx.batch_launch(b, stream=s.cuda_stream)
        for rep in range(2):
            for j, J in enumerate(jobs):
                if len(J["rays"]):
                    J["rays"] = scenes.random_rays(500 + 10 * rep + j, len(J["rays"]))
                    J["d_rays"].copy_(torch.from_numpy(J["rays"]))
                    J["d_hit"].zero_()
            torch.cuda.synchronize()
            g.replay()
            torch.cuda.synchronize()
            _check_against_alone(mctx, native, jobs, True)
        del g
    finally:
        mctx.set_launch_config()
        mctx.batch_destroy(b)


def test_autotune_installs_a_config(mctx, native, world):
    import torch
    built, jobs = world
    b = mctx.batch_create(_outputs(jobs), wide=True)
    try:
        r = mctx.autotune_batch(b, width=False, reps=2)
        assert r["tried"] >= 10 and 0 < r["best_ms"] <= r["start_ms"]
        cfg = mctx.launch_config()
        assert (cfg["block"], cfg["refill_min"], cfg["ray_sort"]) == (r["block"], r["refill_min"], r["ray_sort"])
        for J in jobs:
            J["d_hit"].zero_()
        mctx.batch_launch(b)
        torch.cuda.synchronize()
        _check_against_alone(mctx, native, jobs, True)
    finally:
        mctx.set_launch_config()
        mctx.batch_destroy(b)


def test_batch_near_ties_match_oracle(mctx, native, oracle_mod):
    """A batch whose scene is mostly near-ties (exercises the 8-wide walk's hand-over
    to the binary walk inside the multi-scene kernel), next to an ordinary scene."""
    import torch
    from helpers import near_tie_scene
    from tim_raytracing_b200 import scenes
    s1 = near_tie_scene(41, 3000)
    s2 = scenes.random_triangles(42, 5000)
    imgs = [native.build_bvh(s1), native.build_bvh(s2)]
    sids = [mctx.upload(imgs[0], s1, quant8=True), mctx.upload(imgs[1], s2, quant8=True)]
    b = None
    try:
        rays = [scenes.random_rays(43, 20000, any_fraction=0.3), scenes.random_rays(44, 7000)]
        d = [torch.from_numpy(r).cuda() for r in rays]
        hits = [torch.zeros((len(r), 4), dtype=torch.int32, device="cuda") for r in rays]
        nids = [torch.zeros(len(r), dtype=torch.int32, device="cuda") for r in rays]
        hits_p = [torch.zeros((len(r), 4), dtype=torch.int32, device="cuda") for r in rays]
        b = mctx.batch_create([(sids[k], native.MODE_PER_RAY, len(rays[k]), d[k], hits[k], nids[k], None)
                               for k in range(2)], wide=True)
        bp = mctx.batch_create([(sids[k], native.MODE_PER_RAY, len(rays[k]), d[k], hits_p[k], None, None)
                                for k in range(2)], wide=False)
        for refill, sw in ((16, 10), (1, 0), (4, 31)):
            mctx.set_launch_config(block=128, refill_min=refill, phase_switch=sw)
            mctx.batch_launch(b)
            mctx.batch_launch(bp)
            torch.cuda.synchronize()
            for k, (s, img) in enumerate(((s1, imgs[0]), (s2, imgs[1]))):
                oh, on, _, _ = oracle_mod.trace(oracle_mod.Scene(img, s.positions, s.normals), rays[k], 2)
                assert np.array_equal(hits[k].cpu().numpy().view(np.uint32), oh), (k, refill, sw)
                assert np.array_equal(nids[k].cpu().numpy().view(np.uint32), on), (k, refill, sw)
                assert np.array_equal(hits_p[k].cpu().numpy().view(np.uint32), oh), (k, refill, sw)
    finally:
        mctx.set_launch_config()
        if b is not None:
            mctx.batch_destroy(b)
            mctx.batch_destroy(bp)
        for sid in sids:
            mctx.free_scene(sid)


def test_batch_errors(mctx, native, world):
    built, jobs = world
    b = mctx.batch_create(_outputs(jobs[:2]))
    try:
        with pytest.raises(native.TimRtError) as e:
            mctx.free_scene(jobs[0]["sid"])      # still used by the batch
        assert e.value.code == native.EINVAL
        with pytest.raises(native.TimRtError) as e:
            mctx.batch_create([(12345, 0, 1, jobs[0]["d_rays"], jobs[0]["d_hit"], None, None)])
        assert e.value.code == native.ENOTFOUND
        with pytest.raises(native.TimRtError) as e:
            mctx.batch_create([(jobs[0]["sid"], 7, 1, jobs[0]["d_rays"], jobs[0]["d_hit"], None, None)])
        assert e.value.code == native.EINVAL
    finally:
        mctx.batch_destroy(b)
