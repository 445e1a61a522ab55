"""Splitting one job across ranks (tim_raytracing_b200.shard) on the host.

Two gloo ranks stand in for two GPUs: each builds its own copy of the scene,
traces only its contiguous range of the job -- rays of a batch, output rows of a
camera frame, probes of a field -- and the ranges are all-gathered back in input
order. The tracing here is the oracle (the C restatement of the reference's
traversal), the host stand-in for each rank's GPU trace; the check is that the
reassembled records equal one rank tracing the whole job, bit for bit. Serving's
scene affinity is checked the same way: every job runs on its scene's rank and
the gathered results equal the single-rank results.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tim_raytracing_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


# ---------------------------------------------------------------- range arithmetic

@pytest.mark.parametrize("n,parts,align", [(0, 2, 1), (1, 3, 1), (10, 3, 1), (1080, 8, 4), (1079, 2, 4),
                                           (20_865_466, 8, 1), (7, 8, 4)])
def test_ranges_cover_in_order(n, parts, align):
    r = shard.contiguous_ranges(n, parts, align)
    assert len(r) == parts
    assert r[0][0] == 0 and r[-1][1] == n
    for (b0, e0), (b1, e1) in zip(r, r[1:]):
        assert e0 == b1
    for b, e in r:
        assert b <= e
        assert b % align == 0 or b == n
    sizes = [e - b for b, e in r]
    if n >= parts * align:
        assert max(sizes) - min(sizes) <= 2 * align


def test_weighted_ranges_balance_cost():
    rng = np.random.default_rng(1)
    w = np.concatenate([np.full(300, 0.1), rng.uniform(1, 5, 780)])   # cheap sky rows, then costly ground rows
    r = shard.row_bands(1080, 4, w)
    costs = [w[b:e].sum() for b, e in r]
    assert max(costs) / min(costs) < 1.05
    plain = shard.row_bands(1080, 4)
    pc = [w[b:e].sum() for b, e in plain]
    assert max(pc) / min(pc) > 2.0          # equal row counts would leave the ranks unbalanced
    assert all(b % 4 == 0 for b, _ in r)


def test_ranges_reject_bad_arguments():
    with pytest.raises(ValueError):
        shard.contiguous_ranges(10, 0)
    with pytest.raises(ValueError):
        shard.contiguous_ranges(3, 2, weights=[1.0, -1.0, 2.0])


def test_scene_router_is_deterministic_and_balanced():
    sizes = {10: 900, 11: 100, 12: 500, 13: 400, 14: 300, 15: 300}
    a = shard.SceneRouter(sizes, 2)
    b = shard.SceneRouter(dict(reversed(list(sizes.items()))), 2)
    assert a.rank_of_scene == b.rank_of_scene
    assert sorted(a.load) == [1200, 1300]
    assert sorted(a.scenes_of(0) + a.scenes_of(1)) == sorted(sizes)
    jobs = [(12, "x"), (10, "y"), (11, "z"), (12, "w")]
    routed = a.route(jobs)
    assert sorted(routed[0] + routed[1]) == [0, 1, 2, 3]
    for r in range(2):
        assert routed[r] == sorted(routed[r])
        assert all(a.rank_of(jobs[j][0]) == r for j in routed[r])
    with pytest.raises(KeyError):
        a.rank_of(99)


def test_frame_row_weights_follow_the_records():
    W, H = 32, 8
    rec = np.zeros((W * H, 8), np.uint32)
    rec[:, 3] = np.float32(100.0).view(np.uint32)         # misses
    rec[4 * W:, 3] = np.float32(3.0).view(np.uint32)      # rows 4..7 hit
    w = shard.frame_row_weights(rec, W, H)
    assert w[0] == 0.0
    assert np.all(w[1:4] == W) and np.all(w[4:] == W * 4.0)


# ---------------------------------------------------------------- two gloo ranks

def _rank(rank, world, port, out):
    import datetime
    import sys
    from pathlib import Path
    import torch
    import torch.distributed as dist
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    from oracle import oracle as O
    from tim_raytracing_b200 import _native as N, scenes, shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        res = {}
        # every rank holds its own copy of the scene
        s = scenes.heightfield_scene(seed=5, grid=24, n_spheres=6, n_lights=16, light_radius=5.0)
        img = N.build_bvh(s)
        sc = O.Scene(img, s.positions, s.normals)
        # (1) a ray batch split into contiguous ray ranges
        rays = scenes.serving_rays(7, 5003, extent=20.0)

        def trace_rays(b, e):
            hit, nid, _, _ = O.trace(sc, rays[b:e], mode=N.MODE_PER_RAY, threads=2)
            return torch.from_numpy(np.concatenate([hit, nid[:, None]], 1).view(np.int32))

        got, mine = S.trace_sharded(trace_rays, len(rays))
        res["rays"] = (got.numpy().view(np.uint32), mine)
        # (2) one camera frame split into bands of output rows, balanced by a cost
        # estimate that every rank computes from the same previous frame
        W, H = 96, 70
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        tx, ty = (W + 15) // 16, (H + 15) // 16
        counts, lists = O.cull_lights(sc, pd, tx, ty, threads=2)
        prev, _, _ = O.camera(sc, pd, flags=2 | 4, seed=3, tile_counts=counts, tile_lists=lists, threads=2)
        weights = S.frame_row_weights(prev, W, H, counts)
        bands = S.row_bands(H, world, weights)

        def trace_rows(b, e):
            out, bounce, _ = O.camera(sc, pd, flags=2 | 4, seed=3, tile_counts=counts, tile_lists=lists,
                                      pix_range=(b * W, e * W), threads=2)
            both = np.concatenate([out.reshape(H, W, 8), bounce.reshape(H, W, 4)], 2)[b:e]
            return torch.from_numpy(np.ascontiguousarray(both).view(np.int32))

        got_f, _ = S.trace_sharded(trace_rows, H, weights=weights, align=S.ROW_ALIGN)
        res["frame"] = (got_f.numpy().view(np.uint32), bands)
        # (3) a probe field update split into contiguous probe ranges
        res_xyz = (8, 8, 4)
        dirs = scenes.octahedral_dirs(8)
        od = O.probe_desc(img.aabb[:3], img.aabb[3:], res_xyz, (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), len(dirs))

        def trace_probes(b, e):
            tr, irr, _ = O.probe_trace(sc, od, dirs, b, e, threads=2)
            return torch.from_numpy(np.concatenate([tr.reshape(e - b, -1), irr.reshape(e - b, -1).view(np.uint32)],
                                                   1).view(np.int32))

        got_p, _ = S.trace_sharded(trace_probes, res_xyz[0] * res_xyz[1] * res_xyz[2])
        res["probes"] = got_p.numpy().view(np.uint32)
        # (4) serving: scenes by affinity, jobs routed to their scene's rank
        scs = [scenes.random_triangles(30 + k, 400 + 300 * k) for k in range(4)]
        imgs = [N.build_bvh(x) for x in scs]
        router = S.SceneRouter({k: imgs[k].data.nbytes for k in range(4)}, world)
        jobs = [(k % 4, scenes.random_rays(50 + k, 300 + 17 * k)) for k in range(10)]
        mine_jobs = router.route(jobs)[rank]
        local = {}
        for j in mine_jobs:
            k, r = jobs[j]
            assert router.rank_of(k) == rank
            osc = O.Scene(imgs[k], scs[k].positions, scs[k].normals)
            hit, _, _, _ = O.trace(osc, r, mode=N.MODE_PER_RAY, threads=2)
            local[j] = hit
        parts = [None] * world
        dist.all_gather_object(parts, local)
        merged = {}
        for p in parts:
            merged.update(p)
        res["serving"] = [merged[j] for j in range(len(jobs))]
        res["serving_ranks"] = [router.rank_of(k) for k, _ in jobs]
        out[rank] = res
    finally:
        dist.destroy_process_group()


def _whole_job():
    """The same four jobs traced by one rank."""
    from oracle import oracle as O
    from tim_raytracing_b200 import _native as N, scenes
    s = scenes.heightfield_scene(seed=5, grid=24, n_spheres=6, n_lights=16, light_radius=5.0)
    img = N.build_bvh(s)
    sc = O.Scene(img, s.positions, s.normals)
    rays = scenes.serving_rays(7, 5003, extent=20.0)
    hit, nid, _, _ = O.trace(sc, rays, mode=N.MODE_PER_RAY)
    want_rays = np.concatenate([hit, nid[:, None]], 1)
    W, H = 96, 70
    pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    counts, lists = O.cull_lights(sc, pd, (W + 15) // 16, (H + 15) // 16)
    out, bounce, _ = O.camera(sc, pd, flags=2 | 4, seed=3, tile_counts=counts, tile_lists=lists)
    want_frame = np.concatenate([out.reshape(H, W, 8), bounce.reshape(H, W, 4)], 2)
    dirs = scenes.octahedral_dirs(8)
    od = O.probe_desc(img.aabb[:3], img.aabb[3:], (8, 8, 4), (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), len(dirs))
    tr, irr, _ = O.probe_trace(sc, od, dirs, 0, 256)
    want_probes = np.concatenate([tr.reshape(256, -1), irr.reshape(256, -1).view(np.uint32)], 1)
    scs = [scenes.random_triangles(30 + k, 400 + 300 * k) for k in range(4)]
    imgs = [N.build_bvh(x) for x in scs]
    want_serving = []
    for k in range(10):
        osc = O.Scene(imgs[k % 4], scs[k % 4].positions, scs[k % 4].normals)
        h, _, _, _ = O.trace(osc, scenes.random_rays(50 + k, 300 + 17 * k), mode=N.MODE_PER_RAY)
        want_serving.append(h)
    return want_rays, want_frame, want_probes, want_serving


def test_two_ranks_reassemble_the_one_rank_result(oracle_mod, native):
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    want_rays, want_frame, want_probes, want_serving = _whole_job()
    for r in range(world):
        got, mine = out[r]["rays"]
        assert np.array_equal(got, want_rays)
        got_f, bands = out[r]["frame"]
        assert np.array_equal(got_f, want_frame)
        assert np.array_equal(out[r]["probes"], want_probes)
        assert len(out[r]["serving"]) == len(want_serving)
        for g, w in zip(out[r]["serving"], want_serving):
            assert np.array_equal(g, w)
    # the ranks really split the work: disjoint, non-empty ranges covering the job
    r0, r1 = out[0]["rays"][1], out[1]["rays"][1]
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] == 5003 and r0[1] > 0
    bands = out[0]["frame"][1]
    assert bands[0][0] == 0 and bands[0][1] == bands[1][0] and bands[1][1] == 70 and bands[0][1] % 4 == 0
    assert set(out[0]["serving_ranks"]) == {0, 1}
