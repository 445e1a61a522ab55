"""GPU tests of the serving loop (tim_rt_server_*): requests submitted from
several threads, admitted against a small device arena and traced in chunks
across many batched steps, must each give exactly the outputs of tracing them
alone (tim_rt_trace on the same scene, rays and mode)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(ctx, native):
    from tim_raytracing_b200 import scenes
    sids = []
    for k, n in enumerate([500, 5000, 30000]):
        s = scenes.random_triangles(300 + k, n)
        sids.append(ctx.upload(native.build_bvh(s), s, quant8=True))
    hf = scenes.heightfield_scene(seed=3, grid=32, n_spheres=4)
    sids.append(ctx.upload(native.build_bvh(hf), hf, quant8=True))
    yield sids
    for sid in sids:
        ctx.free_scene(sid)


def _pinned(shape, dtype):
    import torch
    t = torch.empty(shape, dtype=dtype, pin_memory=True)
    return t, t.numpy()


def _requests(sids, count, seed):
    import torch
    from tim_raytracing_b200 import scenes
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(0, np.log(20000))))
        sid = sids[int(rng.integers(len(sids)))]
        mode = int(rng.integers(3))
        rays = scenes.random_rays(seed * 1000 + i, n)
        if sid == sids[-1]:   # the heightfield spans [0, 20]^2 x [0, 2]
            rays[:, 0:3] *= np.array([20, 20, 4], np.float32)
        tr, r = _pinned((n, 8), torch.float32)
        r[:] = rays
        th, h = _pinned((n, 4), torch.int32)
        tn, nid = _pinned((n,), torch.int32)
        tb, b = _pinned((n, 2), torch.float32)
        want_nid = i % 3 != 0
        want_bary = i % 4 != 1
        reqs.append(dict(sid=sid, mode=mode, rays=r, hit=h, nid=nid if want_nid else None,
                         bary=b if want_bary else None, keep=(tr, th, tn, tb)))
    return reqs


def _check(ctx, native, reqs, wide):
    for q in reqs:
        mode = q["mode"] | (native.TRACE_WIDE if wide else 0)
        h, nid, b, _ = ctx.trace(q["sid"], q["rays"], mode)
        assert np.array_equal(q["hit"].view(np.uint32), h)
        if q["nid"] is not None:
            assert np.array_equal(q["nid"].view(np.uint32), nid)
        if q["bary"] is not None:
            assert np.array_equal(q["bary"].view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("wide", [False, True])
def test_server_mix_matches_alone(ctx, native, served, wide):
    reqs = _requests(served, 48, seed=11 + wide)
    srv = native.Server(ctx, memory_budget_bytes=4 << 20, max_rays_per_step=16384, max_inflight_steps=2,
                        wide=wide)
    try:
        def submit(part):
            for q in part:
                q["ticket"] = srv.submit(q["sid"], q["rays"], q["mode"], q["hit"], q["nid"], q["bary"])

        threads = [threading.Thread(target=submit, args=(reqs[k::3],)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        srv.wait(reqs[0]["ticket"], timeout_ms=60000)
        srv.drain(timeout_ms=120000)
        st = srv.stats()
        assert st["completed"] == st["submitted"] == len(reqs)
        assert st["rays_completed"] == sum(len(q["rays"]) for q in reqs)
        assert st["steps"] >= st["rays_completed"] // 16384
        assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
        assert 0 < st["arena_peak_bytes"] <= st["arena_bytes"]
        # continuous batching: steps held several requests, and the worker queued the
        # next step while the previous one still ran on the GPU
        assert st["max_step_requests"] >= 2
        assert st["step_requests"] > st["steps"]
        assert st["max_inflight"] == 2
        assert 0 < st["gpu_busy_ms"] < 1e3 * st["wall_s"]
    finally:
        srv.close()
    _check(ctx, native, reqs, wide)


def test_server_errors(ctx, native, served):
    import torch
    srv = native.Server(ctx, memory_budget_bytes=1 << 20)
    try:
        n = 40000      # 48 B per ray staged: more than the 1 MiB arena
        _, r = _pinned((n, 8), torch.float32)
        _, h = _pinned((n, 4), torch.int32)
        with pytest.raises(native.TimRtError) as e:
            srv.submit(served[0], r, 0, h)
        assert e.value.code == native.ENOMEM
        with pytest.raises(native.TimRtError) as e:
            srv.submit(99999, r[:10], 0, h[:10])
        assert e.value.code == native.ENOTFOUND
        # a completed request no longer pins its scene; the stats reset
        t = srv.submit(served[0], r[:100], 0, h[:100])
        srv.wait(t, timeout_ms=60000)
        assert srv.stats(reset=True)["completed"] == 1
        assert srv.stats()["completed"] == 0
    finally:
        srv.close()


def test_server_probe_updates_in_the_mix(ctx, native, served):
    """Probe-field update requests (tim_rt_server_submit_probes) submitted while
    trace requests stream in from other threads: each update's FP16 field and
    octahedral texels equal tim_rt_update_probes on the same inputs, and the
    trace requests still equal tracing alone."""
    import torch
    from tim_raytracing_b200 import scenes
    sid = served[-1]
    res = (8, 8, 4)
    dirs = scenes.octahedral_dirs(8)
    basis = scenes.sh9_basis(dirs)
    lo, hi = np.zeros(3, np.float32), np.array([20, 20, 4], np.float32)
    forms = [(0, 0, 64, False), (native.PROBE_WIDE | native.PROBE_PRIMARY_BINARY, 64, 192, True),
             (native.PROBE_WIDE, 16, 48, True), (0, 200, 256, True)]
    probes = []
    rng = np.random.default_rng(4)
    for k, (flag, p0, p1, octa) in enumerate(forms):
        desc = native.probe_desc(lo, hi, res, (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), len(dirs), 0.03,
                                 flag | (native.PROBE_OCTA if octa else 0))
        sh = rng.uniform(-1, 1, size=(7, res[2], res[1], res[0], 4)).astype(np.float16).view(np.uint16)
        want = sh.copy()
        _, _, _, want_octa, _ = ctx.update_probes(sid, desc, dirs, basis, want, p0, p1, want_octa=octa)
        t16, got = _pinned(sh.shape, torch.int16)
        got = got.view(np.uint16)
        got[:] = sh
        to, go = _pinned((p1 - p0, 64, 3), torch.float32) if octa else (None, None)
        probes.append(dict(desc=desc, p0=p0, p1=p1, want=want, want_octa=want_octa, got=got, octa=go,
                           keep=(t16, to)))
    reqs = _requests(served, 24, seed=29)
    srv = native.Server(ctx, memory_budget_bytes=16 << 20, max_rays_per_step=16384, max_inflight_steps=2, wide=True)
    try:
        def submit(part):
            for q in part:
                q["ticket"] = srv.submit(q["sid"], q["rays"], q["mode"], q["hit"], q["nid"], q["bary"])

        def submit_probes():
            for P in probes:
                P["ticket"] = srv.submit_probes(sid, P["desc"], dirs, basis, P["got"], P["p0"], P["p1"], P["octa"])

        threads = [threading.Thread(target=submit, args=(reqs[k::2],)) for k in range(2)]
        threads.append(threading.Thread(target=submit_probes))
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        srv.drain(timeout_ms=120000)
        st = srv.stats()
        assert st["completed"] == st["submitted"] == len(reqs) + len(probes)
        assert st["rays_completed"] == sum(len(q["rays"]) for q in reqs) + sum(
            (P["p1"] - P["p0"]) * len(dirs) for P in probes)
    finally:
        srv.close()
    for P in probes:
        assert np.array_equal(P["got"], P["want"])
        if P["octa"] is not None:
            assert np.array_equal(P["octa"].view(np.uint32), P["want_octa"].view(np.uint32))
    _check(ctx, native, reqs, True)


def test_server_probe_request_errors(ctx, native, served):
    from tim_raytracing_b200 import scenes
    dirs = scenes.octahedral_dirs(8)
    basis = scenes.sh9_basis(dirs)
    sh = np.zeros((7, 4, 8, 8, 4), np.uint16)
    srv = native.Server(ctx, memory_budget_bytes=1 << 20)
    try:
        bad_res = native.probe_desc((0, 0, 0), (1, 1, 1), (8, 8, 6), (0, 0, -1), (1, 1, 1), len(dirs), 0.03, 0)
        with pytest.raises(native.TimRtError) as e:
            srv.submit_probes(served[-1], bad_res, dirs, basis, sh, 0, 64)
        assert e.value.code == native.EINVAL
        desc = native.probe_desc((0, 0, 0), (1, 1, 1), (8, 8, 4), (0, 0, -1), (1, 1, 1), len(dirs), 0.03, 0)
        with pytest.raises(native.TimRtError) as e:
            srv.submit_probes(served[-1], desc, dirs, basis, sh, 0, 256)    # ~17 MB of staging
        assert e.value.code == native.ENOMEM
        with pytest.raises(native.TimRtError) as e:
            srv.submit_probes(served[-1], desc, dirs, basis, sh, 10, 5)
        assert e.value.code == native.EINVAL
    finally:
        srv.close()


def _sentinel_hits(n):
    import torch
    th, h = _pinned((n, 4), torch.int32)
    h[:] = 0x7F7F7F7F
    return th, h


def test_server_cancel(ctx, native, served):
    """tim_rt_server_cancel on a request still waiting for admission and on an
    admitted one that many steps still have to trace: both complete as cancelled
    (wait reports ECANCELLED) without writing their outputs, the other requests
    are served as if alone, and tickets that are unknown or done are refused."""
    import torch
    from tim_raytracing_b200 import scenes
    sid = served[2]
    big_n, wait_n = 1_000_000, 200_000      # 48 B staged per ray: 48 MB and 9.6 MB
    tb, big_rays = _pinned((big_n, 8), torch.float32)
    big_rays[:] = scenes.random_rays(71, big_n)
    tbh, big_hit = _sentinel_hits(big_n)
    tw, wait_rays = _pinned((wait_n, 8), torch.float32)
    wait_rays[:] = scenes.random_rays(72, wait_n)
    twh, wait_hit = _sentinel_hits(wait_n)
    reqs = _requests(served, 8, seed=43)
    srv = native.Server(ctx, memory_budget_bytes=56 << 20, max_rays_per_step=4096, max_inflight_steps=2)
    try:
        t_big = srv.submit(sid, big_rays, native.MODE_PER_RAY, big_hit)
        t_wait = srv.submit(sid, wait_rays, native.MODE_PER_RAY, wait_hit)   # cannot fit beside the big one
        assert srv.cancel(t_wait) == native.OK        # still waiting: gone at once
        assert srv.cancel(t_big) == native.OK         # admitted, most of its ~245 steps still to come
        assert srv.cancel(t_big) in (native.OK, native.ENOTFOUND)   # again: still draining, or already done
        for t in (t_wait, t_big):
            with pytest.raises(native.TimRtError) as e:
                srv.wait(t, timeout_ms=60000)
            assert e.value.code == native.ECANCELLED
        for q in reqs:
            q["ticket"] = srv.submit(q["sid"], q["rays"], q["mode"], q["hit"], q["nid"], q["bary"])
        srv.drain(timeout_ms=120000)
        assert srv.cancel(reqs[0]["ticket"]) == native.ENOTFOUND    # completed
        assert srv.cancel(10 ** 9) == native.ENOTFOUND             # never issued
        st = srv.stats()
        assert st["cancelled"] == 2
        assert st["completed"] == len(reqs)
    finally:
        srv.close()
    assert np.all(big_hit == 0x7F7F7F7F) and np.all(wait_hit == 0x7F7F7F7F)
    _check(ctx, native, reqs, False)


def test_server_stalled_submitter(ctx, native, served):
    """Host-side fault injection: one client thread submits requests and then
    stalls (blocks without ever waiting for them) while two other clients keep
    submitting and waiting. The server does not depend on its clients: the other
    clients' requests complete while the stalled one is blocked, so do the
    stalled client's own requests (checked from the main thread), and every
    result equals tracing alone."""
    import time
    stalled = _requests(served, 6, seed=51)
    others = _requests(served, 24, seed=52)
    srv = native.Server(ctx, memory_budget_bytes=8 << 20, max_rays_per_step=16384, max_inflight_steps=2)
    release = threading.Event()
    submitted = threading.Event()
    errors = []

    def stalled_client():
        for q in stalled:
            q["ticket"] = srv.submit(q["sid"], q["rays"], q["mode"], q["hit"], q["nid"], q["bary"])
        submitted.set()
        release.wait(120)       # the stall: no waits, no further calls

    def client(part):
        try:
            for q in part:
                t = srv.submit(q["sid"], q["rays"], q["mode"], q["hit"], q["nid"], q["bary"])
                srv.wait(t, timeout_ms=60000)
                q["done_while_stalled"] = not release.is_set()
        except Exception as e:     # noqa: BLE001 -- reported below
            errors.append(e)

    ts = threading.Thread(target=stalled_client)
    ts.start()
    try:
        assert submitted.wait(60)
        workers = [threading.Thread(target=client, args=(others[k::2],)) for k in range(2)]
        for w in workers:
            w.start()
        for w in workers:
            w.join(120)
        assert not errors, errors
        assert all(q["done_while_stalled"] for q in others)
        t0 = time.perf_counter()
        for q in stalled:
            srv.wait(q["ticket"], timeout_ms=60000)   # served without the stalled client's help
        assert time.perf_counter() - t0 < 60
        assert ts.is_alive()       # the stalled client is still blocked
    finally:
        release.set()
        ts.join(60)
        srv.close()
    _check(ctx, native, stalled + others, False)
