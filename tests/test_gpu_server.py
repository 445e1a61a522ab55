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
