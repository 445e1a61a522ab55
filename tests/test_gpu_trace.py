"""GPU parity: the sm_100a kernels, called through the C ABI, against the oracle
and the golden vectors. Integer outputs (hit records, leaf ids, masks) and the
FP32 t / barycentrics must be bit-identical for the plain (reference layout)
form and for the 8-wide quantised form alike (the 8-wide walk re-traces the rays
whose answer it cannot prove equal with the binary walk)."""
import numpy as np
import pytest

from helpers import load_room, load_room_golden, near_tie_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def room(ctx):
    s, img = load_room()
    sid = ctx.upload(img, s, quant8=True)
    yield s, img, sid
    ctx.free_scene(sid)


def test_trace_room_matches_golden(ctx, native, room):
    s, img, sid = room
    g = load_room_golden()
    hit, nid, bary, st = ctx.trace(sid, g["rays"], native.MODE_CLOSEST)
    assert np.array_equal(hit, g["hit_closest"])
    assert np.array_equal(nid, g["nid_closest"])
    assert np.array_equal(bary.view(np.uint32), g["bary_closest"].view(np.uint32))
    ha, _, _, _ = ctx.trace(sid, g["rays"], native.MODE_ANY)
    assert np.array_equal(ha, g["hit_any"])
    assert st.rays == len(g["rays"])


def test_trace_per_ray_mode(ctx, native, room, oracle_mod):
    s, img, sid = room
    g = load_room_golden()
    rays = g["rays"]
    hit, nid, bary, _ = ctx.trace(sid, rays, native.MODE_PER_RAY)
    sc = oracle_mod.Scene(img, s.positions, s.normals)
    oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
    assert np.array_equal(hit, oh)
    assert np.array_equal(nid, on)
    assert np.array_equal(bary.view(np.uint32), ob.view(np.uint32))


def test_camera_room_matches_golden(ctx, native, room):
    """cameraPass.comp TRACING_STEP with USE_LPF_MASK on the reference-built BVH."""
    from tim_raytracing_b200 import scenes
    s, img, sid = room
    g = load_room_golden()
    pd = g["pass_data"].view(scenes.PASS_DATA_DTYPE)
    out, _, st = ctx.trace_camera(sid, pd, flags=native.CAM_PROB_MASK)
    assert np.array_equal(out, g["camera"])
    assert st.primary_rays == 256 * 255


@pytest.mark.parametrize("wide", [0, 1, 2])
def test_camera_heightfield_tile_lights_bounce(ctx, native, oracle_mod, wide):
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=9, grid=32, n_spheres=6, n_lights=16, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=wide)
    try:
        W, H = 160, 120
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        tx, ty = (W + 15) // 16, (H + 15) // 16
        counts, lists = ctx.cull_lights(sid, pd, tx, ty)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oc, ol = oracle_mod.cull_lights(sc, pd, tx, ty)
        assert np.array_equal(counts, oc)
        assert np.array_equal(lists, ol)
        flags = native.CAM_TILE_LIGHTS | native.CAM_BOUNCE | native.CAM_PROB_MASK
        form = [0, native.CAM_WIDE, native.CAM_WIDE | native.CAM_PRIMARY_BINARY][wide]
        out, bounce, st = ctx.trace_camera(sid, pd, flags=flags | form, seed=17,
                                           tile_counts=counts, tile_lists=lists)
        o_out, o_bounce, o_counts = oracle_mod.camera(sc, pd, flags=flags, seed=17, tile_counts=oc, tile_lists=ol)
        assert np.array_equal(out, o_out)
        assert np.array_equal(bounce, o_bounce)
        assert st.rays == int(o_counts.sum())
    finally:
        ctx.free_scene(sid)


@pytest.mark.parametrize("H", [257, 400])
def test_camera_pipelined_bands_match_oracle(ctx, native, oracle_mod, H):
    """TIM_RT_CAM_PIPELINED (bands of rows, copies overlapped with tracing) gives the
    oracle's records, bounce records and ray count, frame heights with and without
    a partial last tile row."""
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=10, grid=32, n_spheres=6, n_lights=16, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        W = 200
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        tx, ty = (W + 15) // 16, (H + 15) // 16
        counts, lists = ctx.cull_lights(sid, pd, tx, ty)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        flags = native.CAM_TILE_LIGHTS | native.CAM_BOUNCE | native.CAM_PROB_MASK
        o_out, o_bounce, o_counts = oracle_mod.camera(sc, pd, flags=flags, seed=5, tile_counts=counts,
                                                      tile_lists=lists)
        for form in (0, native.CAM_WIDE | native.CAM_PRIMARY_BINARY):
            out, bounce, st = ctx.trace_camera(sid, pd, flags=flags | form | native.CAM_PIPELINED, seed=5,
                                               tile_counts=counts, tile_lists=lists)
            assert np.array_equal(out, o_out)
            assert np.array_equal(bounce, o_bounce)
            assert st.rays == int(o_counts.sum())
    finally:
        ctx.free_scene(sid)


@pytest.mark.parametrize("n_tris,seed", [(2000, 1), (50000, 2)])
def test_random_scene_mixed_rays(ctx, native, oracle_mod, n_tris, seed):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(seed, n_tris)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rays = scenes.random_rays(seed + 100, 60000)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
        for form in (0, native.TRACE_WIDE):
            hit, nid, bary, _ = ctx.trace(sid, rays, native.MODE_PER_RAY | form)
            assert np.array_equal(hit, oh), form
            assert np.array_equal(nid, on), form
            assert np.array_equal(bary.view(np.uint32), ob.view(np.uint32)), form
    finally:
        ctx.free_scene(sid)


def _margin_rays(img, aabb, seed, n_per_kind):
    """Rays whose child-box tests fall inside or near the error margin of the binary
    walk's filtered box test (origins on box planes, rays grazing box corners and
    edges, axis-parallel and near-axis-parallel directions, far origins, extreme
    tmax), mixed closest / any-hit."""
    rng = np.random.default_rng(seed)
    f = img.nodes().view(np.float32)
    lo = np.concatenate([f[:, [4, 5, 12]], f[:, [8, 9, 14]]])
    hi = np.concatenate([f[:, [6, 7, 13]], f[:, [10, 11, 15]]])
    keep = (hi > lo).any(axis=1)
    lo, hi = lo[keep], hi[keep]
    amin, amax = np.asarray(aabb[:3], np.float64), np.asarray(aabb[3:], np.float64)
    span = amax - amin

    def unit(k):
        d = rng.normal(size=(k, 3))
        return d / np.linalg.norm(d, axis=1, keepdims=True)

    def boxes(k):
        i = rng.integers(0, len(lo), k)
        return lo[i].astype(np.float64), hi[i].astype(np.float64)

    k = n_per_kind
    out = []
    # origin on a plane of a child box, inside the box on the other axes
    bl, bh = boxes(k)
    o = bl + rng.uniform(size=(k, 3)) * (bh - bl)
    ax = rng.integers(0, 3, k)
    side = rng.integers(0, 2, k).astype(bool)
    o[np.arange(k), ax] = np.where(side, bh[np.arange(k), ax], bl[np.arange(k), ax])
    out.append((o, unit(k)))
    # aimed at a box corner or at a point on a box edge
    bl, bh = boxes(k)
    corner = np.where(rng.integers(0, 2, (k, 3)).astype(bool), bh, bl)
    free = rng.integers(0, 4, k)
    for a in range(3):
        m = free == a
        corner[m, a] = bl[m, a] + rng.uniform(size=m.sum()) * (bh[m, a] - bl[m, a])
    o = amin - 0.2 * span + rng.uniform(size=(k, 3)) * 1.4 * span
    out.append((o, corner - o))
    # axis-parallel (one or two zero components, signed zeros) from box planes
    bl, bh = boxes(k)
    o = bl + rng.uniform(size=(k, 3)) * (bh - bl)
    o[:, 0] = np.where(rng.integers(0, 2, k).astype(bool), bl[:, 0], o[:, 0])
    d = unit(k)
    z = rng.integers(0, 3, (k, 3)) == 0
    z[z.all(axis=1), 0] = False
    d[z] = 0.0
    d[z & (rng.integers(0, 2, (k, 3)) == 0)] = -0.0
    out.append((o, d))
    # tiny (subnormal-range and 1e-20) components
    o = amin + rng.uniform(size=(k, 3)) * span
    d = unit(k)
    t = rng.integers(0, 3, (k, 3)) == 0
    d[t] = np.choose(rng.integers(0, 3, t.sum()), [1e-35, -1e-20, 1e-42])
    out.append((o, d))
    # far origins looking back at the scene
    c = 0.5 * (amin + amax)
    o = c + unit(k) * rng.choice([1e3, 1e5, 1e7], size=(k, 1))
    out.append((o, c + (rng.uniform(size=(k, 3)) - 0.5) * span - o))
    rays = []
    for o, d in out:
        r = np.zeros((len(o), 8), np.float32)
        r[:, 0:3] = o
        r[:, 4:7] = d
        r[:, 3] = rng.choice(np.array([100.0, 1e-3, 7.5, 1e31, np.inf], np.float32), size=len(o))
        r.view(np.uint32)[:, 7] = rng.integers(0, 2, len(o)).astype(np.uint32)
        rays.append(r)
    return np.concatenate(rays)


@pytest.mark.parametrize("which", ["room", "heightfield"])
def test_box_filter_margin_cases(ctx, native, oracle_mod, which):
    """The binary walk's filtered child-box test decides only outside its error
    margin and takes the reference's divisions inside it; rays built to sit on
    that boundary must give the oracle's records bit for bit in both forms."""
    from tim_raytracing_b200 import scenes
    if which == "room":
        s, img = load_room()
    else:
        s = scenes.heightfield_scene(5, grid=64, n_spheres=12)
        img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rays = _margin_rays(img, img.aabb, 11, 6000)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
        assert (oh[:, 3] != np.float32(100.0).view(np.uint32)).sum() > 1000   # plenty of hits
        for form in (0, native.TRACE_WIDE):
            hit, nid, bary, _ = ctx.trace(sid, rays, native.MODE_PER_RAY | form)
            assert np.array_equal(hit, oh), form
            assert np.array_equal(nid, on), form
            assert np.array_equal(bary.view(np.uint32), ob.view(np.uint32)), form
    finally:
        ctx.free_scene(sid)


def test_fp64_verification(ctx, native, oracle_mod):
    """tim_rt_verify_hits re-intersects every reported closest hit in FP64: all
    hits are counted, and the FP32 t of the reference arithmetic is close to FP64."""
    import torch
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=6, grid=32, n_spheres=5)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        n = 50000
        rays = scenes.random_rays(61, n, any_fraction=0.0)
        rays[:, 0:3] = np.random.default_rng(62).uniform((0, 0, 0.5), (20, 20, 5), size=(n, 3))
        d_rays = torch.from_numpy(rays).cuda()
        d_hit = torch.empty((n, 4), dtype=torch.int32, device="cuda")
        ctx.trace_dev(sid, d_rays, n, native.MODE_CLOSEST | native.TRACE_WIDE, d_hit)
        torch.cuda.synchronize()
        r = ctx.verify_hits(sid, d_rays, n, d_hit)
        h = d_hit.cpu().numpy().view(np.uint32)
        n_hit = int((h[:, 3].view(np.float32) != rays[:, 3]).sum())
        assert r["hits_checked"] == n_hit and r["misses"] == n - n_hit and n_hit > 10000
        assert r["fp64_misses"] <= n_hit * 1e-3
        assert 0 < r["max_rel_t_err"] < 1e-3 and r["max_abs_t_err"] < 1e-2
    finally:
        ctx.free_scene(sid)


def test_wide_near_ties_match_oracle(ctx, native, oracle_mod):
    """Scenes built to be mostly near-ties: the 8-wide walk must still return the
    binary walk's (the reference's order-dependent) answer on every ray."""
    from tim_raytracing_b200 import scenes
    s = near_tie_scene(31, 4000)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rays = scenes.random_rays(32, 50000, any_fraction=0.3)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
        assert (oh[:, 3].view(np.float32) < 100).sum() > 3000   # plenty of hits
        hw, nw, bw, _ = ctx.trace(sid, rays, native.MODE_PER_RAY | native.TRACE_WIDE)
        assert np.array_equal(hw, oh)
        assert np.array_equal(nw, on)
        assert np.array_equal(bw.view(np.uint32), ob.view(np.uint32))
    finally:
        ctx.free_scene(sid)


@pytest.mark.parametrize("want_nid", [True, False])
def test_wide_duplicated_triangles_match_oracle(ctx, native, oracle_mod, want_nid):
    """The reference builder copies a triangle into every leaf it straddles. Without
    a leaf-id output the 8-wide walk takes a second reference to its nearest
    triangle as the same hit (only the leaf id could differ); with one it keeps
    deciding such rays by the binary walk. Records, barycentrics and (when asked
    for) leaf ids equal the oracle on a reference-built scene full of copies."""
    from tim_raytracing_b200 import scenes
    if not oracle_mod.have_refbuild():
        pytest.skip("the reference builder is not built (oracle/_ref)")
    s = scenes.random_triangles(41, 20000)
    img = oracle_mod.ref_build(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rays = scenes.random_rays(42, 60000, any_fraction=0.25)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
        assert (oh[:, 3].view(np.float32) < 100).sum() > 5000
        hw, nw, bw, _ = ctx.trace(sid, rays, native.MODE_PER_RAY | native.TRACE_WIDE, want_nid=want_nid)
        assert np.array_equal(hw, oh)
        assert np.array_equal(bw.view(np.uint32), ob.view(np.uint32))
        if want_nid:
            assert np.array_equal(nw, on)
    finally:
        ctx.free_scene(sid)


@pytest.mark.parametrize("grid,spheres", [(64, 12), (128, 53)])
def test_wide_form_matches_plain(ctx, native, grid, spheres):
    """8-wide quantised BVH: hit records, leaf ids and barycentrics identical to the
    binary walk's for every ray, near-ties included; any-hit results identical. The
    larger scene (61K binary nodes) is collapsed on worker threads, subtree by subtree."""
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=4, grid=grid, n_spheres=spheres)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rng = np.random.default_rng(8)
        n = 100000
        rays = np.zeros((n, 8), np.float32)
        rays[:, 0:3] = rng.uniform((0, 0, 0.5), (20, 20, 6), size=(n, 3))
        d = rng.normal(size=(n, 3))
        rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
        rays[:, 3] = 100.0
        hp, np_, bp, _ = ctx.trace(sid, rays, native.MODE_CLOSEST)
        hw, nw, bw, _ = ctx.trace(sid, rays, native.MODE_CLOSEST | native.TRACE_WIDE)
        assert np.array_equal(hp, hw)
        assert np.array_equal(np_, nw)
        assert np.array_equal(bp.view(np.uint32), bw.view(np.uint32))
        ap, _, _, _ = ctx.trace(sid, rays, native.MODE_ANY)
        aw, _, _, _ = ctx.trace(sid, rays, native.MODE_ANY | native.TRACE_WIDE)
        assert np.array_equal(ap, aw)
    finally:
        ctx.free_scene(sid)


def test_wide_camera_room_matches_golden(ctx, native, room):
    from tim_raytracing_b200 import scenes
    s, img, sid = room
    g = load_room_golden()
    pd = g["pass_data"].view(scenes.PASS_DATA_DTYPE)
    out, _, _ = ctx.trace_camera(sid, pd, flags=native.CAM_PROB_MASK | native.CAM_WIDE)
    assert np.array_equal(out, g["camera"])


def test_trace_dev_with_torch_buffers(ctx, native, room):
    import torch
    s, img, sid = room
    g = load_room_golden()
    d_rays = torch.from_numpy(g["rays"]).cuda()
    n = d_rays.shape[0]
    d_hit = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    d_nid = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    ctx.trace_dev(sid, d_rays, n, native.MODE_CLOSEST, d_hit, d_nid, None, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_hit.cpu().numpy().view(np.uint32), g["hit_closest"])
    assert np.array_equal(d_nid.cpu().numpy().view(np.uint32), g["nid_closest"])


def test_errors(ctx, native, room):
    from tim_raytracing_b200 import scenes
    s, img, sid = room
    with pytest.raises(native.TimRtError) as e:
        ctx.trace(12345, np.zeros((4, 8), np.float32))
    assert e.value.code == native.ENOTFOUND
    bad = native.BvhImage(img.data.copy(), img.ranges.copy(), img.pc, img.aabb)
    bad.ranges[native.RANGE_NODE][0] += 4          # misaligned node range
    with pytest.raises(native.TimRtError) as e:
        ctx.upload(bad, s)
    assert e.value.code == native.EINVAL
    small = native.Context(0, mem_budget_bytes=64 * 1024)   # room for the context, not the scene
    try:
        with pytest.raises(native.TimRtError) as e:
            small.upload(img, s)
        assert e.value.code == native.ENOMEM
    finally:
        small.close()


@pytest.mark.parametrize("wide", [False, True])
def test_camera_leaf_lights_and_counts(ctx, native, oracle_mod, wide):
    """Leaf light lists (no tile culling) on a scene where about half the hit
    pixels are shadowed, against the oracle, and the counting variant: the same
    records, and work counts whose secondary rays are the traced rays less the
    primary ones."""
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=4, grid=40, n_spheres=12, n_lights=24, light_radius=6.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=wide)
    try:
        W, H = 136, 90
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        flags = native.CAM_PROB_MASK | native.CAM_BOUNCE
        o_out, o_bounce, o_counts = oracle_mod.camera(sc, pd, flags=flags, seed=3)
        masked = (o_out[:, 4] != 0).mean()
        assert 0.05 < masked < 0.95            # both outcomes occur
        form = native.CAM_WIDE if wide else 0
        for extra in (0, native.CAM_COUNT):
            out, bounce, st = ctx.trace_camera(sid, pd, flags=flags | form | extra, seed=3)
            assert np.array_equal(out, o_out)
            assert np.array_equal(bounce, o_bounce)
            assert st.rays == int(o_counts.sum())
            if extra & native.CAM_COUNT:
                assert st.secondary_rays_counted == st.rays - st.primary_rays
    finally:
        ctx.free_scene(sid)


def test_camera_pipelined_bands_without_secondary_rays(ctx, native, oracle_mod):
    """TIM_RT_CAM_PIPELINED on a frame whose hits fall in a few of its 8 bands: the
    bands without secondary rays are flagged final before the secondary trace and
    copied at once, the others as they complete; records equal the oracle's."""
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(31, 300)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s)
    try:
        W, H = 96, 512
        lo, hi = img.aabb[:3], img.aabb[3:]
        c, e = (lo + hi) / 2, hi - lo
        pd = scenes.pass_data(s, W, H, cam_pos=c + np.array([0.0, -4.0 * e[1], 0.0]), cam_target=c, aabb=(lo, hi))
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        o_out, o_bounce, o_counts = oracle_mod.camera(sc, pd, flags=native.CAM_BOUNCE, seed=1)
        hit_rows = (o_out[:, 3].view(np.float32).reshape(H, W) < 100.0).sum(1)
        band_hits = hit_rows.reshape(8, 64).sum(1)
        assert (band_hits == 0).sum() >= 3 and (band_hits > 0).sum() >= 2
        for form in (0, native.CAM_WIDE):
            if form:
                ctx.free_scene(sid)
                sid = ctx.upload(img, s, quant8=True)
            for _ in range(2):
                out, bounce, st = ctx.trace_camera(sid, pd, flags=native.CAM_BOUNCE | native.CAM_PIPELINED | form,
                                                   seed=1)
                assert np.array_equal(out, o_out)
                assert np.array_equal(bounce, o_bounce)
                assert st.rays == int(o_counts.sum())
    finally:
        ctx.free_scene(sid)


@pytest.mark.gpu
def test_camera_device_cull(ctx, native, oracle_mod):
    """TIM_RT_CAM_DEVICE_CULL: tim_rt_trace_camera culls the tile lights on the device
    itself (no host tile lists) and gives the oracle's records with the oracle's
    culling, pipelined or not; it needs TIM_RT_CAM_TILE_LIGHTS and is refused by the
    device-pointer forms."""
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=12, grid=32, n_spheres=6, n_lights=16, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        W, H = 184, 136
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        tx, ty = (W + 15) // 16, (H + 15) // 16
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        counts, lists = oracle_mod.cull_lights(sc, pd, tx, ty)
        flags = native.CAM_TILE_LIGHTS | native.CAM_BOUNCE
        o_out, o_bounce, o_counts = oracle_mod.camera(sc, pd, flags=flags, seed=3, tile_counts=counts,
                                                      tile_lists=lists)
        assert int(counts.max()) > 0
        for form in (0, native.CAM_WIDE | native.CAM_PRIMARY_BINARY):
            for extra in (0, native.CAM_PIPELINED):
                out, bounce, st = ctx.trace_camera(sid, pd, flags=flags | form | extra | native.CAM_DEVICE_CULL,
                                                   seed=3)
                assert np.array_equal(out, o_out)
                assert np.array_equal(bounce, o_bounce)
                assert st.rays == int(o_counts.sum())
        with pytest.raises(native.TimRtError) as e:
            ctx.trace_camera(sid, pd, flags=native.CAM_BOUNCE | native.CAM_DEVICE_CULL, seed=3)
        assert e.value.code == native.EINVAL
        import torch
        d_out = torch.zeros((W * H, 8), dtype=torch.int32, device="cuda")
        d_b = torch.zeros((W * H, 4), dtype=torch.int32, device="cuda")
        d_c = torch.zeros(tx * ty, dtype=torch.int32, device="cuda")
        d_l = torch.zeros(tx * ty * 16, dtype=torch.int32, device="cuda")
        with pytest.raises(native.TimRtError) as e:
            ctx.trace_camera_dev(sid, pd, flags | native.CAM_DEVICE_CULL, 3, d_c, d_l, d_out, d_b)
        assert e.value.code == native.EINVAL
    finally:
        ctx.free_scene(sid)
