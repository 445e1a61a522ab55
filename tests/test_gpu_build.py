"""The GPU BVH builder (tim_rt_build_bvh_gpu): its image passes the reference-layout
validation, holds every triangle exactly once in leaves of at most max_leaf_size,
stores the light lists of the sphere-vs-leaf-box rule, is the same byte for byte
on every build, and traces (both forms) exactly like the oracle on that image."""
import numpy as np
import pytest

from helpers import near_tie_scene

pytestmark = pytest.mark.gpu


def _leaves(img):
    """(node id, leaf offset, parent id, is right child) of every leaf."""
    nodes = img.nodes()
    out = []
    for i in range(img.num_nodes):
        c = nodes[i, 2]
        if c == 0x3FFFFFFF:
            continue
        left = int(c & 0x3FFFFFFF)
        for k, leaf_bit in ((0, 0x80000000), (1, 0x40000000)):
            if c & leaf_bit:
                out.append((left + k, int(nodes[left + k, 3]), i, k))
    return out


def _check_image(native, s, img, max_leaf=4):
    depth = native.validate(img, s.num_vertex)
    assert depth <= 30
    words = img.leaf_words()
    nodes = img.nodes()
    boxes = nodes[:, 4:16].view(np.float32)
    lights = np.frombuffer(s.packed_lights_bytes(), np.float32).reshape(-1, 14) if len(s.lights) else np.zeros((0, 14), np.float32)
    seen = []
    for nid, off, parent, k in _leaves(img):
        hdr = int(words[off])
        cnt, nl = hdr & 0xFFF, hdr >> 28
        assert 1 <= cnt <= max_leaf
        seen.append(words[off + 1: off + 1 + 3 * cnt].reshape(-1, 3))
        # light list: sphere vs the leaf's widened box as its parent stores it
        b = boxes[parent]
        lo = np.array([b[0], b[1], b[8]] if k == 0 else [b[4], b[5], b[10]], np.float32)
        hi = np.array([b[2], b[3], b[9]] if k == 0 else [b[6], b[7], b[11]], np.float32)
        want = []
        for l in range(len(lights)):
            if len(want) == 15:
                break
            f = lights[l, 1:5]
            d2 = np.float32(0)
            for a in range(3):
                c = np.minimum(np.maximum(f[a], lo[a]), hi[a])
                d2 = np.float32(d2 + (c - f[a]) * (c - f[a]))
            if d2 < f[3] * f[3]:
                want.append(l)
        assert list(words[off + 1 + 3 * cnt: off + 1 + 3 * cnt + nl]) == want
    got = np.concatenate(seen)
    ref = s.tri_records()
    key = lambda r: np.lexsort(r.T[::-1])
    assert np.array_equal(got[key(got)], ref[key(ref)])


@pytest.mark.parametrize("kind", ["heightfield", "random", "near_ties", "tiny"])
def test_gpu_builder(ctx, native, oracle_mod, kind):
    from tim_raytracing_b200 import scenes
    if kind == "heightfield":
        s = scenes.heightfield_scene(seed=12, grid=48, n_spheres=8, n_lights=16, light_radius=4.0)
    elif kind == "random":
        s = scenes.random_triangles(21, 40000)
    elif kind == "near_ties":
        s = near_tie_scene(5, 3000)
    else:
        s = scenes.random_triangles(22, 5)
    img = native.build_bvh(s, ctx=ctx)
    _check_image(native, s, img)
    again = native.build_bvh(s, ctx=ctx)
    assert np.array_equal(img.data, again.data) and np.array_equal(img.ranges, again.ranges)
    sid = ctx.upload(img, s, quant8=True)
    try:
        rays = scenes.random_rays(40, 30000, any_fraction=0.4)
        lo, hi = img.aabb[:3], img.aabb[3:]
        rays[:, 0:3] = lo + (hi - lo) * rays[:, 0:3]
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, ob, _ = oracle_mod.trace(sc, rays, 2)
        for mode in (2, 2 | native.TRACE_WIDE):
            h, nid, b, _ = ctx.trace(sid, rays, mode)
            assert np.array_equal(h, oh) and np.array_equal(nid, on)
            assert np.array_equal(b.view(np.uint32), ob.view(np.uint32))
    finally:
        ctx.free_scene(sid)


def test_gpu_builder_small_scene_uses_host_builder(ctx, native):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(23, 3)
    img = native.build_bvh(s, ctx=ctx)
    assert img.num_nodes == 1 and np.array_equal(img.data, native.build_bvh(s).data)


def test_gpu_builder_errors(ctx, native):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(24, 100)
    with pytest.raises(native.TimRtError) as e:
        native.build_bvh(s, ctx=ctx, max_depth=40)
    assert e.value.code == native.EINVAL
    with pytest.raises(native.TimRtError) as e:
        native.build_bvh(s, ctx=ctx, max_depth=3)      # 100 triangles need more than 3 levels
    assert e.value.code == native.EUNSUPPORTED
    for kw in ({"traversal_cost": 0.0}, {"intersection_cost": float("nan")}, {"intersection_cost": -1.0}):
        with pytest.raises(native.TimRtError) as e:
            native.build_bvh(s, ctx=ctx, **kw)
        assert e.value.code == native.EINVAL
    bad = scenes.random_triangles(25, 100)
    bad.positions[7, 1] = np.nan
    with pytest.raises(native.TimRtError) as e:
        native.build_bvh(bad, ctx=ctx)
    assert e.value.code == native.EINVAL


def test_gpu_builder_depth_fallback(ctx, native, oracle_mod):
    """A max_depth below the restructured tree's depth but not below the
    Morton-code tree's gives the Morton-code tree (its subtrees of at most
    max_leaf_size triangles as leaves), still a valid image that traces like the
    oracle on it."""
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(21, 40000)
    deep = native.validate(native.build_bvh(s, ctx=ctx, max_depth=32), s.num_vertex)
    img = None
    for md in range(deep - 1, 0, -1):
        try:
            img = native.build_bvh(s, ctx=ctx, max_depth=md)
            break
        except native.TimRtError as e:
            assert e.code == native.EUNSUPPORTED
    assert img is not None, "the Morton-code tree was never shallower than the restructured one"
    assert native.validate(img, s.num_vertex) <= md
    _check_image(native, s, img)
    sid = ctx.upload(img, s)
    try:
        rays = scenes.random_rays(41, 20000, any_fraction=0.4)
        lo, hi = img.aabb[:3], img.aabb[3:]
        rays[:, 0:3] = lo + (hi - lo) * rays[:, 0:3]
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        oh, on, _, _ = oracle_mod.trace(sc, rays, 2)
        h, nid, _, _ = ctx.trace(sid, rays, 2)
        assert np.array_equal(h, oh) and np.array_equal(nid, on)
    finally:
        ctx.free_scene(sid)
