"""Product-side builder (tim_rt_build_bvh): emits a valid image in the reference
layout, and the reference traversal over it finds the brute-force closest hits."""
import numpy as np
import pytest

from helpers import brute_closest, tri_positions, OFFSET


def leaves(img):
    nodes = img.nodes()
    leaf = img.leaf_words()
    out = {}
    for i in range(img.num_nodes):
        if (nodes[i, 2] & 0x3FFFFFFF) == 0x3FFFFFFF:
            off = nodes[i, 3]
            if off == 0xFFFFFFFF:
                out[i] = np.zeros((0, 3), np.uint32)
            else:
                n = leaf[off] & 0xFFF
                out[i] = leaf[off + 1:off + 1 + 3 * n].reshape(-1, 3)
    return out


@pytest.mark.parametrize("n", [1, 3, 5, 1000, 20000])
def test_every_triangle_in_exactly_one_leaf(native, n):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(11, n)
    img = native.build_bvh(s)
    depth = native.validate(img, s.num_vertex)
    assert depth <= 30
    recs = np.concatenate(list(leaves(img).values()))
    assert recs.shape[0] == n
    want = s.tri_records()
    key = lambda a: np.sort(a.view(np.dtype((np.void, 12))).ravel())
    assert np.array_equal(key(np.ascontiguousarray(recs)), key(np.ascontiguousarray(want)))


def test_links_and_boxes(native):
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=3, grid=24, n_spheres=4)
    img = native.build_bvh(s)
    nodes = img.nodes()
    f = nodes.view(np.float32)
    lv = leaves(img)
    n = img.num_nodes
    for i in range(n):
        left = nodes[i, 2] & 0x3FFFFFFF
        if left == 0x3FFFFFFF:
            continue
        assert left > i
        for k, c in enumerate((left, left + 1)):
            assert nodes[c, 0] == i                               # parent
            assert (nodes[c, 1] & 0x3FFFFFFF) == (left + 1 - k)    # sibling
            is_leaf = (nodes[c, 2] & 0x3FFFFFFF) == 0x3FFFFFFF
            assert bool(nodes[i, 2] & (0x80000000 if k == 0 else 0x40000000)) == is_leaf
            lo = f[i, [4, 5, 12]] if k == 0 else f[i, [8, 9, 14]]
            hi = f[i, [6, 7, 13]] if k == 0 else f[i, [10, 11, 15]]
            if is_leaf:
                P = tri_positions(s, lv[c]).reshape(-1, 3)
                assert np.all(P >= lo) and np.all(P <= hi)


def test_deterministic(native):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(5, 100000)
    a = native.build_bvh(s)
    b = native.build_bvh(s)
    assert np.array_equal(a.data, b.data)


def test_traversal_over_product_bvh_is_bruteforce_min(native, oracle_mod):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(21, 3000)
    img = native.build_bvh(s)
    rays = scenes.random_rays(4, 2000, any_fraction=0.0)
    sc = oracle_mod.Scene(img, s.positions, s.normals)
    hit, _, _, _ = oracle_mod.trace(sc, rays, 0)
    tmin, arg = brute_closest(s, rays)
    t = hit[:, 3].view(np.float32)
    hits = t < 100
    assert np.array_equal(hits, np.isfinite(tmin))
    assert np.all(np.abs(t[hits] + OFFSET - tmin[hits]) <= 1.1e-5)
    ha, _, _, _ = oracle_mod.trace(sc, rays, 1)
    assert np.array_equal(ha[:, 0] == 1, hits)


def test_malformed_images_are_rejected(native):
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(2, 500)
    img = native.build_bvh(s)
    native.validate(img, s.num_vertex)

    def bad(mutate):
        d = img.data.copy()
        r = img.ranges.copy()
        mutate(d, r)
        with pytest.raises(native.TimRtError) as e:
            native.validate(native.BvhImage(d, r, img.pc, img.aabb), s.num_vertex)
        assert e.value.code == native.EINVAL

    node_off = int(img.ranges[native.RANGE_NODE][0])
    leaf_off = int(img.ranges[native.RANGE_LEAF][0])

    def child_loop(d, r):      # child id pointing back at the root (a cycle)
        w = d[node_off:node_off + 64].view(np.uint32)
        w[2] = (w[2] & 0xC0000000)

    def leaf_past_end(d, r):
        nodes = d[node_off:].view(np.uint32)[:16 * img.num_nodes].reshape(-1, 16)
        i = int(np.nonzero(nodes[:, 3] != 0xFFFFFFFF)[0][0])
        nodes[i, 3] = img.ranges[native.RANGE_LEAF][1] // 4 + 5

    def vertex_oob(d, r):
        lw = d[leaf_off:].view(np.uint32)
        lw[1] = s.num_vertex + 10

    def range_oob(d, r):
        r[native.RANGE_LEAF][1] = len(d)

    for m in (child_loop, leaf_past_end, vertex_oob, range_oob):
        bad(m)


def test_bad_builder_inputs_are_refused(native):
    """tim_rt_build_bvh refuses inputs it cannot build from, with EINVAL and a
    message, instead of building a tree that indexes out of range."""
    import ctypes
    from tim_raytracing_b200 import scenes
    s = scenes.random_triangles(4, 200)
    L = native.lib()
    pos = np.ascontiguousarray(s.positions, np.float32)
    rec = np.ascontiguousarray(s.tri_records())
    mats = s.materials_bytes()
    nmat = len(mats) // 48

    def build(pos, rec, **params):
        p = native.build_params(**params)
        out = ctypes.c_void_p()
        rc = L.tim_rt_build_bvh(pos.ctypes.data, pos.shape[0], rec.ctypes.data, rec.shape[0], mats, nmat, None, 0,
                                ctypes.byref(p), ctypes.byref(out))
        if rc == native.OK:
            L.tim_rt_bvh_blob_free(out)
        return rc, L.tim_rt_last_error().decode()

    assert build(pos, rec)[0] == native.OK
    bad = rec.copy()
    bad[7, 0] = pos.shape[0]                      # vertex offset past the vertex array
    rc, msg = build(pos, bad)
    assert rc == native.EINVAL and "num_vertex" in msg
    nanpos = pos.copy()
    nanpos[5, 1] = np.nan
    rc, msg = build(nanpos, rec)
    assert rc == native.EINVAL and "non-finite" in msg
    for params in ({"max_leaf_size": 0}, {"max_depth": 33}, {"max_depth": 0}):
        rc, msg = build(pos, rec, **params)
        assert rc == native.EINVAL and "max_leaf_size" in msg, params
    rc, msg = build(pos, rec[:0])
    assert rc == native.EINVAL
