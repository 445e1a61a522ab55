"""Two-level (TLAS/BLAS) scenes on the host: the image tim_rt_build_bvh_tlas
writes, and the oracle's any-hit walk of USE_TRAVERSE_TLAS scenes
(traverseTlasFast + tlas_collide_fast, src/Shaders/bvh/bvhCollision.glsl:321-348)
pinned to the reference's own shader code compiled for the host, directly where
oracle/_ref/librefglsl.so is built and through the committed fixture
(tests/golden/tlas_golden.npz, made by tests/golden/make_golden.py) everywhere."""
import numpy as np
import pytest

from helpers import GOLDEN


def _fixture(native):
    z = np.load(GOLDEN / "tlas_golden.npz")
    img = native.BvhImage(z["data"], z["ranges"], tuple(int(x) for x in z["pc"]), z["aabb"])
    return z, img


def test_two_level_image_layout(native):
    from tim_raytracing_b200 import scenes
    s = scenes.instanced_clusters(3, 12, 400)
    img = native.build_bvh_tlas(s)
    assert np.array_equal(img.data, native.build_bvh_tlas(s).data)      # deterministic
    assert img.pc[1] == 12 and img.pc[0] == s.num_tris
    native.validate(img, s.num_vertex)
    z, fx = _fixture(native)
    assert np.array_equal(img.data, fx.data)                              # the fixture is this image
    nodes = img.data[img.ranges[native.RANGE_NODE][0]:].view(np.uint32)[: 16 * img.pc[4]].reshape(-1, 16)
    blas = img.data[img.ranges[native.RANGE_BLAS][0]:].view(np.uint32)[: 8 * 12].reshape(12, 8)
    roots = blas[:, 7]
    assert np.all(roots < img.pc[4])
    assert np.all((nodes[roots, 2] & 0x3FFFFFFF) != 0x3FFFFFFF)          # every BLAS root is an inner node
    assert np.all(np.diff(roots.astype(np.int64)) > 0)                    # BLAS node ranges in instance order
    # top-level leaves hold instance ids and no triangles
    leaf = img.data[img.ranges[native.RANGE_LEAF][0]:].view(np.uint32)
    top = roots.min()
    for i in range(top):
        off = nodes[i, 3]
        if (nodes[i, 2] & 0x3FFFFFFF) == 0x3FFFFFFF and off != 0xFFFFFFFF:
            hdr = leaf[off]
            assert hdr & 0xFFF == 0 and 1 <= (hdr >> 12) & 0xFF <= 2
            assert np.all(leaf[off + 1: off + 1 + ((hdr >> 12) & 0xFF)] < 12)


def test_two_level_builder_refuses_bad_instances(native):
    from tim_raytracing_b200 import scenes
    s = scenes.instanced_clusters(4, 3, 50)
    s.chunks[1, 3] = 1          # an instance of one triangle cannot have an inner root
    s.local_idx = s.local_idx   # (the chunk table alone changes)
    with pytest.raises(native.TimRtError) as e:
        native.build_bvh_tlas(s)
    assert e.value.code == native.EINVAL


def test_oracle_matches_the_fixture(native, oracle_mod):
    from tim_raytracing_b200 import scenes
    z, img = _fixture(native)
    s = scenes.instanced_clusters(3, 12, 400)
    sc = oracle_mod.Scene(img, s.positions, s.normals)
    hit, _, _, _ = oracle_mod.trace(sc, z["rays"], oracle_mod.ORC_MODE_ANY | oracle_mod.ORC_MODE_TLAS)
    assert np.array_equal(hit, z["glsl_hit"])     # the reference's own shader, recorded
    assert np.array_equal(hit, z["hit"])
    assert 0.1 < hit[:, 0].mean() < 0.5


def test_oracle_matches_reference_shader(native, oracle_mod):
    from oracle import refglsl
    if not refglsl.available():
        pytest.skip("oracle/_ref/librefglsl.so not built (reference tree absent)")
    from tim_raytracing_b200 import scenes
    for seed, (nc, nt) in ((11, (6, 300)), (12, (20, 150))):
        s = scenes.instanced_clusters(seed, nc, nt)
        img = native.build_bvh_tlas(s, tlas_max_leaf=1 + seed % 2)
        rays = scenes.occlusion_rays(seed, 6000, targets=s.meta["centres"])
        rays[:32, 4:7] = 0.0                                   # axis-aligned rays: zero direction components
        rays[:32, 4 + (np.arange(32) % 3)] = 1.0
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        hit, _, _, _ = oracle_mod.trace(sc, rays, oracle_mod.ORC_MODE_ANY | oracle_mod.ORC_MODE_TLAS)
        g = refglsl.trace_tlas(refglsl.Scene(img, s.positions, s.normals), rays)
        assert np.array_equal(hit, g)
