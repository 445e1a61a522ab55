"""GPU parity of the two-level any-hit walk (TIM_RT_TRACE_TLAS): the
reference's USE_TRAVERSE_TLAS shadow traversal (traverseTlasFast +
tlas_collide_fast, src/Shaders/bvh/bvhCollision.glsl:321-348) on the committed
two-level fixture, against the occlusion results its own shader code gave on
the host (tests/golden/tlas_golden.npz) and the oracle; through the host and the
device-pointer entry points and the counting kernel; and the refusals."""
import numpy as np
import pytest

from helpers import GOLDEN

pytestmark = pytest.mark.gpu


def _fixture(native):
    z = np.load(GOLDEN / "tlas_golden.npz")
    img = native.BvhImage(z["data"], z["ranges"], tuple(int(x) for x in z["pc"]), z["aabb"])
    return z, img


def test_two_level_any_hit_matches_reference_shader(ctx, native, oracle_mod):
    import torch
    from tim_raytracing_b200 import scenes
    z, img = _fixture(native)
    s = scenes.instanced_clusters(3, 12, 400)
    sid = ctx.upload(img, s)
    try:
        rays = z["rays"]
        mode = native.MODE_ANY | native.TRACE_TLAS
        hit, _, _, st = ctx.trace(sid, rays, mode)
        assert np.array_equal(hit, z["glsl_hit"])
        hit_c, _, _, stc = ctx.trace(sid, rays, mode | native.TRACE_COUNT)
        assert np.array_equal(hit_c, z["glsl_hit"])
        assert stc.node_visits > 0 and stc.leaf_visits > 0
        d_rays = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
        d_hit = torch.full((len(rays), 4), -1, dtype=torch.int32, device="cuda")
        ctx.trace_dev(sid, d_rays, len(rays), mode, d_hit)
        torch.cuda.synchronize()
        assert np.array_equal(d_hit.cpu().numpy().view(np.uint32), z["glsl_hit"])
        # more rays on the same image, checked against the oracle
        more = scenes.occlusion_rays(77, 50000, targets=s.meta["centres"])
        more[:64, 4:7] = 0.0
        more[:64, 4 + (np.arange(64) % 3)] = -1.0
        got, _, _, _ = ctx.trace(sid, more, mode)
        sc = oracle_mod.Scene(img, s.positions, s.normals)
        want, _, _, _ = oracle_mod.trace(sc, more, oracle_mod.ORC_MODE_ANY | oracle_mod.ORC_MODE_TLAS)
        assert np.array_equal(got, want)
        # the one-level walk of the same image (BLAS boxes only) differs: the flag matters
        one, _, _, _ = ctx.trace(sid, rays, native.MODE_ANY)
        assert not np.array_equal(one, hit)
        # closest-hit two-level rays: the reference's variant does not compile
        with pytest.raises(native.TimRtError) as e:
            ctx.trace(sid, rays[:10], native.MODE_CLOSEST | native.TRACE_TLAS)
        assert e.value.code == native.EUNSUPPORTED
    finally:
        ctx.free_scene(sid)


def test_two_level_walk_refuses_a_leaf_blas_root(ctx, native):
    from tim_raytracing_b200 import scenes
    z, img = _fixture(native)
    data = img.data.copy()
    blas = data[img.ranges[native.RANGE_BLAS][0]:].view(np.uint32)
    nodes = data[img.ranges[native.RANGE_NODE][0]:].view(np.uint32)[: 16 * img.pc[4]].reshape(-1, 16)
    leaf_ids = np.nonzero((nodes[:, 2] & 0x3FFFFFFF) == 0x3FFFFFFF)[0]
    blas[7] = leaf_ids[-1]            # instance 0's root now names a leaf node
    bad = native.BvhImage(data, img.ranges.copy(), img.pc, img.aabb)
    s = scenes.instanced_clusters(3, 12, 400)
    sid = ctx.upload(bad, s)
    try:
        with pytest.raises(native.TimRtError) as e:
            ctx.trace(sid, z["rays"][:10], native.MODE_ANY | native.TRACE_TLAS)
        assert e.value.code == native.EINVAL
    finally:
        ctx.free_scene(sid)
