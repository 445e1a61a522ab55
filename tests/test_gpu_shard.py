"""GPU side of splitting a frame across GPUs: tim_rt_trace_camera_rows_dev.

One GPU traces the frame as the contiguous row bands that N ranks would each
trace (tim_raytracing_b200.shard.row_bands, balanced by a previous frame's
per-row cost), each band into the whole frame's arrays; the assembled records
must equal one whole-frame tim_rt_trace_camera_dev call bit for bit, in both
forms, and the whole-frame call must equal the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("parts,wide", [(3, False), (8, True)])
def test_row_bands_assemble_the_frame(ctx, native, oracle_mod, parts, wide):
    import torch
    from tim_raytracing_b200 import scenes, shard
    s = scenes.heightfield_scene(seed=17, grid=32, n_spheres=6, n_lights=16, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        W, H = 200, 150
        pd = scenes.pass_data(s, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
        tx, ty = (W + 15) // 16, (H + 15) // 16
        flags = native.CAM_TILE_LIGHTS | native.CAM_BOUNCE | (native.CAM_WIDE if wide else 0)
        dev = torch.device("cuda", 0)
        d_counts = torch.zeros(tx * ty, dtype=torch.int32, device=dev)
        d_lists = torch.zeros(tx * ty * 16, dtype=torch.int32, device=dev)
        ctx.cull_lights_dev(sid, pd, tx, ty, d_counts, d_lists)
        whole = torch.zeros(W * H * 8, dtype=torch.int32, device=dev)
        whole_b = torch.zeros(W * H * 4, dtype=torch.int32, device=dev)
        n_whole = torch.zeros(1, dtype=torch.int64, device=dev)
        ctx.trace_camera_dev(sid, pd, flags, 5, d_counts, d_lists, whole, whole_b, n_whole)
        torch.cuda.synchronize()
        rec = whole.cpu().numpy().view(np.uint32).reshape(-1, 8)
        bands = shard.row_bands(H, parts, shard.frame_row_weights(rec, W, H, d_counts.cpu().numpy()))
        assert all(b % 4 == 0 for b, _ in bands) and bands[-1][1] == H
        got = torch.full((W * H * 8,), -1, dtype=torch.int32, device=dev)
        got_b = torch.full((W * H * 4,), -1, dtype=torch.int32, device=dev)
        n_bands = torch.zeros(1, dtype=torch.int64, device=dev)
        for b, e in bands:
            if b < e:
                ctx.trace_camera_rows_dev(sid, pd, flags, 5, b, e, d_counts, d_lists, got, got_b, n_bands)
        torch.cuda.synchronize()
        assert torch.equal(got, whole) and torch.equal(got_b, whole_b)
        assert int(n_bands.item()) == int(n_whole.item())
        # the whole frame itself against the oracle
        O = oracle_mod
        sc = O.Scene(img, s.positions, s.normals)
        counts = d_counts.cpu().numpy().view(np.uint32)
        lists = d_lists.cpu().numpy().view(np.uint32).reshape(-1, 16)
        ref, ref_b, _ = O.camera(sc, pd, flags=flags & 7, seed=5, tile_counts=counts, tile_lists=lists)
        assert np.array_equal(rec, ref)
        assert np.array_equal(whole_b.cpu().numpy().view(np.uint32).reshape(-1, 4), ref_b)
        # a band must start on a 4-row tile boundary and lie inside the frame
        for b, e in ((2, 10), (8, 8), (0, H + 4)):
            with pytest.raises(native.TimRtError) as ex:
                ctx.trace_camera_rows_dev(sid, pd, flags, 5, b, e, d_counts, d_lists, got, got_b)
            assert ex.value.code == native.EINVAL
    finally:
        ctx.free_scene(sid)
