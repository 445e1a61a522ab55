"""The allocation-free camera trace (tim_rt_trace_camera_noalloc).

It exists for callers that may not allocate device memory while tracing -- an
engine that owns a fixed device budget, a plugin host that forbids allocation
from its callbacks, or a frame loop that cannot absorb cudaMalloc's
synchronisation. Here the test plays that caller: it owns the device copies of
the BVH buffer, positions, tile lists and outputs (torch tensors), calls the
entry point through the C ABI twice in a row, and checks both calls against the
context-based tim_rt_trace_camera on the same inputs (integer records:
bit-identical). Frames include one whose sides are not multiples of the 8x4
tile (50x37), so partial tiles meet the fixed-stride scratch layout, and each
case is also captured in a CUDA graph on a side stream and replayed. This file is
collected last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from helpers import load_room

pytestmark = pytest.mark.gpu


def _device(t):
    import torch
    return torch.from_numpy(np.ascontiguousarray(t)).cuda()


def test_noalloc_camera_matches_context_path(native):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tim_raytracing_b200 import scenes
    L = native.lib()
    cases = []
    s, img = load_room()
    cases.append((s, img, scenes.pass_data(s, 64, 64, lpf_res=(8, 8, 8), aabb=(img.aabb[:3], img.aabb[3:])),
                  native.CAM_PROB_MASK, 0))
    h = scenes.heightfield_scene(seed=13, grid=24, n_spheres=5, n_lights=16, light_radius=5.0)
    himg = native.build_bvh(h)
    cases.append((h, himg, scenes.pass_data(h, 48, 40, aabb=(himg.aabb[:3], himg.aabb[3:])),
                  native.CAM_TILE_LIGHTS | native.CAM_BOUNCE | native.CAM_PROB_MASK, 7))
    # 50 x 37 = 1850 pixels: partial 8x4 tiles on the right and bottom edges
    cases.append((h, himg, scenes.pass_data(h, 50, 37, aabb=(himg.aabb[:3], himg.aabb[3:])),
                  native.CAM_TILE_LIGHTS | native.CAM_BOUNCE, 3))
    with native.Context(0) as ctx:
        for scene, im, pd, flags, seed in cases:
            depth = native.validate(im, scene.num_vertex)
            sid = ctx.upload(im, scene)
            W, H = (int(x) for x in pd["frameSize"].reshape(-1))
            tx, ty = (W + 15) // 16, (H + 15) // 16
            counts, lists = ctx.cull_lights(sid, pd, tx, ty)
            want, want_b, _ = ctx.trace_camera(sid, pd, flags=flags, seed=seed, tile_counts=counts, tile_lists=lists)
            d_bvh = _device(im.data)
            d_pos = _device(scene.positions.astype(np.float32))
            d_counts = _device(counts)
            d_lists = _device(lists)
            ranges = np.ascontiguousarray(im.ranges, np.uint32)
            pc = native.PushConstants(*[int(x) for x in im.pc])
            pdc = np.ascontiguousarray(pd)
            for call in range(2):
                d_out = torch.full((W * H * 8,), -1, dtype=torch.int32, device="cuda")
                d_bounce = torch.full((W * H * 4,), -1, dtype=torch.int32, device="cuda")
                rc = L.tim_rt_trace_camera_noalloc(d_bvh.data_ptr(), ranges.ctypes.data, ctypes.byref(pc),
                                                   d_pos.data_ptr(), scene.num_vertex, depth, pdc.ctypes.data, flags,
                                                   seed, d_counts.data_ptr(), d_lists.data_ptr(), d_out.data_ptr(),
                                                   d_bounce.data_ptr(), None)
                assert rc == native.OK, L.tim_rt_last_error().decode()
                torch.cuda.synchronize()
                got = d_out.cpu().numpy().view(np.uint32).reshape(-1, 8)
                assert np.array_equal(got, want), f"call {call}: {np.sum(np.any(got != want, axis=1))} pixels differ"
                if flags & native.CAM_BOUNCE:
                    gb = d_bounce.cpu().numpy().view(np.uint32).reshape(-1, 4)
                    assert np.array_equal(gb, want_b), f"call {call}: bounce records differ"
            # the same call captured in a CUDA graph on a side stream (after the warm
            # calls above), then replayed twice
            side = torch.cuda.Stream()
            g_out = torch.full((W * H * 8,), -1, dtype=torch.int32, device="cuda")
            g_bounce = torch.full((W * H * 4,), -1, dtype=torch.int32, device="cuda")
            graph = torch.cuda.CUDAGraph()
            torch.cuda.synchronize()
            with torch.cuda.graph(graph, stream=side):
                rc = L.tim_rt_trace_camera_noalloc(d_bvh.data_ptr(), ranges.ctypes.data, ctypes.byref(pc),
                                                   d_pos.data_ptr(), scene.num_vertex, depth, pdc.ctypes.data, flags,
                                                   seed, d_counts.data_ptr(), d_lists.data_ptr(), g_out.data_ptr(),
                                                   g_bounce.data_ptr(), ctypes.c_void_p(side.cuda_stream))
            assert rc == native.OK, L.tim_rt_last_error().decode()
            for rep in range(2):
                g_out.fill_(-1)
                g_bounce.fill_(-1)
                graph.replay()
                torch.cuda.synchronize()
                got = g_out.cpu().numpy().view(np.uint32).reshape(-1, 8)
                assert np.array_equal(got, want), f"replay {rep}: {np.sum(np.any(got != want, axis=1))} pixels differ"
                if flags & native.CAM_BOUNCE:
                    gb = g_bounce.cpu().numpy().view(np.uint32).reshape(-1, 4)
                    assert np.array_equal(gb, want_b), f"replay {rep}: bounce records differ"
            del graph
            ctx.free_scene(sid)


def test_noalloc_rejects_frames_above_the_limit(native):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tim_raytracing_b200 import scenes
    L = native.lib()
    s, img = load_room()
    pd = np.ascontiguousarray(scenes.pass_data(s, 128, 64))    # 8192 pixels > 4096
    d_bvh = _device(img.data)
    d_pos = _device(s.positions.astype(np.float32))
    d_out = torch.empty(128 * 64 * 8, dtype=torch.int32, device="cuda")
    ranges = np.ascontiguousarray(img.ranges, np.uint32)
    pc = native.PushConstants(*[int(x) for x in img.pc])
    rc = L.tim_rt_trace_camera_noalloc(d_bvh.data_ptr(), ranges.ctypes.data, ctypes.byref(pc), d_pos.data_ptr(),
                                       s.num_vertex, 0, pd.ctypes.data, 0, 0, None, None, d_out.data_ptr(), None, None)
    assert rc == native.EINVAL
    assert b"exceeds the allocation-free limit" in L.tim_rt_last_error()
    # a materials range that is not 4-byte aligned is refused before any launch
    bad = ranges.copy()
    bad[3][0] += 2
    pd_ok = np.ascontiguousarray(scenes.pass_data(s, 32, 32))
    rc = L.tim_rt_trace_camera_noalloc(d_bvh.data_ptr(), bad.ctypes.data, ctypes.byref(pc), d_pos.data_ptr(),
                                       s.num_vertex, 0, pd_ok.ctypes.data, 0, 0, None, None, d_out.data_ptr(), None,
                                       None)
    assert rc == native.EINVAL
    assert b"misaligned" in L.tim_rt_last_error()
