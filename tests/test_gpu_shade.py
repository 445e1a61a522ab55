"""GPU parity of the camera pass's lighting step (tim_rt_shade_camera): the RGBA16F
image and the FP32 lit values must equal the oracle's (which equals the
reference's own cameraPass.comp lighting step, tests/test_refglsl.py) bit for bit,
on the reference builder's room buffer with the committed fixture and on a frame
whose light-probe field comes from tim_rt_update_probes."""
import numpy as np
import pytest

from helpers import load_room, load_room_golden

pytestmark = pytest.mark.gpu


def test_room_fixture(ctx, native):
    from tim_raytracing_b200 import scenes
    s, img = load_room()
    g = load_room_golden()
    sid = ctx.upload(img, s)
    try:
        pd = g["pass_data"].view(scenes.PASS_DATA_DTYPE)
        out, _, st = ctx.shade_camera(sid, pd, g["camera"], g["lpf16"])
        assert np.array_equal(out, g["shade16"])
        assert np.array_equal(out, g["glsl_shade16"])
        assert st.kernel_ms > 0
    finally:
        ctx.free_scene(sid)


def test_frame_with_updated_probe_field(ctx, native, oracle_mod):
    import torch
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s = scenes.heightfield_scene(seed=31, grid=24, n_spheres=6, n_lights=12, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        res = (8, 8, 4)
        lo, hi = img.aabb[:3], img.aabb[3:]
        dirs = scenes.octahedral_dirs(8)
        basis = scenes.sh9_basis(dirs)
        desc = native.probe_desc(lo, hi, res, (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), len(dirs), 0.03,
                                 native.PROBE_WIDE | native.PROBE_PRIMARY_BINARY)
        sh16 = np.zeros((7, res[2], res[1], res[0], 4), np.uint16)
        for _ in range(3):                                   # a few updates blend the field in
            ctx.update_probes(sid, desc, dirs, basis, sh16)
        pd = scenes.pass_data(s, 200, 120, lpf_res=res, aabb=(lo, hi))
        cam, _, _ = ctx.trace_camera(sid, pd, native.CAM_PROB_MASK | native.CAM_WIDE | native.CAM_PRIMARY_BINARY)
        sc = O.Scene(img, s.positions, s.normals)
        for flags in (0, native.SHADE_NO_LPF):
            out, f32, _ = ctx.shade_camera(sid, pd, cam, sh16, flags=flags, want_f32=True)
            o16, of32 = O.shade_camera(sc, pd, cam, sh16, no_lpf=bool(flags))
            assert np.array_equal(out, o16), flags
            assert np.array_equal(f32.view(np.uint32), of32.view(np.uint32)), flags
        lit = f32.reshape(-1, 3)
        assert np.isfinite(lit).all() and (out[:, 3] == 0x3C00).sum() == 200 * 119
        # the device entry point on caller-owned buffers and stream
        d_cam = torch.from_numpy(cam.view(np.int32)).cuda()
        d_sh = torch.from_numpy(sh16.view(np.int16)).cuda()
        d_out = torch.zeros((len(out), 4), dtype=torch.int16, device="cuda")
        stream = torch.cuda.Stream()
        pdc = np.ascontiguousarray(pd)
        native._check(native.lib().tim_rt_shade_camera_dev(ctx._c, sid, pdc.ctypes.data, 0, d_cam.data_ptr(),
                                                           d_sh.data_ptr(), d_out.data_ptr(), None,
                                                           stream.cuda_stream))
        stream.synchronize()
        out0, _, _ = ctx.shade_camera(sid, pd, cam, sh16)
        assert np.array_equal(d_out.cpu().numpy().view(np.uint16), out0)
    finally:
        ctx.free_scene(sid)


def test_shade_errors(ctx, native):
    from tim_raytracing_b200 import scenes
    s, img = load_room()
    g = load_room_golden()
    sid = ctx.upload(img, s)
    try:
        pd = g["pass_data"].view(scenes.PASS_DATA_DTYPE).copy()
        with pytest.raises(native.TimRtError) as e:
            ctx.shade_camera(sid, pd, g["camera"], None)              # the probe term needs the field
        assert e.value.code == native.EINVAL
        pd["lpfResolution"][0, 0] = 1
        with pytest.raises(native.TimRtError) as e:
            ctx.shade_camera(sid, pd, g["camera"], g["lpf16"])
        assert e.value.code == native.EINVAL
        out, _, _ = ctx.shade_camera(sid, pd, g["camera"], None, flags=native.SHADE_NO_LPF)
        assert out.shape == (256 * 256, 4)
    finally:
        ctx.free_scene(sid)
