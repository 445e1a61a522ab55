"""GPU parity of the light-probe update (tim_rt_update_probes) against the oracle:
trace records and shadow masks, per-ray lit values, SH9 (FP32 and the FP16
images) and octahedral texels are all computed in the oracle's operation order,
so they must be bit-identical."""
import numpy as np
import pytest
from helpers import probe_coord, sh16_to_prev27

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wide", [0, 1, 2])
def test_probe_update_matches_oracle(ctx, native, oracle_mod, wide):
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s = scenes.heightfield_scene(seed=21, grid=24, n_spheres=5, n_lights=16, light_radius=5.0)
    img = native.build_bvh(s)
    sid = ctx.upload(img, s, quant8=True)
    try:
        res = (8, 8, 4)
        total = res[0] * res[1] * res[2]
        dirs = scenes.octahedral_dirs(16)
        basis = scenes.sh9_basis(dirs)
        lo, hi = img.aabb[:3], img.aabb[3:]
        sun = np.array([-0.4, 0.3, -1.0], np.float32)      # not normalised, as the reference passes it
        sunc = np.array([1.0, 0.95, 0.9], np.float32)
        flags = native.PROBE_OCTA | [0, native.PROBE_WIDE, native.PROBE_WIDE | native.PROBE_PRIMARY_BINARY][wide]
        desc = native.probe_desc(lo, hi, res, sun, sunc, len(dirs), 0.03, flags)
        rng = np.random.default_rng(5)
        sh16 = rng.uniform(-1, 1, size=(7, res[2], res[1], res[0], 4)).astype(np.float16).view(np.uint16).copy()
        prev16 = sh16.copy()
        p0, p1 = 16, total - 8
        tr, irr, s32, octa, st = ctx.update_probes(sid, desc, dirs, basis, sh16, p0, p1, want_trace=True,
                                                   want_irr=True, want_sh32=True, want_octa=True)
        sc = O.Scene(img, s.positions, s.normals)
        od = O.probe_desc(lo, hi, res, sun, sunc, len(dirs), 0.03)
        otr, oirr, ocounts = O.probe_trace(sc, od, dirs, p0, p1)
        otr = otr.reshape(tr.shape)
        oirr = oirr.reshape(irr.shape)
        assert np.array_equal(tr, otr)
        assert np.array_equal(irr.view(np.uint32), oirr.view(np.uint32))
        assert st.rays == int(ocounts[0] + ocounts[1])
        prev27 = sh16_to_prev27(prev16, res, list(range(p0, p1)))
        osh = O.probe_sh9(od, basis, oirr.reshape(-1, 3), p0, p1, prev27)
        assert np.array_equal(s32.reshape(-1, 27).view(np.uint32), osh.view(np.uint32))
        oocta = O.probe_octa(od, oirr.reshape(-1, 3), p0, p1)
        assert np.array_equal(octa.view(np.uint32), oocta.view(np.uint32))
        # the FP16 images: updated probes hold fp16(new), the rest are untouched
        new = sh16.view(np.float16).astype(np.float32).reshape(7, res[2], res[1], res[0], 4)
        got27 = sh16_to_prev27(sh16, res, list(range(p0, p1)))
        assert np.array_equal(got27, osh.astype(np.float16).astype(np.float32))
        for p in list(range(0, p0)) + list(range(p1, total)):
            x, y, z = probe_coord(p, res)
            assert np.array_equal(sh16.reshape(7, res[2], res[1], res[0], 4)[:, z, y, x],
                                  prev16.reshape(7, res[2], res[1], res[0], 4)[:, z, y, x])
        assert np.all(np.isfinite(new))
    finally:
        ctx.free_scene(sid)
