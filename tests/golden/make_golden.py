"""Generates the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py [room|tlas|all]

* room_refbvh.npz -- the reference's own BVHBuilder (compiled from the reference
  sources by oracle/Makefile, single-threaded so node numbering is stable) run
  on the config-1 room scene (scenes.room_scene(1)): the fillGpuBuffer bytes,
  the seven ranges and the push constants. GPU tests trace this exact buffer.
* room_golden.npz -- camera (tracing and lighting steps), random-ray and
  light-probe results on that buffer
  from the C restatement (oracle/reftrace.c) and, under the glsl_* keys, from the
  reference's own compute shaders compiled as C++ (oracle/refglsl, built by
  oracle/Makefile from the reference tree); the tests check the two against each
  other and the CUDA kernels against them.
* tlas_golden.npz -- a two-level scene (scenes.instanced_clusters(3, 12, 400):
  12 BLAS instances) written by the product's tim_rt_build_bvh_tlas (the
  reference's own builder cannot write a two-level image, see include/tim_rt.h),
  8,000 any-hit rays aimed at the instances, and the occlusion results of the
  reference's USE_TRAVERSE_TLAS shader compiled as C++ (glsl_hit) and of the C
  restatement (hit).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from tim_raytracing_b200 import scenes  # noqa: E402


def room_rays(seed=7, n=4096):
    rng = np.random.default_rng(seed)
    o = rng.uniform((0.2, 0.2, 0.2), (3.8, 3.8, 2.8), size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = 100.0
    r[:, 4:7] = d
    r.view(np.uint32)[:, 7] = (rng.uniform(size=n) < 0.5).astype(np.uint32)
    # a few axis-aligned directions exercise the division-by-zero slab cases
    r[:64, 4:7] = 0.0
    r[:64, 4 + (np.arange(64) % 3)] = np.where(np.arange(64) % 2 == 0, 1.0, -1.0)
    return r


def tlas_fixture():
    from tim_raytracing_b200 import _native as N
    s = scenes.instanced_clusters(3, 12, 400)
    img = N.build_bvh_tlas(s)
    sc = O.Scene(img, s.positions, s.normals)
    rays = scenes.occlusion_rays(5, 8000, targets=s.meta["centres"])
    hit, _, _, _ = O.trace(sc, rays, 1 | 4)
    out = dict(data=img.data, ranges=img.ranges, pc=np.array(img.pc, np.uint32), aabb=img.aabb, rays=rays, hit=hit)
    from oracle import refglsl
    if not refglsl.available():
        raise SystemExit("tlas_golden.npz needs oracle/_ref/librefglsl.so (make -C oracle REF=<reference tree>)")
    out["glsl_hit"] = refglsl.trace_tlas(refglsl.Scene(img, s.positions, s.normals), rays)
    np.savez_compressed(HERE / "tlas_golden.npz", **out)
    print("wrote", HERE / "tlas_golden.npz", "occluded:", float(hit[:, 0].mean()))


def main():
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    O.build()
    if what in ("tlas", "all"):
        tlas_fixture()
    if what == "tlas":
        return
    s = scenes.room_scene(1)
    img = O.ref_build(s, multithread=False)
    np.savez_compressed(HERE / "room_refbvh.npz", data=img.data, ranges=img.ranges, pc=np.array(img.pc, np.uint32),
                        aabb=img.aabb)
    sc = O.Scene(img, s.positions, s.normals)
    rays = room_rays()
    hit_c, nid_c, bary_c, _ = O.trace(sc, rays, 0)
    hit_a, _, _, _ = O.trace(sc, rays, 1)
    pd = scenes.pass_data(s, 256, 256, lpf_res=(8, 8, 8), aabb=(img.aabb[:3], img.aabb[3:]))
    cam, _, _ = O.camera(sc, pd, flags=1)
    out = dict(rays=rays, hit_closest=hit_c, nid_closest=nid_c, bary_closest=bary_c, hit_any=hit_a,
               pass_data=pd.view(np.uint8).reshape(-1), camera=cam)
    # light-probe field of the room: 4x4x4 probes, 64 octahedral directions
    res = (4, 4, 4)
    total = res[0] * res[1] * res[2]
    dirs = scenes.octahedral_dirs(8)
    basis = scenes.sh9_basis(dirs)
    sun = np.array([-0.4, 0.3, -1.0], np.float32)
    sunc = np.array([1.0, 0.95, 0.9], np.float32)
    od = O.probe_desc(img.aabb[:3], img.aabb[3:], res, sun, sunc, len(dirs), 0.03)
    ptr, pirr, _ = O.probe_trace(sc, od, dirs, 0, total)
    prev16 = np.random.default_rng(11).uniform(-1, 1, size=(7, res[2], res[1], res[0], 4)).astype(np.float16)
    # camera lighting step over the camera records, with a seeded FP16 probe field
    lpf16 = np.random.default_rng(13).uniform(-0.5, 1.5, size=(7, 8, 8, 8, 4)).astype(np.float16).view(np.uint16)
    shade16, _ = O.shade_camera(sc, pd, cam, lpf16)
    out.update(lpf16=lpf16, shade16=shade16)
    out.update(probe_res=np.array(res, np.uint32), probe_dirs=dirs, probe_basis=basis,
               probe_sun=np.stack([sun, sunc]), probe_prev16=prev16.view(np.uint16),
               probe_trace=ptr.reshape(-1, 8), probe_irradiance=pirr.reshape(-1, 3))
    try:
        from oracle import refglsl
        g = refglsl.available()
    except Exception:
        g = False
    if g:
        gs = refglsl.Scene(img, s.positions, s.normals)
        gh, gn = refglsl.trace(gs, rays, 0)
        ga, _ = refglsl.trace(gs, rays, 1)
        gcam = refglsl.camera(gs, pd)
        gptr = refglsl.probe_trace(gs, od, dirs)
        girr = refglsl.probe_light(gs, od, dirs, gptr)
        gimg = refglsl.probe_update(od, basis, girr, prev16.view(np.uint16))
        out.update(glsl_shade16=refglsl.shade(gs, pd, cam, lpf16))
        out.update(glsl_hit_closest=gh, glsl_nid_closest=gn, glsl_hit_any=ga, glsl_camera=gcam,
                   glsl_probe_trace=gptr, glsl_probe_irradiance=girr, glsl_probe_images16=gimg)
    np.savez_compressed(HERE / "room_golden.npz", **out)
    print("wrote", HERE / "room_refbvh.npz", HERE / "room_golden.npz", "glsl:", bool(g))


if __name__ == "__main__":
    main()
