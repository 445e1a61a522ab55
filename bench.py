"""Benchmark: Mrays/s of the ray-tracing hot path on B200.

Headline workload (one "step" = one frame, identical every step):
  scene   128x128-quad heightfield (32,768 tris, heights U[0,2]) + 53 icospheres of
          1,280 tris (centres U in 20x20x5, radii log-U[0.2,1.5]) = 100,608 tris,
          16 point lights; BVH built once by the product builder (reference layout).
  rays    1920x1080 pinhole primary closest-hit rays (cameraPass.comp row mapping:
          rows 1..1079), then per hit: the sun shadow ray, one shadow ray per
          tile-culled light in range (16x16-pixel tiles, 120x68 tiles), and one
          cosine-weighted diffuse bounce ray (closest hit).
Both the plain form (reference 64-B binary nodes) and the quantised form (8-wide,
8-bit child bounds) are timed; `value` is the faster form's Mrays/s (their records
are identical), device time of the frame's CUDA graph (tile culling + primary +
secondary generation + secondary trace) with the BVH resident in HBM and L2 flushed
before each step. `e2e` runs the same frame through the host-pointer C-ABI call,
one per frame (tim_rt_trace_camera with pinned host buffers, the lights culled on the
device, TIM_RT_CAM_DEVICE_CULL, and the records copied back band by band while the
frame traces, TIM_RT_CAM_PIPELINED), copies included.

On N GPUs (torchrun, one process per GPU) the same frame is split into N
contiguous bands of output rows, balanced by a per-row cost estimate from a
warm-up frame (tim_raytracing_b200.shard); every rank holds its own copy of the
scene and traces its band (tim_rt_trace_camera_rows_dev); value = the frame's
rays / the slowest rank's time (strong scaling). The bands are all-gathered over
NCCL afterwards, outside the timed region, and checked against rank 0's
whole-frame trace.

Beside the headline (1 GPU only): the room at 256x256 (reference-built BVH), the
64-scene batched launch, the 1M-triangle probe field, the serving loop, a stream
of small jobs, the builders and the lighting step. Outside every timed region,
the oracle (C restatement of the reference's traversal, pinned to its shaders)
checks the records of each of those workloads at full size: `parity`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H = 1920, 1080
# the quantised form of the frame: 8-wide walk for the secondary rays, binary walk
# for the coherent primary rays (faster there; both walks give identical results)
WIDE_FORM_FLAGS = 0x100 | 0x400   # TIM_RT_CAM_WIDE | TIM_RT_CAM_PRIMARY_BINARY
FRAME_FLAGS = 2 | 4               # TIM_RT_CAM_TILE_LIGHTS | TIM_RT_CAM_BOUNCE
METRIC = "Mrays/s"
TRAFFIC_FILE = ROOT / "profiles" / "ncu_dram_bytes.json"


def make_workload():
    from tim_raytracing_b200 import scenes
    return scenes.heightfield_scene(seed=2, grid=128, n_spheres=53, extent=20.0, n_lights=16, light_radius=6.0)


def config_dict(scene, world):
    """The workload of both arms (the GPU arm and --impl reference report the same dict)."""
    return {"workload": "heightfield_100k_frame_1080p", "triangles": int(scene.num_tris), "width": W, "height": H,
            "rays": "primary + sun shadow + tile-culled point-light shadows (16 lights, 16x16 tiles) + 1 diffuse bounce",
            "bvh": "product binned-SAH builder (tim_rt_build_bvh), reference fillGpuBuffer layout",
            "l2": "GPU timing: flushed (256 MiB write) before each step",
            "parallelism": ("1 GPU" if world == 1 else
                            f"frame rows in {world} contiguous cost-balanced bands, one per GPU, scene replicated")}


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else the fallback."""
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


def measured_traffic(key):
    """DRAM bytes (read + write) of one launch of a kernel, as an ncu capture of the
    same launch measured them (profiles/ncu_dram_bytes.json, entry `key`), or None."""
    try:
        e = json.loads(TRAFFIC_FILE.read_text())["kernels"][key]
        return int(e["dram_bytes_per_launch"]), e
    except Exception:
        return None, None


def roofline(abytes, launch_ms, l2_gbs, traffic_key, kernel, bytes_per_unit):
    """Roofline object of one kernel launch: algorithmic bytes per launch over its
    CUDA-event duration, against the bound its bytes actually come from. The bound
    is HBM when the ncu capture of the launch shows DRAM carrying at least half of
    the algorithmic bytes, else L2 (the scene's nodes and triangles are L2-resident
    and DRAM carries only the ray streams): the denominator is then the L2 read
    bandwidth this run measured with its own probe kernel."""
    achieved = abytes / (launch_ms * 1e-3) / 1e9
    hbm, hbm_src = hbm_peak()
    traffic, rec = measured_traffic(traffic_key)
    hbm_bound = traffic is not None and traffic >= 0.5 * abytes
    peak = hbm if hbm_bound else l2_gbs
    out = {"bound": "hbm" if hbm_bound else "l2", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
           "algorithmic_bytes_per_launch": int(abytes), "launch_ms": launch_ms, "bytes_per_unit": bytes_per_unit,
           "peak_source": (hbm_src if hbm_bound else
                           "L2 read bandwidth measured in this run (tim_rt_measure_l2_bandwidth: 16-B loads over an "
                           "L2-resident 32 MB buffer), of measured"),
           "frac_of_hbm": achieved / hbm, "hbm_peak_gbs": hbm, "l2_peak_gbs_measured": l2_gbs}
    if rec is not None:
        out["traffic_source"] = f"ncu dram__bytes_read.sum + dram__bytes_write.sum: {rec.get('capture', '')}"
    return out


def wide_bytes(st, prefix=""):
    g = lambda k: getattr(st, prefix + k)   # noqa: E731
    return 80 * g("node_visits") + 32 * g("node_reloads") + 48 * g("tri_tests")


def plain_bytes(st, prefix=""):
    g = lambda k: getattr(st, prefix + k)   # noqa: E731
    return 64 * g("node_visits") + 16 * g("leaf_visits") + 48 * g("tri_tests")


BYTES_WIDE = "80 per 8-wide node + 32 per node-header reload + 48 per triangle test (device counts)"
BYTES_PLAIN = "64 per node + 16 per leaf record + 48 per triangle test (device counts)"


# ---------------------------------------------------------------- the oracle: checker and CPU baseline only
#
# Everything in this section runs outside the timed regions. The oracle is the C
# restatement of the reference's traversal (oracle/reftrace.c, pinned bit for bit
# to the reference's own shaders compiled for the host); it is the checker of the
# GPU records and the timed CPU baseline, never on the measured path.

def _differing(a, b):
    a = np.asarray(a).view(np.uint32).reshape(len(a), -1)
    b = np.asarray(b).view(np.uint32).reshape(len(b), -1)
    if a.shape != b.shape:
        return -1
    return int(np.any(a != b, axis=1).sum())


def cpu_baseline_and_frame_parity(scene, img, pd, gpu, threads):
    """The oracle on the same frame (same BVH buffer, same tile lists): three
    whole-frame passes on all host threads, the best one timed as the CPU
    baseline; the first pass's records are compared word for word with the GPU's
    frame records of both forms (hit record + masks, bounce record) and the GPU's
    tile lists with the oracle's culling."""
    from oracle import oracle as O
    sc = O.Scene(img, scene.positions, scene.normals)
    tx, ty = (W + 15) // 16, (H + 15) // 16
    counts, lists = O.cull_lights(sc, pd, tx, ty, threads=threads)
    passes, rays = [], 0
    ref = ref_b = None
    O.camera(sc, pd, flags=FRAME_FLAGS, seed=1, tile_counts=counts, tile_lists=lists, pix_range=(W, 9 * W),
             threads=threads)   # warm-up: page in the scene and the worker threads
    for k in range(3):
        t0 = time.perf_counter()
        out, bounce, c = O.camera(sc, pd, flags=FRAME_FLAGS, seed=1, tile_counts=counts, tile_lists=lists,
                                  threads=threads)
        passes.append(time.perf_counter() - t0)
        rays = int(c.sum())
        if k == 0:
            ref, ref_b = out, bounce
    best = min(passes)
    base = {"value": rays / best / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"whole frame ({rays} rays, the same BVH buffer and tile lists), best of 3 passes "
                      f"({', '.join(f'{t:.2f}' for t in passes)} s)"}
    par = {"records": W * H, "rays": rays,
           "tile_lists_differing": _differing(np.concatenate([gpu["counts"][:, None], gpu["lists"]], 1),
                                              np.concatenate([counts[:, None], lists], 1))}
    for form in ("plain", "wide"):
        par[f"{form}_differing_vs_oracle"] = _differing(gpu["out"][form], ref)
        par[f"{form}_bounce_differing_vs_oracle"] = _differing(gpu["bounce"][form], ref_b)
    par["differing_vs_oracle"] = max(v for k, v in par.items() if k.endswith("differing_vs_oracle") or
                                     k == "tile_lists_differing")
    return base, par


def reference_builder_frame(N, ctx, scene, threads):
    """The drop-in case: the reference's own CPU builder (BVHBuilder::build, compiled
    from its sources into oracle/_ref, deterministic single-threaded order) makes
    the frame scene's fillGpuBuffer image, and the GPU traces that exact buffer in
    both forms (kernel time of tim_rt_trace_camera, median of 5); its records are
    checked against the oracle on the same buffer. Also the builder's own time with
    its worker threads."""
    from oracle import oracle as O
    from tim_raytracing_b200 import scenes
    if not O.have_refbuild():
        return {"unavailable": "oracle/_ref/libtimref_build.so not built"}
    t0 = time.perf_counter()
    O.ref_build(scene, multithread=True)
    t_mt = time.perf_counter() - t0
    t0 = time.perf_counter()
    img = O.ref_build(scene, multithread=False)
    t_st = time.perf_counter() - t0
    sid = ctx.upload(img, scene, quant8=True)
    pd = scenes.pass_data(scene, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    tx, ty = (W + 15) // 16, (H + 15) // 16
    counts, lists = ctx.cull_lights(sid, pd, tx, ty)
    out = {"builder_s": {"threads": round(t_mt, 3), "single_thread": round(t_st, 3)}, "nodes": int(img.pc[4]),
           "bytes": int(img.data.nbytes)}
    recs = {}
    for form, fl in (("plain_binary", 0), ("quantised_8wide", WIDE_FORM_FLAGS)):
        ks = []
        for _ in range(6):
            o, b, st = ctx.trace_camera(sid, pd, FRAME_FLAGS | fl, 1, counts, lists)
            ks.append(st.kernel_ms)
        recs[form] = (o, b)
        ms = float(np.median(ks[1:]))
        out[form] = {"value": st.rays / ms / 1e3, "kernel_ms": ms, "rays": int(st.rays)}
    ctx.free_scene(sid)
    sc = O.Scene(img, scene.positions, scene.normals)
    ref, ref_b, _ = O.camera(sc, pd, flags=FRAME_FLAGS, seed=1, tile_counts=counts, tile_lists=lists, threads=threads)
    out["parity"] = {"records": W * H}
    for form, (o, b) in recs.items():
        out["parity"][f"{form}_differing_vs_oracle"] = _differing(o, ref) + _differing(b, ref_b)
    return out


def parity_room(room, threads):
    """Config 1 records (both forms) against the oracle on the reference-built room."""
    from oracle import oracle as O
    scene, img, pd, flags, recs = room
    sc = O.Scene(img, scene.positions, scene.normals)
    ref, _, _ = O.camera(sc, pd, flags=flags, threads=threads)
    r = {"records": int(len(ref))}
    for form, o in recs.items():
        r[f"{form}_differing_vs_oracle"] = _differing(o, ref)
    r["differing_vs_oracle"] = max(v for k, v in r.items() if k.endswith("_vs_oracle"))
    return r


def parity_batched(jobs, threads):
    """Config 3: every ray of every job (20.9M rays, 64 scenes) traced by the
    oracle and compared with both forms' k_multi records."""
    from oracle import oracle as O
    from tim_raytracing_b200 import _native as N
    diff = {"plain": 0, "wide": 0}
    rays_total = 0
    t0 = time.perf_counter()
    for scene, img, rays, got in jobs:
        sc = O.Scene(img, scene.positions, scene.normals)
        hit, _, _, _ = O.trace(sc, rays, mode=N.MODE_PER_RAY, threads=threads)
        rays_total += len(rays)
        for form in diff:
            diff[form] += _differing(got[form], hit)
    return {"records": rays_total, "plain_differing_vs_oracle": diff["plain"],
            "wide_differing_vs_oracle": diff["wide"], "differing_vs_oracle": max(diff.values()),
            "oracle_s": round(time.perf_counter() - t0, 1)}


def parity_probes(checks, threads):
    """Config 4: one full update of the 32x32x8 field (256 directions per probe,
    octahedral and sampleRays-stratified sets) on the GPU in both forms against the
    oracle: trace records with their shadow masks, per-ray lit values, the new
    SH9 in FP32, the FP16 images and the octahedral texels."""
    from oracle import oracle as O
    from tim_raytracing_b200 import scenes
    out = {}
    for name, c in checks.items():
        scene, img, lo, hi, res, dirs, basis, sun, sunc, gpu = c
        sc = O.Scene(img, scene.positions, scene.normals)
        od = O.probe_desc(lo, hi, res, sun, sunc, len(dirs), 0.03)
        total = res[0] * res[1] * res[2]
        t0 = time.perf_counter()
        otr, oirr, ocnt = O.probe_trace(sc, od, dirs, 0, total, threads=threads)
        prev = np.zeros((total, 27), np.float32)
        osh = O.probe_sh9(od, basis, oirr.reshape(-1, 3), 0, total, prev)
        oocta = O.probe_octa(od, oirr.reshape(-1, 3), 0, total) if name == "octahedral" else None
        r = {"probes": total, "directions": len(dirs), "rays": int(ocnt[0] + ocnt[1]),
             "oracle_s": round(time.perf_counter() - t0, 1)}
        for form, (tr, irr, s32, octa, sh16) in gpu.items():
            d = _differing(tr.reshape(-1, 8), otr.reshape(-1, 8))
            d += _differing(irr.reshape(-1, 3), oirr.reshape(-1, 3))
            d += _differing(s32.reshape(-1, 27), osh)
            got16 = scenes.sh9_from_images16(sh16, res, np.arange(total))
            d += _differing(got16, osh.astype(np.float16).astype(np.float32))
            if oocta is not None:
                d += _differing(octa.reshape(total, -1), oocta.reshape(total, -1))
            r[f"{form}_differing_vs_oracle"] = d
        r["differing_vs_oracle"] = max(v for k, v in r.items() if k.endswith("_vs_oracle"))
        r["compared"] = ("trace records + masks, lit values, SH9 FP32, FP16 images" +
                         (", octahedral texels" if oocta is not None else "") + " (all probes)")
        out[name] = r
    return out


def parity_serving(sample, threads):
    """Config 5: a sample of served ray jobs (completed through the serving loop
    while other jobs ran) against the oracle."""
    from oracle import oracle as O
    from tim_raytracing_b200 import _native as N
    diff = rays = 0
    for scene, img, r, hit in sample:
        sc = O.Scene(img, scene.positions, scene.normals)
        want, _, _, _ = O.trace(sc, r, mode=N.MODE_PER_RAY, threads=threads)
        diff += _differing(hit, want)
        rays += len(r)
    return {"jobs": len(sample), "records": rays, "differing_vs_oracle": diff}


def run_reference(args, rank, world):
    """--impl reference: the reference's trace path on the host cores -- the
    oracle restatement of its GLSL traversal, which is bit-identical to its
    shaders compiled for the host (their Vulkan path cannot run here) -- over the
    same BVH buffer, tile lists and frame as the GPU arm, on all host threads. Step
    k traces quarter k mod 4 of the frame's traced rows [1, H) in one call (about
    0.18 s of work), so 4 consecutive steps trace the whole frame once. (One call per
    row let at most 8 threads work on a row's 1920 pixels and cost about 6x the
    time per ray.) The reference's own CPU builder is timed separately."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    from tim_raytracing_b200 import _native as N, scenes
    scene = make_workload()
    img = N.build_bvh(scene)
    pd = scenes.pass_data(scene, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    threads = O.threads_available()
    sc = O.Scene(img, scene.positions, scene.normals)
    tx, ty = (W + 15) // 16, (H + 15) // 16
    counts, lists = O.cull_lights(sc, pd, tx, ty, threads=threads)
    builder = {}
    if O.have_refbuild():
        t0 = time.perf_counter()
        rimg = O.ref_build(scene, multithread=True)
        builder = {"reference_builder": {"s": time.perf_counter() - t0, "nodes": int(rimg.pc[4]),
                                         "threads": "BVHBuilder::build(true) workers"}}

    quarter = [1 + (H - 1) * q // 4 for q in range(5)]

    def step(k):
        q = k % 4
        _, _, c = O.camera(sc, pd, flags=FRAME_FLAGS, seed=1, tile_counts=counts, tile_lists=lists,
                           pix_range=(quarter[q] * W, quarter[q + 1] * W), threads=threads)
        return int(c.sum())

    for k in range(args.warmup):
        step(k)
    t0 = time.perf_counter()
    rays = sum(step(args.warmup + k) for k in range(args.steps))
    dt = time.perf_counter() - t0
    v = rays / dt / 1e6
    sample = ("one quarter of the frame's traced rows per step, in one call (quarter = step mod 4; "
              "4 steps = the whole frame)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(scene, world),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample,
                             **builder},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU workloads

def aggregate(t, rays, dist, dev):
    """Whole-job figures of a multi-rank run: the slowest rank's time and the rays
    of all ranks (every rank calls this with its own numbers; no-op on one rank)."""
    if not dist:
        return float(t), float(rays)
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    rr = torch.tensor([float(rays)], dtype=torch.float64, device=dev)
    dist.all_reduce(rr)
    return float(tt.item()), float(rr.item())


def bench_room(N, ctx):
    """Config 1: the room (5 wall quads, 2 boxes, a 1,280-triangle icosphere) with
    the reference builder's own BVH buffer (tests/golden/room_refbvh.npz, made by
    tests/golden/make_golden.py), 256x256 primary rays plus per hit the sun ray and
    the shadow ray to the ceiling light (its leaf light list); both forms, kernel
    time of tim_rt_trace_camera, median of 20."""
    from tim_raytracing_b200 import scenes
    z = np.load(ROOT / "tests" / "golden" / "room_refbvh.npz")
    img = N.BvhImage(z["data"], z["ranges"], tuple(int(x) for x in z["pc"]), z["aabb"])
    scene = scenes.room_scene(1)
    sid = ctx.upload(img, scene, quant8=True)
    pd = scenes.pass_data(scene, 256, 256, aabb=(img.aabb[:3], img.aabb[3:]))
    out, recs = {"workload": "room 1,314 tris (reference-built BVH), 256x256 primary + sun + point-light shadow"}, {}
    for form, fl in (("plain_binary", 0), ("quantised_8wide", N.CAM_WIDE)):
        ks = []
        for _ in range(22):
            o, _, st = ctx.trace_camera(sid, pd, fl)
            ks.append(st.kernel_ms)
        ms = float(np.median(ks[2:]))
        out[form] = {"value": st.rays / ms / 1e3, "kernel_ms": ms, "rays": int(st.rays)}
        recs[form] = o
    ctx.free_scene(sid)
    return out, (scene, img, pd, 0, recs)


def batched_workload():
    """Triangle and ray counts of the 64 scenes of the batched workload."""
    rng = np.random.default_rng(3)
    tris = np.exp(rng.uniform(np.log(1e3), np.log(1e6), 64)).astype(np.int64)
    nrays = np.exp(rng.uniform(np.log(4e3), np.log(2e6), 64)).astype(np.int64)
    return tris, nrays


def bench_batched(N, ctx, dev, steps, warmup, l2_gbs, keep_for_parity):
    """Batched multi-scene workload: 64 scenes of random triangles (counts log-U
    [1K, 1M], edges log-U [1e-3, 1e-1] in the unit cube), each with its own batch
    of log-U [4K, 2M] rays (origins uniform in the cube, directions uniform, half
    closest-hit, half any-hit), traced by ONE persistent launch captured in a CUDA
    graph with the autotuner's configuration; plain and 8-wide forms. Inputs
    (~0.7 GB of rays) exceed L2, so no flush between steps. Algorithmic bytes of
    the launch from the counting kernel run per job (same rays, same form)."""
    import torch
    from tim_raytracing_b200 import scenes
    tris, nrays = batched_workload()
    t0 = time.perf_counter()
    sids, d_rays, h_rays, sc_list = [], [], [], []
    for k in range(64):
        s = scenes.random_triangles(10_000 + k, int(tris[k]))
        img = N.build_bvh(s)
        sids.append(ctx.upload(img, s, quant8=True))
        r = scenes.random_rays(20_000 + k, int(nrays[k]))
        d_rays.append(torch.from_numpy(r).to(dev))
        h_rays.append(r)
        sc_list.append((s, img))
    setup_s = time.perf_counter() - t0
    total = int(nrays.sum())
    stream = torch.cuda.Stream(device=dev)
    out = {}
    hits = {}
    for form in ("plain", "wide"):
        hits[form] = [torch.empty((int(n), 4), dtype=torch.int32, device=dev) for n in nrays]
        jobs = [(sids[k], N.MODE_PER_RAY, int(nrays[k]), d_rays[k], hits[form][k], None, None) for k in range(64)]
        b = ctx.batch_create(jobs, wide=form == "wide")
        ctx.set_launch_config()
        tune = ctx.autotune_batch(b, width=False, reps=3)
        ctx.batch_launch(b, stream=stream.cuda_stream)      # sizes the sort scratch before capture
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            ctx.batch_launch(b, stream=stream.cuda_stream)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                g.replay()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for k in range(steps):
                evs[k][0].record(stream)
                g.replay()
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        ms = [a.elapsed_time(c) for a, c in evs]
        # the same rays as 64 separate single-scene launches (default configuration)
        ctx.set_launch_config()
        sep = []
        for rep in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for k in range(64):
                ctx.trace_dev(sids[k], d_rays[k], int(nrays[k]), N.MODE_PER_RAY | (N.TRACE_WIDE if form == "wide" else 0),
                              hits[form][k], stream=stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            sep.append(e0.elapsed_time(e1))
        del g
        ctx.batch_destroy(b)
        med = float(np.median(ms))
        # work of the launch: the counting kernel over every job (outside the timed region)
        abytes = 0
        for k in range(64):
            _, _, _, st = ctx.trace(sids[k], h_rays[k], N.MODE_PER_RAY | N.TRACE_COUNT |
                                    (N.TRACE_WIDE if form == "wide" else 0), want_nid=False, want_bary=False)
            abytes += wide_bytes(st) if form == "wide" else plain_bytes(st)
        out[form] = {"value": total / (sum(ms) / len(ms) / 1e3) / 1e6, "ms_per_launch_median": med,
                     "autotuned": {k: tune[k] for k in ("block", "refill_min", "ray_sort", "stack_depth", "phase_switch")},
                     "autotune_ms": {"start": tune["start_ms"], "best": tune["best_ms"], "tried": tune["tried"]},
                     "separate_launches_ms": float(np.median(sep)),
                     "separate_launches_value": total / (float(np.median(sep)) / 1e3) / 1e6,
                     "roofline": roofline(abytes, med, l2_gbs, f"k_multi_{form}",
                                          f"k_multi<{tune['block']}, {1 if form == 'wide' else 0}> (64 scenes)",
                                          BYTES_WIDE if form == "wide" else BYTES_PLAIN)}
    ctx.set_launch_config()
    differing = 0
    ver = {"hits_checked": 0, "fp64_misses": 0, "max_abs_t_err": 0.0, "max_rel_t_err": 0.0}
    for k in range(64):
        a, c = hits["plain"][k], hits["wide"][k]
        differing += int((a != c).any(dim=1).sum().item())
        v = ctx.verify_hits(sids[k], d_rays[k], int(nrays[k]), hits["wide"][k])
        ver["hits_checked"] += v["hits_checked"]
        ver["fp64_misses"] += v["fp64_misses"]
        ver["max_abs_t_err"] = max(ver["max_abs_t_err"], v["max_abs_t_err"])
        ver["max_rel_t_err"] = max(ver["max_rel_t_err"], v["max_rel_t_err"])
    parity_jobs = None
    if keep_for_parity:
        parity_jobs = [(sc_list[k][0], sc_list[k][1], h_rays[k],
                        {f: hits[f][k].cpu().numpy().view(np.uint32) for f in ("plain", "wide")}) for k in range(64)]
    for sid in sids:
        ctx.free_scene(sid)
    res = {"workload": "64 random-triangle scenes (log-U 1K..1M tris), log-U 4K..2M rays each, 50% any-hit",
           "triangles": int(tris.sum()), "rays": total, "setup_s": round(setup_s, 2),
           "quantised_8wide": out["wide"], "plain_binary": out["plain"],
           "speedup_quantised_over_plain": out["wide"]["value"] / out["plain"]["value"],
           "hit_records_differing": differing, "l2": "not flushed: inputs exceed L2",
           "fp64_check": dict(ver, note="closest-hit records re-intersected in FP64 on the GPU (tim_rt_verify_hits); "
                                        "any-hit records carry no t and are not checked")}
    return res, parity_jobs


def bench_probes(N, ctx, l2_gbs, keep_for_parity, reps=5):
    """Light-probe field workload: the heightfield + icosphere generator at 1M
    triangles, a 32x32x8 probe grid, 256 rays per probe per update (closest hit,
    then sun and leaf-light shadow rays). Two direction sets: octahedral (FP32
    radiance averaged into 8x8 FP32 octahedral texels per probe) and the
    stratified sphere of sampleRays (lightProbFieldPass.cpp:151-202, seeded); SH9
    stored as FP16 in both. Throughput is rays (probe + shadow) per second of the
    update's device time. FP16 storage error: the FP32 texels rounded to FP16
    against texels averaged in FP64 from the same per-ray radiance."""
    from tim_raytracing_b200 import scenes
    t0 = time.perf_counter()
    scene = scenes.scaled_heightfield(77, 1_000_000)
    img = N.build_bvh(scene)
    sid = ctx.upload(img, scene, quant8=True)
    setup_s = time.perf_counter() - t0
    res = (32, 32, 8)
    side = 16
    total = res[0] * res[1] * res[2]
    lo, hi = img.aabb[:3], img.aabb[3:]
    sun, sunc = (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9)
    sets = {"octahedral": (scenes.octahedral_dirs(side), None),
            "stratified": N.probe_directions(256, N.DIRS_STRATIFIED, seed=9)}
    out = {"workload": "probe field 32x32x8, 256 rays per probe, heightfield+icospheres",
           "triangles": int(scene.num_tris), "setup_s": round(setup_s, 2)}
    forms = (("quantised_8wide", N.PROBE_WIDE | N.PROBE_PRIMARY_BINARY), ("plain_binary", 0))
    checks = {}
    for set_name, (dirs, basis) in sets.items():
        if basis is None:
            basis = scenes.sh9_basis(dirs)
        octa_flag = N.PROBE_OCTA if set_name == "octahedral" else 0
        row = {"directions": len(dirs)}
        gpu = {}
        for form, flag in forms:
            desc = N.probe_desc(lo, hi, res, sun, sunc, len(dirs), 0.03, octa_flag | flag)
            sh16 = np.zeros((7, res[2], res[1], res[0], 4), np.uint16)
            ms, pms, rays = [], [], 0
            for k in range(reps + 2):
                _, _, _, _, st = ctx.update_probes(sid, desc, dirs, basis, sh16)
                if k >= 2:
                    ms.append(st.kernel_ms)
                    pms.append(st.primary_ms)
                    rays = st.rays
            med = float(np.median(ms))
            row[form] = {"value": rays / (med / 1e3) / 1e6, "update_ms": med, "rays_per_update": int(rays),
                         "probe_ray_launch_ms": float(np.median(pms))}
            if flag:
                row[form]["walks"] = "binary for the probe rays, 8-wide for their shadow rays"
            if keep_for_parity:
                sh16 = np.zeros((7, res[2], res[1], res[0], 4), np.uint16)
                tr, irr, s32, octa, _ = ctx.update_probes(sid, desc, dirs, basis, sh16, want_trace=True,
                                                          want_irr=True, want_sh32=True, want_octa=bool(octa_flag))
                gpu[form] = (tr, irr, s32, octa, sh16)
        row["speedup_quantised_over_plain"] = row["quantised_8wide"]["value"] / row["plain_binary"]["value"]
        out[set_name] = row
        if keep_for_parity:
            checks[set_name] = (scene, img, lo, hi, res, dirs, basis, sun, sunc, gpu)
    # roofline of the probe-ray launch (closest hit, binary walk in both forms) of each
    # direction set: its rays traced once more by the counting kernel
    origins = scenes.probe_positions(lo, hi, res, np.arange(total))
    for set_name, key in (("octahedral", "probe_rays_plain"), ("stratified", "probe_rays_plain_stratified")):
        dirs = sets[set_name][0]
        rays = np.zeros((total * len(dirs), 8), np.float32)
        rays[:, 0:3] = np.repeat(origins, len(dirs), axis=0)
        rays[:, 3] = np.float32(100.0)
        rays[:, 4:7] = np.tile(dirs[:, :3], (total, 1))
        _, _, _, stc = ctx.trace(sid, rays, N.MODE_CLOSEST | N.TRACE_COUNT, want_nid=False, want_bary=False)
        out[set_name]["roofline_probe_rays"] = roofline(
            plain_bytes(stc), out[set_name]["plain_binary"]["probe_ray_launch_ms"], l2_gbs, key,
            "k_persistent<256, 0, 0, ProbePolicy> (probe rays, binary walk)", BYTES_PLAIN)
        del rays
    dirs = sets["octahedral"][0]
    # FP16 texel storage error against FP64 averaging of the same radiance
    desc = N.probe_desc(lo, hi, res, sun, sunc, len(dirs), 0.03, N.PROBE_OCTA | N.PROBE_WIDE)
    sh16 = np.zeros((7, res[2], res[1], res[0], 4), np.uint16)
    _, irr, _, octa, _ = ctx.update_probes(sid, desc, dirs, scenes.sh9_basis(dirs), sh16, want_irr=True,
                                           want_octa=True)
    step = side // 8
    tex64 = irr.astype(np.float64).reshape(total, 8, step, 8, step, 3).mean(axis=(2, 4)).reshape(total, 64, 3)
    tex16 = octa.astype(np.float16).astype(np.float64)
    mag = np.maximum(np.abs(tex64), 1e-6)
    rel16 = np.abs(tex16 - tex64) / mag
    rel32 = np.abs(octa.astype(np.float64) - tex64) / mag
    out["octa_texels"] = {"texels": int(tex64.size // 3), "fp16_max_rel_err": float(rel16.max()),
                          "fp16_mean_rel_err": float(rel16.mean()), "fp32_max_rel_err": float(rel32.max()),
                          "reference": "FP64 mean of the same per-ray FP32 radiance"}
    ctx.free_scene(sid)
    return out, checks


def bench_serving(N, ctx, dev, keep_for_parity, jobs_per_rate=1500, pool_size=256):
    """Serving workload: 16 resident heightfield + icosphere scenes (log-U [10K, 2M]
    tris), Poisson arrivals of jobs, a 40 GB device arena. A job is a ray batch of
    log-U [1K, 1M] mixed primary / shadow / probe-direction rays, or, one job in
    16, a probe-field update (tim_rt_server_submit_probes) of 64 probes x 256
    directions of a 16x16x8 field on its scene. First the saturation throughput
    (jobs submitted back to back), then p50/p99 latency at 0.5x, 0.8x and 1.0x of
    the saturation job rate. Host buffers are pinned. The server's own counters
    show the continuous batching: requests per step, steps in flight, GPU-busy
    time."""
    import torch
    from tim_raytracing_b200 import scenes
    rng = np.random.default_rng(5)
    tris = np.exp(rng.uniform(np.log(1e4), np.log(2e6), 16)).astype(np.int64)
    t0 = time.perf_counter()
    sids, ntris, descs, scs = [], 0, [], []
    for k in range(16):
        s = scenes.scaled_heightfield(40 + k, int(tris[k]))
        img = N.build_bvh(s)
        sids.append(ctx.upload(img, s, quant8=True))
        scs.append((s, img))
        ntris += s.num_tris
        descs.append(N.probe_desc(img.aabb[:3], img.aabb[3:], (16, 16, 8), (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), 256,
                                  0.03, N.PROBE_WIDE | N.PROBE_PRIMARY_BINARY))
    dirs = scenes.octahedral_dirs(16)
    basis = scenes.sh9_basis(dirs)
    fields = [torch.zeros((7, 8, 16, 16, 4), dtype=torch.int16).pin_memory() for _ in range(32)]
    field_owner = [0] * len(fields)
    pool = []   # reusable pinned ray / hit buffers: up to pool_size requests in flight
    for e in range(pool_size):
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        r = torch.from_numpy(scenes.serving_rays(60_000 + e, n)).pin_memory()
        h = torch.empty((n, 4), dtype=torch.int32).pin_memory()
        pool.append((r, h))
    setup_s = time.perf_counter() - t0
    srv = N.Server(ctx, memory_budget_bytes=40 << 30, max_rays_per_step=4 << 20, max_inflight_steps=2, wide=True)
    owner = [0] * len(pool)           # ticket of the job that last used each pool entry

    def run(n_jobs, rate, seed):
        """Submits n_jobs at Poisson times of `rate` jobs/s (0 = back to back)."""
        rg = np.random.default_rng(seed)
        srv.stats(reset=True)
        gaps = rg.exponential(1.0 / rate, n_jobs) if rate else np.zeros(n_jobs)
        t_next = time.perf_counter()
        probe_jobs = 0
        for j in range(n_jobs):
            t_next += gaps[j]
            while time.perf_counter() < t_next:
                pass
            k = int(rg.integers(16))
            if rg.uniform() < 1.0 / 16:
                f = int(rg.integers(len(fields)))
                if field_owner[f]:
                    srv.wait(field_owner[f])
                p0 = 64 * int(rg.integers(32))
                field_owner[f] = srv.submit_probes(sids[k], descs[k], dirs, basis,
                                                   fields[f].numpy().view(np.uint16), p0, p0 + 64)
                probe_jobs += 1
                continue
            e = j % len(pool)   # the entry least recently handed out: its job is long done at saturation
            if owner[e]:
                srv.wait(owner[e])
            r, h = pool[e]
            owner[e] = srv.submit(sids[k], r, N.MODE_PER_RAY, h)
        srv.drain()
        st = srv.stats()
        return {"jobs": n_jobs, "probe_update_jobs": probe_jobs, "rate_jobs_per_s": rate,
                "value": st["rays_completed"] / st["wall_s"] / 1e6,
                "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
                "queue_p50_ms": st["queue_p50_ms"], "queue_p99_ms": st["queue_p99_ms"], "steps": st["steps"],
                "requests_per_step_mean": st["step_requests"] / max(st["steps"], 1),
                "requests_per_step_max": st["max_step_requests"], "max_steps_in_flight": st["max_inflight"],
                "gpu_busy_frac": st["gpu_busy_ms"] / max(st["wall_s"] * 1e3, 1e-9),
                "arena_peak_gb": st["arena_peak_bytes"] / 1e9, "wall_s": st["wall_s"]}

    def burst(seed):
        """Every pool buffer's job submitted at once, then drained: the server's own
        capacity, without the closed loop's waits for buffers."""
        rg = np.random.default_rng(seed)
        srv.drain()
        srv.stats(reset=True)
        for e in range(len(pool)):
            if owner[e]:
                srv.wait(owner[e])
        srv.stats(reset=True)
        for e in range(len(pool)):
            r, h = pool[e]
            owner[e] = srv.submit(sids[int(rg.integers(16))], r, N.MODE_PER_RAY, h)
        srv.drain()
        st = srv.stats()
        return {"jobs": len(pool), "value": st["rays_completed"] / st["wall_s"] / 1e6, "wall_s": st["wall_s"],
                "steps": st["steps"], "gpu_busy_frac": st["gpu_busy_ms"] / max(st["wall_s"] * 1e3, 1e-9)}

    run(64, 0, 1)    # warm-up
    sat = run(jobs_per_rate, 0, 2)
    sat_rate = sat["jobs"] / sat["wall_s"]
    rates = [run(jobs_per_rate, f * sat_rate, 10 + i) | {"load": f} for i, f in enumerate((0.5, 0.8, 1.0))]
    bursts = [burst(40 + i) for i in range(3)]
    sample = None
    if keep_for_parity:
        # 12 served jobs, submitted together so that they share steps, then kept
        srv.drain()
        rg = np.random.default_rng(77)
        picks = []
        for e in rg.choice(len(pool), 12, replace=False):
            k = int(rg.integers(16))
            r, h = pool[int(e)]
            picks.append((k, int(e), srv.submit(sids[k], r, N.MODE_PER_RAY, h)))
        srv.drain()
        sample = [(scs[k][0], scs[k][1], pool[e][0].numpy(), pool[e][1].numpy().view(np.uint32).copy())
                  for k, e, _ in picks]
    srv.close()
    for sid in sids:
        ctx.free_scene(sid)
    return ({"workload": "16 heightfield+icosphere scenes (log-U 10K..2M tris), Poisson jobs: log-U 1K..1M mixed "
                         "primary/shadow/probe rays, or (1 in 16) a probe-field update of 64 probes x 256 rays, "
                         "40 GB arena, 8-wide BVHs",
             "note": "value counts traced rays: ray-batch rays plus the probe rays of probe updates (their shadow "
                     "rays are traced but not counted)",
             "triangles": int(ntris), "setup_s": round(setup_s, 2), "saturation": sat,
             "saturation_jobs_per_s": sat_rate, "rates": rates,
             "burst": max(bursts, key=lambda b: b["value"]) | {"runs": [round(b["value"], 1) for b in bursts]}}, sample)


def bench_build(N, ctx, frame_scene, pd, tx, ty):
    """Builders: the binned-SAH host builder (tim_rt_build_bvh, all host threads)
    against the GPU builder (tim_rt_build_bvh_gpu: Morton-code tree over single
    triangles, four treelet-restructuring passes that also choose the leaves by
    surface-area cost, max_depth 32; wall time including the copies of the triangles in
    and of the image out) on the benchmark frame's scene and on
    the 1M-triangle probe scene, and the frame's trace time on each tree (kernel
    time of tim_rt_trace_camera, median of 5, both forms)."""
    from tim_raytracing_b200 import scenes
    out = {}
    for name, sc in (("frame_100k", frame_scene), ("heightfield_1m", scenes.scaled_heightfield(77, 1_000_000))):
        row = {"triangles": int(sc.num_tris)}
        # the GPU builder may use the full 32 levels the traversal's stack holds (its
        # restructured trees lean deeper than the Morton-code tree it starts from)
        for label, kw in (("host_sah", {}), ("gpu_lbvh", {"ctx": ctx, "max_depth": 32})):
            ts = []
            for _ in range(3):
                t0 = time.perf_counter()
                img = N.build_bvh(sc, **kw)
                ts.append(time.perf_counter() - t0)
            row[label] = {"build_ms": 1e3 * min(ts), "nodes": int(img.num_nodes)}
            if name == "frame_100k":
                sid = ctx.upload(img, sc, quant8=True)
                counts, lists = ctx.cull_lights(sid, pd, tx, ty)
                for form, fl in (("plain", 0), ("wide", WIDE_FORM_FLAGS)):
                    ks = []
                    for _ in range(6):
                        _, _, st = ctx.trace_camera(sid, pd, FRAME_FLAGS | fl, 1, counts, lists)
                        ks.append(st.kernel_ms)
                    row[label][f"frame_trace_ms_{form}"] = float(np.median(ks[1:]))
                ctx.free_scene(sid)
        row["gpu_speedup"] = row["host_sah"]["build_ms"] / row["gpu_lbvh"]["build_ms"]
        out[name] = row
    return out


def bench_jobs_100k(N, ctx, dev, frame_scene, sid, steps=10):
    """A stream of ray jobs on the ~100K-triangle benchmark scene: 512 jobs of
    log-U [1K, 64K] mixed primary / shadow / probe-direction rays (the serving
    generator), traced (a) in the plain form as one binary-BVH launch per job, the
    way a caller without batching dispatches them (each launch then lasts at least
    one ray's chain of dependent node loads), and (b) in the quantised batched form
    as one 8-wide k_multi launch over all jobs in a CUDA graph; also the two mixed
    cases. Device-resident rays; hit records must be identical. Most of the gain
    of (b) over (a) is the batching, not the quantisation: the plain batched form
    is reported beside it."""
    import torch
    from tim_raytracing_b200 import scenes
    rng = np.random.default_rng(31)
    nr = np.exp(rng.uniform(np.log(1e3), np.log(6.4e4), 512)).astype(np.int64)
    d_rays = [torch.from_numpy(scenes.serving_rays(90_000 + k, int(n))).to(dev) for k, n in enumerate(nr)]
    total = int(nr.sum())
    stream = torch.cuda.Stream(device=dev)
    res, hits = {}, {}

    def time_it(fn):
        with torch.cuda.stream(stream):   # graph replays go to the current stream
            for _ in range(2):
                fn()
            torch.cuda.synchronize()
            ms = []
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    ctx.set_launch_config()
    for form, wide in (("plain", False), ("wide", True)):
        hits[form] = [torch.empty((int(n), 4), dtype=torch.int32, device=dev) for n in nr]
        mode = N.MODE_PER_RAY | (N.TRACE_WIDE if wide else 0)

        def per_job():
            for k in range(len(nr)):
                ctx.trace_dev(sid, d_rays[k], int(nr[k]), mode, hits[form][k], stream=stream.cuda_stream)

        res[f"{form}_per_job_launches"] = time_it(per_job)
        b = ctx.batch_create([(sid, N.MODE_PER_RAY, int(nr[k]), d_rays[k], hits[form][k], None, None)
                              for k in range(len(nr))], wide=wide)
        ctx.batch_launch(b, stream=stream.cuda_stream)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            ctx.batch_launch(b, stream=stream.cuda_stream)
        res[f"{form}_batched_graph"] = time_it(lambda: g.replay())
        del g
        ctx.batch_destroy(b)
    torch.cuda.synchronize()
    differing = sum(int((hits["plain"][k] != hits["wide"][k]).any(dim=1).sum().item()) for k in range(len(nr)))
    out = {"workload": "512 jobs of log-U 1K..64K mixed rays on the 100,608-triangle benchmark scene",
           "rays": total, "hit_records_differing": differing}
    for key, ms in res.items():
        out[key] = {"ms": ms, "value": total / (ms / 1e3) / 1e6}
    out["speedup_quantised_batched_over_plain_per_job"] = res["plain_per_job_launches"] / res["wide_batched_graph"]
    out["speedup_quantised_batched_over_plain_batched"] = res["plain_batched_graph"] / res["wide_batched_graph"]
    return out


# ---------------------------------------------------------------- small fixed launch sequences for ncu

def profile_frames(form):
    """Two frames of the benchmark workload in one form (tim_rt_trace_camera;
    pipelined: the binary form with TIM_RT_CAM_PIPELINED, results copied in bands)."""
    from tim_raytracing_b200 import _native as N, scenes
    scene = make_workload()
    img = N.build_bvh(scene)
    ctx = N.Context(0)
    sid = ctx.upload(img, scene, quant8=True)
    pd = scenes.pass_data(scene, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    tx, ty = (W + 15) // 16, (H + 15) // 16
    counts, lists = ctx.cull_lights(sid, pd, tx, ty)
    flags = FRAME_FLAGS | (N.CAM_WIDE if form == "wide" else 0) | (N.CAM_PIPELINED if form == "pipelined" else 0)
    for _ in range(2):
        _, _, st = ctx.trace_camera(sid, pd, flags, 1, counts, lists)
    print(json.dumps({"form": form, "kernel_ms": st.kernel_ms, "rays": int(st.rays)}))
    ctx.close()
    return 0


def profile_batched(wide, scenes_used=16):
    """Two launches of one batch over the first scenes_used scenes of the batched
    workload (same generators and seeds; a few hundred MB on the device)."""
    import torch
    from tim_raytracing_b200 import _native as N, scenes
    tris, nrays = batched_workload()
    ctx = N.Context(0)
    dev = torch.device("cuda", 0)
    sids, jobs = [], []
    for k in range(scenes_used):
        s = scenes.random_triangles(10_000 + k, int(tris[k]))
        sids.append(ctx.upload(N.build_bvh(s), s, quant8=True))
        r = torch.from_numpy(scenes.random_rays(20_000 + k, int(nrays[k]))).to(dev)
        h = torch.empty((int(nrays[k]), 4), dtype=torch.int32, device=dev)
        jobs.append((sids[k], N.MODE_PER_RAY, int(nrays[k]), r, h, None, None))
    b = ctx.batch_create(jobs, wide=wide)
    for _ in range(2):
        ctx.batch_launch(b)
    torch.cuda.synchronize()
    print(json.dumps({"wide": wide, "scenes": scenes_used, "rays": int(nrays[:scenes_used].sum()),
                      "triangles": int(tris[:scenes_used].sum())}))
    ctx.batch_destroy(b)
    ctx.close()
    return 0


def profile_probes(wide, stratified=False):
    """Two updates of the probe-field workload in one walk (pure 8-wide or binary), with the
    octahedral directions or (binary only) the stratified sampleRays set."""
    from tim_raytracing_b200 import _native as N, scenes
    scene = scenes.scaled_heightfield(77, 1_000_000)
    img = N.build_bvh(scene)
    ctx = N.Context(0)
    sid = ctx.upload(img, scene, quant8=True)
    res = (32, 32, 8)
    if stratified:
        dirs, basis = N.probe_directions(256, N.DIRS_STRATIFIED, seed=9)
        flags = 0
    else:
        dirs = scenes.octahedral_dirs(16)
        basis = scenes.sh9_basis(dirs)
        flags = N.PROBE_OCTA | (N.PROBE_WIDE if wide else 0)
    desc = N.probe_desc(img.aabb[:3], img.aabb[3:], res, (-0.4, 0.3, -1.0), (1.0, 0.95, 0.9), len(dirs), 0.03,
                        flags)
    sh16 = np.zeros((7, res[2], res[1], res[0], 4), np.uint16)
    for _ in range(2):
        _, _, _, _, st = ctx.update_probes(sid, desc, dirs, basis, sh16)
    print(json.dumps({"wide": wide, "probe_ms": st.primary_ms, "shadow_ms": st.secondary_ms, "rays": int(st.rays)}))
    ctx.close()
    return 0


def profile_shade():
    """The benchmark frame traced once (quantised form), then two lighting steps
    (tim_rt_shade_camera) over its records with a seeded 12x12x12 FP16 probe field."""
    from tim_raytracing_b200 import _native as N, scenes
    scene = make_workload()
    img = N.build_bvh(scene)
    ctx = N.Context(0)
    sid = ctx.upload(img, scene, quant8=True)
    pd = scenes.pass_data(scene, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    tx, ty = (W + 15) // 16, (H + 15) // 16
    counts, lists = ctx.cull_lights(sid, pd, tx, ty)
    cam, _, _ = ctx.trace_camera(sid, pd, FRAME_FLAGS | WIDE_FORM_FLAGS, 1, counts, lists)
    lres = [int(x) for x in np.asarray(pd["lpfResolution"]).reshape(-1)[:3]]
    field = np.random.default_rng(3).uniform(0.0, 1.0, size=(7, lres[2], lres[1], lres[0], 4)).astype(np.float16)
    for _ in range(2):
        _, _, st = ctx.shade_camera(sid, pd, cam, field.view(np.uint16))
    print(json.dumps({"shade_kernel_ms": st.kernel_ms}))
    ctx.close()
    return 0


def profile_build():
    """Two GPU builds (tim_rt_build_bvh_gpu, max_depth 32) of the 1M-triangle
    heightfield scene of the builder comparison: the first warms the context's
    build scratch, the second is the one to read."""
    from tim_raytracing_b200 import _native as N, scenes
    ctx = N.Context(0)
    scene = scenes.scaled_heightfield(77, 1_000_000)
    out = []
    for _ in range(2):
        t0 = time.perf_counter()
        img = N.build_bvh(scene, ctx=ctx, max_depth=32)
        out.append(1e3 * (time.perf_counter() - t0))
    print(json.dumps({"build_wall_ms": out, "nodes": int(img.num_nodes)}))
    ctx.close()
    return 0


# ---------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="tim")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline and every oracle check")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-size oracle checks of the side workloads")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched multi-scene workload")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving workload")
    ap.add_argument("--no-probes", action="store_true", help="skip the light-probe field workload")
    ap.add_argument("--no-build", action="store_true", help="skip the BVH builder comparison")
    ap.add_argument("--profile", choices=["plain", "wide", "pipelined", "batched-plain", "batched-wide",
                                          "probes-plain", "probes-wide", "probes-stratified", "shade", "build"],
                    help="only run a small, fixed launch sequence for ncu and exit: plain / wide = two frames of "
                         "one form (per frame one primary and one secondary k_persistent launch); pipelined = two "
                         "binary frames whose results are copied in bands while they trace; batched-* = two "
                         "launches of one k_multi batch over the first 16 scenes of the batched workload; "
                         "probes-* = two probe-field updates of one form (per update one probe-ray and one "
                         "shadow-ray k_persistent launch; probes-stratified: binary, stratified directions); shade = one quantised frame, then two k_shade_camera "
                         "launches; build = two GPU builds of the 1M-triangle scene")
    args = ap.parse_args()
    if args.profile in ("plain", "wide", "pipelined"):
        return profile_frames(args.profile)
    if args.profile in ("batched-plain", "batched-wide"):
        return profile_batched(args.profile == "batched-wide")
    if args.profile == "shade":
        return profile_shade()
    if args.profile == "build":
        return profile_build()
    if args.profile:
        return profile_probes(args.profile == "probes-wide", args.profile == "probes-stratified")
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from tim_raytracing_b200 import _native as N, scenes, shard
    scene = make_workload()
    t0 = time.perf_counter()
    img = N.build_bvh(scene)
    build_s = time.perf_counter() - t0
    ctx = N.Context(local)
    sid = ctx.upload(img, scene, quant8=True)
    pd = scenes.pass_data(scene, W, H, aabb=(img.aabb[:3], img.aabb[3:]))
    tx, ty = (W + 15) // 16, (H + 15) // 16
    dev = torch.device("cuda", local)
    d_counts = torch.zeros(tx * ty, dtype=torch.int32, device=dev)
    d_lists = torch.zeros(tx * ty * 16, dtype=torch.int32, device=dev)
    outs = {f: torch.zeros(W * H * 8, dtype=torch.int32, device=dev) for f in ("plain", "wide")}
    bounces = {f: torch.zeros(W * H * 4, dtype=torch.int32, device=dev) for f in ("plain", "wide")}
    d_rays = torch.zeros(1, dtype=torch.int64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    # this rank's band of output rows: the whole frame on one GPU; on N GPUs N
    # contiguous bands balanced by the per-row cost of a warm-up frame, which every
    # rank traces whole and so computes the same bands
    whole = None
    if world > 1:
        ctx.cull_lights_dev(sid, pd, tx, ty, d_counts, d_lists, stream=stream.cuda_stream)
        ctx.trace_camera_dev(sid, pd, FRAME_FLAGS, 1, d_counts, d_lists, outs["plain"], bounces["plain"],
                             stream=stream.cuda_stream)
        stream.synchronize()
        whole = outs["plain"].view(H, W * 8).clone(), bounces["plain"].view(H, W * 4).clone()
        weights = shard.frame_row_weights(whole[0].cpu().numpy().view(np.uint32), W, H,
                                          d_counts.cpu().numpy().view(np.uint32))
        bands = shard.row_bands(H, world, weights)
    else:
        bands = [(0, H)]
    row_b, row_e = bands[rank]

    def frame(form, s):
        flags = FRAME_FLAGS | (WIDE_FORM_FLAGS if form == "wide" else 0)
        ctx.cull_lights_dev(sid, pd, tx, ty, d_counts, d_lists, stream=s.cuda_stream)
        if row_b < row_e:
            ctx.trace_camera_rows_dev(sid, pd, flags, 1, row_b, row_e, d_counts, d_lists, outs[form], bounces[form],
                                      d_rays, stream=s.cuda_stream)

    results = {}
    graphs = {}
    for form in ("plain", "wide"):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                frame(form, stream)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            frame(form, stream)
        graphs[form] = g
        for _ in range(2):
            g.replay()
        torch.cuda.synchronize()

    def timed(form, steps):
        g = graphs[form]
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        r0 = int(d_rays.item())
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(float(k))
                evs[k][0].record(stream)
                g.replay()
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        rays = int(d_rays.item()) - r0
        return ms, rays

    sampler = ClockSampler(local)
    with sampler:
        for form in ("plain", "wide"):
            ms, rays = timed(form, args.steps)
            results[form] = (ms, rays)
    clocks = sampler.summary()

    # the bands of all ranks make one frame: rays of all ranks, the slowest rank's time
    ms_w, rays_w = aggregate(*results["wide"], dist, dev)
    ms_p, rays_p = aggregate(*results["plain"], dist, dev)
    v_w = rays_w / (ms_w / 1e3) / 1e6
    v_p = rays_p / (ms_p / 1e3) / 1e6
    rays_per_frame = rays_w / args.steps

    sharding = None
    if world > 1:
        # reassembly of the frame from the bands (NCCL all-gather, outside the timed
        # region) and its check against the whole-frame trace of this rank
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        got = shard.gather_in_order(outs["wide"].view(H, W * 8)[row_b:row_e], bands)
        got_b = shard.gather_in_order(bounces["wide"].view(H, W * 4)[row_b:row_e], bands)
        e1.record()
        torch.cuda.synchronize()
        diff = int((got[1:] != whole[0][1:]).any(dim=1).sum().item()) + \
            int((got_b[1:] != whole[1][1:]).any(dim=1).sum().item())
        sharding = {"bands": bands, "gather_ms": e0.elapsed_time(e1),
                    "gathered_rows_differing_vs_whole_frame": diff,
                    "per_rank_ms": {"plain": results["plain"][0] / args.steps, "wide": results["wide"][0] / args.steps}}
        if dist:
            parts = [None] * world
            dist.all_gather_object(parts, sharding["per_rank_ms"])
            sharding["per_rank_ms"] = parts

    # hit-id agreement of the two forms on this rank's rows of the frame
    op = outs["plain"].view(H, W, 8)[row_b:row_e].reshape(-1, 8)
    ow = outs["wide"].view(H, W, 8)[row_b:row_e].reshape(-1, 8)
    prim_mismatch = int((op[:, :4] != ow[:, :4]).any(dim=1).sum().item())
    bnc_mismatch = int((bounces["plain"].view(H, W, 4)[row_b:row_e] != bounces["wide"].view(H, W, 4)[row_b:row_e])
                       .any(dim=2).sum().item())
    mask_mismatch = int((op[:, 4] != ow[:, 4]).sum().item())

    # end to end through the host-pointer C ABI (pinned buffers, copies included)
    counts_h = torch.empty(tx * ty, dtype=torch.int32).pin_memory()
    lists_h = torch.empty(tx * ty * 16, dtype=torch.int32).pin_memory()
    out_h = torch.empty(W * H * 8, dtype=torch.int32).pin_memory()
    bounce_h = torch.empty(W * H * 4, dtype=torch.int32).pin_memory()
    L = N.lib()
    import ctypes
    pdc = np.ascontiguousarray(pd)

    # the headline is the faster of the two forms (identical records); the end-to-end
    # run and the roofline use that form
    best = "plain" if v_p > v_w else "wide"
    best_flags = WIDE_FORM_FLAGS if best == "wide" else 0

    def e2e_step():
        if world == 1:
            # one call per frame: the pass data goes in, the lights are culled on the
            # device, and the records come back to the pinned host buffers band by band
            st = N.Stats()
            N._check(L.tim_rt_trace_camera(ctx.handle, sid, pdc.ctypes.data,
                                           FRAME_FLAGS | best_flags | N.CAM_PIPELINED | N.CAM_DEVICE_CULL, 1,
                                           None, None, out_h.data_ptr(), bounce_h.data_ptr(), ctypes.byref(st)))
            return st.rays
        # one band per rank: tile lists up, the band traced, the band's records down
        r0 = int(d_rays.item())
        d_counts.copy_(counts_h, non_blocking=True)
        d_lists.copy_(lists_h, non_blocking=True)
        ctx.trace_camera_rows_dev(sid, pd, FRAME_FLAGS | best_flags, 1, row_b, row_e, d_counts, d_lists, outs[best],
                                  bounces[best], d_rays)
        out_h.view(H, W * 8)[row_b:row_e].copy_(outs[best].view(H, W * 8)[row_b:row_e])
        bounce_h.view(H, W * 4)[row_b:row_e].copy_(bounces[best].view(H, W * 4)[row_b:row_e])
        torch.cuda.synchronize()
        return int(d_rays.item()) - r0

    if world > 1:
        c_np, l_np = ctx.cull_lights(sid, pd, tx, ty)
        counts_h.copy_(torch.from_numpy(c_np.view(np.int32)))
        lists_h.copy_(torch.from_numpy(l_np.reshape(-1).view(np.int32)))
    for _ in range(2):
        e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_rays = sum(e2e_step() for _ in range(args.steps))
    e2e_s = time.perf_counter() - t0
    e2e_s, e2e_rays = aggregate(e2e_s, e2e_rays, dist, dev)
    e2e_v = e2e_rays / e2e_s / 1e6
    band_rows = row_e - row_b
    # the host-pointer path's records (pipelined bands on two streams) against the
    # device path's records of the same frame, this rank's rows
    e2e_diff = int((out_h.view(H, W, 8)[row_b:row_e] != outs[best].cpu().view(H, W, 8)[row_b:row_e]).any(-1).sum() +
                   (bounce_h.view(H, W, 4)[row_b:row_e] != bounces[best].cpu().view(H, W, 4)[row_b:row_e]).any(-1).sum())
    # world 1: the pass data (240 B, the call's by-value kernel arguments) in, the
    # frame's records out; N ranks: each rank's tile lists in, its band's records out
    e2e_h2d = 240 if world == 1 else int(tx * ty * 68 + 240)
    e2e_d2h = int(W * H * 48) if world == 1 else int(W * band_rows * 48)

    # Dominant kernel (the secondary trace): its launch duration from CUDA events
    # recorded around each phase on the context stream, and its work from the
    # counting kernel variant on the same frame.
    counts_np, lists_np = ctx.cull_lights(sid, pd, tx, ty)
    kern = {}
    for form, flw in (("wide", WIDE_FORM_FLAGS), ("plain", 0)):
        ph = []
        for _ in range(5):
            _, _, st = ctx.trace_camera(sid, pd, FRAME_FLAGS | flw, 1, counts_np, lists_np)
            ph.append((st.primary_ms, st.gen_ms, st.secondary_ms))
        _, _, stc = ctx.trace_camera(sid, pd, FRAME_FLAGS | flw | N.CAM_COUNT, 1, counts_np, lists_np)
        med = np.median(np.array(ph), axis=0)
        abytes = wide_bytes(stc, "secondary_") if form == "wide" else plain_bytes(stc, "secondary_")
        r = max(stc.secondary_rays_counted, 1)
        kern[form] = {"primary_ms": float(med[0]), "gen_ms": float(med[1]), "secondary_ms": float(med[2]),
                      "secondary_rays": int(stc.secondary_rays_counted), "algorithmic_bytes": int(abytes),
                      "per_ray": {"node_visits": stc.secondary_node_visits / r, "leaf_visits": stc.secondary_leaf_visits / r,
                                  "tri_tests": stc.secondary_tri_tests / r, "node_reloads": stc.secondary_node_reloads / r,
                                  "bytes": abytes / r}}
    l2_gbs = N.measure_l2_gbs(local)
    frame_host = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        frame_host = {"out": {f: outs[f].cpu().numpy().view(np.uint32).reshape(-1, 8) for f in outs},
                      "bounce": {f: bounces[f].cpu().numpy().view(np.uint32).reshape(-1, 4) for f in bounces},
                      "counts": d_counts.cpu().numpy().view(np.uint32),
                      "lists": d_lists.cpu().numpy().view(np.uint32).reshape(-1, 16)}
    # the lighting step of the same frame (tim_rt_shade_camera) on the quantised
    # frame's records, with a seeded FP16 light-probe field of the frame's grid
    cam_h = outs["wide"].cpu().numpy().view(np.uint32).reshape(-1, 8)
    lres = [int(x) for x in np.asarray(pd["lpfResolution"]).reshape(-1)[:3]]
    field = np.random.default_rng(3).uniform(0.0, 1.0, size=(7, lres[2], lres[1], lres[0], 4)).astype(np.float16)
    sk = []
    for _ in range(7):
        img16, _, st = ctx.shade_camera(sid, pd, cam_h, field.view(np.uint16))
        sk.append(st.kernel_ms)
    shade_ms = float(np.median(sk[2:]))
    shade = {"kernel_ms": shade_ms, "mpix_per_s": W * H / shade_ms / 1e3,
             "lit_pixels": int((img16[:, 3] != 0).sum()),
             "workload": "cameraPass.comp lighting step of the 1080p frame: direct light of the 16 lights and the "
                         f"sun from the shadow masks, probe-masked SH9 sample of a {lres[0]}x{lres[1]}x{lres[2]} "
                         "FP16 probe field, RGBA16F out"}
    single = world == 1
    checks = single and not args.no_cpu_baseline and not args.no_parity
    room = bench_room(N, ctx) if single else None
    build = bench_build(N, ctx, scene, pd, tx, ty) if single and not args.no_build else None
    jobs_100k = bench_jobs_100k(N, ctx, dev, scene, sid) if single and not args.no_batched else None
    batched = batched_jobs = serving = serving_sample = probes = probe_checks = None
    if single and not args.no_batched:
        batched, batched_jobs = bench_batched(N, ctx, dev, args.steps, args.warmup, l2_gbs, checks)
    if single and not args.no_serving:
        serving, serving_sample = bench_serving(N, ctx, dev, checks)
    if single and not args.no_probes:
        probes, probe_checks = bench_probes(N, ctx, l2_gbs, checks)

    if rank == 0:
        v_best, ms_best = (v_p, ms_p) if best == "plain" else (v_w, ms_w)
        line = {
            "metric": METRIC, "value": v_best, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_best / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(scene, world),
            "form": "plain_binary" if best == "plain" else "quantised_8wide",
            "rays_per_step": rays_per_frame, "bvh_build_s": round(build_s, 3),
            "forms": {"quantised_8wide": {"value": v_w, "ms_per_step": ms_w / args.steps,
                                          "walks": "8-wide for secondary rays, binary for primary rays "
                                                   "(TIM_RT_CAM_WIDE | TIM_RT_CAM_PRIMARY_BINARY)"},
                      "plain_binary": {"value": v_p, "ms_per_step": ms_p / args.steps,
                                       "walks": "binary for every ray (filtered box test, flags 0)"},
                      "speedup_quantised_over_plain": v_w / v_p,
                      "headline": "plain_binary" if best == "plain" else "quantised_8wide"},
            "hit_ids": {"primary_records_differing": prim_mismatch, "bounce_records_differing": bnc_mismatch,
                        "shadow_masks_differing": mask_mismatch, "pixels": W * (row_e - row_b),
                        "compared": "plain vs quantised records of the same frame (rank 0's rows)"},
            "e2e": {"value": e2e_v, "unit": METRIC, "h2d_bytes_per_step": e2e_h2d, "d2h_bytes_per_step": e2e_d2h,
                    "records_differing_vs_device_path": e2e_diff,
                    "inputs": ("per step the frame's pass data (camera and sun, 240 B) goes in with the call and "
                               "the lights are culled on the device (TIM_RT_CAM_DEVICE_CULL); the scene's BVH "
                               "stays resident, uploaded once as the reference uploads it once per scene"
                               if world == 1 else
                               "per step each rank's tile lists and pass data go in; the scene stays resident"),
                    "outputs": "the hit records (32 B) and bounce records (16 B) of every pixel of the frame "
                               "(of the rank's band for N > 1), copied into pinned host buffers"},
            "gpu_launches": None, "clocks": clocks,
        }
        # our kernels per frame: cull, primary trace, secondary generation, kind prefix, secondary trace, ray count
        line["gpu_launches"] = 6 * args.steps * world
        kw = kern[best]
        wide_k = best == "wide"
        line["roofline"] = roofline(
            kw["algorithmic_bytes"], kw["secondary_ms"], l2_gbs, f"frame_secondary_{best}",
            (f"k_persistent<256, {1 if wide_k else 0}, 0, SecondaryPolicy> "
             f"({'8-wide' if wide_k else 'binary'} secondary trace of the frame)"),
            BYTES_WIDE if wide_k else BYTES_PLAIN)
        line["roofline"]["note"] = ("the 11 MB scene is L2-resident: the algorithmic node and triangle bytes are L2 "
                                    "reads, and DRAM carries only the secondary-ray queue (traffic << algorithmic "
                                    "bytes); the kernel is issue-bound (ncu: instructions and lanes per instruction)")
        line["kernels"] = kern
        if sharding:
            line["sharding"] = sharding
        if room:
            line["room"] = room[0]
        if batched:
            line["batched"] = batched
        if probes:
            line["probes"] = probes
        line["shade"] = shade
        if build:
            line["build"] = build
        if jobs_100k:
            line["jobs_100k"] = jobs_100k
        if serving:
            line["serving"] = serving
            r8 = serving["rates"][1]
            line["latency"] = {"p50_ms": r8["p50_ms"], "p99_ms": r8["p99_ms"], "unit": "ms",
                               "arrival": f"Poisson, {r8['rate_jobs_per_s']:.0f} jobs/s (0.8x saturation)",
                               "throughput": r8["value"]}
        if not args.no_cpu_baseline and single:
            # the oracle: timed CPU baseline and checker (outside every timed region)
            from oracle import oracle as O
            threads = O.threads_available()
            base, par_frame = cpu_baseline_and_frame_parity(scene, img, pd, frame_host, threads)
            line["cpu_baseline"] = base
            parity = {"frame_1080p_100k": par_frame}
            if not args.no_parity:
                ref_tree = reference_builder_frame(N, ctx, scene, threads)
                line["reference_tree"] = ref_tree
                if "parity" in ref_tree:
                    rp = ref_tree["parity"]
                    rp["differing_vs_oracle"] = max(v for k, v in rp.items() if k.endswith("_vs_oracle"))
                    parity["frame_1080p_reference_builder_tree"] = rp
                parity["room_256"] = parity_room(room[1], threads)
                if batched_jobs:
                    parity["batched_64_scenes"] = parity_batched(batched_jobs, threads)
                if probe_checks:
                    for k, v in parity_probes(probe_checks, threads).items():
                        parity[f"probes_1m_{k}"] = v
                if serving_sample:
                    parity["serving_sample"] = parity_serving(serving_sample, threads)
            parity["all_zero"] = all(v.get("differing_vs_oracle", 0) == 0 for v in parity.values()
                                     if isinstance(v, dict))
            line["parity"] = parity
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
