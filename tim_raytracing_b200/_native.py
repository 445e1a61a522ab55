"""ctypes binding of the C ABI in include/tim_rt.h (libtim_rt.so, built in-tree).

This is the Python view of the same entry points a C++ caller binds; it adds
no computation of its own. Loading fails loudly if the shared library is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libtim_rt.so"

OK, EINVAL, ENOMEM, ETIMEOUT, EDEVICE, ENOTFOUND, EUNSUPPORTED, ECANCELLED, EBUSY = range(9)
MODE_CLOSEST, MODE_ANY, MODE_PER_RAY = 0, 1, 2
TRACE_WIDE = 0x100
TRACE_COUNT = 0x400
TRACE_TLAS = 0x800
UPLOAD_QUANT8 = 0x2
CAM_PROB_MASK, CAM_TILE_LIGHTS, CAM_BOUNCE, CAM_WIDE, CAM_COUNT = 1, 2, 4, 0x100, 0x200
CAM_PRIMARY_BINARY = 0x400
CAM_PIPELINED = 0x800
CAM_DEVICE_CULL = 0x1000
RANGE_BLAS, RANGE_TRI, RANGE_PRIM, RANGE_MAT, RANGE_LIGHT, RANGE_NODE, RANGE_LEAF = range(7)

EXPORTED = [
    "tim_rt_version", "tim_rt_last_error", "tim_rt_create", "tim_rt_destroy", "tim_rt_memory_used",
    "tim_rt_upload_bvh", "tim_rt_free_scene", "tim_rt_scene_bytes", "tim_rt_trace", "tim_rt_trace_dev",
    "tim_rt_trace_camera", "tim_rt_cull_lights", "tim_rt_build_params_default", "tim_rt_build_bvh",
    "tim_rt_bvh_blob_info", "tim_rt_bvh_blob_free", "tim_rt_validate_bvh", "tim_rt_trace_camera_dev",
    "tim_rt_cull_lights_dev", "tim_rt_get_launch_config", "tim_rt_set_launch_config", "tim_rt_trace_camera_noalloc",
    "tim_rt_measure_l2_bandwidth", "tim_rt_update_probes", "tim_rt_batch_create", "tim_rt_batch_launch",
    "tim_rt_batch_info", "tim_rt_batch_destroy", "tim_rt_autotune_batch", "tim_rt_server_create",
    "tim_rt_server_submit", "tim_rt_server_wait", "tim_rt_server_drain", "tim_rt_server_stats_get",
    "tim_rt_server_destroy", "tim_rt_verify_hits", "tim_rt_server_submit_probes", "tim_rt_bvh_file_write",
    "tim_rt_bvh_file_read", "tim_rt_bvh_file_info", "tim_rt_bvh_file_free", "tim_rt_upload_bvh_file",
    "tim_rt_shade_camera", "tim_rt_shade_camera_dev", "tim_rt_build_bvh_gpu", "tim_rt_probe_directions",
    "tim_rt_wide_check", "tim_rt_trace_camera_rows_dev", "tim_rt_server_cancel", "tim_rt_build_bvh_tlas",
]
SORT_NONE, SORT_OCTANT, SORT_MORTON = 0, 1, 2
BATCH_WIDE = 0x100
TUNE_WIDTH = 1
PROBE_OCTA, PROBE_WIDE, PROBE_PRIMARY_BINARY = 1, 0x100, 0x400
SHADE_NO_LPF = 1


class ProbeDesc(ctypes.Structure):
    _fields_ = [("aabbMin", ctypes.c_float * 4), ("aabbMax", ctypes.c_float * 4), ("resolution", ctypes.c_uint32 * 4),
                ("sunDir", ctypes.c_float * 4), ("sunColor", ctypes.c_float * 4), ("hysteresis", ctypes.c_float),
                ("num_dirs", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


def probe_desc(aabb_min, aabb_max, res, sun_dir, sun_color, num_dirs, hysteresis=0.03, flags=0) -> ProbeDesc:
    d = ProbeDesc()
    for i in range(3):
        d.aabbMin[i] = float(aabb_min[i])
        d.aabbMax[i] = float(aabb_max[i])
        d.resolution[i] = int(res[i])
        d.sunDir[i] = float(sun_dir[i])
        d.sunColor[i] = float(sun_color[i])
    d.hysteresis = hysteresis
    d.num_dirs = num_dirs
    d.flags = flags
    return d


class TimRtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tim_rt error {code}: {msg}")
        self.code = code


class PushConstants(ctypes.Structure):
    _fields_ = [("numTriangles", ctypes.c_uint32), ("numBlas", ctypes.c_uint32), ("numPrimitives", ctypes.c_uint32),
                ("numLights", ctypes.c_uint32), ("numNodes", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_uint64), ("primary_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("probe_rays", ctypes.c_uint64), ("bounce_rays", ctypes.c_uint64), ("kernel_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("node_visits", ctypes.c_uint64), ("leaf_visits", ctypes.c_uint64),
                ("tri_tests", ctypes.c_uint64), ("node_reloads", ctypes.c_uint64), ("primary_ms", ctypes.c_float),
                ("gen_ms", ctypes.c_float), ("secondary_ms", ctypes.c_float), ("secondary_rays_counted", ctypes.c_uint64),
                ("secondary_node_visits", ctypes.c_uint64), ("secondary_leaf_visits", ctypes.c_uint64),
                ("secondary_tri_tests", ctypes.c_uint64), ("secondary_node_reloads", ctypes.c_uint64)]


class LaunchConfig(ctypes.Structure):
    _fields_ = [("block", ctypes.c_uint32), ("stack_depth", ctypes.c_uint32), ("refill_min", ctypes.c_uint32),
                ("ray_sort", ctypes.c_uint32), ("phase_switch", ctypes.c_uint32)]


class Job(ctypes.Structure):
    """tim_rt_job: one ray buffer of a batch, traced against one resident scene (device pointers)."""
    _fields_ = [("scene", ctypes.c_uint32), ("mode", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("d_rays", ctypes.c_void_p), ("d_hit", ctypes.c_void_p),
                ("d_leaf_nid", ctypes.c_void_p), ("d_bary", ctypes.c_void_p)]


class ServerParams(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_uint64), ("max_rays_per_step", ctypes.c_uint32),
                ("max_inflight_steps", ctypes.c_uint32), ("max_jobs_per_step", ctypes.c_uint32),
                ("flags", ctypes.c_uint32)]


class Request(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("mode", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("rays", ctypes.c_void_p), ("hit", ctypes.c_void_p),
                ("leaf_nid", ctypes.c_void_p), ("bary", ctypes.c_void_p)]


class ProbeRequest(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("probe_begin", ctypes.c_uint32), ("probe_end", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("desc", ctypes.c_void_p), ("dirs", ctypes.c_void_p),
                ("sh_basis", ctypes.c_void_p), ("sh9_fp16", ctypes.c_void_p), ("octa", ctypes.c_void_p)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rays_completed", ctypes.c_uint64),
                ("steps", ctypes.c_uint64), ("arena_bytes", ctypes.c_uint64), ("arena_peak_bytes", ctypes.c_uint64),
                ("p50_ms", ctypes.c_float), ("p99_ms", ctypes.c_float), ("mean_ms", ctypes.c_float),
                ("max_ms", ctypes.c_float), ("queue_p50_ms", ctypes.c_float), ("queue_p99_ms", ctypes.c_float),
                ("wall_s", ctypes.c_float), ("cancelled", ctypes.c_uint64), ("step_requests", ctypes.c_uint64),
                ("max_step_requests", ctypes.c_uint32), ("max_inflight", ctypes.c_uint32),
                ("gpu_busy_ms", ctypes.c_float)]


class VerifyResult(ctypes.Structure):
    _fields_ = [("hits_checked", ctypes.c_uint64), ("misses", ctypes.c_uint64), ("fp64_misses", ctypes.c_uint64),
                ("max_abs_t_err", ctypes.c_double), ("max_rel_t_err", ctypes.c_double)]


class TuneResult(ctypes.Structure):
    _fields_ = [("best", LaunchConfig), ("wide", ctypes.c_uint32), ("tried", ctypes.c_uint32),
                ("best_ms", ctypes.c_float), ("start_ms", ctypes.c_float)]


class BuildParams(ctypes.Structure):
    _fields_ = [("max_leaf_size", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("traversal_cost", ctypes.c_float),
                ("intersection_cost", ctypes.c_float), ("num_threads", ctypes.c_uint32)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m tim_raytracing_b200.build` "
                          "(the CUDA library is required; there is no CPU fallback)")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    L.tim_rt_version.restype = ctypes.c_char_p
    L.tim_rt_last_error.restype = ctypes.c_char_p
    L.tim_rt_create.argtypes = [i32, u64, ctypes.POINTER(vp)]
    L.tim_rt_destroy.argtypes = [vp]
    L.tim_rt_memory_used.argtypes = [vp, ctypes.POINTER(u64)]
    L.tim_rt_upload_bvh.argtypes = [vp, vp, u64, vp, vp, vp, vp, u32, u32, ctypes.POINTER(PushConstants), u32,
                                    ctypes.POINTER(u32)]
    L.tim_rt_free_scene.argtypes = [vp, u32]
    L.tim_rt_scene_bytes.argtypes = [vp, u32, ctypes.POINTER(u64)]
    L.tim_rt_trace.argtypes = [vp, u32, vp, u32, u32, vp, vp, vp, ctypes.POINTER(Stats)]
    L.tim_rt_trace_dev.argtypes = [vp, u32, vp, u32, u32, vp, vp, vp, vp]
    L.tim_rt_trace_camera.argtypes = [vp, u32, vp, u32, u32, vp, vp, vp, vp, ctypes.POINTER(Stats)]
    L.tim_rt_cull_lights.argtypes = [vp, u32, vp, u32, u32, vp, vp]
    L.tim_rt_build_params_default.argtypes = [ctypes.POINTER(BuildParams)]
    L.tim_rt_build_params_default.restype = None
    L.tim_rt_build_bvh.argtypes = [vp, u32, vp, u32, vp, u32, vp, u32, ctypes.POINTER(BuildParams), ctypes.POINTER(vp)]
    L.tim_rt_build_bvh_tlas.argtypes = [vp, u32, vp, u32, vp, vp, u32, vp, u32, vp, u32, ctypes.POINTER(BuildParams), u32,
                                        ctypes.POINTER(vp)]
    L.tim_rt_bvh_blob_info.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(u64), vp, ctypes.POINTER(PushConstants), vp]
    L.tim_rt_bvh_blob_free.argtypes = [vp]
    L.tim_rt_bvh_blob_free.restype = None
    L.tim_rt_validate_bvh.argtypes = [vp, u64, vp, ctypes.POINTER(PushConstants), u32, ctypes.POINTER(u32)]
    L.tim_rt_trace_camera_dev.argtypes = [vp, u32, vp, u32, u32, vp, vp, vp, vp, vp, vp]
    L.tim_rt_trace_camera_rows_dev.argtypes = [vp, u32, vp, u32, u32, u32, u32, vp, vp, vp, vp, vp, vp]
    L.tim_rt_cull_lights_dev.argtypes = [vp, u32, vp, u32, u32, vp, vp, vp]
    L.tim_rt_get_launch_config.argtypes = [vp, ctypes.POINTER(LaunchConfig)]
    L.tim_rt_measure_l2_bandwidth.argtypes = [i32, u64, i32, ctypes.POINTER(ctypes.c_float)]
    L.tim_rt_update_probes.argtypes = [vp, u32, ctypes.POINTER(ProbeDesc), vp, vp, u32, u32, vp, vp, vp, vp, vp,
                                       ctypes.POINTER(Stats)]
    L.tim_rt_trace_camera_noalloc.argtypes = [vp, vp, ctypes.POINTER(PushConstants), vp, u32, u32, vp, u32, u32, vp,
                                              vp, vp, vp, vp]
    L.tim_rt_set_launch_config.argtypes = [vp, ctypes.POINTER(LaunchConfig)]
    L.tim_rt_batch_create.argtypes = [vp, ctypes.POINTER(Job), u32, u32, ctypes.POINTER(vp)]
    L.tim_rt_batch_launch.argtypes = [vp, vp, vp]
    L.tim_rt_batch_info.argtypes = [vp, vp, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.tim_rt_batch_destroy.argtypes = [vp, vp]
    L.tim_rt_autotune_batch.argtypes = [vp, vp, u32, u32, ctypes.POINTER(TuneResult)]
    L.tim_rt_server_create.argtypes = [vp, ctypes.POINTER(ServerParams), ctypes.POINTER(vp)]
    L.tim_rt_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(u64)]
    L.tim_rt_server_submit_probes.argtypes = [vp, ctypes.POINTER(ProbeRequest), ctypes.POINTER(u64)]
    L.tim_rt_server_wait.argtypes = [vp, u64, u32]
    L.tim_rt_server_cancel.argtypes = [vp, u64]
    L.tim_rt_server_drain.argtypes = [vp, u32]
    L.tim_rt_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats), i32]
    L.tim_rt_server_destroy.argtypes = [vp]
    L.tim_rt_verify_hits.argtypes = [vp, u32, vp, u32, vp, ctypes.POINTER(VerifyResult)]
    L.tim_rt_bvh_file_write.argtypes = [ctypes.c_char_p, vp, u64, vp, ctypes.POINTER(PushConstants), vp, vp, vp, vp,
                                        u32, u32]
    L.tim_rt_bvh_file_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
    L.tim_rt_bvh_file_info.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(u64), vp, ctypes.POINTER(PushConstants),
                                       vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                       ctypes.POINTER(u32), ctypes.POINTER(u32)]
    L.tim_rt_bvh_file_free.argtypes = [vp]
    L.tim_rt_bvh_file_free.restype = None
    L.tim_rt_upload_bvh_file.argtypes = [vp, ctypes.c_char_p, u32, ctypes.POINTER(u32)]
    L.tim_rt_shade_camera.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, ctypes.POINTER(Stats)]
    L.tim_rt_build_bvh_gpu.argtypes = [vp, vp, u32, vp, u32, vp, u32, vp, u32, ctypes.POINTER(BuildParams),
                                       ctypes.POINTER(vp)]
    L.tim_rt_shade_camera_dev.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp]
    L.tim_rt_probe_directions.argtypes = [u32, u32, u64, vp, vp]
    L.tim_rt_wide_check.argtypes = [vp, u64, vp, ctypes.POINTER(PushConstants), vp, u32, ctypes.POINTER(WideReport)]
    for name in EXPORTED:
        if name not in ("tim_rt_version", "tim_rt_last_error", "tim_rt_build_params_default", "tim_rt_bvh_blob_free",
                        "tim_rt_bvh_file_free"):
            getattr(L, name).restype = i32
    _lib = L
    return L


def _check(rc: int):
    if rc != OK:
        raise TimRtError(rc, lib().tim_rt_last_error().decode())


def _host_buf(a, dtype, count: int, name: str):
    """A caller-provided host array that the C call reads or writes `count` elements
    of: checked (type, layout, size) and passed as it is, never copied."""
    if not isinstance(a, np.ndarray) or a.dtype != np.dtype(dtype) or not a.flags["C_CONTIGUOUS"] or a.size < count:
        raise ValueError(f"{name}: needs a C-contiguous {np.dtype(dtype).name} array of at least {count} elements")
    return a


def _need_bytes(a, nbytes: int, name: str) -> None:
    """A caller-provided host buffer (numpy array or torch tensor, any element
    type) that the request reads or writes `nbytes` of."""
    if a is None:
        return
    have = a.nbytes if isinstance(a, np.ndarray) else (a.numel() * a.element_size() if hasattr(a, "numel") else None)
    contiguous = a.flags["C_CONTIGUOUS"] if isinstance(a, np.ndarray) else (a.is_contiguous() if hasattr(a, "is_contiguous") else True)
    if have is None or have < nbytes or not contiguous:
        raise ValueError(f"{name}: needs a contiguous buffer of at least {nbytes} bytes")


def _ray_records(rays) -> np.ndarray:
    """Rays as the C ABI reads them: 32-byte records, float32 [n, 8] (flags as raw
    u32 bits in column 7)."""
    r = np.ascontiguousarray(rays, np.float32)
    if r.ndim != 2 or r.shape[1] != 8:
        raise ValueError(f"rays: needs shape [n, 8] (32-byte tim_rt_ray records), got {r.shape}")
    return r


def _copy_bytes(ptr: int, n: int) -> np.ndarray:
    """A uint8 copy of n bytes at a C pointer (one copy, no intermediate bytes object)."""
    if n == 0:
        return np.zeros(0, np.uint8)
    return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(n,)).copy()


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    if hasattr(a, "data_ptr"):   # torch tensor (host or device)
        return a.data_ptr()
    return int(a)


@dataclass
class BvhImage:
    """A BVHBuilder::fillGpuBuffer-layout image: bytes, 7 {offset, size} ranges in
    memory order (blas, tri, prim, mat, light, node, leaf), push constants, AABB."""
    data: np.ndarray        # uint8
    ranges: np.ndarray      # uint32 [7, 2]
    pc: tuple               # (numTriangles, numBlas, numPrimitives, numLights, numNodes)
    aabb: np.ndarray        # float32 [6]

    @property
    def num_nodes(self) -> int:
        return int(self.pc[4])

    def nodes(self) -> np.ndarray:
        o, _ = self.ranges[RANGE_NODE]
        return self.data[o:o + 64 * self.num_nodes].view(np.uint32).reshape(-1, 16)

    def leaf_words(self) -> np.ndarray:
        o, s = self.ranges[RANGE_LEAF]
        return self.data[o:o + s].view(np.uint32)


def validate(img: BvhImage, num_vertex: int) -> int:
    """tim_rt_validate_bvh: raises TimRtError(EINVAL) on a malformed image, returns the tree depth."""
    pc = PushConstants(*[int(x) for x in img.pc])
    depth = ctypes.c_uint32()
    ranges = np.ascontiguousarray(img.ranges, np.uint32)
    data = np.ascontiguousarray(img.data, np.uint8)
    _check(lib().tim_rt_validate_bvh(data.ctypes.data, data.nbytes, ranges.ctypes.data, ctypes.byref(pc), num_vertex,
                                     ctypes.byref(depth)))
    return depth.value


class WideReport(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_uint32), ("depth", ctypes.c_uint32), ("triangles", ctypes.c_uint32),
                ("leaf_slots", ctypes.c_uint32), ("internal_slots", ctypes.c_uint32),
                ("slot_histogram", ctypes.c_uint32 * 9), ("reserved", ctypes.c_uint32 * 2),
                ("device_bytes", ctypes.c_uint64)]


def wide_check(img: BvhImage, positions) -> dict:
    """tim_rt_wide_check: builds the 8-wide quantised form on the host as the upload
    does and checks it against the binary tree; raises TimRtError(EINVAL) on the
    first violation, returns the report as a dict."""
    pc = PushConstants(*[int(x) for x in img.pc])
    ranges = np.ascontiguousarray(img.ranges, np.uint32)
    data = np.ascontiguousarray(img.data, np.uint8)
    pos = np.ascontiguousarray(positions, np.float32)
    r = WideReport()
    _check(lib().tim_rt_wide_check(data.ctypes.data, data.nbytes, ranges.ctypes.data, ctypes.byref(pc),
                                   pos.ctypes.data, pos.size // 3, ctypes.byref(r)))
    return {"nodes": r.nodes, "depth": r.depth, "triangles": r.triangles, "leaf_slots": r.leaf_slots,
            "internal_slots": r.internal_slots, "slot_histogram": list(r.slot_histogram),
            "device_bytes": int(r.device_bytes)}


def measure_l2_gbs(device: int = 0, nbytes: int = 32 << 20, passes: int = 50) -> float:
    v = ctypes.c_float()
    _check(lib().tim_rt_measure_l2_bandwidth(device, nbytes, passes, ctypes.byref(v)))
    return float(v.value)


def build_params(**kw) -> BuildParams:
    p = BuildParams()
    lib().tim_rt_build_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def build_bvh(scene, ctx: "Context" = None, **params) -> BvhImage:
    """Product-side builder over a scenes.Scene: tim_rt_build_bvh (binned SAH on the
    host), or tim_rt_build_bvh_gpu on ctx's GPU when a context is given."""
    L = lib()
    pos = np.ascontiguousarray(scene.positions, np.float32)
    rec = np.ascontiguousarray(scene.tri_records())
    mats = scene.materials_bytes()
    lights = scene.packed_lights_bytes()
    nmat = len(mats) // 48
    nl = len(lights) // 56
    p = build_params(**params)
    out = ctypes.c_void_p()
    if ctx is not None:
        _check(L.tim_rt_build_bvh_gpu(ctx._c, pos.ctypes.data, pos.shape[0], rec.ctypes.data, rec.shape[0], mats, nmat,
                                      lights if nl else None, nl, ctypes.byref(p), ctypes.byref(out)))
    else:
        _check(L.tim_rt_build_bvh(pos.ctypes.data, pos.shape[0], rec.ctypes.data, rec.shape[0], mats, nmat,
                                  lights if nl else None, nl, ctypes.byref(p), ctypes.byref(out)))
    return _take_blob(L, out)


def build_bvh_tlas(scene, tlas_max_leaf: int = 2, **params) -> BvhImage:
    """tim_rt_build_bvh_tlas over a scenes.Scene: one BLAS instance per chunk, a
    top level over the instances (trace with MODE_ANY | TRACE_TLAS)."""
    L = lib()
    pos = np.ascontiguousarray(scene.positions, np.float32)
    rec = np.ascontiguousarray(scene.tri_records())
    first = np.ascontiguousarray(scene.chunks[:, 2], np.uint32)
    count = np.ascontiguousarray(scene.chunks[:, 3], np.uint32)
    mats = scene.materials_bytes()
    lights = scene.packed_lights_bytes()
    nl = len(lights) // 56
    p = build_params(**params)
    out = ctypes.c_void_p()
    _check(L.tim_rt_build_bvh_tlas(pos.ctypes.data, pos.shape[0], rec.ctypes.data, rec.shape[0], first.ctypes.data,
                                   count.ctypes.data, len(first), mats, len(mats) // 48, lights if nl else None, nl,
                                   ctypes.byref(p), tlas_max_leaf, ctypes.byref(out)))
    return _take_blob(L, out)


def _take_blob(L, out) -> BvhImage:
    """Wraps a tim_rt_bvh_blob as a BvhImage without copying its bytes: the image's
    data array reads the blob's memory, and the blob is freed when the last array
    over it is collected (freed at once when there is nothing to wrap)."""
    try:
        bp, size = ctypes.c_void_p(), ctypes.c_uint64()
        ranges = np.zeros((7, 2), np.uint32)
        pc = PushConstants()
        aabb = np.zeros(6, np.float32)
        _check(L.tim_rt_bvh_blob_info(out, ctypes.byref(bp), ctypes.byref(size), ranges.ctypes.data, ctypes.byref(pc),
                                      aabb.ctypes.data))
    except BaseException:
        L.tim_rt_bvh_blob_free(out)
        raise
    if size.value == 0 or not bp.value:
        L.tim_rt_bvh_blob_free(out)
        data = np.zeros(0, np.uint8)
    else:
        buf = (ctypes.c_uint8 * size.value).from_address(bp.value)
        weakref.finalize(buf, L.tim_rt_bvh_blob_free, ctypes.c_void_p(out.value))
        data = np.frombuffer(buf, np.uint8)
    return BvhImage(data, ranges, (pc.numTriangles, pc.numBlas, pc.numPrimitives, pc.numLights, pc.numNodes), aabb)


DIRS_STRATIFIED, DIRS_OCTAHEDRAL = 0, 1


def probe_directions(count: int, kind: int = DIRS_STRATIFIED, seed: int = 0):
    """tim_rt_probe_directions: (dirs float32 [count, 4], SH9 basis float32 [count, 9])."""
    dirs = np.zeros((count, 4), np.float32)
    basis = np.zeros((count, 9), np.float32)
    _check(lib().tim_rt_probe_directions(count, kind, seed, dirs.ctypes.data, basis.ctypes.data))
    return dirs, basis


def save_bvh_file(path, img: BvhImage, positions, normals=None, uvs=None) -> None:
    """tim_rt_bvh_file_write: the BVH image and the vertex arrays to a versioned file."""
    pos = np.ascontiguousarray(positions, np.float32)
    nrm = np.ascontiguousarray(normals, np.float32) if normals is not None else None
    uv = np.ascontiguousarray(uvs, np.float32) if uvs is not None else None
    ranges = np.ascontiguousarray(img.ranges, np.uint32)
    aabb = np.ascontiguousarray(img.aabb, np.float32)
    pc = PushConstants(*[int(x) for x in img.pc])
    data = np.ascontiguousarray(img.data, np.uint8)
    _check(lib().tim_rt_bvh_file_write(str(path).encode(), data.ctypes.data, data.nbytes, ranges.ctypes.data,
                                       ctypes.byref(pc), aabb.ctypes.data, pos.ctypes.data, _ptr(nrm), _ptr(uv),
                                       pos.shape[0], pos.shape[0]))


def load_bvh_file(path):
    """tim_rt_bvh_file_read: (BvhImage, positions, normals or None, uvs or None), copied out of the file."""
    L = lib()
    f = ctypes.c_void_p()
    _check(L.tim_rt_bvh_file_read(str(path).encode(), ctypes.byref(f)))
    try:
        bp, size = ctypes.c_void_p(), ctypes.c_uint64()
        ranges = np.zeros((7, 2), np.uint32)
        pc = PushConstants()
        aabb = np.zeros(6, np.float32)
        pp, pn, pu = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        mx, nv = ctypes.c_uint32(), ctypes.c_uint32()
        _check(L.tim_rt_bvh_file_info(f, ctypes.byref(bp), ctypes.byref(size), ranges.ctypes.data, ctypes.byref(pc),
                                      aabb.ctypes.data, ctypes.byref(pp), ctypes.byref(pn), ctypes.byref(pu),
                                      ctypes.byref(mx), ctypes.byref(nv)))
        data = _copy_bytes(bp.value, size.value)
        n = nv.value

        def arr(ptr, k):
            if not ptr.value:
                return None
            return np.frombuffer(ctypes.string_at(ptr.value, 4 * k * n), dtype=np.float32).reshape(n, k).copy()

        pos, nrm, uv = arr(pp, 3), arr(pn, 3), arr(pu, 2)
    finally:
        L.tim_rt_bvh_file_free(f)
    img = BvhImage(data, ranges, (pc.numTriangles, pc.numBlas, pc.numPrimitives, pc.numLights, pc.numNodes), aabb)
    return img, pos, nrm, uv


class Context:
    """A tim_rt_ctx: one device, one CUDA stream, resident scenes."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        self._L = lib()
        self._c = ctypes.c_void_p()
        _check(self._L.tim_rt_create(device, mem_budget_bytes, ctypes.byref(self._c)))

    def close(self):
        if self._c:
            self._L.tim_rt_destroy(self._c)
            self._c = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._c

    def launch_config(self) -> dict:
        c = LaunchConfig()
        _check(self._L.tim_rt_get_launch_config(self._c, ctypes.byref(c)))
        return {"block": c.block, "stack_depth": c.stack_depth, "refill_min": c.refill_min, "ray_sort": c.ray_sort,
                "phase_switch": c.phase_switch}

    def set_launch_config(self, block: int = 256, stack_depth: int = 0, refill_min: int = 16, ray_sort: int = 0,
                          phase_switch: int = 10):
        c = LaunchConfig(block, stack_depth, refill_min, ray_sort, phase_switch)
        _check(self._L.tim_rt_set_launch_config(self._c, ctypes.byref(c)))

    def verify_hits(self, sid: int, d_rays, n: int, d_hit) -> dict:
        """tim_rt_verify_hits: FP64 re-intersection of closest-hit records (device buffers)."""
        r = VerifyResult()
        _check(self._L.tim_rt_verify_hits(self._c, sid, _ptr(d_rays), n, _ptr(d_hit), ctypes.byref(r)))
        return {name: getattr(r, name) for name, _ in VerifyResult._fields_}

    # -- batched multi-scene trace
    def batch_create(self, jobs, wide: bool = False):
        """jobs: iterable of (scene_id, mode, n, d_rays, d_hit, d_leaf_nid, d_bary); device buffers are
        torch tensors or raw pointers. Returns an opaque batch handle."""
        jobs = list(jobs)
        arr = (Job * max(1, len(jobs)))()
        for i, (sid, mode, n, r, h, nid, bary) in enumerate(jobs):
            arr[i] = Job(sid, mode, n, 0, _ptr(r), _ptr(h), _ptr(nid), _ptr(bary))
        out = ctypes.c_void_p()
        _check(self._L.tim_rt_batch_create(self._c, arr, len(jobs), BATCH_WIDE if wide else 0, ctypes.byref(out)))
        return out

    def batch_launch(self, batch, stream=None):
        _check(self._L.tim_rt_batch_launch(self._c, batch, _ptr(stream) if stream is not None else None))

    def batch_info(self, batch) -> tuple:
        rays, nbytes = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self._L.tim_rt_batch_info(self._c, batch, ctypes.byref(rays), ctypes.byref(nbytes)))
        return rays.value, nbytes.value

    def batch_destroy(self, batch):
        _check(self._L.tim_rt_batch_destroy(self._c, batch))

    def autotune_batch(self, batch, width: bool = False, reps: int = 3) -> dict:
        r = TuneResult()
        _check(self._L.tim_rt_autotune_batch(self._c, batch, TUNE_WIDTH if width else 0, reps, ctypes.byref(r)))
        return {"block": r.best.block, "stack_depth": r.best.stack_depth, "refill_min": r.best.refill_min,
                "ray_sort": r.best.ray_sort, "phase_switch": r.best.phase_switch, "wide": bool(r.wide),
                "tried": r.tried, "best_ms": r.best_ms,
                "start_ms": r.start_ms}

    def memory_used(self) -> int:
        v = ctypes.c_uint64()
        _check(self._L.tim_rt_memory_used(self._c, ctypes.byref(v)))
        return v.value

    def upload(self, img: BvhImage, scene, quant8: bool = False) -> int:
        pos = np.ascontiguousarray(scene.positions, np.float32)
        nrm = np.ascontiguousarray(scene.normals, np.float32)
        pc = PushConstants(*[int(x) for x in img.pc])
        sid = ctypes.c_uint32()
        ranges = np.ascontiguousarray(img.ranges, np.uint32)
        _check(self._L.tim_rt_upload_bvh(self._c, img.data.ctypes.data, img.data.nbytes, ranges.ctypes.data,
                                         pos.ctypes.data, nrm.ctypes.data, None, pos.shape[0], pos.shape[0],
                                         ctypes.byref(pc), UPLOAD_QUANT8 if quant8 else 0, ctypes.byref(sid)))
        return sid.value

    def upload_file(self, path, quant8: bool = False) -> int:
        """tim_rt_upload_bvh_file: a scene straight from a BVH file."""
        sid = ctypes.c_uint32()
        _check(self._L.tim_rt_upload_bvh_file(self._c, str(path).encode(), UPLOAD_QUANT8 if quant8 else 0,
                                              ctypes.byref(sid)))
        return sid.value

    def free_scene(self, sid: int):
        _check(self._L.tim_rt_free_scene(self._c, sid))

    def scene_bytes(self, sid: int) -> int:
        v = ctypes.c_uint64()
        _check(self._L.tim_rt_scene_bytes(self._c, sid, ctypes.byref(v)))
        return v.value

    def trace(self, sid: int, rays: np.ndarray, mode: int = MODE_CLOSEST, want_nid=True, want_bary=True,
              hit=None, nid=None, bary=None):
        rays = _ray_records(rays)
        n = rays.shape[0]
        hit = np.empty((n, 4), np.uint32) if hit is None else _host_buf(hit, np.uint32, 4 * n, "hit")
        nid = (np.empty(n, np.uint32) if want_nid else None) if nid is None else _host_buf(nid, np.uint32, n, "nid")
        bary = ((np.empty((n, 2), np.float32) if want_bary else None) if bary is None
                else _host_buf(bary, np.float32, 2 * n, "bary"))
        st = Stats()
        _check(self._L.tim_rt_trace(self._c, sid, rays.ctypes.data, n, mode, _ptr(hit), _ptr(nid), _ptr(bary),
                                    ctypes.byref(st)))
        return hit, nid, bary, st

    def trace_dev(self, sid: int, d_rays, n: int, mode: int, d_hit, d_nid=None, d_bary=None, stream=None):
        _check(self._L.tim_rt_trace_dev(self._c, sid, _ptr(d_rays), n, mode, _ptr(d_hit), _ptr(d_nid), _ptr(d_bary),
                                        _ptr(stream) if stream is not None else None))

    def cull_lights(self, sid: int, pd: np.ndarray, tiles_x: int, tiles_y: int):
        counts = np.empty(tiles_x * tiles_y, np.uint32)
        lists = np.empty((tiles_x * tiles_y, 16), np.uint32)
        pd = np.ascontiguousarray(pd)
        _check(self._L.tim_rt_cull_lights(self._c, sid, pd.ctypes.data, tiles_x, tiles_y, counts.ctypes.data,
                                          lists.ctypes.data))
        return counts, lists

    def cull_lights_dev(self, sid: int, pd: np.ndarray, tiles_x: int, tiles_y: int, d_counts, d_lists, stream=None):
        pd = np.ascontiguousarray(pd)
        _check(self._L.tim_rt_cull_lights_dev(self._c, sid, pd.ctypes.data, tiles_x, tiles_y, _ptr(d_counts),
                                              _ptr(d_lists), _ptr(stream) if stream is not None else None))

    def trace_camera_dev(self, sid: int, pd: np.ndarray, flags: int, seed: int, d_tile_counts, d_tile_lists, d_out,
                         d_bounce=None, d_ray_count=None, stream=None):
        pd = np.ascontiguousarray(pd)
        _check(self._L.tim_rt_trace_camera_dev(self._c, sid, pd.ctypes.data, flags, seed, _ptr(d_tile_counts),
                                               _ptr(d_tile_lists), _ptr(d_out), _ptr(d_bounce), _ptr(d_ray_count),
                                               _ptr(stream) if stream is not None else None))

    def trace_camera_rows_dev(self, sid: int, pd: np.ndarray, flags: int, seed: int, row_begin: int, row_end: int,
                              d_tile_counts, d_tile_lists, d_out, d_bounce=None, d_ray_count=None, stream=None):
        """tim_rt_trace_camera_rows_dev: output rows [row_begin, row_end) of the frame
        into the whole frame's device arrays."""
        pd = np.ascontiguousarray(pd)
        _check(self._L.tim_rt_trace_camera_rows_dev(self._c, sid, pd.ctypes.data, flags, seed, row_begin, row_end,
                                                    _ptr(d_tile_counts), _ptr(d_tile_lists), _ptr(d_out),
                                                    _ptr(d_bounce), _ptr(d_ray_count),
                                                    _ptr(stream) if stream is not None else None))

    def update_probes(self, sid: int, desc: ProbeDesc, dirs: np.ndarray, sh_basis: np.ndarray, sh16: np.ndarray,
                      probe_begin: int = 0, probe_end: int = None, want_trace=False, want_irr=False, want_sh32=False,
                      want_octa=False):
        """tim_rt_update_probes. sh16 (uint16 [7, rz, ry, rx, 4]) is updated in place."""
        res = [int(desc.resolution[i]) for i in range(3)]
        total = res[0] * res[1] * res[2]
        probe_end = total if probe_end is None else probe_end
        np_ = probe_end - probe_begin
        nd = int(desc.num_dirs)
        _host_buf(sh16, np.uint16, 7 * total * 4, "sh16")
        dirs = np.ascontiguousarray(dirs, np.float32)
        basis = np.ascontiguousarray(sh_basis, np.float32)
        if dirs.size < 4 * nd or basis.size < 9 * nd:
            raise ValueError(f"dirs / sh_basis: need {nd} directions (float4) and {nd} x 9 basis weights")
        tr = np.empty((np_, nd, 8), np.uint32) if want_trace else None
        irr = np.empty((np_, nd, 3), np.float32) if want_irr else None
        s32 = np.empty((np_, 9, 3), np.float32) if want_sh32 else None
        octa = np.empty((np_, 64, 3), np.float32) if want_octa else None
        st = Stats()
        _check(self._L.tim_rt_update_probes(self._c, sid, ctypes.byref(desc), dirs.ctypes.data, basis.ctypes.data,
                                            probe_begin, probe_end, _ptr(tr), _ptr(irr), sh16.ctypes.data, _ptr(s32),
                                            _ptr(octa), ctypes.byref(st)))
        return tr, irr, s32, octa, st

    def shade_camera(self, sid: int, pd: np.ndarray, tracing: np.ndarray, sh16=None, flags: int = 0,
                     want_f32: bool = False):
        """tim_rt_shade_camera: (RGBA16F u16 [W*H, 4], FP32 rgb [W*H, 3] or None, Stats)."""
        W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
        pd = np.ascontiguousarray(pd)
        tr = np.ascontiguousarray(tracing, np.uint32)
        if tr.size < 8 * W * H:
            raise ValueError(f"tracing: needs the {W}x{H} frame's 32-byte records ({8 * W * H} words)")
        sh = np.ascontiguousarray(sh16, np.uint16) if sh16 is not None else None
        if sh is not None:
            lres = [int(x) for x in np.asarray(pd["lpfResolution"]).reshape(-1)[:3]]
            _host_buf(sh, np.uint16, 7 * lres[0] * lres[1] * lres[2] * 4, "sh16")
        out = np.empty((W * H, 4), np.uint16)
        f32 = np.empty((W * H, 3), np.float32) if want_f32 else None
        st = Stats()
        _check(self._L.tim_rt_shade_camera(self._c, sid, pd.ctypes.data, flags, tr.ctypes.data, _ptr(sh),
                                           out.ctypes.data, _ptr(f32), ctypes.byref(st)))
        return out, f32, st

    def trace_camera(self, sid: int, pd: np.ndarray, flags: int = 0, seed: int = 0, tile_counts=None, tile_lists=None,
                     out=None, bounce_out=None):
        W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
        out = np.empty((W * H, 8), np.uint32) if out is None else _host_buf(out, np.uint32, 8 * W * H, "out")
        if (flags & CAM_BOUNCE) and bounce_out is None:
            bounce_out = np.empty((W * H, 4), np.uint32)
        elif bounce_out is not None:
            _host_buf(bounce_out, np.uint32, 4 * W * H, "bounce_out")
        tiles = ((W + 15) // 16) * ((H + 15) // 16)
        if tile_counts is not None:
            _host_buf(tile_counts, np.uint32, tiles, "tile_counts")
        if tile_lists is not None:
            _host_buf(tile_lists, np.uint32, 16 * tiles, "tile_lists")
        st = Stats()
        pd = np.ascontiguousarray(pd)
        _check(self._L.tim_rt_trace_camera(self._c, sid, pd.ctypes.data, flags, seed, _ptr(tile_counts),
                                           _ptr(tile_lists), _ptr(out), _ptr(bounce_out), ctypes.byref(st)))
        return out, bounce_out, st


class Server:
    """tim_rt_server_*: a serving loop over a context's resident scenes. Host
    buffers passed to submit() are kept referenced until the request completes."""

    def __init__(self, ctx: "Context", memory_budget_bytes: int = 1 << 30, max_rays_per_step: int = 0,
                 max_inflight_steps: int = 0, max_jobs_per_step: int = 0, wide: bool = False):
        self._L = lib()
        self._ctx = ctx
        p = ServerParams(memory_budget_bytes, max_rays_per_step, max_inflight_steps, max_jobs_per_step,
                         BATCH_WIDE if wide else 0)
        h = ctypes.c_void_p()
        _check(self._L.tim_rt_server_create(ctx._c, ctypes.byref(p), ctypes.byref(h)))
        self._s = h
        self._keep = {}

    def submit(self, sid: int, rays, mode: int, hit, nid=None, bary=None) -> int:
        n = int(rays.shape[0])
        for buf, per, name in ((rays, 32, "rays"), (hit, 16, "hit"), (nid, 4, "nid"), (bary, 8, "bary")):
            _need_bytes(buf, per * n, name)
        r = Request(sid, mode, n, 0, _ptr(rays), _ptr(hit), _ptr(nid), _ptr(bary))
        t = ctypes.c_uint64()
        _check(self._L.tim_rt_server_submit(self._s, ctypes.byref(r), ctypes.byref(t)))
        self._keep[t.value] = (rays, hit, nid, bary)
        return t.value

    def submit_probes(self, sid: int, desc: "ProbeDesc", dirs, sh_basis, sh16, probe_begin: int, probe_end: int,
                      octa=None) -> int:
        """A probe-field update request (tim_rt_server_submit_probes): sh16 (uint16
        [7][rz][ry][rx][4], host) is read at admission and rewritten on completion;
        octa (float32 [probes][64][3]) is optional."""
        dirs = np.ascontiguousarray(dirs, np.float32)
        basis = np.ascontiguousarray(sh_basis, np.float32)
        res = [int(desc.resolution[i]) for i in range(3)]
        if all(x > 0 and x % 4 == 0 for x in res):   # other grids the library refuses before reading sh16
            _host_buf(sh16, np.uint16, 7 * res[0] * res[1] * res[2] * 4, "sh16")
        nd = int(desc.num_dirs)
        if dirs.size < 4 * nd or basis.size < 9 * nd:
            raise ValueError(f"dirs / sh_basis: need {nd} directions (float4) and {nd} x 9 basis weights")
        if octa is not None:
            _host_buf(octa, np.float32, (probe_end - probe_begin) * 64 * 3, "octa")
        r = ProbeRequest(sid, probe_begin, probe_end, 0, ctypes.cast(ctypes.byref(desc), ctypes.c_void_p), _ptr(dirs),
                         _ptr(basis), _ptr(sh16), _ptr(octa))
        t = ctypes.c_uint64()
        _check(self._L.tim_rt_server_submit_probes(self._s, ctypes.byref(r), ctypes.byref(t)))
        self._keep[t.value] = (desc, dirs, basis, sh16, octa)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 0):
        """tim_rt_server_wait; raises TimRtError (code ECANCELLED for a cancelled request)."""
        rc = self._L.tim_rt_server_wait(self._s, ticket, timeout_ms)
        if rc in (OK, ECANCELLED):
            self._keep.pop(ticket, None)
        _check(rc)

    def cancel(self, ticket: int) -> int:
        """tim_rt_server_cancel: OK (taken back; wait() then raises ECANCELLED), EBUSY
        (too late, completes normally) or ENOTFOUND (unknown or completed)."""
        rc = self._L.tim_rt_server_cancel(self._s, ticket)
        if rc not in (OK, EBUSY, ENOTFOUND):
            _check(rc)
        return rc

    def drain(self, timeout_ms: int = 0):
        _check(self._L.tim_rt_server_drain(self._s, timeout_ms))
        self._keep.clear()

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        _check(self._L.tim_rt_server_stats_get(self._s, ctypes.byref(st), 1 if reset else 0))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if self._s:
            _check(self._L.tim_rt_server_destroy(self._s))
            self._s = None
            self._keep.clear()
