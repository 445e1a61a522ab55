"""oracle/oracle.py -- TEST INFRASTRUCTURE ONLY.

ctypes wrappers around
  * oracle/lib/liboracle.so       -- the C restatement of the reference's GLSL
                                     traversal (oracle/reftrace.c), and
  * oracle/_ref/libtimref_build.so -- the reference's own CPU BVH builder
                                     compiled from its sources (oracle/Makefile).
Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as a checker / baseline. The shipped library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from collections import namedtuple
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "lib" / "liboracle.so"
REFBUILD_SO = HERE / "_ref" / "libtimref_build.so"

Image = namedtuple("Image", "data ranges pc aabb")   # same fields as tim_raytracing_b200.BvhImage


# orc_trace modes (oracle/reftrace.h); ORC_MODE_TLAS is or'ed into the mode
ORC_MODE_CLOSEST, ORC_MODE_ANY, ORC_MODE_PER_RAY, ORC_MODE_TLAS = 0, 1, 2, 4

# Where this container keeps the reference's source tree (read-only). Only the
# build recipe reads it; the GPU box has no such tree and uses the prebuilt _ref.
REFERENCE_TREE = Path(os.environ.get("TIM_RT_REFERENCE_TREE", "/root/reference"))


def build(quiet: bool = True) -> None:
    """Compiles the restatement, and the reference builder and shaders when the
    reference tree is present."""
    cmd = ["make", "-C", str(HERE)]
    if (REFERENCE_TREE / "src" / "Renderer" / "BVHBuilder.cpp").exists():
        cmd.append(f"REF={REFERENCE_TREE}")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(r.stdout)


class OrcScene(ctypes.Structure):
    _fields_ = [("blob", ctypes.c_void_p), ("blob_size", ctypes.c_uint64), ("ranges", (ctypes.c_uint32 * 2) * 7),
                ("pos", ctypes.c_void_p), ("nrm", ctypes.c_void_p), ("num_vertex", ctypes.c_uint32),
                ("num_nodes", ctypes.c_uint32), ("num_lights", ctypes.c_uint32)]


class OrcProbeDesc(ctypes.Structure):
    _fields_ = [("aabbMin", ctypes.c_float * 4), ("aabbMax", ctypes.c_float * 4), ("resolution", ctypes.c_uint32 * 4),
                ("sunDir", ctypes.c_float * 4), ("sunColor", ctypes.c_float * 4), ("hysteresis", ctypes.c_float),
                ("num_dirs", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class RefResult(ctypes.Structure):
    _fields_ = [("blob", ctypes.c_void_p), ("blob_size", ctypes.c_uint64), ("ranges", (ctypes.c_uint32 * 2) * 7),
                ("num_triangles", ctypes.c_uint32), ("num_blas", ctypes.c_uint32), ("num_primitives", ctypes.c_uint32),
                ("num_lights", ctypes.c_uint32), ("num_nodes", ctypes.c_uint32), ("aabb_min", ctypes.c_float * 3),
                ("aabb_max", ctypes.c_float * 3), ("vertex_offsets_count", ctypes.c_uint32),
                ("vertex_offsets", ctypes.c_void_p)]


class RefParams(ctypes.Structure):
    _fields_ = [("maxDepth", ctypes.c_uint32), ("minObjPerNode", ctypes.c_uint32), ("minObjGain", ctypes.c_uint32),
                ("expandNodeVolumeThreshold", ctypes.c_float), ("expandNodeDimensionFactor", ctypes.c_float)]


_orc = None
_ref = None


def orc():
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build()
        L = ctypes.CDLL(str(ORACLE_SO))
        vp, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        L.orc_trace.argtypes = [vp, vp, u64, u32, vp, vp, vp, vp, i32]
        L.orc_trace.restype = None
        L.orc_camera.argtypes = [vp, vp, u32, u32, vp, vp, vp, vp, vp, u64, u64, i32]
        L.orc_camera.restype = None
        L.orc_cull_lights.argtypes = [vp, vp, u32, u32, vp, vp, i32]
        L.orc_cull_lights.restype = None
        L.orc_probe_trace.argtypes = [vp, vp, vp, u32, u32, vp, vp, vp, i32]
        L.orc_probe_trace.restype = None
        L.orc_probe_sh9.argtypes = [vp, vp, vp, u32, u32, vp, vp]
        L.orc_probe_sh9.restype = None
        L.orc_probe_octa.argtypes = [vp, vp, u32, u32, vp]
        L.orc_probe_octa.restype = None
        L.orc_bounce_dir.argtypes = [vp, u32, u32, vp]
        L.orc_bounce_dir.restype = None
        L.orc_shade_camera.argtypes = [vp, vp, u32, vp, vp, vp, vp, i32]
        L.orc_shade_camera.restype = None
        L.orc_hash32.argtypes = [u32]
        L.orc_hash32.restype = u32
        _orc = L
    return _orc


def have_refbuild() -> bool:
    return REFBUILD_SO.exists()


def refbuild_lib():
    global _ref
    if _ref is None:
        if not REFBUILD_SO.exists():
            build()
        if not REFBUILD_SO.exists():
            raise RuntimeError("the reference builder is not built (reference tree absent when oracle/ was built)")
        L = ctypes.CDLL(str(REFBUILD_SO))
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        L.timref_build.argtypes = [vp, vp, u32, vp, u32, vp, vp, vp, u32, vp, ctypes.c_int, vp]
        L.timref_build.restype = ctypes.c_int
        L.timref_free.argtypes = [vp]
        L.timref_free.restype = None
        L.timref_default_params.argtypes = [vp]
        L.timref_default_params.restype = None
        _ref = L
    return _ref


def _ref_params(L, params):
    p = RefParams()
    L.timref_default_params(ctypes.byref(p))
    for k, v in params.items():
        setattr(p, k, v)
    return p


def _ref_call(L, scene, build):
    pos = np.ascontiguousarray(scene.positions, np.float32)
    nrm = np.ascontiguousarray(scene.normals, np.float32)
    chunks = np.ascontiguousarray(scene.chunks, np.uint32)
    idx = np.ascontiguousarray(scene.local_idx, np.uint32)
    colors = np.ascontiguousarray(scene.colors, np.float32)
    lights = np.ascontiguousarray(scene.lights, np.float32)
    res = RefResult()
    rc = build(pos.ctypes.data, nrm.ctypes.data, pos.shape[0], chunks.ctypes.data, chunks.shape[0], idx.ctypes.data,
               colors.ctypes.data, lights.ctypes.data if len(lights) else None, len(lights), res)
    if rc != 0:
        raise RuntimeError("the reference builder failed")
    try:
        data = np.frombuffer(ctypes.string_at(res.blob, res.blob_size), np.uint8).copy()
        ranges = np.array([[res.ranges[i][0], res.ranges[i][1]] for i in range(7)], np.uint32)
        voffs = np.frombuffer(ctypes.string_at(res.vertex_offsets, 4 * res.vertex_offsets_count), np.uint32)
        assert np.array_equal(voffs, scene.chunks[:, 0]), "vertex offsets differ from the chunk layout"
        pc = (res.num_triangles, res.num_blas, res.num_primitives, res.num_lights, res.num_nodes)
        aabb = np.array(list(res.aabb_min) + list(res.aabb_max), np.float32)
    finally:
        L.timref_free(ctypes.byref(res))
    return Image(data, ranges, pc, aabb)


def ref_build(scene, multithread: bool = False, **params) -> Image:
    """Runs the reference's own BVHBuilder (single-threaded by default: its threaded
    build numbers nodes in thread order, BVHBuilder.cpp:851-857,880-894)."""
    L = refbuild_lib()
    p = _ref_params(L, params)
    return _ref_call(L, scene, lambda *a: L.timref_build(*a[:9], ctypes.byref(p), 1 if multithread else 0,
                                                         ctypes.byref(a[9])))


class Scene:
    """Keeps the arrays of one traced scene alive next to its orc_scene struct."""

    def __init__(self, img, positions, normals=None):
        self.data = np.ascontiguousarray(img.data, np.uint8)
        self.pos = np.ascontiguousarray(positions, np.float32)
        self.nrm = np.ascontiguousarray(normals if normals is not None else positions, np.float32)
        self.s = OrcScene()
        self.s.blob = self.data.ctypes.data
        self.s.blob_size = self.data.nbytes
        for i in range(7):
            self.s.ranges[i][0] = int(img.ranges[i][0])
            self.s.ranges[i][1] = int(img.ranges[i][1])
        self.s.pos = self.pos.ctypes.data
        self.s.nrm = self.nrm.ctypes.data
        self.s.num_vertex = self.pos.shape[0]
        self.s.num_nodes = int(img.pc[4])
        self.s.num_lights = int(img.pc[3])

    @property
    def ref(self):
        return ctypes.byref(self.s)


def trace(sc: Scene, rays: np.ndarray, mode: int = 0, threads: int = 0, stats: bool = False):
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hit = np.empty((n, 4), np.uint32)
    nid = np.empty(n, np.uint32)
    bary = np.empty((n, 2), np.float32)
    st = np.empty((n, 4), np.uint32) if stats else None
    orc().orc_trace(sc.ref, rays.ctypes.data, n, mode, hit.ctypes.data, nid.ctypes.data, bary.ctypes.data,
                    st.ctypes.data if stats else None, threads)
    return hit, nid, bary, st


def camera(sc: Scene, pd: np.ndarray, flags: int = 0, seed: int = 0, tile_counts=None, tile_lists=None,
           pix_range=None, threads: int = 0):
    W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
    out = np.zeros((W * H, 8), np.uint32)
    bounce = np.zeros((W * H, 4), np.uint32)
    counts = np.zeros(4, np.uint64)
    b, e = pix_range if pix_range else (0, W * H)
    pd = np.ascontiguousarray(pd)
    tc = np.ascontiguousarray(tile_counts, np.uint32) if tile_counts is not None else None
    tl = np.ascontiguousarray(tile_lists, np.uint32) if tile_lists is not None else None
    orc().orc_camera(sc.ref, pd.ctypes.data, flags, seed, tc.ctypes.data if tc is not None else None,
                     tl.ctypes.data if tl is not None else None, out.ctypes.data, bounce.ctypes.data,
                     counts.ctypes.data, b, e, threads)
    return out, bounce, counts


def shade_camera(sc: Scene, pd: np.ndarray, tracing: np.ndarray, sh16: np.ndarray, no_lpf: bool = False,
                 threads: int = 0):
    """orc_shade_camera: the camera pass's lighting step -> (RGBA16F u16 [W*H, 4], FP32 rgb [W*H, 3])."""
    W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
    pd = np.ascontiguousarray(pd)
    tr = np.ascontiguousarray(tracing, np.uint32)
    sh = np.ascontiguousarray(sh16, np.uint16)
    out = np.zeros((W * H, 4), np.uint16)
    f32 = np.zeros((W * H, 3), np.float32)
    orc().orc_shade_camera(sc.ref, pd.ctypes.data, 1 if no_lpf else 0, tr.ctypes.data, sh.ctypes.data,
                           out.ctypes.data, f32.ctypes.data, threads)
    return out, f32


def cull_lights(sc: Scene, pd: np.ndarray, tiles_x: int, tiles_y: int, threads: int = 0):
    counts = np.empty(tiles_x * tiles_y, np.uint32)
    lists = np.empty((tiles_x * tiles_y, 16), np.uint32)
    pd = np.ascontiguousarray(pd)
    orc().orc_cull_lights(sc.ref, pd.ctypes.data, tiles_x, tiles_y, counts.ctypes.data, lists.ctypes.data, threads)
    return counts, lists


def probe_desc(aabb_min, aabb_max, res, sun_dir, sun_color, num_dirs, hysteresis=0.03) -> OrcProbeDesc:
    d = OrcProbeDesc()
    for i in range(3):
        d.aabbMin[i] = float(aabb_min[i])
        d.aabbMax[i] = float(aabb_max[i])
        d.resolution[i] = int(res[i])
        d.sunDir[i] = float(sun_dir[i])
        d.sunColor[i] = float(sun_color[i])
    d.hysteresis = hysteresis
    d.num_dirs = num_dirs
    return d


def probe_trace(sc: Scene, desc: OrcProbeDesc, dirs: np.ndarray, probe_begin: int, probe_end: int, threads: int = 0):
    nd = desc.num_dirs
    npb = probe_end - probe_begin
    out = np.zeros((npb * nd, 8), np.uint32)
    irr = np.zeros((npb * nd, 3), np.float32)
    counts = np.zeros(4, np.uint64)
    dirs = np.ascontiguousarray(dirs, np.float32)
    orc().orc_probe_trace(sc.ref, ctypes.byref(desc), dirs.ctypes.data, probe_begin, probe_end, out.ctypes.data,
                          irr.ctypes.data, counts.ctypes.data, threads)
    return out, irr, counts


def probe_sh9(desc: OrcProbeDesc, sh_basis: np.ndarray, irr: np.ndarray, probe_begin: int, probe_end: int, prev=None):
    npb = probe_end - probe_begin
    out = np.zeros((npb, 27), np.float32)
    b = np.ascontiguousarray(sh_basis, np.float32)
    irr = np.ascontiguousarray(irr, np.float32)
    pv = np.ascontiguousarray(prev, np.float32) if prev is not None else None
    orc().orc_probe_sh9(ctypes.byref(desc), b.ctypes.data, irr.ctypes.data, probe_begin, probe_end,
                        pv.ctypes.data if pv is not None else None, out.ctypes.data)
    return out


def probe_octa(desc: OrcProbeDesc, irr: np.ndarray, probe_begin: int, probe_end: int):
    npb = probe_end - probe_begin
    out = np.zeros((npb, 64, 3), np.float32)
    irr = np.ascontiguousarray(irr, np.float32)
    orc().orc_probe_octa(ctypes.byref(desc), irr.ctypes.data, probe_begin, probe_end, out.ctypes.data)
    return out


def bounce_dir(n, pixel: int, seed: int) -> np.ndarray:
    nn = np.ascontiguousarray(n, np.float32)
    out = np.empty(3, np.float32)
    orc().orc_bounce_dir(nn.ctypes.data, pixel, seed, out.ctypes.data)
    return out


def threads_available() -> int:
    return len(os.sched_getaffinity(0))
