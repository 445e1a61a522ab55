"""oracle/refglsl -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper around oracle/_ref/librefglsl.so: the reference's own compute
shaders (cameraPass.comp in its tracing and lighting steps, genLightProbField.comp,
updateLightProbField.comp and the BVH traversal they include), rewritten mechanically into C++ by
make_refglsl.py and compiled with glsl_shim.h by oracle/Makefile. It is a second
oracle, used only by the tests and the golden-fixture script to pin the C
restatement (oracle/reftrace.c) to the reference's code. Scenes are the same
orc_scene structs as the restatement's (oracle.oracle.Scene).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from oracle.oracle import Scene  # noqa: F401  (same scene struct)

SO = Path(__file__).resolve().parent.parent / "_ref" / "librefglsl.so"
RAYS_PER_PROBE = 64          # NUM_RAYS_PER_PROB, lightprob/lightprob.glsl
_lib = None


def available() -> bool:
    return SO.exists()


def lib():
    global _lib
    if _lib is None:
        if not SO.exists():
            raise FileNotFoundError(f"{SO} is not built (make -C oracle with the reference tree present)")
        L = ctypes.CDLL(str(SO))
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.refglsl_trace.argtypes = [vp, vp, u64, u32, vp, vp]
        L.refglsl_camera.argtypes = [vp, vp, vp]
        L.refglsl_probe_trace.argtypes = [vp, vp, vp, vp]
        L.refglsl_probe_light.argtypes = [vp, vp, vp, vp, vp]
        L.refglsl_probe_update.argtypes = [vp, vp, vp, vp]
        L.refglsl_shade.argtypes = [vp, vp, vp, vp, vp]
        L.refglsl_trace_tlas.argtypes = [vp, vp, u64, vp]
        for f in (L.refglsl_trace, L.refglsl_camera, L.refglsl_probe_trace, L.refglsl_probe_light,
                  L.refglsl_probe_update, L.refglsl_shade, L.refglsl_trace_tlas):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int, what: str) -> None:
    if rc:
        raise RuntimeError(f"refglsl {what}: shader copy reported error bits {rc:#x}")


def trace(sc, rays: np.ndarray, mode: int = 0):
    """(hit records [n,4] u32, nid [n] u32) with the contract of oracle.trace."""
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hit = np.zeros((n, 4), np.uint32)
    nid = np.zeros(n, np.uint32)
    _check(lib().refglsl_trace(sc.ref, _ptr(rays), n, mode, _ptr(hit), _ptr(nid)), "trace")
    return hit, nid


def trace_tlas(sc, rays: np.ndarray) -> np.ndarray:
    """Any-hit rays through the USE_TRAVERSE_TLAS shader (traverseForShadow): hit
    records [n,4] u32 = (occluded, 0, 0, bits(tmax)), as oracle.trace reports them."""
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hit = np.zeros((n, 4), np.uint32)
    _check(lib().refglsl_trace_tlas(sc.ref, _ptr(rays), n, _ptr(hit)), "trace_tlas")
    return hit


def camera(sc, pd: np.ndarray) -> np.ndarray:
    """cameraPass.comp tracing step (probe mask on): [W*H, 8] u32 = g_tracingData."""
    pd = np.ascontiguousarray(pd)
    W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
    out = np.zeros((W * H, 8), np.uint32)
    _check(lib().refglsl_camera(sc.ref, _ptr(pd), _ptr(out)), "camera")
    return out


def probe_trace(sc, desc, dirs: np.ndarray) -> np.ndarray:
    """genLightProbField.comp tracing step over every probe: [probes*64, 8] u32."""
    dirs = np.ascontiguousarray(dirs, np.float32).reshape(RAYS_PER_PROBE, 4)
    n = int(desc.resolution[0] * desc.resolution[1] * desc.resolution[2]) * RAYS_PER_PROBE
    out = np.zeros((n, 8), np.uint32)
    _check(lib().refglsl_probe_trace(sc.ref, ctypes.byref(desc), _ptr(dirs), _ptr(out)), "probe_trace")
    return out


def probe_light(sc, desc, dirs: np.ndarray, trace_records: np.ndarray) -> np.ndarray:
    """genLightProbField.comp lighting step: [probes*64, 3] f32 lit values."""
    dirs = np.ascontiguousarray(dirs, np.float32).reshape(RAYS_PER_PROBE, 4)
    tr = np.ascontiguousarray(trace_records, np.uint32)
    irr = np.zeros((tr.shape[0], 3), np.float32)
    _check(lib().refglsl_probe_light(sc.ref, ctypes.byref(desc), _ptr(dirs), _ptr(tr), _ptr(irr)), "probe_light")
    return irr


def probe_update(desc, sh_basis: np.ndarray, irradiance: np.ndarray, images16: np.ndarray) -> np.ndarray:
    """updateLightProbField.comp: returns the 7 rgba16f images (u16 bits) after the update."""
    b = np.ascontiguousarray(sh_basis, np.float32)
    irr = np.ascontiguousarray(irradiance, np.float32)
    img = np.array(images16, np.uint16, copy=True, order="C")
    _check(lib().refglsl_probe_update(ctypes.byref(desc), _ptr(b), _ptr(irr), _ptr(img)), "probe_update")
    return img


def shade(sc, pd: np.ndarray, tracing: np.ndarray, sh16: np.ndarray) -> np.ndarray:
    """cameraPass.comp lighting step (USE_LPF, USE_LPF_MASK): RGBA16F [W*H, 4] as u16."""
    pd = np.ascontiguousarray(pd)
    W, H = (int(x) for x in np.asarray(pd["frameSize"]).reshape(-1)[:2])
    tr = np.ascontiguousarray(tracing, np.uint32)
    sh = np.ascontiguousarray(sh16, np.uint16)
    out = np.zeros((W * H, 4), np.uint16)
    _check(lib().refglsl_shade(sc.ref, _ptr(pd), _ptr(tr), _ptr(sh), _ptr(out)), "shade")
    return out
