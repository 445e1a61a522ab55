"""The C-ABI library loads and exports every symbol include/tim_rt.h declares (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(tim_rt_\w+)\s*\(", text):
            syms.add(m.group(1))
    return sorted(syms)


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for name in ("tim_rt_upload_bvh", "tim_rt_trace", "tim_rt_cull_lights", "tim_rt_trace_camera", "tim_rt_create",
                 "tim_rt_destroy", "tim_rt_free_scene"):
        assert name in syms


def test_library_exports_every_declared_symbol(native):
    L = ctypes.CDLL(str(native.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_list_matches_header(native):
    assert sorted(native.EXPORTED) == declared_symbols()


def test_binding_constants_match_header(native):
    """Every flag, mode and error code the bindings name has the header's value."""
    text = "\n".join(h.read_text() for h in (ROOT / "include").glob("*.h"))
    defines = {m.group(1): int(m.group(2), 0)
               for m in re.finditer(r"^#define TIM_RT_(\w+)\s+(0x[0-9a-fA-F]+|\d+)u?\b", text, flags=re.M)}
    checked = 0
    for name, value in defines.items():
        if isinstance(getattr(native, name, None), int):
            assert getattr(native, name) == value, name
            checked += 1
    for name in ("CAM_DEVICE_CULL", "CAM_PIPELINED", "CAM_PRIMARY_BINARY", "TRACE_TLAS", "PROBE_OCTA", "EINVAL"):
        assert name in defines and getattr(native, name) == defines[name], name
    assert checked >= 20


def test_version_and_no_error(native):
    L = native.lib()
    assert b"sm_100a" in L.tim_rt_version()


def test_create_without_gpu_fails_cleanly(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.TimRtError) as e:
        native.Context(0)
    assert e.value.code == native.EDEVICE


def test_struct_sizes(native):
    from tim_raytracing_b200 import scenes
    assert ctypes.sizeof(native.PushConstants) == 20
    assert scenes.PASS_DATA_DTYPE.itemsize == 240
    assert np.zeros((1, 8), np.float32).nbytes == 32   # tim_rt_ray


def test_python_bindings_check_host_buffers(native):
    """The bindings refuse host arrays the C call would read or write past,
    before any call is made."""
    r = native._ray_records(np.zeros((5, 8), np.float64))
    assert r.dtype == np.float32 and r.shape == (5, 8)
    for bad in (np.zeros((5, 7), np.float32), np.zeros(40, np.float32), np.zeros((2, 4, 8), np.float32)):
        with pytest.raises(ValueError):
            native._ray_records(bad)
    ok = np.zeros((10, 4), np.uint32)
    assert native._host_buf(ok, np.uint32, 40, "hit") is ok
    for bad, count in ((np.zeros((10, 4), np.uint32), 41), (np.zeros((10, 4), np.int64), 40),
                       (np.zeros((4, 10), np.uint32).T, 40), ([0] * 40, 40)):
        with pytest.raises(ValueError):
            native._host_buf(bad, np.uint32, count, "hit")


def test_header_is_c99_and_host_calls_work_from_c(native, tmp_path):
    """include/tim_rt.h compiles as strict C99 (what a cgo or FFI binding parses),
    and a C program linked with libtim_rt.so builds, validates and wide-checks a
    BVH and has a malformed image refused (tests/c/abi_c_check.c; no GPU)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "abi_c_check"
    lib_dir = str(Path(native.LIB_PATH).parent)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"),
                        str(ROOT / "tests" / "c" / "abi_c_check.c"), "-L", lib_dir, "-ltim_rt",
                        f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("ok ")
