"""Sanitizer fuzzing of the host code that reads untrusted input (no GPU needed):
image validation and the 8-wide collapse, the BVH file reader, the host builder.
tests/c/host_fuzz.cpp is compiled with those library sources under
AddressSanitizer and UBSan; a memory error or undefined behaviour aborts it."""
import shutil
import subprocess
from pathlib import Path

import pytest

from helpers import load_room

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = ROOT / "tim_raytracing_b200" / "csrc"


@pytest.fixture(scope="module")
def fuzzer(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path_factory.mktemp("fuzz") / "host_fuzz"
    cmd = [cxx, "-g", "-O1", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-I", str(ROOT / "include"), "-I", str(CSRC), str(HERE / "c" / "host_fuzz.cpp"),
           str(CSRC / "bvh_layout.cpp"), str(CSRC / "bvh_file.cpp"), str(CSRC / "bvh_build.cpp"), "-o", str(exe),
           "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("sanitizer build unavailable: " + r.stderr[-300:])
    return exe


def _run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600,
                       env={"ASAN_OPTIONS": "detect_leaks=0:abort_on_error=1", "UBSAN_OPTIONS": "print_stacktrace=1"})
    assert r.returncode == 0, r.stdout + r.stderr[-3000:]
    words = r.stdout.split()
    return dict(zip(words[0::2], map(int, words[1::2])))


@pytest.fixture(scope="module")
def room_file(native, tmp_path_factory):
    s, img = load_room()
    p = tmp_path_factory.mktemp("fuzzfiles") / "room.timbvh"
    native.save_bvh_file(p, img, s.positions, s.normals)
    return p


@pytest.mark.parametrize("seed", [1, 2])
def test_corrupt_images(fuzzer, room_file, seed):
    c = _run(fuzzer, "image", room_file, seed, 1500)
    assert c["accepted"] > 0 and c["refused"] > 0 and c["failures"] == 0


def test_corrupt_files(fuzzer, room_file):
    c = _run(fuzzer, "file", room_file, 3, 1500)
    assert c["accepted"] > 0 and c["refused"] > 0 and c["failures"] == 0


def test_degenerate_builds(fuzzer):
    c = _run(fuzzer, "build", 4, 120)
    assert c["accepted"] == 120 and c["failures"] == 0
