"""CPU property test of the margin argument behind the binary walk's filtered
child-box test (no GPU needed): tests/c/box_filter_check.c restates the kernel's
arithmetic (csrc/trace_plain.cuh: box_filter, plain_children) and compares each
decision it takes with the reference's CollideBox on boxes and rays built to sit
on the decision boundary. The GPU parity tests check the kernel itself."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path_factory.mktemp("boxcheck") / "box_filter_check"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-fno-fast-math", str(HERE / "c" / "box_filter_check.c"), "-o",
                    str(exe), "-lm"], check=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_filtered_box_test_never_decides_wrong(checker, seed):
    r = subprocess.run([str(checker), "1000000", str(seed)], capture_output=True, text=True)
    counts = dict(zip(r.stdout.split()[0::2], map(int, r.stdout.split()[1::2])))
    assert r.returncode == 0, r.stdout
    assert counts["wrong"] == 0 and counts["order_wrong"] == 0
    # the boundary cases are really exercised: many undecided tests, many decided ones
    assert counts["undecided"] > 0.05 * counts["tests"]
    assert counts["tests"] - counts["undecided"] > 0.3 * counts["tests"]
    assert counts["orders"] > 1000
