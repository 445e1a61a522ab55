"""CPU property tests of the two margin arguments the traversal kernels rest on
(no GPU needed). Each C program under tests/c restates a kernel's arithmetic and
checks, on seeded cases built to sit on the decision boundary, the property the
kernel's exactness depends on:

* tests/c/box_filter_check.c -- the binary walk's filtered child-box test
  (csrc/trace_plain.cuh: box_filter, plain_children) takes only decisions that
  CollideBox (the reference's divisions) takes too;
* tests/c/wide_slab_check.c -- the 8-wide walk's quantised slot test
  (csrc/trace_wide.cuh: wide_visit) accepts every slot whose reference box
  CollideBox accepts, for the rays the 8-wide walk trusts;
* tests/c/ebox_check.c -- the 8-wide walk's cheap proof that the binary walk
  reaches a hit's leaf (csrc/trace_wide.cuh: wide_finish) succeeds only where
  CollideBox on the leaf's ancestor-intersection box agrees;
* tests/c/tie_window_check.c -- the window in which the 8-wide walk keeps
  testing triangles after its nearest hit t1 holds every t2 that could still
  change the reference's answer (RN(t2 - 1e-5) <= t1).

The GPU parity tests check the kernels themselves against the oracle."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


def _build(tmp_path_factory, name):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path_factory.mktemp(name) / name
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-fno-fast-math", str(HERE / "c" / f"{name}.c"), "-o", str(exe),
                    "-lm"], check=True)
    return exe


def _run(exe, cases, seed):
    r = subprocess.run([str(exe), str(cases), str(seed)], capture_output=True, text=True)
    words = r.stdout.split()
    return r.returncode, dict(zip(words[0::2], map(float, words[1::2]))), r.stdout + r.stderr


@pytest.fixture(scope="module")
def box_filter_check(tmp_path_factory):
    return _build(tmp_path_factory, "box_filter_check")


@pytest.fixture(scope="module")
def wide_slab_check(tmp_path_factory):
    return _build(tmp_path_factory, "wide_slab_check")


@pytest.fixture(scope="module")
def ebox_check(tmp_path_factory):
    return _build(tmp_path_factory, "ebox_check")


@pytest.fixture(scope="module")
def tie_window_check(tmp_path_factory):
    return _build(tmp_path_factory, "tie_window_check")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_filtered_box_test_never_decides_wrong(box_filter_check, seed):
    rc, c, out = _run(box_filter_check, 1000000, seed)
    assert rc == 0 and c["wrong"] == 0 and c["order_wrong"] == 0, out
    # the boundary is really exercised: many undecided tests, many decided ones, many orders
    assert c["undecided"] > 0.05 * c["tests"]
    assert c["tests"] - c["undecided"] > 0.3 * c["tests"]
    assert c["orders"] > 1000


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_quantised_slot_test_never_loses_a_hit(wide_slab_check, seed):
    rc, c, out = _run(wide_slab_check, 1000000, seed)
    assert rc == 0 and c["lost"] == 0 and c["nonfinite"] == 0, out
    assert c["ref_hits"] > 0.2 * c["cases"]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_reachability_proof_is_never_false(ebox_check, seed):
    rc, c, out = _run(ebox_check, 1000000, seed)
    assert rc == 0 and c["false_proofs"] == 0, out
    assert c["proofs"] > 0.02 * c["cases"]


@pytest.mark.parametrize("seed", [1, 2])
def test_near_tie_window_holds_every_blocking_hit(tie_window_check, seed):
    rc, c, out = _run(tie_window_check, 300000, seed)
    assert rc == 0 and c["missed"] == 0, out
    assert c["min_gap_ulps"] >= 2


def test_nearest_hit_is_order_independent_outside_the_window():
    """Rule (a) of the 8-wide walk: if no other hit t2 has RN(t2 - 1e-5) <= t1
    (t1 the smallest hit t), the reference's shrinking acceptance (accept t iff
    t < c, then c = RN(t - 1e-5)) ends on t1 in every visit order; and when some
    t2 is inside that window, some order gives another answer (so the walk must
    hand such rays to the binary walk). Simulated in float32 over random hit sets
    with many near-ties."""
    import numpy as np
    rng = np.random.default_rng(5)
    off = np.float32(1e-5)
    tmax = np.float32(100.0)

    def final(order):
        c, best = tmax, None
        for i in order:
            if ts[i] < c:
                c, best = np.float32(ts[i] - off), i
        return best

    outside = inside = 0
    for _ in range(20000):
        n = int(rng.integers(2, 6))
        base = np.float32(rng.uniform(0.01, 50.0))
        ts = (base + rng.choice([0.0, 2e-6, 5e-6, 9.9e-6, 1e-5, 1.1e-5, 3e-5, 1.0], size=n)
              * rng.choice([1.0, -1.0], size=n)).astype(np.float32)
        ts = ts[ts > 0]
        if len(ts) < 2:
            continue
        i1 = int(np.argmin(ts))
        t1 = ts[i1]
        others = np.delete(ts, i1)
        window = bool(np.any((others - off).astype(np.float32) <= t1))
        answers = {ts[final(rng.permutation(len(ts)))] for _ in range(12)}
        answers.add(ts[final(range(len(ts)))])
        if not window:
            outside += 1
            assert answers == {t1}, (ts, answers)
        else:
            inside += 1
            # a hit j in the window visited before t1 lowers c to RN(t_j - 1e-5) <= t1,
            # so t1 is rejected and the answer is another triangle: the rule is tight
            j = next(i for i in range(len(ts)) if i != i1 and np.float32(ts[i] - off) <= t1)
            order = [j, i1] + [i for i in range(len(ts)) if i not in (j, i1)]
            assert final(order) != i1
    assert outside > 1000 and inside > 1000
