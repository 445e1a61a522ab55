"""tim_rt_probe_directions (host only): the stratified directions follow
LightProbFieldPass::sampleRays cell by cell, the octahedral ones and both SH9
bases match the Python helpers the GPU tests use."""
import numpy as np
import pytest


@pytest.mark.parametrize("side", [8, 16])
def test_stratified_directions(native, side):
    n = side * side
    d, b = native.probe_directions(n, native.DIRS_STRATIFIED, seed=7)
    d2, _ = native.probe_directions(n, native.DIRS_STRATIFIED, seed=7)
    assert np.array_equal(d, d2)                                   # reproducible for a seed
    assert not np.array_equal(d, native.probe_directions(n, native.DIRS_STRATIFIED, seed=8)[0])
    assert np.allclose(np.linalg.norm(d[:, :3], axis=1), 1.0, atol=1e-6) and np.all(d[:, 3] == 0)
    # ray i * side + j lies in cell (i, j) of (theta / 2pi, (1 - cos phi) / 2)
    u = np.mod(np.arctan2(d[:, 1], d[:, 0]), 2 * np.pi) / (2 * np.pi)
    v = (1.0 - d[:, 2]) / 2.0
    i, j = np.divmod(np.arange(n), side)
    assert np.all(np.abs(u * side - (i + 0.5)) <= 0.5 + 1e-4)
    assert np.all(np.abs(v * side - (j + 0.5)) <= 0.5 + 1e-4)


def test_octahedral_directions_and_basis(native):
    from tim_raytracing_b200 import scenes
    for side in (8, 16):
        d, b = native.probe_directions(side * side, native.DIRS_OCTAHEDRAL)
        ref = scenes.octahedral_dirs(side)
        assert np.array_equal(d.view(np.uint32), ref.view(np.uint32))
        assert np.array_equal(b.view(np.uint32), scenes.sh9_basis(ref).view(np.uint32))
    ds, bs = native.probe_directions(64, native.DIRS_STRATIFIED, seed=3)
    assert np.array_equal(bs.view(np.uint32), scenes.sh9_basis(ds).view(np.uint32))


def test_bad_counts(native):
    for n in (0, 63, 5000):
        with pytest.raises(native.TimRtError):
            native.probe_directions(n)
