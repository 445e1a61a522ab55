"""Host-side checks of the 8-wide quantised form (no GPU needed).

tim_rt_wide_check builds the 8-wide form exactly as tim_rt_upload_bvh does with
TIM_RT_UPLOAD_QUANT8 and verifies it against the binary tree: each slot's 8-bit
box contains the reference's box of that subtree (the property that makes the
8-wide walk conservative), every binary leaf's triangles appear once with the
reference's records and rounded edges, and every wide node is reachable once.
The GPU parity tests then only have to show that the kernels walk this form
correctly."""
import numpy as np
import pytest

from helpers import load_room, near_tie_scene

INVALID = 0x3FFFFFFF


def binary_leaf_stats(img):
    """(triangles in binary leaves, binary leaves holding triangles) of a fillGpuBuffer image."""
    nodes = img.nodes()
    words = img.leaf_words()
    if img.num_nodes == 1:
        leaves = [0]
    else:
        leaves = []
        for i in range(img.num_nodes):
            left = int(nodes[i, 2]) & INVALID
            if left == INVALID:
                continue
            if nodes[i, 2] & 0x80000000:
                leaves.append(left)
            if nodes[i, 2] & 0x40000000:
                leaves.append(left + 1)
    tris = nonempty = 0
    for n in leaves:
        off = int(nodes[n, 3])
        if off == 0xFFFFFFFF or off >= len(words):
            continue
        k = int(words[off]) & 0xFFF
        tris += k
        nonempty += k > 0
    return tris, nonempty


def triangle_soup(P, name="soup"):
    """A scene from float32 triangle corners P [n, 3, 3] (one material per 21,845 triangles)."""
    from tim_raytracing_b200 import scenes
    b = scenes._Builder()
    Q = P.astype(np.float64) / max(float(np.abs(P).max()), 1e-300)   # normals from a rescaled copy
    e1, e2 = Q[:, 1] - Q[:, 0], Q[:, 2] - Q[:, 0]
    nf = np.cross(e1, e2)
    nf /= np.maximum(np.linalg.norm(nf, axis=1, keepdims=True), 1e-30)
    per = 21845
    for s0 in range(0, len(P), per):
        q = P[s0:s0 + per]
        b.add(q.reshape(-1, 3).astype(np.float32), np.repeat(nf[s0:s0 + per], 3, 0).astype(np.float32),
              np.arange(3 * len(q), dtype=np.uint32).reshape(-1, 3), (0.7, 0.7, 0.7))
    return b.scene(name, [], seed=0)


def random_corners(seed, n, scale=1.0, offset=0.0, flat_axis=None):
    rng = np.random.default_rng(seed)
    p0 = rng.uniform(0.0, 1.0, size=(n, 1, 3))
    e = rng.normal(size=(n, 2, 3)) * 0.05
    P = np.concatenate([p0, p0 + e], axis=1)
    if flat_axis is not None:
        P[:, :, flat_axis] = 0.25
    return (P * scale + offset).astype(np.float32)


def check(native, img, scene):
    rep = native.wide_check(img, scene.positions)
    tris, leaves = binary_leaf_stats(img)
    assert rep["triangles"] == tris
    assert rep["leaf_slots"] == leaves
    assert rep["internal_slots"] == rep["nodes"] - 1
    assert sum(rep["slot_histogram"]) == rep["nodes"]
    assert rep["device_bytes"] == 80 * rep["nodes"] + 80 * rep["triangles"]
    assert 1 <= rep["depth"] <= 32
    return rep


def test_reference_room_fixture(native):
    s, img = load_room()
    rep = check(native, img, s)
    assert rep["nodes"] > 10


def test_product_builder_heightfield(native):
    """61K binary nodes: the collapse splits the tree over worker threads and
    merges their parts, which the check walks as one tree."""
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene()
    img = native.build_bvh(s)
    rep = check(native, img, s)
    assert rep["triangles"] == 100608 and rep["nodes"] > 1000


@pytest.mark.parametrize("kind", ["random", "near_ties", "heightfield"])
def test_reference_builder_scenes(native, oracle_mod, kind):
    from tim_raytracing_b200 import scenes
    if not oracle_mod.have_refbuild():
        pytest.skip("the reference builder is not built here")
    if kind == "random":
        s = scenes.random_triangles(31, 3000)
    elif kind == "near_ties":
        s = near_tie_scene(8, 800)
    else:
        s = scenes.heightfield_scene(seed=5, grid=16, n_spheres=4, n_lights=6, light_radius=4.0)
    r = oracle_mod.ref_build(s)
    check(native, native.BvhImage(r.data, r.ranges, r.pc, r.aabb), s)


def test_single_leaf_root(native):
    s = triangle_soup(random_corners(3, 1))
    img = native.build_bvh(s)
    assert img.num_nodes == 1
    rep = check(native, img, s)
    assert rep["nodes"] == 1 and rep["slot_histogram"][1] == 1


@pytest.mark.parametrize("scale,offset,flat", [(1.0, 0.0, 2), (1.0, 1.0e6, None), (1.0e-30, 0.0, None),
                                               (1.0e12, -3.0e12, None), (1.0, -7.5, 0)])
def test_extreme_coordinates(native, scale, offset, flat):
    """Flat scenes (zero extent on one axis), far offsets and tiny and huge scales:
    the quantisation must still round every slot box outward."""
    s = triangle_soup(random_corners(9, 4000, scale, offset, flat))
    img = native.build_bvh(s)
    check(native, img, s)


def test_too_wide_for_8_bit_boxes_is_refused(native):
    """Slot planes are origin + q * 2^e with e at most 40 (so that the kernel's
    plane coefficients stay finite); a node wider than 255 * 2^40 cannot be
    quantised and the 8-wide form is refused with an error, never built wrong."""
    s = triangle_soup(random_corners(9, 200, 1.0e30, -3.0e30))
    img = native.build_bvh(s)
    with pytest.raises(native.TimRtError) as e:
        native.wide_check(img, s.positions)
    assert e.value.code == native.EINVAL and "quantised" in str(e.value)


def test_malformed_image_is_refused(native):
    s, img = load_room()
    bad = native.BvhImage(img.data.copy(), img.ranges.copy(), img.pc, img.aabb)
    o, _ = bad.ranges[native.RANGE_NODE]
    bad.data[o + 8:o + 12] = np.frombuffer(np.uint32(0x3FFFFFF0).tobytes(), np.uint8)   # root's child id out of range
    with pytest.raises(native.TimRtError) as e:
        native.wide_check(bad, s.positions)
    assert e.value.code == native.EINVAL


def test_corrupt_images_never_crash_the_host(native):
    """Validation and the host-side 8-wide collapse on corrupted images: every
    corruption is either refused (EINVAL) or yields a checked 8-wide form; none
    may crash the process. A NaN or infinite child box once made the slot
    assignment write outside its array."""
    s, img = load_room()
    rng = np.random.default_rng(17)
    o, size = img.ranges[native.RANGE_NODE]
    lo_, lsize = img.ranges[native.RANGE_LEAF]
    # the regression: non-finite child boxes. A NaN plane cannot be quantised and is
    # refused; an infinite one is refused or, where the collapse opens that child
    # (its box is then not stored), checked like any other image.
    for val in (np.nan, np.inf, -np.inf):
        bad = native.BvhImage(img.data.copy(), img.ranges.copy(), img.pc, img.aabb)
        bad.data[o + 16:o + 20] = np.frombuffer(np.float32(val).tobytes(), np.uint8)   # root's child 0 min.x
        try:
            native.wide_check(bad, s.positions)
            assert not np.isnan(val)
        except native.TimRtError as e:
            assert e.code == native.EINVAL
    refused = checked = 0
    for _ in range(400):
        data = img.data.copy()
        words = data.view(np.uint32)
        for _ in range(int(rng.integers(1, 5))):
            base, n = (o, size) if rng.integers(0, 2) else (lo_, lsize)
            i = (int(base) + 4 * int(rng.integers(0, int(n) // 4))) // 4
            words[i] = rng.choice([0, 0xFFFFFFFF, 0x3FFFFFFF, 0x80000000, 0x7FC00000, int(rng.integers(0, 2**32)),
                                   (int(words[i]) + 1) & 0xFFFFFFFF, int(words[i]) ^ (1 << int(rng.integers(0, 32)))])
        try:
            native.wide_check(native.BvhImage(data, img.ranges.copy(), img.pc, img.aabb), s.positions)
            checked += 1
        except native.TimRtError as e:
            assert e.code == native.EINVAL
            refused += 1
    assert refused > 0 and checked > 0
