"""The on-disk BVH file (tim_rt_bvh_file_*): a round trip returns the same bytes,
ranges, push constants, bounds and vertex arrays; damaged, truncated or foreign
files are refused; a scene loaded from a file traces like the original."""
import numpy as np
import pytest

from helpers import load_room


def _same(img, pos, nrm, other):
    img2, pos2, nrm2, uv2 = other
    assert np.array_equal(img.data, img2.data)
    assert np.array_equal(np.asarray(img.ranges, np.uint32), img2.ranges)
    assert tuple(int(x) for x in img.pc) == tuple(int(x) for x in img2.pc)
    assert np.array_equal(np.asarray(img.aabb, np.float32).view(np.uint32), img2.aabb.view(np.uint32))
    assert np.array_equal(pos.view(np.uint32), pos2.view(np.uint32))
    if nrm is None:
        assert nrm2 is None
    else:
        assert np.array_equal(nrm.view(np.uint32), nrm2.view(np.uint32))
    assert uv2 is None


def test_round_trip_reference_buffer(native, tmp_path):
    s, img = load_room()
    p = tmp_path / "room.timbvh"
    pos = np.ascontiguousarray(s.positions, np.float32)
    nrm = np.ascontiguousarray(s.normals, np.float32)
    native.save_bvh_file(p, img, pos, nrm)
    _same(img, pos, nrm, native.load_bvh_file(p))
    q = tmp_path / "room_pos_only.timbvh"
    native.save_bvh_file(q, img, pos)
    _same(img, pos, None, native.load_bvh_file(q))


def test_round_trip_product_builder(native, tmp_path):
    from tim_raytracing_b200 import scenes
    s = scenes.heightfield_scene(seed=4, grid=16, n_spheres=3, n_lights=5)
    img = native.build_bvh(s)
    p = tmp_path / "hf.timbvh"
    pos = np.ascontiguousarray(s.positions, np.float32)
    uv = np.random.default_rng(0).uniform(size=(pos.shape[0], 2)).astype(np.float32)
    native.save_bvh_file(p, img, pos, s.normals, uv)
    img2, pos2, nrm2, uv2 = native.load_bvh_file(p)
    assert np.array_equal(img.data, img2.data) and np.array_equal(uv.view(np.uint32), uv2.view(np.uint32))


def test_damaged_files_are_refused(native, tmp_path):
    s, img = load_room()
    p = tmp_path / "room.timbvh"
    native.save_bvh_file(p, img, s.positions, s.normals)
    raw = bytearray(p.read_bytes())
    cases = {
        "flip": lambda b: b.__setitem__(200, b[200] ^ 0x10),          # a blob byte: checksum
        "trunc": lambda b: b.__delitem__(slice(len(b) - 9, len(b))),   # size vs header
        "magic": lambda b: b.__setitem__(0, ord("X")),
    }
    for name, damage in cases.items():
        b = bytearray(raw)
        damage(b)
        q = tmp_path / f"{name}.timbvh"
        q.write_bytes(bytes(b))
        with pytest.raises(native.TimRtError) as e:
            native.load_bvh_file(q)
        assert e.value.code == native.EINVAL, name
    b = bytearray(raw)
    b[8] = 99                                                          # version
    q = tmp_path / "version.timbvh"
    q.write_bytes(bytes(b))
    with pytest.raises(native.TimRtError) as e:
        native.load_bvh_file(q)
    assert e.value.code == native.EUNSUPPORTED
    with pytest.raises(native.TimRtError):
        native.load_bvh_file(tmp_path / "missing.timbvh")


def test_invalid_bvh_is_not_written(native, tmp_path):
    s, img = load_room()
    bad = native.BvhImage(np.zeros_like(img.data), img.ranges, img.pc, img.aabb)
    with pytest.raises(native.TimRtError) as e:
        native.save_bvh_file(tmp_path / "bad.timbvh", bad, s.positions)
    assert e.value.code == native.EINVAL
    assert not (tmp_path / "bad.timbvh").exists()


@pytest.mark.gpu
def test_scene_from_file_traces_like_original(ctx, native, tmp_path):
    from helpers import load_room_golden
    s, img = load_room()
    p = tmp_path / "room.timbvh"
    native.save_bvh_file(p, img, s.positions, s.normals)
    sid = ctx.upload_file(p, quant8=True)
    try:
        g = load_room_golden()
        for mode in (0, 0 | native.TRACE_WIDE):
            h, nid, _, _ = ctx.trace(sid, g["rays"], mode)
            assert np.array_equal(h, g["hit_closest"]) and np.array_equal(nid, g["nid_closest"])
    finally:
        ctx.free_scene(sid)
