"""The C restatement (oracle/reftrace.c) against the reference's own compute
shaders compiled as C++ (oracle/refglsl): BVH traversal (closest and any hit),
the camera pass's tracing step with its shadow and probe masks, and the three
light-probe passes must agree bit for bit on the reference builder's BVHs.
The committed fixture's glsl_* vectors pin the restatement where the shader
library is not built; the rest needs oracle/_ref/librefglsl.so."""
import numpy as np
import pytest

from helpers import load_room, load_room_golden, near_tie_scene, sh16_to_prev27, sh27_to_images16

O_CAM_PROB_MASK = 1        # ORC_CAM_PROB_MASK: the camera pass with USE_LPF_MASK


@pytest.fixture(scope="module")
def G():
    from oracle import refglsl
    if not refglsl.available():
        pytest.skip("oracle/_ref/librefglsl.so not built (needs the reference tree at build time)")
    return refglsl


def _probe_inputs(g):
    res = tuple(int(x) for x in g["probe_res"])
    sun, sunc = g["probe_sun"]
    return res, g["probe_dirs"], g["probe_basis"], sun, sunc, g["probe_prev16"]


def test_fixture_pins_restatement(oracle_mod):
    """Restatement == the glsl_* vectors the shader copies wrote into the fixture."""
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s, img = load_room()
    g = load_room_golden()
    assert "glsl_hit_closest" in g, "fixture lacks the shader-copy vectors (rerun tests/golden/make_golden.py)"
    sc = O.Scene(img, s.positions, s.normals)
    hit, nid, _, _ = O.trace(sc, g["rays"], 0)
    assert np.array_equal(hit, g["glsl_hit_closest"]) and np.array_equal(nid, g["glsl_nid_closest"])
    ha, _, _, _ = O.trace(sc, g["rays"], 1)
    assert np.array_equal(ha, g["glsl_hit_any"])
    pd = g["pass_data"].view(scenes.PASS_DATA_DTYPE)
    cam, _, _ = O.camera(sc, pd, flags=O_CAM_PROB_MASK)
    assert np.array_equal(cam, g["glsl_camera"])
    shade16, _ = O.shade_camera(sc, pd, cam, g["lpf16"])
    assert np.array_equal(shade16, g["glsl_shade16"])
    res, dirs, basis, sun, sunc, prev16 = _probe_inputs(g)
    total = res[0] * res[1] * res[2]
    od = O.probe_desc(img.aabb[:3], img.aabb[3:], res, sun, sunc, len(dirs), 0.03)
    tr, irr, _ = O.probe_trace(sc, od, dirs, 0, total)
    assert np.array_equal(tr.reshape(-1, 8), g["glsl_probe_trace"])
    assert np.array_equal(irr.reshape(-1, 3).view(np.uint32), g["glsl_probe_irradiance"].view(np.uint32))
    probes = list(range(total))
    sh = O.probe_sh9(od, basis, irr.reshape(-1, 3), 0, total, sh16_to_prev27(prev16, res, probes))
    assert np.array_equal(sh27_to_images16(sh, res, probes, prev16), g["glsl_probe_images16"])



def _rays_with_edge_cases(seed, n, lo, hi):
    """Random rays in a box plus axis-aligned, zero-component and short-tmax rays."""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 4:7] = d
    r[:, 3] = 100.0
    r.view(np.uint32)[:, 7] = (rng.uniform(size=n) < 0.4).astype(np.uint32)
    k = n // 8
    r[:k, 4:7] = 0.0                                              # axis-aligned (0/0 slab cases)
    r[:k, 4 + (np.arange(k) % 3)] = np.where(np.arange(k) % 2 == 0, 1.0, -1.0)
    r[k:2 * k, 4 + (np.arange(k) % 3)] = 0.0                      # one zero component
    r[2 * k:3 * k, 3] = rng.uniform(0.0, 0.5, size=k).astype(np.float32)   # short tmax
    return r


def _check_trace(O, G, sc, gs, rays):
    for mode in (0, 1, 2):
        oh, on, _, _ = O.trace(sc, rays, mode)
        gh, gn = G.trace(gs, rays, mode)
        bad = np.flatnonzero((oh != gh).any(1) | (on != gn))
        assert bad.size == 0, (mode, bad[:8])


def test_trace_room(oracle_mod, G):
    s, img = load_room()
    sc = oracle_mod.Scene(img, s.positions, s.normals)
    rays = _rays_with_edge_cases(3, 20000, (0.2, 0.2, 0.2), (3.8, 3.8, 2.8))
    _check_trace(oracle_mod, G, sc, G.Scene(img, s.positions, s.normals), rays)


@pytest.mark.parametrize("kind,n", [("random", 1), ("random", 3), ("random", 2000), ("random", 30000),
                                    ("near_ties", 1500), ("heightfield", 0)])
def test_trace_reference_builder_scenes(oracle_mod, G, kind, n):
    """Scenes built by the reference's own BVH builder, including one-node trees
    (numNodes == 1 roots at a leaf) and near-tie triangles."""
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    if kind == "random":
        s = scenes.random_triangles(100 + n, n)
    elif kind == "near_ties":
        s = near_tie_scene(7, n)
    else:
        s = scenes.heightfield_scene(seed=5, grid=16, n_spheres=4, n_lights=6, light_radius=4.0)
    img = O.ref_build(s)
    sc = O.Scene(img, s.positions, s.normals)
    lo, hi = img.aabb[:3] - 0.1, img.aabb[3:] + 0.1
    rays = _rays_with_edge_cases(11 + n, 6000, lo, hi)
    _check_trace(O, G, sc, G.Scene(img, s.positions, s.normals), rays)


@pytest.mark.parametrize("size", [(64, 48), (37, 21)])
def test_camera_tracing_step(oracle_mod, G, size):
    """cameraPass.comp TRACING_STEP (closest hit, leaf-light shadow mask, probe
    mask) over whole frames, sizes not multiples of the 16x16 work group."""
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s = scenes.heightfield_scene(seed=9, grid=20, n_spheres=6, n_lights=12, light_radius=5.0)
    img = O.ref_build(s)
    sc = O.Scene(img, s.positions, s.normals)
    pd = scenes.pass_data(s, size[0], size[1], lpf_res=(8, 8, 4), aabb=(img.aabb[:3], img.aabb[3:]))
    cam, _, _ = O.camera(sc, pd, flags=O_CAM_PROB_MASK)
    gcam = G.camera(G.Scene(img, s.positions, s.normals), pd)
    bad = np.flatnonzero((cam != gcam).any(1))
    assert bad.size == 0, bad[:8]
    hits = cam[:, 3].view(np.float32) < 100.0
    assert hits.mean() > 0.05 and (cam[hits, 4] != 0).any() and (cam[hits, 5] != 0).any()


def test_probe_passes(oracle_mod, G):
    """genLightProbField.comp (tracing and lighting steps) and updateLightProbField.comp."""
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s = scenes.heightfield_scene(seed=21, grid=24, n_spheres=5, n_lights=16, light_radius=5.0)
    img = O.ref_build(s)
    sc = O.Scene(img, s.positions, s.normals)
    gs = G.Scene(img, s.positions, s.normals)
    res = (8, 8, 4)
    total = res[0] * res[1] * res[2]
    dirs = scenes.octahedral_dirs(8)
    basis = scenes.sh9_basis(dirs)
    sun, sunc = np.array([-0.4, 0.3, -1.0], np.float32), np.array([1.0, 0.95, 0.9], np.float32)
    od = O.probe_desc(img.aabb[:3], img.aabb[3:], res, sun, sunc, len(dirs), 0.03)
    tr, irr, _ = O.probe_trace(sc, od, dirs, 0, total)
    gtr = G.probe_trace(gs, od, dirs)
    assert np.array_equal(tr.reshape(-1, 8), gtr)
    girr = G.probe_light(gs, od, dirs, gtr)
    assert np.array_equal(irr.reshape(-1, 3).view(np.uint32), girr.view(np.uint32))
    prev16 = np.random.default_rng(2).uniform(-1, 1, size=(7, res[2], res[1], res[0], 4)).astype(np.float16).view(np.uint16)
    probes = list(range(total))
    sh = O.probe_sh9(od, basis, irr.reshape(-1, 3), 0, total, sh16_to_prev27(prev16, res, probes))
    assert np.array_equal(G.probe_update(od, basis, girr, prev16), sh27_to_images16(sh, res, probes, prev16))


@pytest.mark.parametrize("mask_frac", [0.0, 0.5])
def test_camera_lighting_step(oracle_mod, G, mask_frac):
    """cameraPass.comp lighting step (USE_LPF, USE_LPF_MASK): direct light from the
    tracing step's shadow masks, the probe-masked SH9 sample of the FP16 field,
    evalSH and computeIndirectLighting, stored as RGBA16F."""
    from tim_raytracing_b200 import scenes
    O = oracle_mod
    s = scenes.heightfield_scene(seed=9, grid=20, n_spheres=6, n_lights=12, light_radius=5.0)
    img = O.ref_build(s)
    sc = O.Scene(img, s.positions, s.normals)
    pd = scenes.pass_data(s, 80, 56, lpf_res=(8, 8, 4), aabb=(img.aabb[:3], img.aabb[3:]))
    cam, _, _ = O.camera(sc, pd, flags=O_CAM_PROB_MASK)
    rng = np.random.default_rng(17)
    if mask_frac:   # random probe masks exercise every branch of the masked trilinear tree
        hit = cam[:, 3].view(np.float32) < 100.0
        cam[hit, 5] = rng.integers(0, 256, size=int(hit.sum())).astype(np.uint32)
    sh16 = rng.uniform(-0.5, 1.5, size=(7, 4, 8, 8, 4)).astype(np.float16).view(np.uint16)
    o16, _ = O.shade_camera(sc, pd, cam, sh16)
    g16 = G.shade(G.Scene(img, s.positions, s.normals), pd, cam, sh16)
    bad = np.flatnonzero((o16 != g16).any(1))
    assert bad.size == 0, bad[:8]
    hit = cam[:, 3].view(np.float32) < 100.0
    assert hit.sum() > 100
