"""Shared test helpers: fixture loading, float32 brute force and FP64 adjudication."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
OFFSET = np.float32(1e-5)      # OFFSET_RAY_COLLISION, system.glsl:45
EPS = np.float32(1e-7)         # CollideTriangle EPSILON, collision.glsl:62


def load_room():
    from tim_raytracing_b200 import _native as N, scenes
    z = np.load(GOLDEN / "room_refbvh.npz")
    img = N.BvhImage(z["data"], z["ranges"], tuple(int(x) for x in z["pc"]), z["aabb"])
    return scenes.room_scene(1), img


def load_room_golden():
    return dict(np.load(GOLDEN / "room_golden.npz"))


def tri_positions(scene, rec):
    """Vertex positions (float32 [n,3,3]) of triangle records (vertexOffset, i01, i2m)."""
    rec = np.asarray(rec, np.uint32).reshape(-1, 3)
    i0 = rec[:, 0] + (rec[:, 1] & 0xFFFF)
    i1 = rec[:, 0] + (rec[:, 1] >> 16)
    i2 = rec[:, 0] + (rec[:, 2] & 0xFFFF)
    P = scene.positions.astype(np.float32)
    return np.stack([P[i0], P[i1], P[i2]], 1)


def mt_float32(o, d, P, tmax):
    """CollideTriangle (collision.glsl:58-95) vectorised in float32, same operation
    order as the kernels; o, d: [n,3]; P: [m,3,3] -> t [n,m] (-1 = no hit)."""
    f32 = np.float32
    o = o.astype(f32)[:, None, :]
    d = d.astype(f32)[:, None, :]
    p0, p1, p2 = P[None, :, 0, :], P[None, :, 1, :], P[None, :, 2, :]
    e1 = p1 - p0
    e2 = p2 - p0
    hx = d[..., 1] * e2[..., 2] - d[..., 2] * e2[..., 1]
    hy = d[..., 2] * e2[..., 0] - d[..., 0] * e2[..., 2]
    hz = d[..., 0] * e2[..., 1] - d[..., 1] * e2[..., 0]
    a = e1[..., 0] * hx + e1[..., 1] * hy + e1[..., 2] * hz
    with np.errstate(all="ignore"):
        f = f32(1.0) / a
        s = o - p0
        u = f * (s[..., 0] * hx + s[..., 1] * hy + s[..., 2] * hz)
        qx = s[..., 1] * e1[..., 2] - s[..., 2] * e1[..., 1]
        qy = s[..., 2] * e1[..., 0] - s[..., 0] * e1[..., 2]
        qz = s[..., 0] * e1[..., 1] - s[..., 1] * e1[..., 0]
        v = f * (d[..., 0] * qx + d[..., 1] * qy + d[..., 2] * qz)
        t = f * (e2[..., 0] * qx + e2[..., 1] * qy + e2[..., 2] * qz)
        ok = (np.abs(a) >= EPS) & (np.minimum(np.maximum(u, f32(0)), f32(1)) == u) & ~(v < 0) & ~(u + v > 1)
        ok &= (t > EPS) & (t < np.asarray(tmax, f32).reshape(-1, 1))
    return np.where(ok, t, f32(-1.0))


def brute_closest(scene, rays, chunk=512):
    """Closest hit over all scene triangles (min t, index), float32."""
    P = tri_positions(scene, scene.tri_records())
    n = rays.shape[0]
    tmin = np.full(n, np.inf, np.float32)
    arg = np.full(n, -1, np.int64)
    for s in range(0, n, chunk):
        r = rays[s:s + chunk]
        for m0 in range(0, P.shape[0], 4096):
            t = mt_float32(r[:, 0:3], r[:, 4:7], P[m0:m0 + 4096], r[:, 3])
            t = np.where(t > 0, t, np.inf)
            j = np.argmin(t, axis=1)
            tj = t[np.arange(t.shape[0]), j]
            better = tj < tmin[s:s + chunk]
            tmin[s:s + chunk][better] = tj[better]
            arg[s:s + chunk][better] = m0 + j[better]
    return tmin, arg


def t64(o, d, P):
    """FP64 ray/plane-triangle distance for adjudication (no culling)."""
    o = o.astype(np.float64)
    d = d.astype(np.float64)
    P = P.astype(np.float64)
    e1 = P[:, 1] - P[:, 0]
    e2 = P[:, 2] - P[:, 0]
    h = np.cross(d, e2)
    a = np.einsum("ij,ij->i", e1, h)
    f = 1.0 / a
    s = o - P[:, 0]
    q = np.cross(s, e1)
    return f * np.einsum("ij,ij->i", e2, q)


def adjudicate_closest(scene, rays, hit_a, hit_b, window=2.5e-5):
    """Rays where two closest-hit results differ are accepted as near-ties when both
    are hits whose FP64 distances lie within `window` of each other (the reference
    accepts a later hit only if t < t_prev - 1e-5, so within that window the winner
    depends on visit order). Returns (n_mismatch, n_unexplained, max |dt| FP64)."""
    ta = hit_a[:, 3].view(np.float32)
    tb = hit_b[:, 3].view(np.float32)
    diff = np.any(hit_a != hit_b, axis=1)
    idx = np.nonzero(diff)[0]
    if len(idx) == 0:
        return 0, 0, 0.0
    unexplained = 0
    worst = 0.0
    for i in idx:
        ha, hb = ta[i] < 100.0, tb[i] < 100.0
        if not (ha and hb):
            unexplained += 1
            continue
        Pa = tri_positions(scene, hit_a[i, :3])
        Pb = tri_positions(scene, hit_b[i, :3])
        da = t64(rays[i:i + 1, 0:3], rays[i:i + 1, 4:7], Pa)[0]
        db = t64(rays[i:i + 1, 0:3], rays[i:i + 1, 4:7], Pb)[0]
        worst = max(worst, abs(da - db))
        if abs(da - db) > window:
            unexplained += 1
    return len(idx), unexplained, worst


def near_tie_scene(seed, n):
    """Random triangles, each present three times: as generated, as an exact copy
    (equal t, different record) and moved 3e-6 along its normal (t within the
    reference's 1e-5 acceptance window), so most closest hits are order-dependent
    near-ties."""
    from tim_raytracing_b200 import scenes
    base = scenes.random_triangles(seed, n)
    P = base.positions.reshape(-1, 3, 3)
    N = base.normals.reshape(-1, 3, 3)
    b = scenes._Builder()
    per = 21845
    for shift in (0.0, 0.0, 3e-6):
        Q = (P + N * np.float32(shift)).astype(np.float32)
        for s0 in range(0, len(Q), per):
            q = Q[s0:s0 + per]
            b.add(q.reshape(-1, 3), N[s0:s0 + per].reshape(-1, 3), np.arange(3 * len(q), dtype=np.uint32).reshape(-1, 3),
                  (0.7, 0.7, 0.7))
    return b.scene("near_ties", [], seed=seed)


def sh16_to_prev27(sh16, res, probes):
    """The previous SH9 (FP32, [probe][j][c]) as fetchSH9 reads it from the 7 images
    (lightprob/fetchSH_inline.glsl:6-31)."""
    rx, ry, rz = res
    img = sh16.view(np.float16).astype(np.float32).reshape(7, rz, ry, rx, 4)
    out = np.zeros((len(probes), 27), np.float32)
    for n, p in enumerate(probes):
        x, y, z = probe_coord(p, res)
        out[n, 0:3] = img[0, z, y, x, 0:3]
        for j in range(1, 9):
            for ch in range(3):
                image = 1 + 2 * ch if j <= 4 else 2 + 2 * ch
                comp = j - 1 if j <= 4 else j - 5
                out[n, 3 * j + ch] = img[image, z, y, x, comp]
    return out


def probe_coord(index, res):
    """Probe index -> (x, y, z), lightprobHelpers.glsl getLightProbCoord (4x4x4 tiles)."""
    trx, try_ = res[0] // 4, res[1] // 4
    tile, inn = index // 64, index % 64
    z = tile // (trx * try_)
    tile = tile % (trx * try_)
    y, x = tile // trx, tile % trx
    return x * 4 + inn % 4, y * 4 + (inn // 4) % 4, z * 4 + (inn // 16) % 4


def sh27_to_images16(sh27, res, probes, images16):
    """Inverse of sh16_to_prev27: the 7 rgba16f images (u16 bits) after storeSH9
    (lightprob/storeSH_inline.glsl:6-17) wrote each probe's FP32 SH9, rounded to
    FP16 (w of image 0 is 0); other probes keep their texels."""
    rx, ry, rz = res
    img = np.array(images16, np.uint16).view(np.float16).reshape(7, rz, ry, rx, 4).copy()
    for n, p in enumerate(probes):
        x, y, z = probe_coord(p, res)
        w = np.asarray(sh27[n], np.float32).reshape(9, 3)
        img[0, z, y, x] = (w[0, 0], w[0, 1], w[0, 2], 0.0)
        for ch in range(3):
            img[1 + 2 * ch, z, y, x] = w[1:5, ch]
            img[2 + 2 * ch, z, y, x] = w[5:9, ch]
    return img.view(np.uint16).reshape(np.shape(images16))
