/* ebox_check.c -- property test of the 8-wide walk's fast reachability proof.
 *
 * When the 8-wide walk ends with a nearest hit t1, it keeps its answer only if
 * the reference's binary walk provably reaches the hit's leaf: the ray must pass
 * CollideBox (collision.glsl:23-40) on E, the intersection of the leaf's box and
 * its ancestors' boxes, with tmin <= t1. The kernel (tim_raytracing_b200/csrc/
 * trace_wide.cuh: wide_finish) first tries a cheap proof with inv = RN(1/d)
 * instead of the division, moving every slab entry up and every exit down by
 * 2^-21 of its magnitude (and 2^-100), and calls CollideBox only when that proof
 * fails. This program restates the cheap proof in C and checks that whenever it
 * succeeds, CollideBox on E with an unbounded tmax returns a tmin in [0, t1] --
 * on seeded boxes and rays built so that t1 lies at the entry distance, an ulp
 * either side or close to it, for rays without zero direction components (the
 * kernel sends those to the binary walk).
 *
 * Usage: ebox_check <cases> <seed>; prints counts, exits 1 on a false proof. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef struct { float ox, oy, oz, dx, dy, dz; } Ray;

static float collide_box(const Ray* r, const float lo[3], const float hi[3], float tmax) {
    const float t0x = (lo[0] - r->ox) / r->dx, t0y = (lo[1] - r->oy) / r->dy, t0z = (lo[2] - r->oz) / r->dz;
    const float t1x = (hi[0] - r->ox) / r->dx, t1y = (hi[1] - r->oy) / r->dy, t1z = (hi[2] - r->oz) / r->dz;
    const float sx = fminf(t0x, t1x), sy = fminf(t0y, t1y), sz = fminf(t0z, t1z);
    const float bx = fmaxf(t0x, t1x), by = fmaxf(t0y, t1y), bz = fmaxf(t0z, t1z);
    const float tmin = fmaxf(0.0f, fmaxf(sx, fmaxf(sy, sz)));
    const float tm = fminf(tmax, fminf(bx, fminf(by, bz)));
    return (tmin < tm) ? tmin : -1.0f;
}

/* wide_finish's fast proof (d has no zero component) */
static int fast_proof(const Ray* r, const float lo[3], const float hi[3], float t1) {
    const float e = 4.76837158203125e-07f;   /* 2^-21 */
    const float a = 7.888609052210118e-31f;  /* 2^-100 */
    const float ix = 1.0f / r->dx, iy = 1.0f / r->dy, iz = 1.0f / r->dz;
    const float ax = (lo[0] - r->ox) * ix, bx = (hi[0] - r->ox) * ix;
    const float ay = (lo[1] - r->oy) * iy, by = (hi[1] - r->oy) * iy;
    const float az = (lo[2] - r->oz) * iz, bz = (hi[2] - r->oz) * iz;
    const float sx = fminf(ax, bx), sy = fminf(ay, by), sz = fminf(az, bz);
    const float fx = fmaxf(ax, bx), fy = fmaxf(ay, by), fz = fmaxf(az, bz);
    const float up = fmaxf(0.0f, fmaxf(sx + fabsf(sx) * e, fmaxf(sy + fabsf(sy) * e, sz + fabsf(sz) * e))) + a;
    const float dn = fminf(fx - fabsf(fx) * e, fminf(fy - fabsf(fy) * e, fz - fabsf(fz) * e)) - a;
    return up <= t1 && up < dn;
}

static uint64_t s_state;
static uint64_t rnd(void) { s_state ^= s_state << 13; s_state ^= s_state >> 7; s_state ^= s_state << 17; return s_state; }
static float uni(void) { return (float)((rnd() >> 11) * (1.0 / 9007199254740992.0)); }
static float near_value(float b) {
    switch (rnd() % 6) {
        case 0: return b;
        case 1: return nextafterf(b, INFINITY);
        case 2: return nextafterf(b, -INFINITY);
        case 3: return b * (1.0f + (uni() - 0.5f) * 1e-5f);
        case 4: return b * (1.0f + (uni() - 0.5f) * 1e-3f);
        default: return b + (uni() - 0.5f) * 2.0f;
    }
}
static float component(void) {
    switch (rnd() % 12) {
        case 0: return 1e-30f;
        case 1: return -3e-12f;
        case 2: return 4e4f;
        default: { const float v = (uni() - 0.5f) * 2.0f; return v == 0.0f ? 0.5f : v; }
    }
}

int main(int argc, char** argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 1000000;
    s_state = 0xA0761D6478BD642Full ^ (uint64_t)(argc > 2 ? atol(argv[2]) : 1);
    long proofs = 0, false_proofs = 0, exact_ok = 0;
    for (long it = 0; it < cases; ++it) {
        const float world = (rnd() % 3 == 0) ? 1e5f : 20.0f;
        Ray r;
        r.ox = (uni() - 0.5f) * world;
        r.oy = (uni() - 0.5f) * world;
        r.oz = (uni() - 0.5f) * world;
        r.dx = component();
        r.dy = component();
        r.dz = component();
        /* a box E around a point on the ray, or with planes through the origin */
        const float tc = uni() * world;
        const float p[3] = {r.ox + r.dx * tc, r.oy + r.dy * tc, r.oz + r.dz * tc};
        const float o[3] = {r.ox, r.oy, r.oz};
        float lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            const float w = (rnd() % 4 == 0) ? 0.0f : uni() * 0.01f * world;
            lo[k] = p[k] - w * uni();
            hi[k] = p[k] + w * uni();
            if (rnd() % 5 == 0) lo[k] = near_value(o[k]);
            if (rnd() % 5 == 0) hi[k] = near_value(o[k]);
            if (lo[k] > hi[k]) { const float t = lo[k]; lo[k] = hi[k]; hi[k] = t; }
        }
        /* t1 at the entry distance (as CollideBox computes it), or near it */
        const float entry = collide_box(&r, lo, hi, INFINITY);
        const float t1 = entry >= 0.0f ? fabsf(near_value(entry)) : uni() * world;
        if (fast_proof(&r, lo, hi, t1)) {
            ++proofs;
            const float d = collide_box(&r, lo, hi, INFINITY);
            if (d >= 0.0f && d <= t1) ++exact_ok;
            else ++false_proofs;
        }
    }
    printf("cases %ld proofs %ld exact_ok %ld false_proofs %ld\n", cases, proofs, exact_ok, false_proofs);
    return false_proofs ? 1 : 0;
}
