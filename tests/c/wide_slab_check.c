/* wide_slab_check.c -- property test of the 8-wide walk's quantised slot test.
 *
 * The 8-wide kernel (tim_raytracing_b200/csrc/trace_wide.cuh: wide_visit) tests a
 * child slot whose planes are origin + 2^(e-127) * q (q an 8-bit value) with
 * per-node coefficients A = RN(RN(origin - o) * inv), B = 2^(e-127) * inv,
 * inv = RN(1/d), both moved outward by 2^-18 of their magnitude, and one FMA per
 * plane, t = RN(q * B' + A'). The walk never loses a hit because this test
 * accepts every slot whose reference box (any box inside the quantised one)
 * CollideBox accepts with the same tmax (collision.glsl:23-40). This program
 * restates the slot test in C and checks exactly that implication on seeded
 * quantised slots, reference boxes as tight as floats allow inside them (and
 * random ones), and rays from and through their planes and corners, for rays
 * the kernel trusts (every direction component at least 2^-60 in magnitude,
 * origin within 2^60). It also checks the slot test's own robustness: every
 * value it computes is finite.
 *
 * Usage: wide_slab_check <cases> <seed>; prints counts, exits 1 on a lost hit.
 * Built with -O2 -ffp-contract=off (the library uses --fmad=false and explicit
 * fused operations only where written). */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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

static float pow2f(int e) {   /* 2^(e-127) from the biased exponent, as the kernel builds it */
    const uint32_t bits = (uint32_t)e << 23;
    float f;
    memcpy(&f, &bits, 4);
    return f;
}
static float wide_inv(float d) { return 1.0f / (d == 0.0f ? copysignf(8.271806125530277e-25f, d) : d); }

/* wide_visit for one slot: 1 when the slot is hit; *finite = 0 if any value is not finite */
static int slot_hit(const Ray* r, const float origin[3], const int e[3], const uint8_t qlo[3], const uint8_t qhi[3],
                    float tcur, int* finite) {
    const float kw = 3.814697265625e-06f;   /* 2^-18 */
    const float inv[3] = {wide_inv(r->dx), wide_inv(r->dy), wide_inv(r->dz)};
    const float o[3] = {r->ox, r->oy, r->oz};
    float tn[3], tf[3];
    for (int a = 0; a < 3; ++a) {
        const float B = pow2f(e[a]) * inv[a];
        const float A = (origin[a] - o[a]) * inv[a];
        const float An = fmaf(-fabsf(A), kw, A), Af = fmaf(fabsf(A), kw, A);
        const float Bn = fmaf(-fabsf(B), kw, B), Bf = fmaf(fabsf(B), kw, B);
        const int neg = signbit(inv[a]) != 0;
        const float qn = (float)(neg ? qhi[a] : qlo[a]), qf = (float)(neg ? qlo[a] : qhi[a]);
        tn[a] = fmaf(qn, Bn, An);
        tf[a] = fmaf(qf, Bf, Af);
        if (!isfinite(tn[a]) || !isfinite(tf[a])) *finite = 0;
    }
    const float tmin = fmaxf(fmaxf(tn[0], fmaxf(tn[1], tn[2])), 0.0f);
    const float tm = fminf(fminf(tf[0], fminf(tf[1], tf[2])), tcur);
    return tmin < tm;
}

static uint64_t s_state;
static uint64_t rnd(void) { s_state ^= s_state << 13; s_state ^= s_state >> 7; s_state ^= s_state << 17; return s_state; }
static float uni(void) { return (float)((rnd() >> 11) * (1.0 / 9007199254740992.0)); }
static float near_value(float b) {
    switch (rnd() % 5) {
        case 0: return b;
        case 1: return nextafterf(b, INFINITY);
        case 2: return nextafterf(b, -INFINITY);
        case 3: return b + (uni() - 0.5f) * 1e-4f * (fabsf(b) + 1.0f);
        default: return b + (uni() - 0.5f) * 3.0f * (fabsf(b) + 1.0f);
    }
}

int main(int argc, char** argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 1000000;
    s_state = 0xD1B54A32D192ED03ull ^ (uint64_t)(argc > 2 ? atol(argv[2]) : 1);
    long ref_hits = 0, lost = 0, nonfinite = 0, slot_hits = 0;
    for (long it = 0; it < cases; ++it) {
        /* a quantised slot: per axis an origin, a scale 2^(e-127) and 8-bit bounds */
        const float world = (rnd() % 3 == 0) ? 1e6f : (rnd() % 2 ? 20.0f : 1e-3f);
        float origin[3], qlo_r[3], qhi_r[3], lo[3], hi[3];
        int e[3];
        uint8_t qlo[3], qhi[3];
        for (int a = 0; a < 3; ++a) {
            origin[a] = (uni() - 0.5f) * world;
            const float extent = world * powf(2.0f, -(float)(rnd() % 12)) * (0.1f + uni());
            e[a] = (int)ceil(log2((double)extent / 255.0)) + 127;
            if (e[a] < 1) e[a] = 1;
            const uint32_t q0 = (uint32_t)(rnd() % 256), q1 = (uint32_t)(rnd() % 256);
            qlo[a] = (uint8_t)(q0 < q1 ? q0 : q1);
            qhi[a] = (uint8_t)(q0 < q1 ? q1 : q0);
            /* the real planes, and a reference box inside them: as tight as floats allow, or random */
            const long double s = ldexpl(1.0L, e[a] - 127);
            const long double pl = (long double)origin[a] + s * qlo[a], ph = (long double)origin[a] + s * qhi[a];
            float fl = (float)pl, fh = (float)ph;
            while ((long double)fl < pl) fl = nextafterf(fl, INFINITY);
            while ((long double)fh > ph) fh = nextafterf(fh, -INFINITY);
            if (fl > fh) { fl = fh = (float)((pl + ph) / 2); if ((long double)fl < pl || (long double)fl > ph) { --it; goto next; } }
            qlo_r[a] = fl;
            qhi_r[a] = fh;
            if (rnd() % 3 == 0) {
                const float u = uni(), v = uni();
                lo[a] = fl + (fh - fl) * fminf(u, v);
                hi[a] = fl + (fh - fl) * fmaxf(u, v);
                if (lo[a] < fl) lo[a] = fl;
                if (hi[a] > fh) hi[a] = fh;
            } else {
                lo[a] = fl;
                hi[a] = fh;
            }
        }
        {
            /* a ray the kernel trusts, from or through the reference box's planes and corners */
            Ray r;
            float o[3], d[3];
            const int kind = (int)(rnd() % 3);
            for (int a = 0; a < 3; ++a) {
                const float c = lo[a] + (hi[a] - lo[a]) * uni();
                o[a] = kind == 0 ? near_value(rnd() % 2 ? lo[a] : hi[a]) : near_value(c);
            }
            if (kind == 2) {   /* aim at a corner or an edge point from outside */
                for (int a = 0; a < 3; ++a) {
                    const float target = (rnd() % 3 == 0) ? lo[a] + (hi[a] - lo[a]) * uni() : (rnd() % 2 ? lo[a] : hi[a]);
                    const float from = target + (uni() - 0.5f) * 4.0f * (hi[a] - lo[a] + world * 1e-3f);
                    d[a] = target - from;
                    o[a] = from;
                }
            } else {
                for (int a = 0; a < 3; ++a) {
                    const uint64_t k = rnd() % 10;
                    d[a] = k == 0 ? 1e-12f : k == 1 ? -8.7e-19f : k == 2 ? 3e5f : (uni() - 0.5f) * 2.0f;
                }
            }
            int ok = 1;
            for (int a = 0; a < 3; ++a)
                if (!(fabsf(d[a]) >= 8.673617379884035e-19f) || !(fabsf(o[a]) <= 1.152921504606847e18f)) ok = 0;
            if (!ok) { --it; goto next; }
            r.ox = o[0]; r.oy = o[1]; r.oz = o[2];
            r.dx = d[0]; r.dy = d[1]; r.dz = d[2];
            const float tmax = (rnd() % 4 == 0) ? 100.0f : (rnd() % 2 ? uni() * world : 1e30f);
            const int h_ref = collide_box(&r, lo, hi, tmax) >= 0.0f;
            int finite = 1;
            const int h_here = slot_hit(&r, origin, e, qlo, qhi, tmax, &finite);
            ref_hits += h_ref;
            slot_hits += h_here;
            if (h_ref && !h_here) {
                ++lost;
                if (lost <= 5)
                    fprintf(stderr, "lost: o %a %a %a d %a %a %a tmax %a box [%a %a %a]-[%a %a %a]\\n", r.ox, r.oy, r.oz,
                            r.dx, r.dy, r.dz, tmax, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
            }
            if (!finite) ++nonfinite;
            (void)qlo_r; (void)qhi_r;
        }
    next:;
    }
    printf("cases %ld ref_hits %ld slot_hits %ld lost %ld nonfinite %ld\n", cases, ref_hits, slot_hits, lost, nonfinite);
    return (lost || nonfinite) ? 1 : 0;
}
