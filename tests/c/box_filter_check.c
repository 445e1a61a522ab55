/* box_filter_check.c -- property test of the binary walk's filtered child-box test.
 *
 * The kernel (tim_raytracing_b200/csrc/trace_plain.cuh: box_filter, plain_children)
 * decides CollideBox's outcome -- hit or miss, and for two hit children whether
 * d1 < d0 -- from slab distances computed by multiplying with RN(1/d) instead of
 * dividing by d, and only when an error margin leaves no doubt; otherwise it
 * calls CollideBox. This program restates that arithmetic in C (same operations,
 * same constants, fmaf for the one fused operation) and compares every decision
 * it takes with CollideBox (collision.glsl:23-40, true division, fminf/fmaxf) on
 * seeded rays and boxes built to sit on the decision boundary: planes through
 * the ray origin and through the point at tmax, one ulp either side, flat boxes,
 * zero, signed-zero, subnormal and tiny direction components, far origins and
 * short or long tmax. Any wrong decision means the margin argument is wrong.
 *
 * Usage: box_filter_check <cases> <seed>; prints one line of counts, exits 1 on a
 * wrong decision. Built with -O2 -ffp-contract=off (no contraction, like the
 * library's --fmad=false). */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef struct { float ox, oy, oz, dx, dy, dz; } Ray;

static float collide_box(const Ray* r, float mnx, float mny, float mnz, float mxx, float mxy, float mxz, float tmax) {
    const float t0x = (mnx - r->ox) / r->dx, t0y = (mny - r->oy) / r->dy, t0z = (mnz - r->oz) / r->dz;
    const float t1x = (mxx - r->ox) / r->dx, t1y = (mxy - r->oy) / r->dy, t1z = (mxz - r->oz) / r->dz;
    const float sx = fminf(t0x, t1x), sy = fminf(t0y, t1y), sz = fminf(t0z, t1z);
    const float bx = fmaxf(t0x, t1x), by = fmaxf(t0y, t1y), bz = fmaxf(t0z, t1z);
    const float tmin = fmaxf(0.0f, fmaxf(sx, fmaxf(sy, sz)));
    const float tm = fminf(tmax, fminf(bx, fminf(by, bz)));
    return (tmin < tm) ? tmin : -1.0f;
}

/* box_dir_ok and the per-ray set-up of trav_init */
static int box_dir_ok(float d) {
    const float a = fabsf(d);
    return a == 0.0f || (a >= 7.888609052210118e-31f && a <= 1.2676506002282294e30f);
}
typedef struct { Ray r; float t, ix, iy, iz, boxabs; } St;
static void init(St* st) {
    st->ix = 1.0f / st->r.dx;
    st->iy = 1.0f / st->r.dy;
    st->iz = 1.0f / st->r.dz;
    st->boxabs = (box_dir_ok(st->r.dx) && box_dir_ok(st->r.dy) && box_dir_ok(st->r.dz) && st->t <= 1.2676506002282294e30f)
                     ? 7.888609052210118e-31f : INFINITY;
}

/* box_filter: 1 when decided (hit, and [lo, hi] holding CollideBox's tmin on a hit) */
static int box_filter(const St* st, float mnx, float mny, float mnz, float mxx, float mxy, float mxz, int* hit,
                      float* lo, float* hi) {
    const float t0x = (mnx - st->r.ox) * st->ix, t0y = (mny - st->r.oy) * st->iy, t0z = (mnz - st->r.oz) * st->iz;
    const float t1x = (mxx - st->r.ox) * st->ix, t1y = (mxy - st->r.oy) * st->iy, t1z = (mxz - st->r.oz) * st->iz;
    const float M = fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z)));
    const float T = fminf(st->t, fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z))));
    const float m = fmaf(fabsf(M) + fabsf(T), 9.5367431640625e-07f, st->boxabs);
    const float tmin = fmaxf(0.0f, M);
    if (tmin + m < T - m) {
        *hit = 1;
        const int zero = M + m <= 0.0f;
        *lo = zero ? 0.0f : fmaxf(0.0f, M - m);
        *hi = zero ? 0.0f : tmin + m;
        return 1;
    }
    *hit = 0;
    *lo = *hi = 0.0f;
    return tmin - m >= T + m;
}

static uint64_t s_state;
static uint64_t rnd(void) { s_state ^= s_state << 13; s_state ^= s_state >> 7; s_state ^= s_state << 17; return s_state; }
static float uni(void) { return (float)((rnd() >> 11) * (1.0 / 9007199254740992.0)); }
static float near_value(float b) {   /* b itself, one ulp either side, or close to it */
    switch (rnd() % 6) {
        case 0: return b;
        case 1: return nextafterf(b, INFINITY);
        case 2: return nextafterf(b, -INFINITY);
        case 3: return b + (uni() - 0.5f) * 1e-5f;
        default: return b + (uni() - 0.5f) * 4.0f;
    }
}
static float direction_component(void) {
    switch (rnd() % 24) {
        case 0: return 0.0f;
        case 1: return -0.0f;
        case 2: return 1e-35f;
        case 3: return -1e-20f;
        case 4: return 1e-42f;
        default: return (uni() - 0.5f) * 2.0f;
    }
}

int main(int argc, char** argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 1000000;
    s_state = 0x9E3779B97F4A7C15ull ^ (uint64_t)(argc > 2 ? atol(argv[2]) : 1);
    long tests = 0, undecided = 0, wrong = 0, orders = 0, order_undecided = 0, order_wrong = 0;
    for (long it = 0; it < cases; ++it) {
        St st;
        const float scale = (rnd() % 4 == 0) ? 2000.0f : 20.0f;
        st.r.ox = (uni() - 0.5f) * scale;
        st.r.oy = (uni() - 0.5f) * scale;
        st.r.oz = (uni() - 0.5f) * scale;
        st.r.dx = direction_component();
        st.r.dy = direction_component();
        st.r.dz = direction_component();
        switch (rnd() % 5) {
            case 0: st.t = 100.0f; break;
            case 1: st.t = 1e-3f; break;
            case 2: st.t = 1e31f; break;
            default: st.t = uni() * 30.0f;
        }
        init(&st);
        const float o[3] = {st.r.ox, st.r.oy, st.r.oz}, d[3] = {st.r.dx, st.r.dy, st.r.dz};
        float b[2][6];
        for (int c = 0; c < 2; ++c) {
            /* a point on the ray, which boxes built around it contain */
            const float tc = uni() * fminf(st.t, 40.0f);
            for (int a = 0; a < 3; ++a) {
                const uint64_t k = rnd() % 4;
                float p1, p2;
                if (k == 3) {
                    const float pc = o[a] + d[a] * tc;
                    p1 = pc - uni() * 2.0f;
                    p2 = pc + uni() * 2.0f;
                } else {
                    p1 = k == 0 ? near_value(o[a]) : k == 1 ? near_value(o[a] + d[a] * fminf(st.t, 40.0f))
                                                            : (uni() - 0.5f) * 20.0f;
                    p2 = p1 + ((rnd() % 8 == 0) ? 0.0f : uni() * 5.0f);
                }
                b[c][a] = p1;
                b[c][3 + a] = p2;
            }
        }
        int h[2], ok[2];
        float lo[2], hi[2], ex[2];
        for (int c = 0; c < 2; ++c) {
            ok[c] = box_filter(&st, b[c][0], b[c][1], b[c][2], b[c][3], b[c][4], b[c][5], &h[c], &lo[c], &hi[c]);
            ex[c] = collide_box(&st.r, b[c][0], b[c][1], b[c][2], b[c][3], b[c][4], b[c][5], st.t);
            ++tests;
            if (!ok[c]) { ++undecided; continue; }
            if (h[c] != (ex[c] >= 0.0f) || (h[c] && !(lo[c] <= ex[c] && ex[c] <= hi[c]))) ++wrong;
        }
        if (ok[0] && ok[1] && h[0] && h[1]) {   /* plain_children's order decision */
            ++orders;
            const int first1 = hi[1] < lo[0];
            if (!first1 && !(lo[1] >= hi[0])) ++order_undecided;
            else if (first1 != (ex[1] < ex[0])) ++order_wrong;
        }
    }
    printf("tests %ld undecided %ld wrong %ld orders %ld order_undecided %ld order_wrong %ld\n", tests, undecided,
           wrong, orders, order_undecided, order_wrong);
    return (wrong || order_wrong) ? 1 : 0;
}
