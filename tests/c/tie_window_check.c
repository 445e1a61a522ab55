/* tie_window_check.c -- property test of the 8-wide walk's near-tie window.
 *
 * The reference accepts a hit at t iff t < c and then sets c = t - 1e-5
 * (bvhCollision.glsl:210, OFFSET_RAY_COLLISION), so of two hits t1 <= t2 the one
 * visited second can still matter whenever RN(t2 - 1e-5) <= t1. The 8-wide walk
 * (tim_raytracing_b200/csrc/trace_wide.cuh: wide_leaf) finds the nearest hit t1
 * and keeps testing every triangle below c = t1 + (1e-5 + (t1 * 2^-20 + 2^-30))
 * (each operation rounded, as the library compiles without contraction), so that
 * it sees every such t2 and can hand the ray to the binary walk. This program
 * checks, for seeded t1 spread over the reference's range (1e-7 .. 100 and
 * beyond), that the largest float t2 with RN(t2 - 1e-5) <= t1 lies below c.
 *
 * Usage: tie_window_check <cases> <seed>; prints counts, exits 1 on a t2 the
 * window would miss. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static uint64_t s_state;
static uint64_t rnd(void) { s_state ^= s_state << 13; s_state ^= s_state >> 7; s_state ^= s_state << 17; return s_state; }
static double uni(void) { return (double)(rnd() >> 11) * (1.0 / 9007199254740992.0); }

int main(int argc, char** argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 1000000;
    s_state = 0xE7037ED1A0B428DBull ^ (uint64_t)(argc > 2 ? atol(argv[2]) : 1);
    const float off = 1e-5f;
    long missed = 0;
    double worst = INFINITY;   /* smallest (c - t2max) / ulp(t2max) seen */
    for (long it = 0; it < cases; ++it) {
        const float t1 = (float)exp(log(1e-7) + uni() * (log(1e3) - log(1e-7)));
        const volatile float a = t1 * 9.5367431640625e-07f;
        const volatile float b = a + 9.313225746154785e-10f;
        const volatile float m = off + b;
        const float c = t1 + m;
        /* the largest t2 with RN(t2 - 1e-5) <= t1: walk up from RN(t1 + 1e-5) */
        float t2 = t1 + off;
        while ((float)(t2 - off) > t1) t2 = nextafterf(t2, 0.0f);
        for (;;) {
            const float next = nextafterf(t2, INFINITY);
            if ((float)(next - off) <= t1) t2 = next; else break;
        }
        if (!(t2 < c)) {
            ++missed;
            if (missed <= 5) fprintf(stderr, "missed: t1 %a t2 %a c %a\n", t1, t2, c);
        }
        const double gap = ((double)c - (double)t2) / (double)(nextafterf(t2, INFINITY) - t2);
        if (gap < worst) worst = gap;
    }
    printf("cases %ld missed %ld min_gap_ulps %.1f\n", cases, missed, worst);
    return missed ? 1 : 0;
}
