/* Checks that div_by_count (smokesim_b200/csrc/common.cuh) returns the same
 * bits as IEEE division a / f (the sign of a zero included) for every count f
 * in 1..6 and every finite float a visited.  Usage: division_check [stride]
 * (stride 1 = all 2^32 bit patterns, about a minute on 8 cores).  Prints the
 * mismatch count and exits non-zero on any mismatch.  Same operations as the
 * device code: RN products and fused multiply-adds. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float div_by_count(float a, int f) {
    if (f == 6) {
        if (fabsf(a) < 7.52316385e-37f) return a / 6.f;
        a = a * 0.5f;
        f = 3;
    } else if (a == 0.f) {
        return a;
    }
    const float y = f == 1 ? 1.f : f == 2 ? 0.5f : f == 3 ? (1.0f / 3.0f) : f == 4 ? 0.25f : (1.0f / 5.0f);
    const float q0 = a * y;
    const float r = fmaf(-(float)f, q0, a);
    return fmaf(r, y, q0);
}

int main(int argc, char** argv) {
    const long long stride = argc > 1 ? atoll(argv[1]) : 1;
    unsigned long long bad = 0, n = 0;
    for (int f = 1; f <= 6; ++f) {
#pragma omp parallel for reduction(+ : bad, n) schedule(static)
        for (long long i = 0; i <= 0xFFFFFFFFLL; i += stride) {
            uint32_t u = (uint32_t)i;
            float a;
            memcpy(&a, &u, 4);
            if (isnan(a) || isinf(a)) continue;
            volatile float ref = a / (float)f;
            const float q = div_by_count(a, f);
            const float rv = ref;
            uint32_t bq, br;
            memcpy(&bq, &q, 4);
            memcpy(&br, &rv, 4);
            ++n;
            if (bq != br) ++bad;
        }
    }
    /* the signed zeros, subnormal and threshold neighbourhoods and the
     * largest finite values, whatever the stride */
    const uint32_t special[] = {0x00000000u, 0x80000000u, 0x00000001u, 0x80000001u, 0x007FFFFFu, 0x807FFFFFu,
                                0x00800000u, 0x80800000u, 0x03800000u, 0x837FFFFFu, 0x03800001u, 0x7F7FFFFFu,
                                0xFF7FFFFFu, 0x3F800000u, 0xBEAAAAABu};
    for (int f = 1; f <= 6; ++f)
        for (size_t k = 0; k < sizeof special / sizeof special[0]; ++k) {
            float a;
            memcpy(&a, &special[k], 4);
            volatile float ref = a / (float)f;
            const float q = div_by_count(a, f), rv = ref;
            uint32_t bq, br;
            memcpy(&bq, &q, 4);
            memcpy(&br, &rv, 4);
            ++n;
            if (bq != br) ++bad;
        }
    printf("checked %llu quotients, %llu bit mismatches\n", n, bad);
    return bad ? 1 : 0;
}
