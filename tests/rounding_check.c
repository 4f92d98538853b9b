/* The forward DCT's rounding identity the encode kernel relies on
 * (h261enc_cuda_b200/csrc/kernels.cu, fdct_round): for every finite float
 * p, floorf((float)((double)p + 0.49999)) -- the reference's expression,
 * mbgpu_kernels.cuh:413-437 -- equals floorf(p + 0.49999f).  Checked here
 * for every float of magnitude below 2^24 (above it, both leave p as it
 * is: p + 0.49999 rounds back to p in float and in double-then-float).
 * Built and run by tests/test_rounding.py; prints the count and exits 0
 * when no float differs. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

int main(void)
{
    long checked = 0, differing = 0;
    float first = 0.0f;
    for (uint32_t u = 0; u < 0x4b800000u; u++) {   /* 0 .. just below 2^24 */
        float p;
        memcpy(&p, &u, sizeof(p));
        for (int sign = 0; sign < 2; sign++) {
            const float q = sign ? -p : p;
            const float ref = floorf((float)((double)q + 0.49999));
            const float alt = floorf(q + 0.49999f);
            checked++;
            if (ref != alt && differing++ == 0)
                first = q;
        }
    }
    /* beyond 2^24: a sample of each binade, both must return p */
    for (uint32_t u = 0x4b800000u; u < 0x7f800000u; u += 4097u) {
        float p;
        memcpy(&p, &u, sizeof(p));
        for (int sign = 0; sign < 2; sign++) {
            const float q = sign ? -p : p;
            checked++;
            if ((floorf((float)((double)q + 0.49999)) != q || floorf(q + 0.49999f) != q) && differing++ == 0)
                first = q;
        }
    }
    printf("%ld %ld %.9g\n", checked, differing, first);
    return differing != 0;
}
