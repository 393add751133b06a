/* CPU check of the arithmetic the GPU's STRICT column walk uses in place of one IEEE
 * division per voxel (xpulse_recon_b200/csrc/xpr_kernels.cu: div_exact, pix_bits2):
 *
 *  (1) q = RN(q0 + RN(a - b*q0) * y), q0 = RN(a*y + RN(a*ylo)), y = RN(1/b),
 *      ylo = RN(RN(1 - b*y) * y) equals the IEEE quotient RN(a/b), for random operands
 *      and for dividends a = RN(b*m) (+-1 ulp) with m a rounding midpoint, the cases
 *      closest to a rounding boundary; divisors with exponents in [-60, 60], including
 *      all-ones and power-of-two significands;
 *  (2) the pixel rule: for an integer row offset off and a window [lo, lo + n), the
 *      reference's in-window test and pixel, round_half_away(RN(q - off)) - lo, equal
 *      bits(RZ(RZ(q + 1/2) + 2^23)) - (bits(2^23) + off + lo) with q = off - 1/2 excluded,
 *      for q around every half-integer border.
 *
 * Built and run by tests/test_host.py (gcc -O2 -mfma -ffp-contract=off -frounding-math).
 * Prints "division <cases> <mismatches>" and "pixel <cases> <mismatches>". */
#include <fenv.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float f_of(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }
static uint32_t u_of(float x) { uint32_t v; memcpy(&v, &x, 4); return v; }
static uint64_t mix(uint64_t r)
{
    r ^= r >> 31; r *= 0xBF58476D1CE4E5B9ull; r ^= r >> 29; r *= 0x94D049BB133111EBull; r ^= r >> 32;
    return r;
}
static float div_exact(float a, float b, float y, float ylo)
{
    const float q0 = fmaf(a, y, a * ylo);
    return fmaf(fmaf(-b, q0, a), y, q0);
}

int main(int argc, char **argv)
{
    const long nb = argc > 1 ? atol(argv[1]) : 2000, na = argc > 2 ? atol(argv[2]) : 50000;
    long bad = 0, tot = 0;
#pragma omp parallel for reduction(+ : bad, tot) schedule(dynamic)
    for (long i = 0; i < nb; ++i) {
        const uint64_t r = mix((uint64_t)i * 0x9E3779B97F4A7C15ull + 5);
        uint32_t bb = ((uint32_t)(127 + (r % 121) - 60) << 23) | (uint32_t)((r >> 8) & 0x7fffff);
        if (i % 5 == 0) bb |= 0x7fffff;
        if (i % 11 == 0) bb = (bb & 0xff800000u) | 0x7ffffe;
        if (i % 13 == 0) bb &= 0xff800000u;
        if (r >> 63) bb |= 0x80000000u;
        const float b = f_of(bb), y = 1.0f / b, ylo = fmaf(-b, y, 1.0f) * y;
        for (long j = 0; j < na; ++j) {
            const uint64_t t = mix((uint64_t)j * 0xD1B54A32D192ED03ull + (uint64_t)i * 7919 + 3);
            float a;
            if (j & 1) {
                const double k = (double)((1u << 23) | (uint32_t)(t & 0x7fffff));
                const int e = (int)((t >> 30) % 60) - 30;
                const double m = ldexp(2.0 * k + 1.0, e - 24);      /* a rounding midpoint */
                a = f_of(u_of((float)((double)b * m)) + (int)((t >> 40) % 3) - 1);
            } else {
                const uint32_t ea = (uint32_t)(127 - 40 + ((t >> 3) % 81));
                a = f_of((ea << 23) | (uint32_t)((t >> 12) & 0x7fffff) | (uint32_t)((t >> 50) & 1) << 31);
            }
            ++tot;
            if (u_of(div_exact(a, b, y, ylo)) != u_of(a / b)) ++bad;
        }
    }
    printf("division %ld %ld\n", tot, bad);

    long bad2 = 0, tot2 = 0;
    for (long i = 0; i < 20000000L; ++i) {
        const uint64_t t = mix((uint64_t)i + 99);
        int off = (t & 1) ? 0 : (int)((t >> 1) % 5000);
        if ((t >> 20) % 7 == 0) off = (int)((t >> 24) % 3);
        int lo = (int)((t >> 30) % 4);
        if ((t >> 33) % 3 == 0) lo = 0;
        const int n = 1 + (int)((t >> 36) % 900);
        float q = (float)((double)off + (double)((int)((t >> 46) % (uint64_t)(n + 8)) - 4) + 0.5);
        q = f_of(u_of(q) + (int)((t >> 56) % 9) - 4);
        if ((t >> 60) == 0) q = (float)off - 0.5f;
        const long long p = (long long)roundf(q - (float)off);
        const int in_ref = p >= lo && p < lo + n;
        fesetround(FE_TOWARDZERO);
        volatile float h = q + 0.5f;
        volatile float bits = h + 8388608.0f;
        fesetround(FE_TONEAREST);
        const uint32_t d = u_of(bits) - (0x4B000000u + (uint32_t)off + (uint32_t)lo);
        const int in_mine = d < (uint32_t)n && q != (float)off - 0.5f;
        ++tot2;
        if (in_ref != in_mine || (in_ref && (long long)d != p - lo)) ++bad2;
    }
    printf("pixel %ld %ld\n", tot2, bad2);
    return 0;
}
