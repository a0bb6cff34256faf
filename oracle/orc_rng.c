/*
 * Counter-based random numbers for the oracle.  Test infrastructure only.
 *
 * The reference draws from per-thread Threefry streams (random_module, an
 * absent submodule), so its values cannot be reproduced.  The oracle and the
 * CUDA implementation instead share a *definition*: Philox4x32-10 from
 * J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11, keyed by the 64-bit seed and countered by
 * (index, step, stream, attempt).  This file is an independent C
 * implementation of that definition.
 *
 * Uniform doubles take the top 53 bits of a 64-bit word times 2^-53.
 * Unit vectors use Marsaglia's 1972 rejection method exactly as
 * rand_sphere does (src/mpcd.f90:43-62).  Normal deviates use Leva's
 * ratio-of-uniforms method with quadratic bounds (J. L. Leva, ACM TOMS 18(4),
 * 449-453, 1992), whose output v/u is pure arithmetic.
 */
#include <math.h>
#include "rmpcd_oracle.h"

static void mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; round++) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u53(uint32_t lo, uint32_t hi)
{
    uint64_t w = ((uint64_t)hi << 32) | (uint64_t)lo;
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

void orc_rng_u2(uint64_t seed, uint64_t step, uint32_t index, uint32_t stream,
                uint32_t attempt, double u[2])
{
    uint32_t ctr[4] = { index, (uint32_t)step, (uint32_t)(step >> 32),
                        (stream << 24) | (attempt & 0xFFFFFFu) };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    u[0] = u53(out[0], out[1]);
    u[1] = u53(out[2], out[3]);
}

void orc_rand_sphere(uint64_t seed, uint64_t step, uint32_t index, double n[3])
{
    for (uint32_t attempt = 0; attempt < 64; attempt++) {
        double u[2];
        orc_rng_u2(seed, step, index, ORC_RNG_AXIS, attempt, u);
        double n1 = 2.0 * u[0] - 1.0;
        double n2 = 2.0 * u[1] - 1.0;
        double s = n1 * n1 + n2 * n2;
        if (s < 1.0) {
            double alpha = 2.0 * sqrt(1.0 - s);
            n[0] = n1 * alpha;
            n[1] = n2 * alpha;
            n[2] = 1.0 - 2.0 * s;
            return;
        }
    }
    n[0] = 0.0; n[1] = 0.0; n[2] = 1.0;
}

double orc_normal(uint64_t seed, uint64_t step, uint32_t index, uint32_t sub)
{
    for (uint32_t attempt = 0; attempt < 256; attempt++) {
        double w[2];
        orc_rng_u2(seed, step, index, ORC_RNG_GAUSS, (sub << 16) | attempt, w);
        double u = 1.0 - w[0];
        double v = 1.7156 * (w[1] - 0.5);
        double x = u - 0.449871;
        double y = fabs(v) + 0.386595;
        double q = x * x + y * (0.19600 * y - 0.25472 * x);
        if (q < 0.27597) return v / u;
        if (q > 0.27846) continue;
        if (v * v <= -4.0 * log(u) * u * u) return v / u;
    }
    return 0.0;
}

void orc_random_shift_values(uint64_t seed, uint64_t step, double origin[3])
{
    double u[2];
    orc_rng_u2(seed, step, 0, ORC_RNG_SHIFT, 0, u);
    origin[0] = u[0] - 1;
    origin[1] = u[1] - 1;
    orc_rng_u2(seed, step, 1, ORC_RNG_SHIFT, 0, u);
    origin[2] = u[0] - 1;
}
