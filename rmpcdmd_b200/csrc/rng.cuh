// Counter-based random numbers (host and device).
//
// Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11): a 128-bit counter is mixed by ten
// multiply/xor rounds under a 64-bit key.  Here the key is the run seed and
// the counter is (index, step_lo, step_hi, stream<<24 | attempt), so every
// draw is addressed by what it is for -- a cell slot, a particle, a random
// shift -- and never depends on thread scheduling.  This replaces the
// reference's per-thread Threefry states (src/mpcd.f90:75,121).
#pragma once
#include <stdint.h>
#include <math.h>

namespace rmpcd {
namespace rng {

enum Stream : uint32_t {
    SHIFT = 1,   // random_shift
    AXIS = 2,    // rand_sphere in the SRD collision
    GAUSS = 3,   // MPC-AT and Maxwell normals
    REACT = 4,   // change_species acceptance
    PLACE = 5,   // random_placement
    BULK = 7,    // bulk_reaction acceptance
};

// step value reserved for the initial Maxwell velocities
constexpr uint64_t kInitStep = 0xFFFFFFFFFFFFFFFFull;

struct U4 {
    uint32_t v[4];
};

__host__ __device__ inline void mul_hi_lo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo)
{
#ifdef __CUDA_ARCH__
    hi = __umulhi(a, b);
    lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

__host__ __device__ inline U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                     uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t h0, l0, h1, l1;
        mul_hi_lo(0xD2511F53u, c0, h0, l0);
        mul_hi_lo(0xCD9E8D57u, c2, h1, l1);
        uint32_t n0 = h1 ^ c1 ^ k0;
        uint32_t n2 = h0 ^ c3 ^ k1;
        c0 = n0;
        c1 = l1;
        c2 = n2;
        c3 = l0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    U4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

__host__ __device__ inline double u53(uint32_t lo, uint32_t hi)
{
    uint64_t w = ((uint64_t)hi << 32) | (uint64_t)lo;
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

// Two uniform doubles in [0, 1).
__host__ __device__ inline void uniform2(uint64_t seed, uint64_t step, uint32_t index,
                                         uint32_t stream, uint32_t attempt, double &a,
                                         double &b)
{
    U4 o = philox(index, (uint32_t)step, (uint32_t)(step >> 32),
                  (stream << 24) | (attempt & 0xFFFFFFu), (uint32_t)seed,
                  (uint32_t)(seed >> 32));
    a = u53(o.v[0], o.v[1]);
    b = u53(o.v[2], o.v[3]);
}

// Uniform point on the unit sphere by Marsaglia's 1972 rejection method, the
// rand_sphere of src/mpcd.f90:43-62; attempts are capped at 64 (acceptance
// probability pi/4 each), after which the z axis is returned.
__host__ __device__ inline void sphere(uint64_t seed, uint64_t step, uint32_t index,
                                       double &n0, double &n1, double &n2)
{
    for (uint32_t t = 0; t < 64u; t++) {
        double a, b;
        uniform2(seed, step, index, AXIS, t, a, b);
        double x = 2.0 * a - 1.0;
        double y = 2.0 * b - 1.0;
        double s = x * x + y * y;
        if (s < 1.0) {
            double f = 2.0 * sqrt(1.0 - s);
            n0 = x * f;
            n1 = y * f;
            n2 = 1.0 - 2.0 * s;
            return;
        }
    }
    n0 = 0.0;
    n1 = 0.0;
    n2 = 1.0;
}

// Attempt t of a standard normal deviate by Leva's ratio-of-uniforms method
// (J. L. Leva, "A fast normal random number generator", ACM TOMS
// 18(4):449-453, 1992): true, with the deviate in *out, when the attempt is
// accepted.  The quadratic bounds decide almost every attempt without a
// logarithm and the returned value v/u is plain arithmetic, so host and
// device agree.
__host__ __device__ inline bool normal_attempt(uint64_t seed, uint64_t step, uint32_t index, uint32_t sub,
                                               uint32_t t, double *out)
{
    double w0, w1;
    uniform2(seed, step, index, GAUSS, (sub << 16) | t, w0, w1);
    double u = 1.0 - w0;
    double v = 1.7156 * (w1 - 0.5);
    double x = u - 0.449871;
    double y = fabs(v) + 0.386595;
    double q = x * x + y * (0.19600 * y - 0.25472 * x);
    if (q < 0.27597 || (q <= 0.27846 && v * v <= -4.0 * log(u) * u * u)) {
        *out = v / u;
        return true;
    }
    return false;
}

// attempts allowed per deviate; after them the deviate is 0
constexpr uint32_t kNormalAttempts = 256u;

// The first accepted of attempts 0, 1, ... (0.0 if none of kNormalAttempts is)
__host__ __device__ inline double normal(uint64_t seed, uint64_t step, uint32_t index,
                                         uint32_t sub)
{
    for (uint32_t t = 0; t < kNormalAttempts; t++) {
        double z;
        if (normal_attempt(seed, step, index, sub, t, &z)) return z;
    }
    return 0.0;
}

}  // namespace rng
}  // namespace rmpcd
