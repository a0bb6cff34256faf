// Compact Hilbert index of a cell, host and device.
//
// This is Hamilton's compact Hilbert index (C. Hamilton, "Compact Hilbert
// indices", Dalhousie Univ. TR CS-2006-07) for 3 dimensions with per-axis
// bit counts M[3], with the conventions of src/hilbert.f90:241-307
// (initial entry e = 0, direction d = 2, axis j contributes bit j of the
// level word, levels from max(M)-1 down to 0).  The key defines the cell
// order of the whole solvent layout, so it has to reproduce the reference's
// ordering bit for bit; the code below is an independent formulation of the
// published algorithm.  Positions outside [0, 2^M) are hashed exactly as the
// reference hashes them (bits above M still enter the level words).
#pragma once
#include <stdint.h>

namespace rmpcd {
namespace hilbert {

constexpr unsigned kMask = 7u;

__host__ __device__ inline unsigned rotr3(unsigned x, unsigned r)
{
    return ((x >> r) | (x << (3u - r))) & kMask;
}
__host__ __device__ inline unsigned rotl3(unsigned x, unsigned r)
{
    return ((x << r) | (x >> (3u - r))) & kMask;
}
__host__ __device__ inline unsigned gray(unsigned i) { return i ^ (i >> 1); }
__host__ __device__ inline unsigned gray_inv(unsigned g) { return g ^ (g >> 1) ^ (g >> 2); }

// entry point of sub-cube i along the curve
__host__ __device__ inline unsigned entry_of(unsigned i)
{
    return i == 0u ? 0u : gray(2u * ((i - 1u) / 2u));
}

__host__ __device__ inline unsigned ctz32(unsigned x)
{
    unsigned n = 0;
    while (n < 32u && !((x >> n) & 1u)) n++;
    return n;
}

// intra-sub-cube direction of sub-cube i
__host__ __device__ inline unsigned dir_of(unsigned i)
{
    if (i == 0u) return 0u;
    unsigned j = (i & 1u) ? i : i - 1u;
    return ctz32(gray(j) ^ gray(j + 1u)) % 3u;
}

// bit mask of the axes still active at level i (bit j set when M[j] > i)
__host__ __device__ inline unsigned active_axes(int i, const int M[3])
{
    return (M[0] > i ? 1u : 0u) | (M[1] > i ? 2u : 0u) | (M[2] > i ? 4u : 0u);
}

// gather the bits of w selected by mu, from the top axis down
__host__ __device__ inline unsigned gather_bits(unsigned w, unsigned mu)
{
    unsigned r = 0;
    for (int k = 2; k >= 0; k--)
        if ((mu >> k) & 1u) r = (r << 1) | ((w >> k) & 1u);
    return r;
}

__host__ __device__ inline int max3(const int M[3])
{
    int m = M[0] > M[1] ? M[0] : M[1];
    return m > M[2] ? m : M[2];
}

// compact_p_to_h
__host__ __device__ inline int compact_index(const int p[3], const int M[3])
{
    unsigned h = 0, e = 0, d = 2;
    for (int i = max3(M) - 1; i >= 0; i--) {
        unsigned act = active_axes(i, M);
        unsigned nact = (act & 1u) + ((act >> 1) & 1u) + ((act >> 2) & 1u);
        unsigned mu = rotr3(act, d + 1u);
        unsigned l = (((unsigned)p[0] >> i) & 1u) | ((((unsigned)p[1] >> i) & 1u) << 1) |
                     ((((unsigned)p[2] >> i) & 1u) << 2);
        unsigned w = gray_inv(rotr3(l ^ e, d + 1u));
        h = (h << nact) | gather_bits(w, mu);
        e ^= rotl3(entry_of(w), d + 1u);
        d = (d + dir_of(w) + 1u) % 3u;
    }
    return (int)h;
}

// compact_h_to_p
__host__ __device__ inline void compact_point(int h, const int M[3], int p[3])
{
    unsigned e = 0, d = 2;
    int k = 0;
    int sum_m = M[0] + M[1] + M[2];
    p[0] = p[1] = p[2] = 0;
    for (int i = max3(M) - 1; i >= 0; i--) {
        unsigned act = active_axes(i, M);
        int nact = (int)((act & 1u) + ((act >> 1) & 1u) + ((act >> 2) & 1u));
        unsigned mu = rotr3(act, d + 1u);
        unsigned pi = rotr3(e, d + 1u) & (~mu & kMask);
        unsigned r = 0;
        for (int j = 0; j < nact; j++)
            r |= (((unsigned)h >> (sum_m - k - nact + j)) & 1u) << j;
        k += nact;
        // rebuild the gray-coded word from its free bits and the implied ones
        unsigned w = 0, g = 0;
        int j = nact - 1;
        for (int b = 2; b >= 0; b--) {
            unsigned upper = (w >> (b + 1)) & 1u;
            if ((mu >> b) & 1u) {
                w |= ((r >> j) & 1u) << b;
                g |= ((((w >> b) & 1u) + upper) & 1u) << b;
                j--;
            } else {
                g |= ((pi >> b) & 1u) << b;
                w |= ((((g >> b) & 1u) + upper) & 1u) << b;
            }
        }
        // inverse of the level transform rotr3(l ^ e, d + 1)
        unsigned lt = rotl3(gray(w), d + 1u) ^ e;
        p[0] |= (int)((lt & 1u) << i);
        p[1] |= (int)(((lt >> 1) & 1u) << i);
        p[2] |= (int)(((lt >> 2) & 1u) << i);
        e ^= rotl3(entry_of(w), d + 1u);
        d = (d + dir_of(w) + 1u) % 3u;
    }
}

}  // namespace hilbert
}  // namespace rmpcd
