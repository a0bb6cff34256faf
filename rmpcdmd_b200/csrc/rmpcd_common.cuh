// Common definitions for the B200 solvent hot path: status handling, the
// library stream, device error word, and small device helpers.
//
// Every translation unit is compiled with -fmad=false: the FP64 form must
// reproduce the reference's separately-rounded multiply/add sequence
// (gfortran on baseline x86-64 emits no FMA), and association order is kept
// as written in the reference expressions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>

#include "../../include/rmpcd.h"

namespace rmpcd {

// ---------------------------------------------------------------------------
// status / last-error string (thread-local, as rmpcd_last_error_string reads)
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

#define RMPCD_CUDA_TRY(expr)                                                     \
    do {                                                                         \
        cudaError_t e__ = (expr);                                                \
        if (e__ != cudaSuccess)                                                  \
            return ::rmpcd::fail(RMPCD_ERR_CUDA, "%s:%d %s: %s", __FILE__,       \
                                 __LINE__, #expr, cudaGetErrorString(e__));      \
    } while (0)

#define RMPCD_CHECK_LAUNCH()                                                     \
    do {                                                                         \
        cudaError_t e__ = cudaGetLastError();                                    \
        if (e__ != cudaSuccess)                                                  \
            return ::rmpcd::fail(RMPCD_ERR_CUDA, "%s:%d launch: %s", __FILE__,  \
                                 __LINE__, cudaGetErrorString(e__));             \
    } while (0)

#define RMPCD_ARG(cond, msg)                                                     \
    do {                                                                         \
        if (!(cond)) return ::rmpcd::fail(RMPCD_ERR_INVALID, "%s", msg);         \
    } while (0)

// The single library stream every kernel runs on (created on first use for
// the current device).  Host entry points that return device results
// synchronize it.
cudaStream_t stream();
int sync();

// Device error word: kernels OR bits in, never trap.  Checked by
// rmpcd_get_status and by entry points that can raise a reference error.
enum : unsigned {
    DEV_ERR_NLIST_FULL = 1u,   // 'maximum of neighbor list reached'
    DEV_ERR_WALL_LOOP = 2u,    // wall-crossing loop hit its iteration cap
    DEV_ERR_RATTLE = 4u,       // RATTLE square root of a negative number
    DEV_ERR_QUAT_LOOP = 8u,    // rigid_body_vv1's quaternion iteration hit its cap
    DEV_ERR_BULK_WAIT = 16u,   // a bulk copy did not complete within its wait limit
    DEV_ERR_BULK_UNDRAINED = 32u,  // ... nor within a second limit before its block exited
};
unsigned *dev_error_word();
int check_dev_error(unsigned *bits_out);

int sm_count();
// one thread per item for kernels whose items carry serial inner loops
// (cells): no cap, so every cell's loop runs in its own thread
inline int grid_full(long long n, int block)
{
    long long g = (n + block - 1) / block;
    if (g > 0x7fffffffLL) g = 0x7fffffffLL;
    if (g < 1) g = 1;
    return (int)g;
}

inline int grid_for(long long n, int block)
{
    long long g = (n + block - 1) / block;
    long long cap = (long long)sm_count() * 32;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// bit positions, src/common.f90:49-55
constexpr int REAC_BIT = 1;
constexpr int MD_BIT = 2;
constexpr int WALL_BIT = 3;
constexpr int PAST_MD_BIT = 4;
constexpr int CATALYZED_BIT = 6;

constexpr int PERIODIC_BC = 1;
constexpr int BOUNCE_BACK_BC = 2;
constexpr int SPECULAR_BC = 3;

// rel_pos, src/common.f90:162-178: minimum image with strict < and >.
template <typename R>
__host__ __device__ inline R min_image(R r, double L)
{
    double h = 0.5 * L;
    if ((double)r < -h) return (R)((double)r + L);
    if ((double)r > h) return (R)((double)r - L);
    return r;
}
__host__ __device__ inline double min_image_d(double r, double L)
{
    if (r < -0.5 * L) return r + L;
    if (r > 0.5 * L) return r - L;
    return r;
}

// floor of a double as the Fortran default integer
__host__ __device__ inline int ifloor(double x) { return (int)floor(x); }

// floor(x / L) for an edge length L > 0 without a division when x lies in
// [-L, 2L) (always the case for a step shorter than the box): there
// x/L rounds into [-1, 0), [0, 1) or [1, 2) exactly as the comparisons below
// say -- a quotient just below an integer k never rounds up to k because
// x < kL implies x/L <= k - 2^-53 * k in double precision -- so the result
// equals floor of the correctly rounded quotient.  Other x divide, and so do
// negative x so small that x/L would underflow to -0.
__host__ __device__ inline int floor_div_edge(double x, double L)
{
    if (x >= -L && x < 2.0 * L && !(x < 0.0 && x > -1e-290))
        return x < 0.0 ? -1 : (x < L ? 0 : 1);
    return (int)floor(x / L);
}

// Unsigned ordering of non-negative doubles equals their numeric ordering,
// so atomicMax on the bit pattern gives a max-reduction of r^2 values.
__device__ inline void atomic_max_nonneg(unsigned long long *addr, double v)
{
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// warp maximum of non-negative r^2 values into *addr: one atomic per warp,
// skipped when it cannot raise the stored maximum (keeps a single hot
// address from serialising thousands of atomics)
__device__ inline void warp_max_into(unsigned long long *addr, double m);

template <typename T>
__device__ inline T warp_max(T v)
{
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = v > w ? v : w;
    }
    return v;
}

__device__ inline void warp_max_into(unsigned long long *addr, double m)
{
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m > 0 && m > __longlong_as_double((long long)__ldcg(addr)))
        atomic_max_nonneg(addr, m);
}

}  // namespace rmpcd
