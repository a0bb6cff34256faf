// The bulk-fluid interval as one fused pass per interval (plus a slot scan
// and a key scatter), replacing the loop of test/setup_bulk_decay.f90:112-121:
//
//     simple_mpcd_step -> mpcd_stream_periodic(tau) -> random_shift -> sort
//
// Layout: inside the schedule each particle is one packed record holding what
// changes or is needed every interval,
//   FP32 (32 B, two 16-byte chunks):  [vx vy vz species] [px py pz idx]
//   FP64 (56 B, seven 8-byte words):  vx vy vz (species,idx) px py pz
// where idx is the particle's position when the schedule started.  image,
// flags and id do not move: they stay in the API arrays at idx (image is
// updated there, in place, only for the few particles that wrap in an
// interval) and are gathered into sorted order once, at the end.  The velocity
// part (16 / 32 B) is what the collision needs for a whole cell at once; the
// rest is needed particle by particle.
//
// Data flow of interval i (grid G_i, next grid G_{i+1}):
//   P1  k_bulk_interval  one block per tile of consecutive Hilbert slots of
//       G_i.  The tile's particles are a contiguous range in G_i order; the
//       block loads the range's source indices (perm), sorts each cell's
//       indices ascending (the reference's stable scatter order), gathers the
//       velocity parts of the records into shared memory with cp.async
//       (scattered reads in flight without stalling the warp), performs the
//       SRD rotation of each cell in place, then per particle gathers the
//       rest of its record, streams and wraps it, keys it in G_{i+1}, counts
//       it and writes the record in G_i order with coalesced stores.
//   P2  slot scan of the G_{i+1} counts (starts and scatter cursors).
//   P3  k_perm_tiles: perm[place] = j for every particle j of the new arrays
//       (k_perm for boxes of more than 2^22 slots).
// The records written by P1 hold exactly the reference's arrays after
// simple_mpcd_step and mpcd_stream_periodic; the sort into G_{i+1} is
// completed by the gather of the next P1 (or by the final gather).
//
// HBM traffic of P1 per particle: perm 4 + record read + record write +
// key 4 (72 B in FP32, 120 B in FP64), plus 12 B per slot, plus a 12-byte
// image update for each particle that wraps.
#include <algorithm>
#include <cmath>

#include "async_copy.cuh"
#include "cellops.cuh"
#include "keys.cuh"
#include "rng.cuh"
#include "scan.cuh"
#include "sortcore.cuh"
#include "sortnet.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kFusedThreads = 256;

template <typename R>
struct Rec;

template <>
struct Rec<float> {
    static constexpr int kBytes = 32;
    static constexpr int kVelBytes = 16;
    __device__ static float *vel(unsigned char *r) { return (float *)r; }
    __device__ static int &species(unsigned char *r) { return ((int *)r)[3]; }
    __device__ static float *pos(unsigned char *r) { return (float *)r + 4; }
    __device__ static int &idx(unsigned char *r) { return ((int *)r)[7]; }
};

template <>
struct Rec<double> {
    static constexpr int kBytes = 56;
    static constexpr int kVelBytes = 32;
    __device__ static double *vel(unsigned char *r) { return (double *)r; }
    __device__ static int &species(unsigned char *r) { return ((int *)r)[6]; }
    __device__ static int &idx(unsigned char *r) { return ((int *)r)[7]; }
    __device__ static double *pos(unsigned char *r) { return (double *)r + 4; }
};

// Tile shape of k_bulk_interval: slots (cells) per block, staged-particle
// capacity and resident blocks per SM (launch bound).  The capacity is more
// than 7 standard deviations above the mean tile occupancy at density 10; an
// over-full tile takes the global-memory path.  Every shape gives the same
// results bit for bit (the tile size changes only which block handles a
// cell); the shape in use is chosen per precision, by default the first one,
// or by rmpcd_bulk_autotune.
template <int SL_, int CAP_, int MINB_>
struct Shape {
    static constexpr int kSlots = SL_;
    static constexpr int kCap = CAP_;
    static constexpr int kMinBlocks = MINB_;
};

template <typename R>
struct FusedArgs {
    const unsigned char *in;  // records in pre-gather order
    unsigned char *out;       // records in G_i order (written)
    int *perm;                // G_i place -> record index in `in`; null = identity
    const int *count;         // G_i
    const int *start;         // G_i (0-based)
    int S;
    int N;
    int *count_next;          // G_{i+1} histogram (accumulated)
    int *key_out;             // G_{i+1} slot of out[j] (packed with its warp group when pack != 0)
    int *tile_info;           // per tile: first particle and count (written)
    int pack;
    int *ix, *iy, *iz;        // image, indexed by idx (updated in place on a wrap)
    Grid g_next;
    double e0, e1, e2;        // edges
    R dt;
    double sin_a, cos_a;
    uint64_t seed, step;
    const double *axes;
    unsigned *err;            // device error word
};

// rotation matrix of one cell in the working precision: the injected axis or
// rand_sphere (src/mpcd.f90:43-62), then omega (src/mpcd.f90:163-171)
template <typename R>
struct CellRot {
    R m[3][3];
};

template <typename R>
__device__ inline CellRot<R> cell_rotation(int slot, const FusedArgs<R> &A)
{
    double n0, n1, n2;
    if (A.axes) {
        n0 = A.axes[3 * (size_t)slot];
        n1 = A.axes[3 * (size_t)slot + 1];
        n2 = A.axes[3 * (size_t)slot + 2];
    } else {
        rng::sphere(A.seed, A.step, (uint32_t)slot, n0, n1, n2);
    }
    Rot o = srd_matrix(n0, n1, n2, A.sin_a, A.cos_a);
    CellRot<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) r.m[i][k] = (R)o.m[i][k];
    return r;
}

// v = lv + matmul(omega, v - lv), the arithmetic of srd_rotate
template <typename R>
__device__ inline void cell_rotate(R &x, R &y, R &z, const R lv[3], const CellRot<R> &o)
{
    R d0 = x - lv[0], d1 = y - lv[1], d2 = z - lv[2];
    R r0 = o.m[0][0] * d0 + o.m[0][1] * d1 + o.m[0][2] * d2;
    R r1 = o.m[1][0] * d0 + o.m[1][1] * d1 + o.m[1][2] * d2;
    R r2 = o.m[2][0] * d0 + o.m[2][1] * d1 + o.m[2][2] * d2;
    x = lv[0] + r0;
    y = lv[1] + r1;
    z = lv[2] + r2;
}

// FP32 cell sums are exact: every velocity component enters as a 64-bit
// fixed-point integer of 2^-40 resolution (exactly for components of
// magnitude 2^-17 and above, rounded to 2^-41 below that; a cell sum may
// reach 2^23 in magnitude), so the cell mean does not depend on the order of
// the cell's particles.  That is what lets the FP32 interval skip ordering each
// cell's particles: the result of every particle is the same for any order.
constexpr float kFixScale = 1099511627776.0f;  // 2^40

__device__ inline long long to_fixed(float v)
{
    return __float2ll_rn(v * kFixScale);
}

__device__ inline float fixed_mean(long long s, int n)
{
    return (float)((double)s / (double)n * (1.0 / 1099511627776.0));
}

// SRD of one cell of n consecutive velocity parts (src/mpcd.f90:127-178);
// stride is the distance between consecutive particles in bytes
template <typename R>
__device__ inline void srd_cell(unsigned char *v0, int stride, int n, const CellRot<R> &o)
{
    if constexpr (sizeof(R) == 4) {
        // [vx vy vz species] in the first 16 bytes of every entry
        int n_eff = 0;
        long long sx = 0, sy = 0, sz = 0;
        for (int k = 0; k < n; k++) {
            int4 c = *(const int4 *)(v0 + (size_t)k * stride);
            if (c.w > 0) {
                sx += to_fixed(__int_as_float(c.x));
                sy += to_fixed(__int_as_float(c.y));
                sz += to_fixed(__int_as_float(c.z));
                n_eff++;
            }
        }
        if (n_eff <= 1) return;
        const float lv[3] = {fixed_mean(sx, n_eff), fixed_mean(sy, n_eff), fixed_mean(sz, n_eff)};
        for (int k = 0; k < n; k++) {
            int4 *q = (int4 *)(v0 + (size_t)k * stride);
            int4 c = *q;
            float x = __int_as_float(c.x), y = __int_as_float(c.y), z = __int_as_float(c.z);
            cell_rotate(x, y, z, lv, o);
            *q = make_int4(__float_as_int(x), __float_as_int(y), __float_as_int(z), c.w);
        }
        return;
    }
    int n_eff = 0;
    CellSum<R> sx, sy, sz;
    for (int k = 0; k < n; k++) {
        unsigned char *r = v0 + (size_t)k * stride;
        if (Rec<R>::species(r) > 0) {
            R *v = Rec<R>::vel(r);
            sx.add(v[0]);
            sy.add(v[1]);
            sz.add(v[2]);
            n_eff++;
        }
    }
    if (n_eff <= 1) return;
    R lv[3] = {sx.value() / n_eff, sy.value() / n_eff, sz.value() / n_eff};
    for (int k = 0; k < n; k++) {
        R *v = Rec<R>::vel(v0 + (size_t)k * stride);
        R x = v[0], y = v[1], z = v[2];
        cell_rotate(x, y, z, lv, o);
        v[0] = x;
        v[1] = y;
        v[2] = z;
    }
}

// floor(x / L) of the FP32 form, decided by float comparisons for
// -L <= x < 2L (every streamed position of a wrapped particle)
__device__ inline int floor_div_edge_f(float x, float L)
{
    if (x >= -L && x < 2.0f * L && !(x < 0.0f && x > -1e-30f)) return x < 0.0f ? -1 : (x < L ? 0 : 1);
    return (int)floorf(x / L);
}

template <typename R>
__device__ inline int wrap_jump(R x, double L)
{
    if constexpr (sizeof(R) == 4) return floor_div_edge_f(x, (float)L);
    else return floor_div_edge(x, L);
}

// mpcd_stream_periodic of one particle (src/mpcd.f90:450-455); returns its
// slot in G_{i+1}; a wrap updates the particle's image at its idx
template <typename R>
__device__ inline int stream_values(const FusedArgs<R> &A, R &x, R &y, R &z, R vx, R vy, R vz, int idx)
{
    x = x + vx * A.dt;
    y = y + vy * A.dt;
    z = z + vz * A.dt;
    int jx = wrap_jump<R>(x, A.e0), jy = wrap_jump<R>(y, A.e1), jz = wrap_jump<R>(z, A.e2);
    if (jx) {
        x = x - (R)(jx * A.e0);
        A.ix[idx] += jx;
    }
    if (jy) {
        y = y - (R)(jy * A.e1);
        A.iy[idx] += jy;
    }
    if (jz) {
        z = z - (R)(jz * A.e2);
        A.iz[idx] += jz;
    }
    return slot_of(A.g_next, (double)x, (double)y, (double)z);
}

// room for the 16-byte rounding of the tile's index window
constexpr int kPermPad = 8;
// polls of the index copy's mbarrier before the block gives up on it (far
// above the microseconds one copy takes)
constexpr int kBulkPolls = 1 << 16;

// shared memory of a tile: velocity parts and source indices per particle;
// the FP64 form's in-cell ordering also keeps the tile-local cell of each
// particle (one byte) and each cell's local start and count
template <typename R, typename S>
constexpr size_t fused_smem()
{
    return (size_t)S::kCap * (Rec<R>::kVelBytes + sizeof(int)) + (size_t)kPermPad * sizeof(int) +
           (sizeof(R) == 8 ? (size_t)S::kCap + 2 * (size_t)S::kSlots * sizeof(int) : 0);
}

// the non-velocity part of a record, as loaded from global memory
template <typename R>
struct Rest;
template <>
struct Rest<float> {
    int4 a;  // [px py pz idx]
};
template <>
struct Rest<double> {
    long long w[3];  // px py pz
};

__device__ inline void load_rest(Rest<float> &r, const unsigned char *rec)
{
    r.a = __ldcs((const int4 *)rec + 1);
}
__device__ inline void load_rest(Rest<double> &r, const unsigned char *rec)
{
    const long long *q = (const long long *)rec;
#pragma unroll
    for (int k = 0; k < 3; k++) r.w[k] = __ldcs(q + 4 + k);
}

// stream particle j (velocity part in shared memory at sv, the rest in r),
// write its record at o and return its G_{i+1} slot
__device__ inline int finish_particle(const FusedArgs<float> &A, const unsigned char *sv, const Rest<float> &r,
                                      unsigned char *o)
{
    int4 c0 = *(const int4 *)sv;
    float x = __int_as_float(r.a.x), y = __int_as_float(r.a.y), z = __int_as_float(r.a.z);
    int key = stream_values<float>(A, x, y, z, __int_as_float(c0.x), __int_as_float(c0.y), __int_as_float(c0.z),
                                   r.a.w);
    int4 *q = (int4 *)o;
    __stcs(q, c0);
    __stcs(q + 1, make_int4(__float_as_int(x), __float_as_int(y), __float_as_int(z), r.a.w));
    return key;
}

__device__ inline int finish_particle(const FusedArgs<double> &A, const unsigned char *sv, const Rest<double> &r,
                                      unsigned char *o)
{
    const long long *sw = (const long long *)sv;
    const double *v = (const double *)sv;
    double x = __longlong_as_double(r.w[0]), y = __longlong_as_double(r.w[1]), z = __longlong_as_double(r.w[2]);
    int idx = ((const int *)sv)[7];
    int key = stream_values<double>(A, x, y, z, v[0], v[1], v[2], idx);
    long long *ow = (long long *)o;
    __stcs(ow, sw[0]);
    __stcs(ow + 1, sw[1]);
    __stcs(ow + 2, sw[2]);
    __stcs(ow + 3, sw[3]);
    __stcs(ow + 4, __double_as_longlong(x));
    __stcs(ow + 5, __double_as_longlong(y));
    __stcs(ow + 6, __double_as_longlong(z));
    return key;
}

// The next slot of a particle packed with its place in the warp group of
// equal slots that the counting atomic formed: bits 0-21 slot, 22-26 the
// distance back to the group's first lane, 27-31 the rank in the group (for
// the first lane: the group size - 1).  k_perm_tiles replays the same warp
// chunks and so places every particle without regrouping the keys.
constexpr int kPackSlotBits = 22;

__device__ inline int pack_key(int key, unsigned peers)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lead_off = lane - (unsigned)(__ffs(peers) - 1);
    const unsigned r = lead_off == 0u ? (unsigned)__popc(peers) - 1u : (unsigned)__popc(peers & lanemask_lt());
    return (int)((unsigned)key | (lead_off << kPackSlotBits) | (r << (kPackSlotBits + 5)));
}

template <typename R, typename S>
__global__ void __launch_bounds__(kFusedThreads, S::kMinBlocks) k_bulk_interval(FusedArgs<R> A)
{
    constexpr int SL = S::kSlots;
    constexpr int CAP = S::kCap;
    static_assert(SL <= kFusedThreads, "one thread per slot of the tile");
    constexpr int B = Rec<R>::kBytes;
    constexpr int VB = Rec<R>::kVelBytes;
    static_assert(SL <= 256, "tile-local cell index kept in one byte");
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *s_vel = smem;
    int *s_idx = (int *)(smem + (size_t)CAP * VB);          // the tile's index window
    // FP64 only (the in-cell ordering): cell starts and counts of the tile,
    // tile-local cell of each particle
    int *s_cstart = s_idx + CAP + kPermPad;
    int *s_ccount = s_cstart + SL;
    unsigned char *s_cell = (unsigned char *)(s_ccount + SL);

    __shared__ __align__(8) unsigned long long s_bar;
    const int t = threadIdx.x;
    const int lane = t & 31;
    if (t == 0) mbar_init(&s_bar, 1);
    const int s0 = blockIdx.x * SL;
    const int slot = s0 + t;
    const int last = min(s0 + SL, A.S) - 1;
    int my_n = 0, my_a = 0;
    if (t < SL && slot < A.S) {
        my_n = A.count[slot];
        my_a = A.start[slot];
    }
    const int a0 = A.start[s0];
    const int np = A.start[last] + A.count[last] - a0;
    if (t == 0) {
        A.tile_info[2 * blockIdx.x] = a0;
        A.tile_info[2 * blockIdx.x + 1] = np;
    }

    if (np <= CAP) {
        // ---- staged path ----
        // the tile's source indices perm[a0, a0 + np): one bulk copy of the
        // enclosing 16-byte window (perm is allocated to a multiple of 4)
        int *s_perm = s_idx;
        bool gave_up = false;  // this thread stopped waiting for the index copy
        if (A.perm) {
            const int w0 = a0 & ~3;
            const unsigned bytes = (unsigned)(((a0 - w0 + np + 3) & ~3) * sizeof(int));
            s_perm = s_idx + (a0 - w0);
            __syncthreads();  // the mbarrier's initialisation
            if (t == 0 && bytes) {
                mbar_arrive_expect_tx(&s_bar, bytes);
                bulk_copy_to_smem(s_idx, A.perm + w0, bytes, &s_bar);
            }
            if (bytes && !mbar_wait_bounded(&s_bar, 0, kBulkPolls)) {
                // not delivered in time: report it and load the same values
                // directly.  While the block runs, a late copy writes only
                // this tile's index window, with the values loaded here (at
                // worst undoing their in-cell order, which the error bit
                // already flags); the thread waits for it again before it
                // exits (below), so the copy cannot land in the shared memory
                // of a later block.
                atomicOr(A.err, DEV_ERR_BULK_WAIT);
                gave_up = true;
                for (int j = t; j < np; j += kFusedThreads) s_perm[j] = __ldcs(A.perm + a0 + j);
            }
        } else {
            for (int j = t; j < np; j += kFusedThreads) s_perm[j] = a0 + j;
        }
        if constexpr (sizeof(R) == 8) if (A.perm) {
            // FP64: each cell's indices in ascending order (the reference's
            // stable scatter order): every index is placed at its rank among
            // the cell's indices, one thread per index, so a crowded cell
            // costs no more than its share; the ranks go through the (still
            // unused) velocity buffer and back.  (The FP32 cell sums do not
            // depend on the order, so FP32 keeps the order of arrival.)
            if (t < SL) {
                s_cstart[t] = my_a - a0;
                s_ccount[t] = my_n;
                for (int k = 0; k < my_n; k++) s_cell[my_a - a0 + k] = (unsigned char)t;
            }
            __syncthreads();
            int *s_tmp = (int *)s_vel;
            for (int j = t; j < np; j += kFusedThreads) {
                const int c = s_cell[j], a = s_cstart[c], n = s_ccount[c];
                const int v = s_perm[j];
                int r = 0;
#pragma unroll 4
                for (int k = a; k < a + n; k++) r += s_perm[k] < v;
                s_tmp[a + r] = v;
            }
            __syncthreads();
            for (int j = t; j < np; j += kFusedThreads) s_perm[j] = s_tmp[j];
        }
        __syncthreads();
        // gather the velocity parts (16 B per particle in FP32, 4 x 8 B in FP64)
        if constexpr (VB == 16) {
            for (int j = t; j < np; j += kFusedThreads)
                cp_async16(s_vel + (size_t)j * VB, A.in + (size_t)s_perm[j] * B);
        } else {
            for (int q = t; q < np * 4; q += kFusedThreads) {
                int j = q >> 2, c = q & 3;
                cp_async8(s_vel + (size_t)j * VB + 8 * c, A.in + (size_t)s_perm[j] * B + 8 * c);
            }
        }
        // the cell's rotation is drawn while the gathers are in flight
        CellRot<R> rot;
        if (my_n > 1) rot = cell_rotation<R>(slot, A);
        cp_async_wait_all();
        __syncthreads();
        if (my_n > 1) srd_cell<R>(s_vel + (size_t)(my_a - a0) * VB, VB, my_n, rot);
        __syncthreads();
        // stream, key, count and write every particle; the rest of the next
        // record is fetched while the current one is processed
        int j = t;
        Rest<R> cur;
        if (j < np) load_rest(cur, A.in + (size_t)s_perm[j] * B);
        for (int jb = 0; jb < np; jb += kFusedThreads) {
            bool ok = j < np;
            Rest<R> nxt;
            int jn = j + kFusedThreads;
            if (jn < np) load_rest(nxt, A.in + (size_t)s_perm[jn] * B);
            int key = -1;
            if (ok) key = finish_particle(A, s_vel + (size_t)j * VB, cur, A.out + (size_t)(a0 + j) * B);
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok) A.key_out[a0 + j] = A.pack ? pack_key(key, peers) : key;
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
            cur = nxt;
            j = jn;
        }
        // a copy given up on must land before the block's shared memory is
        // released; if it has not within a second limit either, the block
        // exits with it pending and says so (a separate error bit)
        if (gave_up && !mbar_wait_bounded(&s_bar, 0, kBulkPolls)) atomicOr(A.err, DEV_ERR_BULK_UNDRAINED);
    } else {
        // ---- over-full tile (dense cells): the same steps in global memory ----
        if (sizeof(R) == 8 && A.perm && my_n > 1) sort_small(A.perm + my_a, my_n);
        __syncthreads();
        if (my_n > 0) {
            for (int k = 0; k < my_n; k++) {
                int src = A.perm ? A.perm[my_a + k] : my_a + k;
                const long long *s = (const long long *)(A.in + (size_t)src * B);
                long long *d = (long long *)(A.out + (size_t)(my_a + k) * B);
                for (int w = 0; w < B / 8; w++) d[w] = s[w];
            }
            if (my_n > 1) srd_cell<R>(A.out + (size_t)my_a * B, B, my_n, cell_rotation<R>(slot, A));
        }
        __syncthreads();
        for (int jb = 0; jb < np; jb += kFusedThreads) {
            int j = a0 + jb + t;
            bool ok = jb + t < np;
            int key = -1;
            if (ok) {
                unsigned char *r = A.out + (size_t)j * B;
                R *p = Rec<R>::pos(r), *v = Rec<R>::vel(r);
                R x = p[0], y = p[1], z = p[2];
                key = stream_values<R>(A, x, y, z, v[0], v[1], v[2], Rec<R>::idx(r));
                p[0] = x;
                p[1] = y;
                p[2] = z;
            }
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok) A.key_out[j] = A.pack ? pack_key(key, peers) : key;
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
        }
    }
}

// perm[place] = j for every particle of the new arrays, from keys packed by
// k_bulk_interval: the blocks walk the interval's tiles with the same
// thread-to-particle mapping, so each warp meets exactly the groups the
// interval formed; the first lane of a group takes the group's places with
// one cursor atomic and hands the base to the others by a shuffle (no
// regrouping of the keys).  Rounds of a thread issue their atomics before
// using any result.
constexpr int kPermTileRounds = 4;

__global__ void __launch_bounds__(kFusedThreads) k_perm_tiles(const int *__restrict__ packed,
                                                              const int *__restrict__ tile_info, int ntiles,
                                                              int *__restrict__ cursor, int *__restrict__ perm)
{
    const int t = threadIdx.x, lane = t & 31;
    const int slot_mask = (1 << kPackSlotBits) - 1;
    for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
        const int a0 = tile_info[2 * b], np = tile_info[2 * b + 1];
        for (int jb0 = 0; jb0 < np; jb0 += kFusedThreads * kPermTileRounds) {
            unsigned w[kPermTileRounds];
            int base[kPermTileRounds];
            bool ok[kPermTileRounds];
#pragma unroll
            for (int r = 0; r < kPermTileRounds; r++) {
                const int j = jb0 + r * kFusedThreads + t;
                ok[r] = j < np;
                w[r] = ok[r] ? (unsigned)packed[a0 + j] : 0u;
            }
#pragma unroll
            for (int r = 0; r < kPermTileRounds; r++) {
                base[r] = 0;
                if (ok[r] && ((w[r] >> kPackSlotBits) & 31u) == 0u)
                    base[r] = atomicAdd(cursor + (int)(w[r] & (unsigned)slot_mask),
                                        (int)((w[r] >> (kPackSlotBits + 5)) & 31u) + 1);
            }
#pragma unroll
            for (int r = 0; r < kPermTileRounds; r++) {
                const int off = ok[r] ? (int)((w[r] >> kPackSlotBits) & 31u) : 0;
                const int bb = __shfl_sync(0xffffffffu, base[r], lane - off);
                if (ok[r]) {
                    const int rank = off == 0 ? 0 : (int)((w[r] >> (kPackSlotBits + 5)) & 31u);
                    perm[bb + rank] = a0 + jb0 + r * kFusedThreads + t;
                }
            }
        }
    }
}

// SoA (API layout) -> records with idx = position.  Each block assembles 256
// records in shared memory and writes them out as one contiguous range of
// 8-byte words (coalesced).
constexpr int kPackThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kPackThreads) k_soa_to_rec(PView<R> v, unsigned char *rec, int N)
{
    constexpr int B = Rec<R>::kBytes;
    __shared__ __align__(16) unsigned char s[kPackThreads * B];
    for (long long base = (long long)blockIdx.x * kPackThreads; base < N; base += (long long)gridDim.x * kPackThreads) {
        const long long i = base + threadIdx.x;
        if (i < N) {
            unsigned char *r = s + (size_t)threadIdx.x * B;
            R *p = Rec<R>::pos(r), *w = Rec<R>::vel(r);
            p[0] = v.pos.x[i];
            p[1] = v.pos.y[i];
            p[2] = v.pos.z[i];
            w[0] = v.vel.x[i];
            w[1] = v.vel.y[i];
            w[2] = v.vel.z[i];
            Rec<R>::species(r) = v.species[i];
            Rec<R>::idx(r) = (int)i;
        }
        __syncthreads();
        const int n = (int)min((long long)kPackThreads, N - base);
        long long *dst = (long long *)(rec + (size_t)base * B);
        const long long *src = (const long long *)s;
        for (int q = threadIdx.x; q < n * (B / 8); q += kPackThreads) dst[q] = src[q];
        __syncthreads();
    }
}

// FP32 end of a run: each cell's particles are put in ascending order of
// their position at the start of the run (idx), a canonical order, since the
// FP32 intervals leave them in order of arrival.  perm[j] is replaced by the
// idx of its record (inv[idx] keeps the record), the segments are sorted and
// mapped back to records.
template <typename R>
__global__ void k_perm_to_idx(const unsigned char *rec, int *perm, int *inv, int N)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x) {
        const int r = perm[j];
        const int idx = ((const int *)(rec + (size_t)r * Rec<R>::kBytes))[7];
        inv[idx] = r;
        perm[j] = idx;
    }
}

__global__ void k_idx_to_perm(int *perm, const int *inv, int N)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x)
        perm[j] = inv[perm[j]];
}

// final gather into the API arrays: pos, vel, species from the records
// through perm; image, flags and id from the position-at-start idx
template <typename R>
__global__ void k_rec_gather_to_soa(const unsigned char *rec, const int *perm, PView<R> side, PView<R> d, int N)
{
    constexpr int B = Rec<R>::kBytes;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x) {
        long long w8[B / 8];
        const long long *src = (const long long *)(rec + (size_t)perm[j] * B);
#pragma unroll
        for (int k = 0; k < B / 8; k++) w8[k] = __ldcs(src + k);
        unsigned char *r = (unsigned char *)w8;
        const R *p = Rec<R>::pos(r), *w = Rec<R>::vel(r);
        const int idx = Rec<R>::idx(r);
        int ix = side.ix[idx], iy = side.iy[idx], iz = side.iz[idx], fl = side.flags[idx], id = side.id[idx];
        d.pos.x[j] = p[0];
        d.pos.y[j] = p[1];
        d.pos.z[j] = p[2];
        d.vel.x[j] = w[0];
        d.vel.y[j] = w[1];
        d.vel.z[j] = w[2];
        d.species[j] = Rec<R>::species(r);
        d.ix[j] = ix;
        d.iy[j] = iy;
        d.iz[j] = iz;
        d.flags[j] = fl;
        d.id[j] = id;
    }
}

// the shapes a precision can run with, and the one in use
template <typename R>
struct ShapeEntry {
    void (*kernel)(FusedArgs<R>);
    int slots;
    size_t smem;
    int min_blocks;
};

template <typename R, typename S>
constexpr ShapeEntry<R> entry()
{
    return {k_bulk_interval<R, S>, S::kSlots, fused_smem<R, S>(), S::kMinBlocks};
}

template <typename R>
struct Shapes;
template <>
struct Shapes<float> {
    static constexpr ShapeEntry<float> list[] = {entry<float, Shape<128, 1792, 4>>(),
                                                  entry<float, Shape<128, 1792, 5>>(),
                                                  entry<float, Shape<96, 1408, 5>>(),
                                                  entry<float, Shape<64, 1024, 6>>(),
                                                  entry<float, Shape<160, 2176, 4>>(),
                                                  entry<float, Shape<192, 2560, 3>>()};
};
template <>
struct Shapes<double> {
    static constexpr ShapeEntry<double> list[] = {entry<double, Shape<96, 1408, 4>>(),
                                                   entry<double, Shape<112, 1600, 3>>(),
                                                   entry<double, Shape<128, 1792, 3>>(),
                                                   entry<double, Shape<160, 2176, 2>>(),
                                                   entry<double, Shape<192, 2560, 2>>(),
                                                   entry<double, Shape<96, 1408, 3>>()};
};
template <typename R>
constexpr int n_shapes()
{
    return (int)(sizeof(Shapes<R>::list) / sizeof(Shapes<R>::list[0]));
}

static int g_shape[2] = {0, 0};  // shape in use: [0] FP32, [1] FP64

template <typename R>
static const ShapeEntry<R> &shape_in_use()
{
    return Shapes<R>::list[g_shape[sizeof(R) == 8]];
}

template <typename R>
static int prepare_shapes()
{
    static bool done[2] = {false, false};
    if (done[sizeof(R) == 8]) return RMPCD_OK;
    for (int k = 0; k < n_shapes<R>(); k++)
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(Shapes<R>::list[k].kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)Shapes<R>::list[k].smem));
    done[sizeof(R) == 8] = true;
    return RMPCD_OK;
}

template <typename R>
static int ensure_records(rmpcd_particles *p)
{
    size_t need = (size_t)p->N * Rec<R>::kBytes + 64;
    if (p->rec_bytes >= need && p->rec[0] && p->rec[1]) return RMPCD_OK;
    cudaStreamSynchronize(stream());
    cudaFree(p->rec[0]);
    cudaFree(p->rec[1]);
    p->rec[0] = p->rec[1] = nullptr;
    p->rec_bytes = 0;
    RMPCD_CUDA_TRY(cudaMalloc(&p->rec[0], need));
    RMPCD_CUDA_TRY(cudaMalloc(&p->rec[1], need));
    p->rec_bytes = need;
    return RMPCD_OK;
}

template <typename R>
static int bulk_run_fused(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, double tau, int has_alpha,
                          double alpha, int n_intervals)
{
    cudaStream_t st = stream();
    int rc = prepare_shapes<R>();
    if (rc) return rc;
    const ShapeEntry<R> &shape = shape_in_use<R>();
    rc = ensure_records<R>(p);
    if (rc) return rc;
    double sin_a = 1, cos_a = 0;
    if (has_alpha) {
        sin_a = sin(alpha);
        cos_a = cos(alpha);
    }
    {
        PhaseTimer t("pack");
        k_soa_to_rec<R><<<grid_for(p->N, 256), 256, 0, st>>>(cur<R>(p), p->rec[0], p->N);
        RMPCD_CHECK_LAUNCH();
    }
    // image, flags and id stay in the current API arrays, addressed by idx
    const PView<R> side = cur<R>(p);
    int rb = 0;  // record buffer holding the current arrays
    const int nblocks = (c->S + shape.slots - 1) / shape.slots;
    const int ntiles = nblocks;
    // slots fit the packed key for every box up to 2^22 slots (128^3 is 2^21);
    // larger boxes keep plain keys and regroup them in k_perm
    const int pack = c->S <= (1 << kPackSlotBits) ? 1 : 0;
    int *perm = nullptr;  // identity for the first interval (data sorted on entry)
    for (int it = 0; it < n_intervals; it++) {
        uint64_t step_c = r->step;
        uint64_t step_s = r->step + 1;
        r->step += 2;
        double u0, u1, u2, u3;
        rng::uniform2(r->seed, step_s, 0, rng::SHIFT, 0, u0, u1);
        rng::uniform2(r->seed, step_s, 1, rng::SHIFT, 0, u2, u3);
        FusedArgs<R> A;
        A.in = p->rec[rb];
        A.out = p->rec[1 - rb];
        A.perm = perm;
        A.count = c->count;
        A.start = c->start;
        A.S = c->S;
        A.N = p->N;
        A.count_next = c->count_next;
        A.key_out = p->key;
        A.tile_info = c->start_next;
        A.pack = pack;
        A.ix = side.ix;
        A.iy = side.iy;
        A.iz = side.iz;
        A.g_next = grid_of(c);
        A.g_next.origin[0] = u0 - 1;
        A.g_next.origin[1] = u1 - 1;
        A.g_next.origin[2] = u2 - 1;
        A.e0 = c->edges[0];
        A.e1 = c->edges[1];
        A.e2 = c->edges[2];
        A.dt = (R)tau;
        A.sin_a = sin_a;
        A.cos_a = cos_a;
        A.seed = r->seed;
        A.step = step_c;
        A.axes = c->axes;
        A.err = dev_error_word();
        {
            PhaseTimer t("interval_fused");
            shape.kernel<<<nblocks, kFusedThreads, shape.smem, st>>>(A);
            RMPCD_CHECK_LAUNCH();
        }
        rb = 1 - rb;
        for (int k = 0; k < 3; k++) c->origin[k] = A.g_next.origin[k];
        // the G_i arrays are consumed: the G_{i+1} counts become current
        {
            PhaseTimer t("scan");
            int *tmp = c->count;
            c->count = c->count_next;
            c->count_next = tmp;
            rc = exclusive_scan(c->count, c->start, c->cursor, c->S, c->scan_tmp, c->count_next, st);
            if (rc) return rc;
        }
        {
            PhaseTimer t("perm");
            if (pack) {
                k_perm_tiles<<<ntiles, kFusedThreads, 0, st>>>(p->key, c->start_next,
                                                                                       ntiles, c->cursor, p->perm);
                RMPCD_CHECK_LAUNCH();
            } else {
                rc = build_perm_unsorted(c, p);
                if (rc) return rc;
            }
        }
        perm = p->perm;
    }
    // complete the last sort: order each cell, gather the records into the
    // API arrays (which become current)
    PhaseTimer t("sort");
    if constexpr (sizeof(R) == 4) {
        // the other record buffer is free: it holds inv
        int *inv = (int *)p->rec[1 - rb];
        k_perm_to_idx<R><<<grid_for(p->N, 256), 256, 0, st>>>(p->rec[rb], p->perm, inv, p->N);
        RMPCD_CHECK_LAUNCH();
        rc = sort_perm_segments(c, p);
        if (rc) return rc;
        k_idx_to_perm<<<grid_for(p->N, 256), 256, 0, st>>>(p->perm, inv, p->N);
        RMPCD_CHECK_LAUNCH();
    } else {
        rc = sort_perm_segments(c, p);
        if (rc) return rc;
    }
    k_rec_gather_to_soa<R><<<grid_for(p->N, 256), 256, 0, st>>>(p->rec[rb], p->perm, side, alt<R>(p), p->N);
    RMPCD_CHECK_LAUNCH();
    p->cur = 1 - p->cur;
    return RMPCD_OK;
}

}  // namespace rmpcd

using namespace rmpcd;

// species = 1 for a synthetic fluid
__global__ void k_fill_int(int *a, long long n, int v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = v;
}

template <typename R>
static int autotune_t(const int L[3], double tau, int n_intervals, int *best, float *ms_out)
{
    rmpcd_cells *c = nullptr;
    rmpcd_particles *p = nullptr;
    int rc = rmpcd_cells_init(&c, L, 1.0, 0);
    long long N = 10LL * L[0] * L[1] * L[2];
    if (!rc && N > 2000000000LL) rc = fail(RMPCD_ERR_CAPACITY, "rmpcd_bulk_autotune: box too large");
    if (!rc) rc = rmpcd_particles_init(&p, (int)N, 1, nullptr, sizeof(R) == 4 ? RMPCD_FP32 : RMPCD_FP64);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!rc) {
        const double edges[3] = {c->edges[0], c->edges[1], c->edges[2]};
        const uint64_t seed = 0x5eed;
        rmpcd_rng r{seed, 0};
        rc = rmpcd_particles_random_placement(p, edges, nullptr, nullptr, &r);
        if (!rc) rc = rmpcd_particles_maxwell(p, 1.0 / 3.0, seed);
        if (!rc) {
            k_fill_int<<<grid_for(N, 256), 256, 0, stream()>>>(p->species[p->cur], N, 1);
            rc = rmpcd_cells_random_shift(c, &r);
        }
        if (!rc) rc = rmpcd_particles_sort(p, c);
        if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
            rc = fail(RMPCD_ERR_CUDA, "rmpcd_bulk_autotune: event creation failed");
        const int keep = g_shape[sizeof(R) == 8];
        float best_ms = 0;
        int best_k = keep;
        for (int k = 0; !rc && k < n_shapes<R>(); k++) {
            g_shape[sizeof(R) == 8] = k;
            rc = bulk_run_fused<R>(p, c, &r, tau, 0, 0.0, 1);
            if (rc) break;
            cudaEventRecord(e0, stream());
            rc = bulk_run_fused<R>(p, c, &r, tau, 0, 0.0, n_intervals);
            cudaEventRecord(e1, stream());
            if (!rc) rc = sync();
            float ms = 0;
            if (!rc) cudaEventElapsedTime(&ms, e0, e1);
            if (ms_out) ms_out[k] = ms;
            if (!rc && (k == 0 || ms < best_ms)) {
                best_ms = ms;
                best_k = k;
            }
        }
        g_shape[sizeof(R) == 8] = rc ? keep : best_k;
        if (best) *best = g_shape[sizeof(R) == 8];
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    rmpcd_particles_destroy(p);
    rmpcd_cells_destroy(c);
    return rc;
}

extern "C" int rmpcd_bulk_shapes(int precision, int *n, int *slots, int *min_blocks)
{
    RMPCD_ARG(n, "null argument");
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be 32 or 64");
    const bool f = precision == RMPCD_FP32;
    *n = f ? n_shapes<float>() : n_shapes<double>();
    for (int k = 0; k < *n; k++) {
        if (slots) slots[k] = f ? Shapes<float>::list[k].slots : Shapes<double>::list[k].slots;
        if (min_blocks) min_blocks[k] = f ? Shapes<float>::list[k].min_blocks : Shapes<double>::list[k].min_blocks;
    }
    return RMPCD_OK;
}

extern "C" int rmpcd_bulk_set_shape(int precision, int shape)
{
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be 32 or 64");
    const int n = precision == RMPCD_FP32 ? n_shapes<float>() : n_shapes<double>();
    RMPCD_ARG(shape >= 0 && shape < n, "rmpcd_bulk_set_shape: no such shape");
    g_shape[precision == RMPCD_FP64] = shape;
    return RMPCD_OK;
}

extern "C" int rmpcd_bulk_get_shape(int precision, int *shape)
{
    RMPCD_ARG(shape, "null argument");
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be 32 or 64");
    *shape = g_shape[precision == RMPCD_FP64];
    return RMPCD_OK;
}

extern "C" int rmpcd_bulk_autotune(const int L[3], int precision, double tau, int n_intervals, int *best,
                                   float *ms_per_shape)
{
    RMPCD_ARG(L && L[0] > 0 && L[1] > 0 && L[2] > 0, "rmpcd_bulk_autotune: box sides must be > 0");
    RMPCD_ARG(n_intervals >= 1, "rmpcd_bulk_autotune: n_intervals must be >= 1");
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be 32 or 64");
    if (precision == RMPCD_FP32) return autotune_t<float>(L, tau, n_intervals, best, ms_per_shape);
    return autotune_t<double>(L, tau, n_intervals, best, ms_per_shape);
}

extern "C" int rmpcd_bulk_run(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, double tau, int has_alpha,
                              double alpha, int n_intervals)
{
    RMPCD_ARG(p && c && r, "null argument");
    RMPCD_ARG(n_intervals >= 0, "n_intervals must be >= 0");
    if (p->N == 0 || n_intervals == 0) {
        r->step += 2 * (uint64_t)n_intervals;
        return RMPCD_OK;
    }
    if (c->has_walls)
        return fail(RMPCD_ERR_INVALID, "rmpcd_bulk_run: the bulk schedule is periodic (no walls)");
    if (!p->force_zero || !p->force_old_zero) {
        // forces are carried by the sort: run the unfused sequence
        for (int it = 0; it < n_intervals; it++) {
            int rc = rmpcd_simple_mpcd_step(p, c, r, has_alpha, alpha, 0, 0.0, 1);
            if (!rc) rc = rmpcd_mpcd_stream_periodic(p, c, tau);
            if (!rc) rc = rmpcd_cells_random_shift(c, r);
            if (!rc) rc = rmpcd_particles_sort(p, c);
            if (rc) return rc;
        }
        return RMPCD_OK;
    }
    if (p->precision == RMPCD_FP32) return bulk_run_fused<float>(p, c, r, tau, has_alpha, alpha, n_intervals);
    return bulk_run_fused<double>(p, c, r, tau, has_alpha, alpha, n_intervals);
}
