// Library-wide services: error strings, the library stream, the device
// error word, per-phase timers and event marks, host Hilbert helpers and
// lj_params_t initialisation.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rmpcd_common.cuh"
#include "hilbert.cuh"
#include "rng.cuh"
#include "timers.cuh"

namespace rmpcd {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

static std::mutex g_mu;
static cudaStream_t g_stream = nullptr;
static unsigned *g_err = nullptr;
static int g_sms = 0;

static void init_once()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_stream) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
    cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
    cudaMalloc(&g_err, sizeof(unsigned));
    cudaMemset(g_err, 0, sizeof(unsigned));
}

cudaStream_t stream()
{
    if (!g_stream) init_once();
    return g_stream;
}

int sm_count()
{
    if (!g_stream) init_once();
    return g_sms;
}

unsigned *dev_error_word()
{
    if (!g_stream) init_once();
    return g_err;
}

int sync()
{
    cudaError_t e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "stream synchronize: %s", cudaGetErrorString(e));
    return RMPCD_OK;
}

int check_dev_error(unsigned *bits_out)
{
    unsigned bits = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&bits, dev_error_word(), sizeof(unsigned),
                                   cudaMemcpyDeviceToHost, stream()));
    RMPCD_CUDA_TRY(cudaStreamSynchronize(stream()));
    if (bits_out) *bits_out = bits;
    if (bits) {
        RMPCD_CUDA_TRY(cudaMemsetAsync(dev_error_word(), 0, sizeof(unsigned), stream()));
        if (bits & DEV_ERR_NLIST_FULL)
            return fail(RMPCD_ERR_NLIST_FULL, "maximum of neighbor list reached");
        if (bits & DEV_ERR_WALL_LOOP)
            return fail(RMPCD_ERR_DEVICE, "wall collision loop exceeded 64 crossings in one step");
        if (bits & DEV_ERR_RATTLE)
            return fail(RMPCD_ERR_DEVICE, "rattle: negative discriminant or bead species outside the mass table");
        if (bits & DEV_ERR_QUAT_LOOP)
            return fail(RMPCD_ERR_DEVICE, "rigid_body_vv1: quaternion iteration did not converge");
        if (bits & DEV_ERR_BULK_UNDRAINED)
            return fail(RMPCD_ERR_DEVICE, "a bulk copy was still pending when its block exited; "
                                          "shared memory of later blocks may have been overwritten");
        if (bits & DEV_ERR_BULK_WAIT)
            return fail(RMPCD_ERR_DEVICE, "bulk interval: an index bulk copy did not complete within its wait limit");
        return fail(RMPCD_ERR_DEVICE, "device error bits 0x%x", bits);
    }
    return RMPCD_OK;
}

// ---------------------------------------------------------------------------
// per-phase timers
// ---------------------------------------------------------------------------
struct TimerSlot {
    std::string name;
    double seconds = 0;
    long long calls = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
};
static std::vector<TimerSlot> g_timers;
static bool g_timers_on = false;
static std::vector<cudaEvent_t> g_event_pool;

static cudaEvent_t take_event()
{
    if (!g_event_pool.empty()) {
        cudaEvent_t e = g_event_pool.back();
        g_event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

static void drain(TimerSlot &t)
{
    for (auto &pr : t.pending) {
        cudaEventSynchronize(pr.second);
        float ms = 0;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        t.seconds += ms * 1e-3;
        g_event_pool.push_back(pr.first);
        g_event_pool.push_back(pr.second);
    }
    t.pending.clear();
}

bool timers_on() { return g_timers_on; }

PhaseTimer::PhaseTimer(const char *name)
{
    if (!g_timers_on) return;
    idx_ = -1;
    for (size_t i = 0; i < g_timers.size(); i++)
        if (g_timers[i].name == name) idx_ = (int)i;
    if (idx_ < 0) {
        g_timers.push_back(TimerSlot());
        g_timers.back().name = name;
        idx_ = (int)g_timers.size() - 1;
    }
    a_ = take_event();
    cudaEventRecord(a_, stream());
}

PhaseTimer::~PhaseTimer()
{
    if (idx_ < 0) return;
    cudaEvent_t b = take_event();
    cudaEventRecord(b, stream());
    TimerSlot &t = g_timers[idx_];
    t.pending.push_back({a_, b});
    t.calls++;
    if (t.pending.size() > 256) drain(t);
}

// event marks
static std::vector<cudaEvent_t> g_marks;

}  // namespace rmpcd

using namespace rmpcd;

extern "C" {

const char *rmpcd_last_error_string(void) { return g_last_error.c_str(); }

int rmpcd_version(int *major, int *minor)
{
    if (major) *major = 0;
    if (minor) *minor = 1;
    return RMPCD_OK;
}

int rmpcd_synchronize(void) { return rmpcd::sync(); }

int rmpcd_set_device(int device)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(RMPCD_ERR_NO_DEVICE, "no CUDA device visible");
    RMPCD_ARG(device >= 0 && device < n, "device index out of range");
    if (g_stream) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != device)
            return fail(RMPCD_ERR_INVALID, "rmpcd_set_device(%d) after the library started on device %d", device, cur);
        return RMPCD_OK;
    }
    RMPCD_CUDA_TRY(cudaSetDevice(device));
    return RMPCD_OK;
}

int rmpcd_get_status(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(RMPCD_ERR_NO_DEVICE, "no CUDA device visible");
    int rc = rmpcd::sync();
    if (rc) return rc;
    return check_dev_error(nullptr);
}

int rmpcd_timers_enable(int on)
{
    g_timers_on = on != 0;
    return RMPCD_OK;
}

int rmpcd_timers_reset(void)
{
    for (auto &t : g_timers) {
        drain(t);
        t.seconds = 0;
        t.calls = 0;
    }
    return RMPCD_OK;
}

int rmpcd_timers_read(int idx, char *name, int name_len, double *seconds, long long *calls)
{
    if (idx < 0 || idx >= (int)g_timers.size())
        return fail(RMPCD_ERR_INVALID, "timer index %d out of range (%d timers)", idx,
                    (int)g_timers.size());
    TimerSlot &t = g_timers[idx];
    drain(t);
    if (name && name_len > 0) {
        strncpy(name, t.name.c_str(), (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (seconds) *seconds = t.seconds;
    if (calls) *calls = t.calls;
    return RMPCD_OK;
}

int rmpcd_mark(int *mark_id)
{
    cudaEvent_t e;
    RMPCD_CUDA_TRY(cudaEventCreate(&e));
    RMPCD_CUDA_TRY(cudaEventRecord(e, stream()));
    g_marks.push_back(e);
    if (mark_id) *mark_id = (int)g_marks.size() - 1;
    return RMPCD_OK;
}

int rmpcd_elapsed_ms(int a, int b, float *ms)
{
    if (a < 0 || b < 0 || a >= (int)g_marks.size() || b >= (int)g_marks.size())
        return fail(RMPCD_ERR_INVALID, "unknown mark");
    RMPCD_CUDA_TRY(cudaEventSynchronize(g_marks[b]));
    RMPCD_CUDA_TRY(cudaEventElapsedTime(ms, g_marks[a], g_marks[b]));
    return RMPCD_OK;
}

int rmpcd_host_alloc(size_t bytes, void **ptr)
{
    RMPCD_ARG(ptr, "null argument");
    RMPCD_CUDA_TRY(cudaHostAlloc(ptr, bytes > 0 ? bytes : 1, cudaHostAllocDefault));
    return RMPCD_OK;
}

int rmpcd_host_free(void *ptr)
{
    if (ptr) RMPCD_CUDA_TRY(cudaFreeHost(ptr));
    return RMPCD_OK;
}

int rmpcd_rng_uniform2(uint64_t seed, uint64_t step, uint32_t index, uint32_t stream_id,
                       uint32_t attempt, double out[2])
{
    RMPCD_ARG(out, "null argument");
    rng::uniform2(seed, step, index, stream_id, attempt, out[0], out[1]);
    return RMPCD_OK;
}

int rmpcd_rng_sphere(uint64_t seed, uint64_t step, uint32_t index, double out[3])
{
    RMPCD_ARG(out, "null argument");
    rng::sphere(seed, step, index, out[0], out[1], out[2]);
    return RMPCD_OK;
}

int rmpcd_rng_normal(uint64_t seed, uint64_t step, uint32_t index, uint32_t sub, double *out)
{
    RMPCD_ARG(out, "null argument");
    *out = rng::normal(seed, step, index, sub);
    return RMPCD_OK;
}

int rmpcd_compact_p_to_h(const int p[3], const int M[3], int *h)
{
    RMPCD_ARG(p && M && h, "null argument");
    *h = hilbert::compact_index(p, M);
    return RMPCD_OK;
}

int rmpcd_compact_h_to_p(int h, const int M[3], int p[3])
{
    RMPCD_ARG(p && M, "null argument");
    hilbert::compact_point(h, M, p);
    return RMPCD_OK;
}

// lj_params_init, src/interaction.f90:38-80; integer powers as gfortran
// expands them (x**6 = x**3 * x**3, x**3 = x*(x*x)).
int rmpcd_lj_init(rmpcd_lj *lj, int n1, int n2, const double *epsilon, const double *sigma,
                  const double *cut)
{
    RMPCD_ARG(lj && epsilon && sigma && cut, "null argument");
    RMPCD_ARG(n1 >= 1 && n2 >= 1 && n1 <= RMPCD_MAX_SPECIES && n2 <= RMPCD_MAX_SPECIES,
              "lj_params_init: species counts must be in 1..4");
    memset(lj, 0, sizeof(*lj));
    lj->n1 = n1;
    lj->n2 = n2;
    for (int i = 0; i < n1 * n2; i++) {
        lj->epsilon[i] = epsilon[i];
        lj->sigma[i] = sigma[i];
        lj->sigma_sq[i] = sigma[i] * sigma[i];
        lj->cut[i] = cut[i];
        lj->cut_sq[i] = cut[i] * cut[i];
        double s3 = sigma[i] * (sigma[i] * sigma[i]);
        double r3 = lj->cut_sq[i] * (lj->cut_sq[i] * lj->cut_sq[i]);
        double s6 = (s3 * s3) / r3;
        lj->cut_energy[i] = 4.0 * lj->epsilon[i] * (s6 * s6 - s6) - sigma[i] * 0;
    }
    return RMPCD_OK;
}

}  // extern "C"
