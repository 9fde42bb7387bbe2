// runtime.cu -- status strings, per-thread error messages, device queries.
#include <stdarg.h>

#include "common.cuh"

namespace piro {

static thread_local char g_err[512] = "";

// Polls a bounded device wait makes before it gives up; negative: each
// kernel's built-in bound (about 2 s of polling).
static std::atomic<long long> g_wait_limit{-1};

long long wait_limit(long long builtin)
{
    const long long v = g_wait_limit.load(std::memory_order_relaxed);
    return v < 0 ? builtin : v;
}

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int sm_count()
{
    static thread_local int dev = -1, count = 0;
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return 148;
    if (d != dev) {
        int c = 0;
        if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || c <= 0) c = 148;
        dev = d;
        count = c;
    }
    return count;
}

}  // namespace piro

extern "C" const char *piro_last_error(void) { return piro::g_err; }

extern "C" int piro_set_wait_limit(long long polls)
{
    piro::g_wait_limit.store(polls < 0 ? -1 : polls, std::memory_order_relaxed);
    return PIRO_OK;
}

extern "C" const char *piro_version(void) { return "piro_b200 0.1 (sm_100a)"; }

extern "C" const char *piro_status_string(int status)
{
    switch (status) {
    case PIRO_OK: return "PIRO_OK";
    case PIRO_ERR_ARG: return "PIRO_ERR_ARG";
    case PIRO_ERR_CONFIG: return "PIRO_ERR_CONFIG";
    case PIRO_ERR_DATATYPE: return "PIRO_ERR_DATATYPE";
    case PIRO_ERR_TABLE_FULL: return "PIRO_ERR_TABLE_FULL";
    case PIRO_ERR_TABLE_SIZE: return "PIRO_ERR_TABLE_SIZE";
    case PIRO_ERR_CUDA: return "PIRO_ERR_CUDA";
    case PIRO_STATUS_STALLED: return "PIRO_STATUS_STALLED";
    case PIRO_ERR_NOT_CONVERGED: return "PIRO_ERR_NOT_CONVERGED";
    case PIRO_ERR_SCHEME: return "PIRO_ERR_SCHEME";
    case PIRO_ERR_NOMEM: return "PIRO_ERR_NOMEM";
    case PIRO_ERR_STATE: return "PIRO_ERR_STATE";
    case PIRO_ERR_ZERO_PIVOT: return "PIRO_ERR_ZERO_PIVOT";
    default: return "PIRO_ERR_UNKNOWN";
    }
}
