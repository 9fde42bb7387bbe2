// geam_noalloc.cu -- the v.grad merge (piro_csrgeam3) for callers that may
// not allocate device memory.
//
// Some hosts of this library cannot hand it scratch memory: a simulation that
// reserves its whole device-memory budget before the time loop and forbids
// any further allocation (an allocation can block on the device and fragment
// the pool mid-run), or a caller that runs inside someone else's memory
// manager and only owns the buffers it was given.  For them the merge's only
// scratch -- the per-block partial sums of its row-pointer scan -- lives in a
// fixed array compiled into this library instead of in caller memory.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (36 KB) until the process exits.  It serves merges of up to
// kNoAllocMaxRows rows; larger requests are refused.  All calls share it, and
// it keeps whatever the last call left there: the scan writes every slot it
// later reads, so nothing needs clearing, but two calls whose work overlaps on
// the GPU (different streams, or different host threads on one device) race
// on it and must be serialised by the caller.
//
// Host code cannot use the array's name as a device address (it names a
// host-side stand-in).  The first call on each device, with that device
// current, looks the address up once with cudaGetSymbolAddress and caches it.
// Under CUDA's lazy module loading (the default), that lookup is also where
// the driver loads this file's module onto the device and so reserves the
// array and its code: a caller that fixes its device-memory budget at
// start-up makes one small call per device then, before the budget is fixed
// and before it starts any stream capture.  Later calls touch no allocator.
#include <mutex>

#include "common.cuh"

namespace piro {
size_t scan_workspace_bytes(int64_t N);
}

namespace {

constexpr int64_t kNoAllocMaxRows = 16777216;  // 256^3: 4096 scan blocks of 4096 rows
constexpr size_t kNoAllocBytes = 36864;        // >= the scan's 33,032 bytes at that size
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int scratch_address(void **out)
{
    int dev = -1;
    PIRO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        piro::set_error("piro_csrgeam3_noalloc: device %d beyond the %d devices this build tracks", dev, kMaxDevices);
        return PIRO_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
        if (e != cudaSuccess || !p) {
            piro::set_error("piro_csrgeam3_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return PIRO_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return PIRO_OK;
}

}  // namespace

extern "C" int piro_csrgeam3_noalloc(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA,
                                     const int32_t *rpB, const int32_t *cB, const float *vB, const int32_t *rpC,
                                     const int32_t *cC, const float *vC, const float *v, int32_t *rpD, int32_t *cD,
                                     float *vD, piro_stream_t stream)
{
    if (N <= 0 || N > kNoAllocMaxRows) {
        piro::set_error("piro_csrgeam3_noalloc: %lld rows; this entry point serves 1 to %lld rows "
                        "(its scratch is a fixed %zu-byte array), use piro_csrgeam3 with caller workspace beyond that",
                        (long long)N, (long long)kNoAllocMaxRows, kNoAllocBytes);
        return PIRO_ERR_ARG;
    }
    if (piro::scan_workspace_bytes(N) > kNoAllocBytes) {
        piro::set_error("piro_csrgeam3_noalloc: scan needs %zu bytes, scratch holds %zu",
                        piro::scan_workspace_bytes(N), kNoAllocBytes);
        return PIRO_ERR_ARG;
    }
    if (!(rpA && cA && vA && rpB && cB && vB && rpC && cC && vC && v && rpD && cD && vD)) {
        piro::set_error("piro_csrgeam3_noalloc: a null pointer argument");
        return PIRO_ERR_ARG;
    }
    void *scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc) return rc;
    return piro_csrgeam3(N, rpA, cA, vA, rpB, cB, vB, rpC, cC, vC, v, rpD, cD, vD, scratch, kNoAllocBytes, stream);
}
