// Device memory of the library: one stream-ordered pool per device.
//
// Every allocation the library makes (a tree's arrays, node records, build and
// marching-cubes scratch, CUB temporaries) comes from a pool the library owns,
// created on the first use on a device with an unbounded release threshold:
// freed blocks stay mapped and serve the next call without new page mappings or
// an implicit device synchronisation.  cagr_pool_trim returns memory to the
// CUDA driver; cagr_pool_reserved reports what the pool holds.  The pools are
// separate from the device's default pool and from the framework allocator of
// the caller, so neither trims the other's memory.
#include <atomic>
#include <mutex>
#include <string>

#include "../../include/cagr.h"
#include "internal.h"

namespace cagr {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices] = {};
// fault injection (cagr_debug_fail_allocations_after): allocations still
// allowed before every further one fails; negative = never fail
std::atomic<long long> g_allow{-1};

int current_pool(cudaMemPool_t* out) {
    int dev = 0;
    CAGR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(kErrInvalid, "device index too large");
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        CAGR_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = UINT64_MAX;
        cudaError_t e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return set_error(kErrCuda, std::string("memory pool: ") + cudaGetErrorString(e));
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return kOk;
}

}  // namespace

int pool_alloc(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    long long left = g_allow.load();
    while (left > 0 && !g_allow.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 0)
        return set_error(kErrAlloc, "device allocation of " + std::to_string(bytes) +
                                        " bytes refused (fault injection)");
    cudaMemPool_t pool;
    if (int rc = current_pool(&pool)) return rc;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error(kErrAlloc, "device allocation of " + std::to_string(bytes) +
                                        " bytes: " + cudaGetErrorString(e));
    }
    return kOk;
}

void pool_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

int pool_trim(size_t keep_bytes) {
    cudaMemPool_t pool;
    if (int rc = current_pool(&pool)) return rc;
    CAGR_CUDA(cudaDeviceSynchronize());
    CAGR_CUDA(cudaMemPoolTrimTo(pool, keep_bytes));
    return kOk;
}

int pool_reserved(int64_t* reserved, int64_t* used) {
    cudaMemPool_t pool;
    if (int rc = current_pool(&pool)) return rc;
    uint64_t r = 0, u = 0;
    CAGR_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
    CAGR_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved) *reserved = (int64_t)r;
    if (used) *used = (int64_t)u;
    return kOk;
}

}  // namespace cagr

extern "C" {

int cagr_pool_trim(int64_t keep_bytes) {
    if (keep_bytes < 0) return cagr::set_error(cagr::kErrInvalid, "keep_bytes < 0");
    return cagr::pool_trim((size_t)keep_bytes);
}

int cagr_pool_reserved(int64_t* reserved_bytes, int64_t* used_bytes) {
    return cagr::pool_reserved(reserved_bytes, used_bytes);
}

int cagr_debug_fail_allocations_after(int64_t n) {
    cagr::g_allow.store(n < 0 ? -1 : (long long)n);
    return CAGR_OK;
}

}  // extern "C"
