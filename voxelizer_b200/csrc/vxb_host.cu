// Error reporting and the process-wide device block cache.

#include "vxb.h"
#include "vxb_host.h"

#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>

namespace vxb {

namespace {

thread_local std::string g_lastError;

// Idle device blocks.  Buffers of destroyed voxelizers and batches (and
// buffers outgrown by a larger request) come here instead of cudaFree, and
// the next allocation of a similar size takes them back, so a caller that
// builds one voxelizer per mesh pays cudaMalloc / cudaFree once.  Idle bytes
// are capped; vxb_trim_cache returns them all to the driver.
struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, std::pair<int, void*>> idle;   // bytes -> (device, block)
    size_t idleBytes = 0;
    static constexpr size_t kBudget = 16ull << 30;
};

BlockCache& blockCache() {
    static BlockCache* c = new BlockCache;   // never destroyed: blocks outlive static destructors
    return *c;
}

}  // namespace

int failf(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return code;
}

int recordError(int code, const char* msg) { return failf(code, "%s", msg); }

void* cacheTake(int device, size_t bytes, size_t* got) {
    BlockCache& c = blockCache();
    std::lock_guard<std::mutex> lock(c.mu);
    for (auto it = c.idle.lower_bound(bytes); it != c.idle.end() && it->first <= 2 * bytes + (1u << 20); ++it) {
        if (it->second.first != device) continue;
        void* p = it->second.second;
        *got = it->first;
        c.idleBytes -= it->first;
        c.idle.erase(it);
        return p;
    }
    return nullptr;
}

void cacheGive(int device, void* p, size_t bytes) {
    BlockCache& c = blockCache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (c.idleBytes + bytes <= BlockCache::kBudget) {
            c.idle.emplace(bytes, std::make_pair(device, p));
            c.idleBytes += bytes;
            return;
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(p);
    if (cur != device) cudaSetDevice(cur);
}

int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return 0;
    release();
    cudaGetDevice(&dev);
    size_t got = 0;
    if ((p = cacheTake(dev, bytes, &got))) {
        cap = got;
        return 0;
    }
    const size_t want = bytes + bytes / 2 + 256;
    const cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return failf(VXB_ENOMEM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    cap = want;
    return 0;
}

}  // namespace vxb

extern "C" {

const char* vxb_last_error(void) { return vxb::g_lastError.c_str(); }

vxb_status vxb_trim_cache(void) {
    vxb::BlockCache& c = vxb::blockCache();
    std::multimap<size_t, std::pair<int, void*>> idle;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        idle.swap(c.idle);
        c.idleBytes = 0;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& e : idle) {
        cudaSetDevice(e.second.first);
        cudaFree(e.second.second);
    }
    cudaSetDevice(cur);
    return VXB_OK;
}

}  // extern "C"
