// Host-side support shared by the engine files: error reporting for
// vxb_last_error, and device buffers backed by a process-wide block cache.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vxb {

// Stores a formatted message as the calling thread's vxb_last_error and
// returns `code`.
int failf(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
// Same with a plain message.
int recordError(int code, const char* msg);

#define VXB_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            cudaGetLastError();                                                                         \
            return ::vxb::failf(VXB_ECUDA, "%s @ %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__);    \
        }                                                                                               \
    } while (0)

// Idle device blocks of the process (vxb_host.cu).  cacheTake returns a
// block of at least `bytes` on `device` (its size in *got) or NULL;
// cacheGive takes a block that no queued work uses any more.
void* cacheTake(int device, size_t bytes, size_t* got);
void cacheGive(int device, void* p, size_t bytes);

// A device buffer that only grows, backed by the block cache.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int dev = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    // Owners call this after the device has drained their work.
    void release() {
        if (p) cacheGive(dev, p, cap);
        p = nullptr;
        cap = 0;
    }
    // Grows to at least `bytes` (with headroom).  Callers grow a buffer only
    // while no queued work uses it: every entry point of this library
    // returns with its own work complete, and a call grows its buffers
    // before it queues any.
    int ensure(size_t bytes);
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

}  // namespace vxb
