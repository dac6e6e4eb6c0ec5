// staging.cu — pinned host staging for descriptor uploads.
//
// The entry points build their device records (frame records, call lists,
// tile prefixes) in host vectors.  A cudaMemcpyAsync from pageable memory
// waits for the stream to drain before it starts, which would stall every
// entry point until the GPU caught up and defeat the pipelining of the serving
// engine.  upload() instead copies the bytes into a pinned block and enqueues
// the copy from there (upload_with() lets the caller build the bytes in the
// block directly); a block is reused once the event recorded after its copy
// has completed.
#include <cstring>
#include <functional>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace av1g {

namespace {

struct Block {
    void* p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    int device = -1;
    bool busy = false;  // taken by a caller that has not recorded its event yet
};

constexpr size_t kMinBlock = 64 << 10;
constexpr size_t kMaxPinned = (size_t)2 << 30;  // beyond this, copy from pageable memory

std::mutex g_mu;
std::vector<Block*> g_blocks;  // stable addresses: callers hold a block outside the lock
size_t g_pinned = 0;

}  // namespace

cudaError_t upload_with(void* dev, size_t n, cudaStream_t s, const std::function<void(uint8_t*)>& fill) {
    if (n == 0) return cudaSuccess;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    Block* pick = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (Block* b : g_blocks) {
            if (b->busy || b->device != device || b->cap < n) continue;
            cudaError_t q = cudaEventQuery(b->ev);
            if (q == cudaSuccess) {
                if (!pick || b->cap < pick->cap) pick = b;
            } else if (q != cudaErrorNotReady) {
                return q;
            }
        }
        if (!pick) {
            size_t cap = kMinBlock;
            while (cap < n) cap <<= 1;
            if (g_pinned + cap > kMaxPinned) {
                // beyond the pinned budget: a copy from pageable memory, which
                // returns once the driver has staged the bytes
                std::vector<uint8_t> tmp(n);
                fill(tmp.data());
                return cudaMemcpyAsync(dev, tmp.data(), n, cudaMemcpyHostToDevice, s);
            }
            auto* b = new Block();
            b->device = device;
            b->cap = cap;
            e = cudaHostAlloc(&b->p, cap, cudaHostAllocPortable);
            if (e != cudaSuccess) {
                delete b;
                return e;
            }
            e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
            if (e != cudaSuccess) {
                cudaFreeHost(b->p);
                delete b;
                return e;
            }
            g_pinned += cap;
            g_blocks.push_back(b);
            pick = b;
        }
        pick->busy = true;
    }
    fill(static_cast<uint8_t*>(pick->p));
    e = cudaMemcpyAsync(dev, pick->p, n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(pick->ev, s);
    std::lock_guard<std::mutex> lk(g_mu);
    pick->busy = false;
    return e;
}

cudaError_t upload(void* dev, const void* host, size_t n, cudaStream_t s) {
    return upload_with(dev, n, s, [&](uint8_t* p) { memcpy(p, host, n); });
}

}  // namespace av1g
