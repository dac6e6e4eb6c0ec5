// staging.cu — pinned host staging for descriptor uploads.
//
// The entry points build their device records (frame records, call lists,
// tile prefixes) in host vectors.  A cudaMemcpyAsync from pageable memory
// waits for the stream to drain before it starts, which would stall every
// entry point until the GPU caught up and defeat the pipelining of the serving
// engine.  upload() instead copies the bytes into a pinned block and enqueues
// the copy from there (upload_with() lets the caller build the bytes in the
// block directly); a block is reused once the event recorded after its copy
// has completed.  Idle blocks wait in power-of-two capacity classes; blocks in
// flight queue in enqueue order and only the oldest few are polled per call,
// so an upload costs a handful of event queries however large the pool grows.
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace av1g {

namespace {

struct Block {
    void* p = nullptr;
    size_t cap = 0;  // a power of two
    cudaEvent_t ev = nullptr;
    int device = -1;
};

constexpr size_t kMinBlock = 64 << 10;
constexpr size_t kMaxPinned = (size_t)2 << 30;  // beyond this, copy from pageable memory
constexpr int kClasses = 40;                    // capacity 2^k
constexpr int kPollPerCall = 8;                 // in-flight blocks checked per upload

std::mutex g_mu;
std::vector<Block*> g_free[kClasses];  // idle blocks by capacity class
std::deque<Block*> g_busy;             // blocks whose copy was enqueued, oldest first
size_t g_pinned = 0;

int cls(size_t cap) {
    int k = 0;
    while (((size_t)1 << k) < cap) k++;
    return k;
}

// Moves finished blocks among the oldest kPollPerCall in flight to the free
// lists (streams finish out of order, so a pending block does not stop the
// scan); called with g_mu held.
cudaError_t reap() {
    for (size_t i = 0, polled = 0; i < g_busy.size() && polled < (size_t)kPollPerCall; polled++) {
        Block* b = g_busy[i];
        cudaError_t q = cudaEventQuery(b->ev);
        if (q == cudaErrorNotReady) {
            i++;
            continue;
        }
        if (q != cudaSuccess) return q;
        g_busy.erase(g_busy.begin() + i);
        g_free[cls(b->cap)].push_back(b);
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t upload_with(void* dev, size_t n, cudaStream_t s, const std::function<void(uint8_t*)>& fill) {
    if (n == 0) return cudaSuccess;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    size_t cap = kMinBlock;
    while (cap < n) cap <<= 1;
    Block* pick = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        e = reap();
        if (e != cudaSuccess) return e;
        // the smallest idle block of this device that fits (at most 4x larger)
        for (int k = cls(cap); k < kClasses && k <= cls(cap) + 2 && !pick; k++) {
            auto& fl = g_free[k];
            for (size_t i = 0; i < fl.size(); i++)
                if (fl[i]->device == device) {
                    pick = fl[i];
                    fl[i] = fl.back();
                    fl.pop_back();
                    break;
                }
        }
        if (!pick) {
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
            pick = b;
        }
    }
    fill(static_cast<uint8_t*>(pick->p));
    e = cudaMemcpyAsync(dev, pick->p, n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(pick->ev, s);
    std::lock_guard<std::mutex> lk(g_mu);
    if (e == cudaSuccess) g_busy.push_back(pick);
    else g_free[cls(pick->cap)].push_back(pick);  // nothing was enqueued from it
    return e;
}

cudaError_t upload(void* dev, const void* host, size_t n, cudaStream_t s) {
    return upload_with(dev, n, s, [&](uint8_t* p) { memcpy(p, host, n); });
}

namespace {
struct ParamChunk {
    uint4 w[kUploadChunk / 16];
};
__global__ void __launch_bounds__(256) param_store_kernel(const __grid_constant__ ParamChunk c, uint4* dst, int nvec) {
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = c.w[i];
}
}  // namespace

cudaError_t upload_by_launch(void* dev, const void* host, size_t n, cudaStream_t s) {
    if ((n & 15) || (reinterpret_cast<uintptr_t>(dev) & 15)) return cudaErrorInvalidValue;
    ParamChunk c;
    const uint8_t* src = static_cast<const uint8_t*>(host);
    uint4* dst = static_cast<uint4*>(dev);
    for (size_t off = 0; off < n; off += kUploadChunk) {
        const size_t len = n - off < kUploadChunk ? n - off : kUploadChunk;
        memcpy(c.w, src + off, len);
        param_store_kernel<<<1, 256, 0, s>>>(c, dst + off / 16, static_cast<int>(len / 16));
    }
    return cudaGetLastError();
}

}  // namespace av1g
