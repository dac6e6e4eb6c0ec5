// common.cuh — shared device-side definitions for the AV1 B200 engine.
//
// FrameDev is the per-frame record every post-filter kernel reads: a copy of
// the resolved frame header plus the device pointers of the frame's grids and
// planes, with each stage's effective input/output planes already resolved
// from the header's gating (src/decoder/frame_driver.rs:832-836, 870, 906,
// 971, 1060).  A batch of frames is an array of FrameDev in device memory;
// each stage kernel walks a flattened list of work tiles over all frames of
// the batch (one launch per stage, any mix of sizes and bit depths).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "av1g.h"

namespace av1g {

// An NVTX range over a host scope (a stage's planning and launches), so that
// a profiler's timeline shows each stage by name; free when no tool listens.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr int kSMs = 148;  // B200

struct PlaneDev {
    uint8_t* p;       // base pointer (u8 for 8-bit content, u16 otherwise)
    int32_t stride;   // bytes
    int32_t w, h;     // samples
};

enum Stage { ST_DEBLOCK = 0, ST_CDEF, ST_SUPERRES, ST_LR, ST_GRAIN, ST_COUNT };

struct FrameDev {
    av1g_frame_header h;
    av1g_mi_grid g;
    const int8_t* cdef_idx;
    const av1g_lr_unit* lr_units[3];
    int32_t lr_unit_rows[3], lr_unit_cols[3];
    int32_t hbd;  // 1 when samples are stored as u16
    // effective planes per stage
    PlaneDev recon[3];     // deblock input
    PlaneDev deb[3];       // deblock output / CDEF input
    PlaneDev cdef[3];      // CDEF output
    PlaneDev updeb[3];     // deblocked frame as seen by LR (upscaled when superres)
    PlaneDev upcdef[3];    // CDEF frame as seen by LR (upscaled when superres)
    PlaneDev lr[3];        // LR output (the reference payload, cropped view)
    PlaneDev out[3];       // film grain output
    int32_t do_stage[ST_COUNT];
    // deblock scratch: per-4x4-cell edge codes of each plane
    uint16_t* lf_codes[3];
    // film grain scratch: templates, scaling LUTs, per-stripe offsets
    int16_t* grain_tmpl;   // 3 x 73 x 82
    uint8_t* grain_lut;    // 3 x 256
    uint8_t* grain_offs;   // nstripes x nblocks
    int32_t grain_nblocks;
};

// Flattened tile list of one stage over a batch: frame f owns tiles
// [starts[f], starts[f+1]).
__device__ __forceinline__ int find_frame(const int32_t* starts, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&starts[mid]) <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int clip3(int lo, int hi, int x) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ int round2(int x, int n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }
__device__ __forceinline__ long long round2ll(long long x, int n) {
    return n == 0 ? x : (x + (1LL << (n - 1))) >> n;
}
__device__ __forceinline__ int floor_log2u(unsigned x) { return x ? 31 - __clz(x) : 0; }

// Enqueues a host-to-device copy of n bytes through a pinned staging block
// (returns once enqueued; the host bytes may be reused immediately).
cudaError_t upload(void* dev, const void* host, size_t n, cudaStream_t s);
cudaError_t upload_with(void* dev, size_t n, cudaStream_t s, const std::function<void(uint8_t*)>& fill);
// Writes n bytes (a multiple of 16, dev 16-byte aligned) by kernel launches
// that carry the bytes as their parameters, kUploadChunk bytes per launch:
// no copy engine, so a small record upload on a compute stream never queues
// behind large copies another stream has on the copy engines.
constexpr size_t kUploadChunk = 16384;
cudaError_t upload_by_launch(void* dev, const void* host, size_t n, cudaStream_t s);

__device__ __forceinline__ int ld_px(const PlaneDev& P, int hbd, int y, int x) {
    const uint8_t* row = P.p + (size_t)y * P.stride;
    return hbd ? (int)reinterpret_cast<const uint16_t*>(row)[x] : (int)row[x];
}
__device__ __forceinline__ void st_px(const PlaneDev& P, int hbd, int y, int x, int v) {
    uint8_t* row = P.p + (size_t)y * P.stride;
    if (hbd) reinterpret_cast<uint16_t*>(row)[x] = (uint16_t)v;
    else row[x] = (uint8_t)v;
}

// Launch shape of a post-filter stage: resident CTAs per SM of its
// grid-stride launch and, for superres, the output samples of a row per tile
// (256, 512 or 1024).  autotune.cu holds the current choice per stage and
// sample width; av1g_autotune_postfilter measures the candidates.
struct StageShape {
    int ctas_per_sm;
    int tile;
};
StageShape stage_shape(int stage, int hbd);
void set_stage_shape(int stage, int hbd, const StageShape& sh);
bool shape_valid(int stage, const StageShape& sh);
int shape_grid(const StageShape& sh, int total);  // min(total, SMs x ctas_per_sm)
av1g_status save_shapes(const char* path, std::string& err);
av1g_status load_shapes(const char* path, std::string& err);

// Stage launchers (one per .cu file).  Each takes the batch's device
// FrameDev array, the stage's tile-start array (n+1 entries, device), the
// total tile count and the launch shape.
void launch_deblock(const FrameDev* frames, const int32_t* starts, int n, int total, int max_cells,
                    const StageShape& sh, cudaStream_t s);
void launch_cdef(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
                 cudaStream_t s);
void launch_superres(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
                     cudaStream_t s);
void launch_lr(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
               cudaStream_t s);
void launch_grain(const FrameDev* frames, const int32_t* starts_tmpl, const int32_t* starts_blend,
                  int n, int total_tmpl, int total_blend, const StageShape& sh, cudaStream_t s);

// Host-side tile counts (must match the kernels' tile decomposition).
int tiles_deblock(const FrameDev& f);
int cells_deblock(const FrameDev& f);  // 4x4 cells over all planes (deblock scratch: 2 bytes each)
int tiles_cdef(const FrameDev& f);
int tiles_superres(const FrameDev& f, int tile);
int tiles_lr(const FrameDev& f);
int tiles_grain_blend(const FrameDev& f);

}  // namespace av1g
