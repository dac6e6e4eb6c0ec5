// intra_plan.h — the host-side plan of one intra launch (intra.cu): the
// batch's frames, TU records in level order, per-superblock level tables,
// the superblocks in claim order and their waits.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace av1g {

// One frame of the launch, as the kernel reads it.
struct IntraFrame {
    PlaneDev planes[3];
    const int32_t* coeffs;
    av1g_quant_params q;
    int32_t bd, hbd;
    int32_t ssx, ssy, np;
    const uint8_t* maps;  // palette colour-index pool (device)
    PlaneDev side[3];     // inter halves of inter-intra blocks
};

// One superblock of the launch, in claim order.
struct SbItem {
    int32_t frame;
    int32_t lv_first;   // its level table: nlv + 1 entries {first TU, first large TU}
    int32_t nlv;
    int32_t wait_first; // its waits, by level: {level, claim index, progress, 0}
    int32_t nwait;
    int32_t x0, y0;     // luma-sample origin
    int32_t log2sb;
    int32_t tu_first, tu_end;  // its TU records
};

// TUs of at most this many samples run on one warp; larger ones on the CTA.
constexpr int kIntraSmallPx = 256;
// Level-table flag (in .y): other superblocks wait for this level.
constexpr int kLevelPublished = 1 << 30;

struct IntraPlan {
    std::vector<IntraFrame> frames;     // maps still relative: map_base[frame]
    std::vector<size_t> map_base;
    std::vector<uint8_t> maps;          // palette colour indices of all jobs
    std::vector<av1g_intra_tu> tus;     // per superblock, in level order (small before large)
    std::vector<int2> lvtab;
    std::vector<SbItem> items;          // claim order: a topological order of the waits
    std::vector<int4> waits;            // before level x, superblock y has finished z levels
    size_t cache_bytes = 0;             // the largest superblock copy (all planes, u16)
    int width = 0;                      // most superblocks at one dependency depth
    int depth = 0;                      // dependency depths (the critical path in superblocks)
};

// Validates the jobs and builds the plan.  AV1G_OK with no items when there
// is nothing to do.
av1g_status intra_plan(const av1g_intra_job* jobs, int n, IntraPlan& plan, std::string& err);

}  // namespace av1g
