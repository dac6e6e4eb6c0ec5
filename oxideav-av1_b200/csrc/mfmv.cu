// mfmv.cu — motion-field motion vectors: §7.19 storage of a decoded frame's
// per-cell candidate and §7.9 projection of the stored candidates of up to
// four reference frames onto the current frame's 8x8 grid.
//
// Storage replaces the cell loop of decode_frame_spec_tiles
// (src/decoder/frame_driver.rs:1119-1160): one thread per 4x4 cell of every
// frame of the batch, two list candidates in, one candidate out.
//
// Projection replaces motion_field_estimation_core
// (src/inter_pred.rs:7592-7742).  The reference walks each selected source
// reference's cells in raster order and writes the seven projected MVs at the
// position each cell lands on, so a position keeps the values of the LAST
// cell (in pass order, then raster order) that reached it.  Here every cell of
// every pass of every frame is one thread:
//   claim:  a cell whose projection is valid raises its position's 64-bit key
//           to (pass + 1) << 32 | raster index with atomicMax — the key order
//           is the reference's write order, so the maximum is the last writer;
//   write:  one thread per position re-derives the winner's seven projections
//           (or AV1G_MFMV_INVALID when no cell landed) and writes them.
// The pass list (which sources, their sign, the ref_stamp budget) depends
// only on header scalars and on whether a slot exists, matches the frame's
// mi extent and is an inter frame, so the host builds it exactly as the
// reference's selection does (inter_pred.rs:7716-7741).
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace av1g {

namespace {

constexpr int kMaxFrameDistance = 31;   // MAX_FRAME_DISTANCE
constexpr int kMaxOffsetWidth = 8;      // MAX_OFFSET_WIDTH
constexpr int kMaxOffsetHeight = 0;     // MAX_OFFSET_HEIGHT
constexpr int kRefmvsLimit = (1 << 12) - 1;
constexpr int kThreads = 256;

// §7.9.3 Div_Mult[32] (round(2^14 / d)); a table of the specification.
__constant__ int kDivMult[32] = {0,    16384, 8192, 5461, 4096, 3276, 2730, 2340, 2048, 1820, 1638,
                                 1489, 1365,  1260, 1170, 1092, 1024, 963,  910,  862,  819,  780,
                                 744,  712,   682,  655,  630,  606,  585,  564,  546,  528};

// get_relative_dist (inter_pred.rs:3383): the sign-extended difference of
// two order hints in a window of `bits` bits.
__host__ __device__ __forceinline__ int relative_dist(int a, int b, int bits) {
    if (bits == 0) return 0;
    const int d = a - b, m = 1 << (bits - 1);
    return (d & (m - 1)) - (d & m);
}

// §7.9.3 get_mv_projection (inter_pred.rs:7661-7676): products in 64 bits so
// any int16 input is exact; the stored candidates (|mv| < 2^12) stay in the
// reference's 32-bit range.
__device__ __forceinline__ int mv_project(int mv, int num, int den) {
    const int cden = den < kMaxFrameDistance ? den : kMaxFrameDistance;
    const int cnum = num < -kMaxFrameDistance ? -kMaxFrameDistance : (num > kMaxFrameDistance ? kMaxFrameDistance : num);
    const long long v = (long long)mv * cnum * kDivMult[cden];
    const long long r = v >= 0 ? (v + (1 << 13)) >> 14 : -((-v + (1 << 13)) >> 14);
    const long long lim = (1 << 14) - 1;
    return (int)(r < -lim ? -lim : (r > lim ? lim : r));
}

// ---------------------------------------------------------------------------
// §7.19 storage

struct StoreDev {
    int32_t ref_order_hint[7];
    int32_t order_hint, hint_bits, is_inter;
    const int8_t* refs;
    const int16_t* mvs;
    int8_t* out_refs;
    int16_t* out_mvs;
};

__global__ void __launch_bounds__(kThreads) mf_store_kernel(const StoreDev* __restrict__ jobs,
                                                            const int32_t* __restrict__ starts, int n, int total) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int j = find_frame(starts, n, t);
        const StoreDev& J = jobs[j];
        const int cell = t - __ldg(&starts[j]);
        int ref = -1, mr = 0, mc = 0;
        if (J.is_inter) {
            const char2 r = __ldg(reinterpret_cast<const char2*>(J.refs) + cell);
            const short4 mv = __ldg(reinterpret_cast<const short4*>(J.mvs) + cell);
            const int rl[2] = {r.x, r.y};
            const int vr[2] = {mv.x, mv.z}, vc[2] = {mv.y, mv.w};
#pragma unroll
            for (int list = 0; list < 2; list++) {
                const int rr = rl[list];
                if (rr < 1 || rr > 7) continue;
                if (relative_dist(J.ref_order_hint[rr - 1], J.order_hint, J.hint_bits) >= 0) continue;
                if (abs(vr[list]) > kRefmvsLimit || abs(vc[list]) > kRefmvsLimit) continue;
                ref = rr;
                mr = vr[list];
                mc = vc[list];
            }
        }
        J.out_refs[cell] = (int8_t)ref;
        reinterpret_cast<short2*>(J.out_mvs)[cell] = make_short2((short)mr, (short)mc);
    }
}

// ---------------------------------------------------------------------------
// §7.9 projection

// One project_ref pass: source reference `src` (1..7) read from one slot.
struct Pass {
    const int16_t* mvs;
    const int8_t* refs;
    int32_t saved_hints[8];
    int32_t src, dst_sign, job, key;  // key: pass number within its frame + 1
};

struct ProjDev {
    int32_t order_hints[8];
    int32_t order_hint, hint_bits;
    int32_t mi_cols, w8, h8, pad;
    int16_t* out;
    unsigned long long* win;  // h8 x w8 claim keys
};

// The projection of one stored cell (project_ref body,
// inter_pred.rs:7637-7700): false when the cell has no candidate or the
// projected position is invalid; else the position and the candidate.
__device__ __forceinline__ bool project_cell(const Pass& P, const ProjDev& D, int y8, int x8, int& py, int& px,
                                             int& mvr, int& mvc, int& ref_offset) {
    const int cell = (2 * y8 + 1) * D.mi_cols + (2 * x8 + 1);
    const int sref = __ldg(P.refs + cell);
    if (sref <= 0 || sref > 7) return false;
    const int ref_to_cur = relative_dist(D.order_hints[P.src], D.order_hint, D.hint_bits);
    ref_offset = relative_dist(D.order_hints[P.src], P.saved_hints[sref], D.hint_bits);
    if (abs(ref_to_cur) > kMaxFrameDistance || abs(ref_offset) > kMaxFrameDistance || ref_offset <= 0) return false;
    const short2 mv = __ldg(reinterpret_cast<const short2*>(P.mvs) + cell);
    mvr = mv.x;
    mvc = mv.y;
    const int pr = mv_project(mvr, ref_to_cur * P.dst_sign, ref_offset);
    const int pc = mv_project(mvc, ref_to_cur * P.dst_sign, ref_offset);
    // §7.9.4 get_block_position
    auto off8 = [](int d) { return d >= 0 ? d >> 6 : -((-d) >> 6); };
    const int by = (y8 >> 3) << 3, bx = (x8 >> 3) << 3;
    py = y8 + P.dst_sign * off8(pr);
    px = x8 + P.dst_sign * off8(pc);
    if (py < 0 || py >= D.h8 || py < by - kMaxOffsetHeight || py >= by + 8 + kMaxOffsetHeight) return false;
    if (px < 0 || px >= D.w8 || px < bx - kMaxOffsetWidth || px >= bx + 8 + kMaxOffsetWidth) return false;
    return true;
}

__global__ void __launch_bounds__(kThreads) mf_claim_kernel(const Pass* __restrict__ passes,
                                                            const ProjDev* __restrict__ frames,
                                                            const int32_t* __restrict__ starts, int npass,
                                                            int total) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int p = find_frame(starts, npass, t);
        const Pass& P = passes[p];
        const ProjDev& D = frames[P.job];
        const int r = t - __ldg(&starts[p]);
        const int y8 = r / D.w8, x8 = r - y8 * D.w8;
        int py, px, mvr, mvc, off;
        if (!project_cell(P, D, y8, x8, py, px, mvr, mvc, off)) continue;
        atomicMax(D.win + (size_t)py * D.w8 + px, ((unsigned long long)P.key << 32) | (unsigned)r);
    }
}

__global__ void __launch_bounds__(kThreads) mf_write_kernel(const Pass* __restrict__ passes,
                                                            const int32_t* __restrict__ pass_first,
                                                            const ProjDev* __restrict__ frames,
                                                            const int32_t* __restrict__ starts, int n, int total) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int j = find_frame(starts, n, t);
        const ProjDev& D = frames[j];
        const int pos = t - __ldg(&starts[j]);
        const size_t plane = (size_t)D.h8 * D.w8;
        const unsigned long long w = D.win[pos];
        short2 v[7];
#pragma unroll
        for (int k = 0; k < 7; k++) v[k] = make_short2((short)AV1G_MFMV_INVALID, (short)AV1G_MFMV_INVALID);
        if (w) {
            const Pass& P = passes[__ldg(&pass_first[j]) + (int)(w >> 32) - 1];
            const int r = (int)(w & 0xffffffffu);
            const int y8 = r / D.w8, x8 = r - y8 * D.w8;
            int py, px, mvr, mvc, off;
            project_cell(P, D, y8, x8, py, px, mvr, mvc, off);  // valid: it claimed this position
#pragma unroll
            for (int k = 0; k < 7; k++) {
                const int ref_to_dst = relative_dist(D.order_hint, D.order_hints[k + 1], D.hint_bits);
                v[k] = make_short2((short)mv_project(mvr, ref_to_dst, off), (short)mv_project(mvc, ref_to_dst, off));
            }
        }
        short2* out = reinterpret_cast<short2*>(D.out);
#pragma unroll
        for (int k = 0; k < 7; k++) out[k * plane + pos] = v[k];
    }
}

int grid_for(int total) {
    const int want = (total + kThreads - 1) / kThreads, cap = kSMs * 8;
    return want < cap ? want : cap;
}

size_t align256(size_t off) { return (off + 255) & ~(size_t)255; }

}  // namespace

av1g_status mf_store_run(const av1g_mf_store_job* jobs, int n, cudaStream_t s, std::string& err) {
    std::vector<StoreDev> dev(n);
    std::vector<int32_t> starts(n + 1, 0);
    long long total = 0;
    for (int i = 0; i < n; i++) {
        const av1g_mf_store_job& j = jobs[i];
        const long long cells = (long long)j.mi_rows * j.mi_cols;
        if (j.mi_rows < 0 || j.mi_cols < 0 || j.hint_bits < 0 || j.hint_bits > 8 ||
            (cells > 0 && (!j.mf_ref_frames || !j.mf_mvs || ((uintptr_t)j.mf_mvs & 3) ||
                           (j.is_inter_frame && (!j.ref_frames || !j.mvs || ((uintptr_t)j.ref_frames & 1) ||
                                                 ((uintptr_t)j.mvs & 7)))))) {
            err = "mf store job " + std::to_string(i) +
                  ": negative extent, order-hint bits outside 0..8, or a missing / misaligned array";
            return AV1G_EINVAL;
        }
        StoreDev& d = dev[i];
        memcpy(d.ref_order_hint, j.ref_order_hint, sizeof d.ref_order_hint);
        d.order_hint = j.order_hint;
        d.hint_bits = j.hint_bits;
        d.is_inter = j.is_inter_frame != 0;
        d.refs = j.ref_frames;
        d.mvs = j.mvs;
        d.out_refs = j.mf_ref_frames;
        d.out_mvs = j.mf_mvs;
        starts[i] = (int32_t)total;
        total += cells;
        if (total > 0x7fffffffLL) {
            err = "mf store: more than 2^31 cells in one call";
            return AV1G_EINVAL;
        }
    }
    starts[n] = (int32_t)total;
    if (total == 0) return AV1G_OK;
    const size_t off_starts = align256(sizeof(StoreDev) * n);
    const size_t bytes = off_starts + sizeof(int32_t) * (n + 1);
    uint8_t* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, s);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    e = upload_with(buf, bytes, s, [&](uint8_t* h) {
        memcpy(h, dev.data(), sizeof(StoreDev) * n);
        memcpy(h + off_starts, starts.data(), sizeof(int32_t) * (n + 1));
    });
    if (e == cudaSuccess) {
        mf_store_kernel<<<grid_for((int)total), kThreads, 0, s>>>((const StoreDev*)buf,
                                                                  (const int32_t*)(buf + off_starts), n, (int)total);
        e = cudaGetLastError();
    }
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) {
        err = std::string("mf store launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

av1g_status mf_project_run(const av1g_mf_project_job* jobs, int n, cudaStream_t s, std::string& err) {
    enum { LAST = 1, LAST2 = 2, GOLDEN = 4, BWDREF = 5, ALTREF2 = 6, ALTREF = 7 };
    std::vector<ProjDev> frames(n);
    std::vector<Pass> passes;
    std::vector<int32_t> pass_first(n + 1, 0), pos_starts(n + 1, 0), cell_starts;
    long long positions = 0, cells = 0;
    for (int i = 0; i < n; i++) {
        const av1g_mf_project_job& j = jobs[i];
        bool ok = j.mi_rows >= 0 && j.mi_cols >= 0 && j.hint_bits >= 0 && j.hint_bits <= 8;
        for (int k = 0; k < 7; k++) ok = ok && j.ref_frame_idx[k] >= 0 && j.ref_frame_idx[k] < 8;
        const int w8 = j.mi_cols >> 1, h8 = j.mi_rows >> 1;
        if (ok && w8 > 0 && h8 > 0) ok = j.out && !((uintptr_t)j.out & 3);
        for (int k = 0; k < 8 && ok; k++) {
            const av1g_mf_slot& sl = j.slots[k];
            if (sl.mf_ref_frames && sl.mi_rows == j.mi_rows && sl.mi_cols == j.mi_cols && !sl.frame_is_intra)
                ok = sl.mf_mvs && !((uintptr_t)sl.mf_mvs & 3);
        }
        if (!ok) {
            err = "mf project job " + std::to_string(i) +
                  ": negative extent, order-hint bits outside 0..8, ref_frame_idx outside 0..7, or a missing / "
                  "misaligned array";
            return AV1G_EINVAL;
        }
        ProjDev& D = frames[i];
        memset(&D, 0, sizeof D);
        memcpy(D.order_hints, j.order_hints, sizeof D.order_hints);
        D.order_hint = j.order_hint;
        D.hint_bits = j.hint_bits;
        D.mi_cols = j.mi_cols;
        D.w8 = w8;
        D.h8 = h8;
        D.out = j.out;
        pass_first[i] = (int32_t)passes.size();
        pos_starts[i] = (int32_t)positions;
        positions += (long long)w8 * h8;
        if (w8 > 0 && h8 > 0) {
            // the selection of motion_field_estimation_core (inter_pred.rs:7716-7741);
            // a pass "succeeds" when its slot exists, matches the extent and is inter
            auto add = [&](int src, int sign) {
                const av1g_mf_slot& sl = j.slots[j.ref_frame_idx[src - LAST]];
                if (!sl.mf_ref_frames || sl.mi_rows != j.mi_rows || sl.mi_cols != j.mi_cols || sl.frame_is_intra)
                    return false;
                Pass P;
                memset(&P, 0, sizeof P);
                P.mvs = sl.mf_mvs;
                P.refs = sl.mf_ref_frames;
                memcpy(P.saved_hints, sl.saved_order_hints, sizeof P.saved_hints);
                P.src = src;
                P.dst_sign = sign;
                P.job = i;
                P.key = (int32_t)(passes.size() - pass_first[i]) + 1;
                passes.push_back(P);
                return true;
            };
            const av1g_mf_slot& last = j.slots[j.ref_frame_idx[0]];
            const int last_alt = last.mf_ref_frames ? last.saved_order_hints[ALTREF] : 0;
            if (last_alt != j.order_hints[GOLDEN]) add(LAST, -1);
            int stamp = 1;  // MFMV_STACK_SIZE - 2
            if (relative_dist(j.order_hints[BWDREF], j.order_hint, j.hint_bits) > 0 && add(BWDREF, 1)) stamp--;
            if (relative_dist(j.order_hints[ALTREF2], j.order_hint, j.hint_bits) > 0 && add(ALTREF2, 1)) stamp--;
            if (relative_dist(j.order_hints[ALTREF], j.order_hint, j.hint_bits) > 0 && stamp >= 0 &&
                add(ALTREF, 1))
                stamp--;
            if (stamp >= 0) add(LAST2, -1);
        }
        if (positions > 0x7fffffffLL) {
            err = "mf project: more than 2^31 positions in one call";
            return AV1G_EINVAL;
        }
    }
    pass_first[n] = (int32_t)passes.size();
    pos_starts[n] = (int32_t)positions;
    if (positions == 0) return AV1G_OK;
    const int npass = (int)passes.size();
    cell_starts.assign(npass + 1, 0);
    for (int p = 0; p < npass; p++) {
        cell_starts[p] = (int32_t)cells;
        cells += (long long)frames[passes[p].job].w8 * frames[passes[p].job].h8;
        if (cells > 0x7fffffffLL) {
            err = "mf project: more than 2^31 projected cells in one call";
            return AV1G_EINVAL;
        }
    }
    cell_starts[npass] = (int32_t)cells;
    const size_t off_frames = 0;
    const size_t off_passes = align256(off_frames + sizeof(ProjDev) * n);
    const size_t off_pfirst = align256(off_passes + sizeof(Pass) * npass);
    const size_t off_pstart = align256(off_pfirst + sizeof(int32_t) * (n + 1));
    const size_t off_cstart = align256(off_pstart + sizeof(int32_t) * (n + 1));
    const size_t off_win = align256(off_cstart + sizeof(int32_t) * (npass + 1));
    const size_t bytes = off_win + sizeof(unsigned long long) * (size_t)positions;
    uint8_t* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, s);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    for (int i = 0; i < n; i++) frames[i].win = (unsigned long long*)(buf + off_win) + pos_starts[i];
    e = upload_with(buf, off_win, s, [&](uint8_t* h) {
        memcpy(h + off_frames, frames.data(), sizeof(ProjDev) * n);
        if (npass) memcpy(h + off_passes, passes.data(), sizeof(Pass) * npass);
        memcpy(h + off_pfirst, pass_first.data(), sizeof(int32_t) * (n + 1));
        memcpy(h + off_pstart, pos_starts.data(), sizeof(int32_t) * (n + 1));
        memcpy(h + off_cstart, cell_starts.data(), sizeof(int32_t) * (npass + 1));
    });
    if (e == cudaSuccess) e = cudaMemsetAsync(buf + off_win, 0, sizeof(unsigned long long) * (size_t)positions, s);
    if (e == cudaSuccess && cells > 0) {
        mf_claim_kernel<<<grid_for((int)cells), kThreads, 0, s>>>(
            (const Pass*)(buf + off_passes), (const ProjDev*)(buf + off_frames), (const int32_t*)(buf + off_cstart),
            npass, (int)cells);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        mf_write_kernel<<<grid_for((int)positions), kThreads, 0, s>>>(
            (const Pass*)(buf + off_passes), (const int32_t*)(buf + off_pfirst), (const ProjDev*)(buf + off_frames),
            (const int32_t*)(buf + off_pstart), n, (int)positions);
        e = cudaGetLastError();
    }
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) {
        err = std::string("mf project launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

}  // namespace av1g
