// intra.cu — §7.11.2 intra prediction, §7.11.5 chroma from luma and intra
// reconstruction as one persistent superblock-wavefront launch.
//
// Replaces predict_intra_into_curr_frame (src/cdf.rs:16789),
// intra_predict_block_samples (cdf.rs:16990-17250), the mode kernels
// (cdf.rs:1348-3120) and predict_chroma_from_luma_into_curr_frame
// (cdf.rs:17256) in the order transform_block_emit runs them per TU
// (cdf.rs:32540-32910): predict, CfL, dequant + inverse transform + merge.
//
// Dependencies.  An intra TU reads final samples of the row above and the
// column to its left (up to twice its size), the co-located luma for CfL and,
// for intra block copy, a window of the frame.  The host walks each frame's
// TUs in decode order and records every area a TU reads:
//  - between superblocks, B waits for A when a TU of one of them reads the
//    other's area and A comes first in decode order (a read of a later
//    superblock's area orders the later one after the reader, as sequential
//    decoding does), so the waits form a DAG ordered by decode order;
//  - inside a superblock, a TU's level is one above the last writer of each
//    4x4 cell it reads or writes and the last reader of each cell it writes,
//    so the TUs of one level are independent of one another.
// One persistent launch covers the batch.  A CTA claims superblocks from an
// atomic counter in a topological order (dependency depth, frame, decode
// order), stages the superblock's samples in shared memory, waits (bounded)
// for the superblocks it depends on, runs the levels — a level's small TUs one
// per warp, then its large TUs with the whole CTA — writes the samples back and
// publishes a done flag.  A CTA only waits for superblocks claimed before its
// own, by CTAs that are running, so every wait ends; the time bound only
// guards against a broken invariant: a wait that runs out sets its frame's
// abort word in the launch's control block, every superblock of that frame
// then skips its remaining TUs (still publishing its levels, so no wait of
// the launch is left hanging), and the host reports that frame of that
// launch as AV1G_EDEVICE.  Other frames of the batch are not affected: waits
// never cross frames.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "intra_plan.h"
#include "itx.cuh"
#include "wedge.cuh"

namespace av1g {

namespace {

using namespace itx;

constexpr int kT = 128;             // threads per CTA
constexpr int kNW = kT / 32;        // warps per CTA
constexpr int kSmallPx = kIntraSmallPx;
constexpr int kLvChunk = 64;        // level-table entries staged at a time
constexpr int kTuWin = 128;         // TU records staged at a time
constexpr int kWaitWin = 32;        // waits staged per superblock (more: read from HBM)
constexpr long long kWaitNs = 2000000000LL;  // the bound of one dependency wait

__constant__ AV1T_MODE_TO_ANGLE_TYPE c_mode_angle AV1T_MODE_TO_ANGLE_DIMS = AV1T_MODE_TO_ANGLE_INIT;
__constant__ AV1T_DR_INTRA_DERIVATIVE_TYPE c_dr AV1T_DR_INTRA_DERIVATIVE_DIMS = AV1T_DR_INTRA_DERIVATIVE_INIT;
__constant__ AV1T_INTRA_EDGE_KERNEL_TYPE c_edge_k AV1T_INTRA_EDGE_KERNEL_DIMS = AV1T_INTRA_EDGE_KERNEL_INIT;
__constant__ AV1T_INTRA_FILTER_TAPS_TYPE c_fi_taps AV1T_INTRA_FILTER_TAPS_DIMS = AV1T_INTRA_FILTER_TAPS_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_4X4_TYPE c_sm4 AV1T_SM_WEIGHTS_TX_4X4_DIMS = AV1T_SM_WEIGHTS_TX_4X4_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_8X8_TYPE c_sm8 AV1T_SM_WEIGHTS_TX_8X8_DIMS = AV1T_SM_WEIGHTS_TX_8X8_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_16X16_TYPE c_sm16 AV1T_SM_WEIGHTS_TX_16X16_DIMS = AV1T_SM_WEIGHTS_TX_16X16_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_32X32_TYPE c_sm32 AV1T_SM_WEIGHTS_TX_32X32_DIMS = AV1T_SM_WEIGHTS_TX_32X32_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_64X64_TYPE c_sm64 AV1T_SM_WEIGHTS_TX_64X64_DIMS = AV1T_SM_WEIGHTS_TX_64X64_INIT;
__constant__ AV1T_SUBPEL_FILTERS_TYPE c_subpel AV1T_SUBPEL_FILTERS_DIMS = AV1T_SUBPEL_FILTERS_INIT;

// The superblock's area in each plane and where the shared-memory copy keeps it.
struct SbCtx {
    int x0[3], y0[3], w[3], h[3], off[3];
};

__device__ const AV1T_II_WEIGHTS_1D_TYPE g_ii_w AV1T_II_WEIGHTS_1D_DIMS = AV1T_II_WEIGHTS_1D_INIT;
__device__ const wedge::Master g_wmaster = wedge::kMaster;
// The wait bound in effect (kWaitNs unless a test shortens it, see
// av1g_test_intra_wait_fault).
__device__ long long g_wait_ns = kWaitNs;

// The intra half of an inter-intra block: blend of the intra prediction
// with the inter half (mask_blend_interintra, src/inter_pred.rs:3272).  The
// mask is the §7.11.3.13 smooth mask on the plane block (read at [i][j]
// directly) or the §7.11.3.11 wedge mask on the luma grid (orientation
// resolved by the host into palette_map).
template <int W, int H>
__device__ __forceinline__ int interintra_px(const IntraFrame& F, const av1g_intra_tu& t, int i, int j, int intra,
                                             int inter, int maxv) {
    int m;
    if (t.interintra == 2) {
        const uint32_t o = t.palette_map;
        const wedge::Orient w{(uint8_t)(o & 0xff), (uint8_t)((o >> 8) & 0xff), (uint8_t)((o >> 16) & 0xff),
                              (uint8_t)(o >> 24)};
        m = wedge::mask_px(g_wmaster, w, t.plane ? F.ssx : 0, t.plane ? F.ssy : 0, i, j);
    } else {
        constexpr int scale = 128 / (W > H ? W : H);
        const int mode = t.interintra_mode;
        m = mode == 1 ? __ldg(&g_ii_w[i * scale]) : mode == 2 ? __ldg(&g_ii_w[j * scale])
          : mode == 3 ? __ldg(&g_ii_w[min(i, j) * scale]) : 32;
    }
    return min(max((m * intra + (64 - m) * inter + 32) >> 6, 0), maxv);
}

// A TU is run either by one warp or by the whole CTA; both expose a rank,
// a size and a barrier over exactly the threads that run the TU.
struct WarpG {
    static constexpr int N = 32;
    int r;
    __device__ __forceinline__ void sync() const { __syncwarp(); }
};
struct CtaG {
    static constexpr int N = kT;
    int r;
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Per-group scratch: edge arrays (index 0 == position -2), the dense
// coefficient / residual block, the reduction slots and the TU record.
template <int E, int PX>
struct Scr {
    uint16_t above[E], left[E], dup[E];
    int buf[PX];
    long long red[kNW];
    av1g_intra_tu tu;
};
using WScr = Scr<96, kSmallPx>;  // W + H <= 40 for the small sizes: 2 + 2 * 40 entries at most
using CScr = Scr<272, 64 * 64>;  // 2 * (64 + 64) + 2 rounded up

struct alignas(16) Shared {
    union {
        WScr w[kNW];
        CScr c;
    } s;
    IntraFrame fr;  // the superblock's frame record
    int2 lv[kLvChunk + 1];
    int4 wv[kWaitWin];
    SbCtx sb;
    int idx, abort_seen;
};
static_assert(sizeof(IntraFrame) % 4 == 0, "frame record copied as words");

// The batch's residual blocks (intra_res_kernel); an intra TU's device record
// carries its block's offset in res.coeff_offset.
struct Pool {
    const int32_t* res;
}; 
constexpr size_t kSharedBytes = (sizeof(Shared) + 15) & ~(size_t)15;

__device__ __forceinline__ const uint8_t* sm_weights(int log2n) {
    return log2n == 2 ? c_sm4 : log2n == 3 ? c_sm8 : log2n == 4 ? c_sm16 : log2n == 5 ? c_sm32 : c_sm64;
}

// Sum over the group (every thread of it calls).
template <class G, class S>
__device__ __forceinline__ long long gsum(const G& g, S& s, long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
    if constexpr (G::N > 32) {
        if ((g.r & 31) == 0) s.red[g.r >> 5] = v;
        __syncthreads();
        long long t = 0;
#pragma unroll
        for (int k = 0; k < G::N / 32; k++) t += s.red[k];
        __syncthreads();
        return t;
    } else {
        return v;
    }
}

// A sample of plane p at (y, x), inside the plane: from the shared-memory
// copy when it lies in the current superblock, else from HBM (an earlier
// superblock's final samples, published by its done flag; read past L1).
__device__ __forceinline__ int rdp(const IntraFrame& F, const SbCtx& c, const uint16_t* cache, int p, int y, int x) {
    const int ly = y - c.y0[p], lx = x - c.x0[p];
    if ((unsigned)ly < (unsigned)c.h[p] && (unsigned)lx < (unsigned)c.w[p]) return cache[c.off[p] + ly * c.w[p] + lx];
    const PlaneDev& P = F.planes[p];
    const uint8_t* row = P.p + (size_t)y * P.stride;
    return F.hbd ? (int)__ldcg(reinterpret_cast<const unsigned short*>(row) + x) : (int)__ldcg(row + x);
}

// intra_edge_filter_strength_selection (cdf.rs:2610)
__device__ int strength_sel(int w, int h, int ft, int delta) {
    int d = abs(delta), wh = w + h, st = 0;
    if (ft == 0) {
        if (wh <= 8) { if (d >= 56) st = 1; }
        else if (wh <= 16) { if (d >= 40) st = 1; }
        else if (wh <= 24) { if (d >= 8) st = 1; if (d >= 16) st = 2; if (d >= 32) st = 3; }
        else if (wh <= 32) { st = 1; if (d >= 4) st = 2; if (d >= 32) st = 3; }
        else st = 3;
    } else {
        if (wh <= 8) { if (d >= 40) st = 1; if (d >= 64) st = 2; }
        else if (wh <= 16) { if (d >= 20) st = 1; if (d >= 48) st = 2; }
        else if (wh <= 24) { if (d >= 4) st = 3; }
        else st = 3;
    }
    return st;
}
// intra_edge_upsample_selection (cdf.rs:2588)
__device__ int upsample_sel(int w, int h, int ft, int delta) {
    int d = abs(delta);
    if (d == 0 || d >= 40) return 0;
    return ft == 0 ? (w + h <= 16) : (w + h <= 8);
}

// intra_edge_filter (cdf.rs:2760) on an edge array (index 0 == position -2), in parallel
template <class G, class S>
__device__ void edge_filter(const G& g, S& s, uint16_t* e, int sz, int strength) {
    if (strength == 0 || sz == 0) return;  // uniform over the group
    for (int i = g.r; i < sz; i += G::N) s.dup[i] = e[i + 1];
    g.sync();
    for (int i = 1 + g.r; i < sz; i += G::N) {
        int acc = 0;
#pragma unroll
        for (int j = 0; j < 5; j++) acc += c_edge_k[strength - 1][j] * s.dup[clip3(0, sz - 1, i - 2 + j)];
        e[i + 1] = (uint16_t)max((acc + 8) >> 4, 0);
    }
    g.sync();
}

// intra_edge_upsample (cdf.rs:2700), in parallel
template <class G, class S>
__device__ void edge_upsample(const G& g, S& s, uint16_t* e, int n, int bd) {
    if (g.r == 0) {
        s.dup[0] = e[1];
        s.dup[1] = e[1];
        s.dup[n + 2] = e[n + 1];
    }
    for (int i = g.r; i < n; i += G::N) s.dup[i + 2] = e[i + 2];
    g.sync();
    const int maxv = (1 << bd) - 1;
    if (g.r == 0) e[0] = s.dup[0];
    for (int i = g.r; i < n; i += G::N) {
        int sum = -s.dup[i] + 9 * s.dup[i + 1] + 9 * s.dup[i + 2] - s.dup[i + 3];
        int r = sum >= 0 ? (sum + 8) >> 4 : -(((-sum) + 8) >> 4);
        e[2 * i + 1] = (uint16_t)clip3(0, maxv, r);
        e[2 * i + 2] = (uint16_t)min((int)s.dup[i + 2], maxv);
    }
    g.sync();
}

// Dequantize (dequantize_step1, cdf.rs:13655-13703) and inverse transform
// (transform.rs:707-789) one TU's residual, stored as w*h int32 in sample
// orientation (the FLIPADST flips of curr_frame_step3_merge, cdf.rs:17398-17470,
// already applied).  cf holds the compact levels, cf[q] == level[g.r + q * G::N].
template <int TX, class G, class S>
__device__ __forceinline__ void residual_store(const G& g, S& s, const IntraFrame& R, const av1g_tu& tu, const int* cf,
                                               int32_t* out) {
    constexpr int W = kTxW[TX], H = kTxH[TX];
    constexpr int LW = ilog2<W>(), LH = ilog2<H>();
    constexpr int TW = W < 32 ? W : 32, TH = H < 32 ? H : 32, NC = TW * TH, K = (NC + G::N - 1) / G::N;
    constexpr int ABS_D = LW > LH ? LW - LH : LH - LW;
    const int bd = R.bd;
    const int seg = tu.segment_id > 7 ? 7 : tu.segment_id;
    const bool lossless = R.q.lossless[seg] != 0;
    for (int k = g.r; k < W * H; k += G::N) s.buf[k] = 0;
    g.sync();
    {
        const av1g_quant_params& q = R.q;
        int qidx;
        if (q.segmentation_enabled && q.seg_alt_q_active[seg]) {
            int data = q.seg_alt_q_data[seg];
            qidx = clip3(0, 255, (q.delta_q_present ? tu.current_q_index : q.base_q_idx) + data);
        } else {
            qidx = q.delta_q_present ? tu.current_q_index : q.base_q_idx;
        }
        const int p = tu.plane;
        const int ddc = p == 0 ? q.delta_q_y_dc : (p == 1 ? q.delta_q_u_dc : q.delta_q_v_dc);
        const int dac = p == 0 ? 0 : (p == 1 ? q.delta_q_u_ac : q.delta_q_v_ac);
        const int row = min((max(bd, 8) - 8) >> 1, 2);
        const int dcq = c_dcq[row][clip3(0, 255, qidx + ddc)], acq = c_acq[row][clip3(0, 255, qidx + dac)];
        const int qml = q.seg_qm_level[p][seg];
        const bool qm = q.using_qmatrix && tu.tx_type < 9 && qml < 15;
        constexpr int denom_sh = (TX == 3 || TX == 9 || TX == 10 || TX == 17 || TX == 18) ? 1
                               : (TX == 4 || TX == 11 || TX == 12) ? 2 : 0;
        const long long cmax = (1LL << (7 + bd)) - 1, cmin = -(1LL << (7 + bd));
#pragma unroll
        for (int qq = 0; qq < K; qq++) {
            const int k = g.r + qq * G::N;
            if (NC % G::N == 0 || k < NC) {
                const int i = k / TW, j = k % TW;
                long long qv = k == 0 ? dcq : acq;
                if (qm) qv = (qv * g_qm[qml][p > 0][c_qm_off[TX] + k] + 16) >> 5;
                const long long dq = (long long)cf[qq] * qv;
                const long long mag = (dq < 0 ? -dq : dq) & 0xFFFFFF;
                const long long v = (dq < 0 ? -mag : mag) / (1 << denom_sh);  // truncating division, as the reference
                s.buf[i * W + j] = (int)min(max(v, cmin), cmax);
            }
        }
    }
    g.sync();
    const Clamp rr{-(1 << (bd + 7)), (1 << (bd + 7)) - 1};
    const int crb = bd + 6 > 16 ? bd + 6 : 16;
    const Clamp cr{-(1 << (crb - 1)), (1 << (crb - 1)) - 1};
    if (g.r < H && g.r < 32) {
        int t[W];
        int* rowp = s.buf + g.r * W;
#pragma unroll
        for (int j = 0; j < W; j++) t[j] = j < 32 ? rowp[j] : 0;
        if constexpr (ABS_D == 1) {
#pragma unroll
            for (int j = 0; j < W; j++) t[j] = rnd12((long long)t[j] * 2896);
        }
        constexpr int kRs = kRowShift[TX];
        const int rsh = lossless ? 0 : kRs;
        if (lossless) {
            if constexpr (W == 4) iwht4(t, 2);
        } else {
            tx1d<LW>(t, row_kind(tu.tx_type), rr);
        }
#pragma unroll
        for (int j = 0; j < W; j++) {
            int v = rsh ? (t[j] + (1 << (rsh - 1))) >> rsh : t[j];
            rowp[j] = min(max(v, cr.lo), cr.hi);
        }
    }
    g.sync();
    if (g.r < W) {
        const int lane = g.r;
        int t[H];
#pragma unroll
        for (int i = 0; i < H; i++) t[i] = s.buf[i * W + lane];
        if (lossless) {
            if constexpr (H == 4) iwht4(t, 0);
        } else {
            tx1d<LH>(t, col_kind(tu.tx_type), cr);
        }
        const int csh = lossless ? 0 : 4;
        const int tt = tu.tx_type;
        const bool fud = tt == 4 || tt == 8 || tt == 14 || tt == 6;
        const bool flr = tt == 5 || tt == 7 || tt == 15 || tt == 6;
        const int x = flr ? W - 1 - lane : lane;
#pragma unroll
        for (int i = 0; i < H; i++) {
            const int y = fud ? H - 1 - i : i;
            out[y * W + x] = csh ? (t[i] + (1 << (csh - 1))) >> csh : t[i];
        }
    }
    g.sync();
}

// One residual task: its compact levels, then residual_store.
template <int TX, class G, class S>
__device__ __forceinline__ void residual_task(const G& g, S& s, const IntraFrame& F, const av1g_tu& tu, int32_t* out) {
    constexpr int W = kTxW[TX], H = kTxH[TX];
    constexpr int TW = W < 32 ? W : 32, TH = H < 32 ? H : 32, NC = TW * TH, K = (NC + G::N - 1) / G::N;
    int cf[K];
    const int32_t* lv = F.coeffs + tu.coeff_offset;
#pragma unroll
    for (int q = 0; q < K; q++) {
        const int k = g.r + q * G::N;
        cf[q] = k < NC ? __ldg(lv + k) : 0;
    }
    residual_store<TX>(g, s, F, tu, cf, out);
}

// One TU: prediction (+ inter-intra blend, + CfL), then the residual, all on
// the shared-memory copy of the superblock.
template <int TX, class G, class S>
__device__ void intra_tu(const G& g, S& s, const IntraFrame& F, const SbCtx& c, uint16_t* cache,
                         const av1g_intra_tu* rec, Pool pool) {
    const av1g_intra_tu t = *rec;
    constexpr int W = kTxW[TX], H = kTxH[TX];
    constexpr int LW = ilog2<W>(), LH = ilog2<H>();
    const int tid = g.r;
    const int pl = t.plane;
    const PlaneDev& P = F.planes[pl];
    const int hbd = F.hbd, bd = F.bd;
    const int sx = t.x, sy = t.y;
    const int cs = c.w[pl];
    uint16_t* tp = cache + c.off[pl] + (sy - c.y0[pl]) * cs + (sx - c.x0[pl]);
    const bool has_res = t.flags & AV1G_INTRA_RESIDUAL;
    // a warp fetches its residual first, so that the latency overlaps the
    // prediction (the CTA path reads it at the merge)
    const int32_t* rp = pool.res + t.res.coeff_offset;
    constexpr int KP = G::N == 32 ? (W * H + 31) / 32 : 1;
    int rv[KP];
    if constexpr (G::N == 32) {
#pragma unroll
        for (int q = 0; q < KP; q++) {
            const int k = tid + q * 32;
            rv[q] = (has_res && k < W * H) ? __ldg(rp + k) : 0;
        }
    }
    const int maxv = (1 << bd) - 1;
    if (t.mode < 13) {
        const int max_x = P.w - 1, max_y = P.h - 1;
        auto rd = [&](int yy, int xx) { return rdp(F, c, cache, pl, min(yy, max_y), min(xx, max_x)); };
        const bool ha = (t.flags & AV1G_INTRA_HAVE_ABOVE) && sy > 0;
        const bool hl = (t.flags & AV1G_INTRA_HAVE_LEFT) && sx > 0;
        const bool har = t.flags & AV1G_INTRA_HAVE_ABOVE_RIGHT, hbl = t.flags & AV1G_INTRA_HAVE_BELOW_LEFT;
        const bool eief = t.flags & AV1G_INTRA_EDGE_FILTER;
        const int ft = (t.flags & AV1G_INTRA_FILTER_TYPE) ? 1 : 0;
        const int corner = ha && hl ? rd(sy - 1, sx - 1) : ha ? rd(sy - 1, sx) : hl ? rd(sy, sx - 1) : 1 << (bd - 1);
        constexpr int span = W + H;
        // edge arrays (intra_predict_block_samples, cdf.rs:17030-17075)
        for (int i = tid; i < span; i += G::N) {
            int a, l;
            if (!ha && hl) a = rd(sy, sx - 1);
            else if (!ha && !hl) a = (1 << (bd - 1)) - 1;
            else a = rd(sy - 1, min(min(max_x, sx + (har ? 2 * W : W) - 1), sx + i));
            if (!hl && ha) l = rd(sy - 1, sx);
            else if (!hl && !ha) l = (1 << (bd - 1)) + 1;
            else l = rd(min(min(max_y, sy + (hbl ? 2 * H : H) - 1), sy + i), sx - 1);
            s.above[2 + i] = (uint16_t)a;
            s.left[2 + i] = (uint16_t)l;
        }
        if (tid < 2) s.above[tid] = s.left[tid] = (uint16_t)corner;
        g.sync();
        const bool dir = t.mode >= 1 && t.mode <= 8;
        const int pa = c_mode_angle[t.mode] + t.angle_delta * 3;
        int ua = 0, ul = 0;
        if (dir && eief && pa != 90 && pa != 180) {
            if (pa > 90 && pa < 180 && span >= 24) {
                if (tid == 0) {
                    uint16_t fc = (uint16_t)((s.left[2] * 5 + s.above[1] * 6 + s.above[2] * 5 + 8) >> 4);
                    s.above[1] = fc;
                    s.left[1] = fc;
                }
                g.sync();
            }
            if (ha) edge_filter(g, s, s.above, min(W, max_x - sx + 1) + (pa < 90 ? H : 0) + 1, strength_sel(W, H, ft, pa - 90));
            if (hl) edge_filter(g, s, s.left, min(H, max_y - sy + 1) + (pa > 180 ? W : 0) + 1, strength_sel(W, H, ft, pa - 180));
            ua = upsample_sel(W, H, ft, pa - 90);
            if (ua) edge_upsample(g, s, s.above, W + (pa < 90 ? H : 0), bd);
            ul = upsample_sel(W, H, ft, pa - 180);
            if (ul) edge_upsample(g, s, s.left, H + (pa > 180 ? W : 0), bd);
        }
        const uint16_t* A = s.above + 2;  // A[k] == AboveRow[k]
        const uint16_t* Lc = s.left + 2;
        const int fim = (pl == 0 && t.filter_intra_mode < 5) ? t.filter_intra_mode : -1;
        // the intra half of an inter-intra block is blended as it is stored
        // (only inside the plane: the side plane has the plane's extent)
        auto put = [&](int i, int j, int v) {
            if (t.interintra && sy + i < P.h && sx + j < P.w)
                v = interintra_px<W, H>(F, t, i, j, v, ld_px(F.side[pl], hbd, sy + i, sx + j), maxv);
            tp[i * cs + j] = (uint16_t)v;
        };
        if (fim >= 0) {
            // predict_intra_recursive (cdf.rs:2145): 4x2 cells, wavefront over
            // i2 + j4, reading earlier cells back from the copy
            constexpr int W4 = W >> 2, H2 = H >> 1;
            const int o = tid & 7, i1 = o >> 2, j1 = o & 3;
            for (int d = 0; d < W4 + H2 - 1; d++) {
                for (int bb = tid >> 3;; bb += G::N >> 3) {
                    const int i2 = max(0, d - (W4 - 1)) + bb, j4 = d - i2;
                    if (i2 >= H2 || j4 < 0) break;
                    int p[7];
#pragma unroll
                    for (int i = 0; i < 7; i++) {
                        if (i < 5) {
                            if (i2 == 0) p[i] = A[(j4 << 2) + i - 1];
                            else if (j4 == 0 && i == 0) p[i] = Lc[(i2 << 1) - 1];
                            else p[i] = tp[((i2 << 1) - 1) * cs + (j4 << 2) + i - 1];
                        } else if (j4 == 0) {
                            p[i] = Lc[(i2 << 1) + i - 5];
                        } else {
                            p[i] = tp[((i2 << 1) + i - 5) * cs + (j4 << 2) - 1];
                        }
                    }
                    int acc = 0;
#pragma unroll
                    for (int i = 0; i < 7; i++) acc += c_fi_taps[fim][(i1 << 2) + j1][i] * p[i];
                    int v = acc >= 0 ? (acc + 8) >> 4 : -(((-acc) + 8) >> 4);
                    tp[((i2 << 1) + i1) * cs + (j4 << 2) + j1] = (uint16_t)clip3(0, maxv, v);
                }
                g.sync();
            }
        } else if (t.mode == 0) {
            // predict_intra_dc_pred (cdf.rs:1348)
            long long part = 0;
            for (int i = tid; i < span; i += G::N) {
                if (hl && i < H) part += Lc[i];
                if (ha && i < W) part += A[i];
            }
            long long sum = gsum(g, s, part);
            unsigned avg;
            if (hl && ha) avg = (unsigned)((sum + (span >> 1)) / span);
            else if (hl) avg = min((unsigned)((sum + (H >> 1)) >> LH), (1u << bd) - 1);
            else if (ha) avg = min((unsigned)((sum + (W >> 1)) >> LW), (1u << bd) - 1);
            else avg = 1u << (bd - 1);
            for (int k = tid; k < W * H; k += G::N) put(k >> LW, k & (W - 1), (int)avg);
        } else {
            const int dx = pa < 90 ? c_dr[pa] : (pa < 180 ? c_dr[180 - pa] : 0);
            const int dy = (pa >= 90 && pa < 180) ? c_dr[pa - 90] : (pa > 180 ? c_dr[270 - pa] : 0);
            const uint8_t* swx = sm_weights(LW);
            const uint8_t* swy = sm_weights(LH);
            for (int k = tid; k < W * H; k += G::N) {
                int i = k >> LW, j = k & (W - 1);
                int v;
                if (t.mode == 1 && t.angle_delta == 0) {
                    v = A[j];
                } else if (t.mode == 2 && t.angle_delta == 0) {
                    v = Lc[i];
                } else if (dir) {
                    // predict_intra_directional (cdf.rs:2879-3010)
                    if (pa < 90) {
                        int maxb = (W + H - 1) << ua;
                        int idx = (i + 1) * dx;
                        int base = (idx >> (6 - ua)) + j * (1 << ua);
                        int sh = ((idx * (1 << ua)) >> 1) & 0x1F;
                        v = base < maxb ? (A[base] * (32 - sh) + A[base + 1] * sh + 16) >> 5 : A[maxb];
                    } else if (pa < 180) {
                        int ix = (j << 6) - (i + 1) * dx;
                        int bx = ix >> (6 - ua);
                        if (bx >= -(1 << ua)) {
                            int sh = ((ix * (1 << ua)) >> 1) & 0x1F;
                            v = (A[bx] * (32 - sh) + A[bx + 1] * sh + 16) >> 5;
                        } else {
                            int iy = (i << 6) - (j + 1) * dy;
                            int by = iy >> (6 - ul);
                            int sh = ((iy * (1 << ul)) >> 1) & 0x1F;
                            v = (Lc[by] * (32 - sh) + Lc[by + 1] * sh + 16) >> 5;
                        }
                    } else {
                        int maxb = (W + H - 1) << ul;
                        int idx = (j + 1) * dy;
                        int base = (idx >> (6 - ul)) + i * (1 << ul);
                        int sh = ((idx * (1 << ul)) >> 1) & 0x1F;
                        v = base < maxb ? (Lc[base] * (32 - sh) + Lc[base + 1] * sh + 16) >> 5 : Lc[maxb];
                    }
                } else if (t.mode == 9) {  // SMOOTH (cdf.rs:2267)
                    unsigned sp = swy[i] * A[j] + (256 - swy[i]) * Lc[H - 1] + swx[j] * Lc[i] + (256 - swx[j]) * A[W - 1];
                    v = (int)((sp + 256) >> 9);
                } else if (t.mode == 10) {  // SMOOTH_V
                    v = (int)((swy[i] * A[j] + (256 - swy[i]) * Lc[H - 1] + 128) >> 8);
                } else if (t.mode == 11) {  // SMOOTH_H
                    v = (int)((swx[j] * Lc[i] + (256 - swx[j]) * A[W - 1] + 128) >> 8);
                } else {  // PAETH (cdf.rs:2077)
                    int base = A[j] + Lc[i] - corner;
                    int pl_ = abs(base - Lc[i]), pt = abs(base - A[j]), ptl = abs(base - corner);
                    v = (pl_ <= pt && pl_ <= ptl) ? Lc[i] : (pt <= ptl ? A[j] : corner);
                }
                put(i, j, v);
            }
        }
        g.sync();
    }
    if (t.mode == AV1G_INTRA_MODE_PALETTE) {
        // predict_palette (cdf.rs:11907); indices checked on the host
        const uint8_t* m = F.maps + t.palette_map;
        for (int k = tid; k < W * H; k += G::N) {
            int i = k >> LW, j = k & (W - 1);
            tp[i * cs + j] = rec->palette_colors[m[i * t.palette_stride + j]];
        }
        g.sync();
    } else if (t.mode == AV1G_INTRA_MODE_INTRABC) {
        // predict_intrabc_leaf_into_curr_frame (cdf.rs:19235): BILINEAR
        // block_inter_prediction from the pre-filter plane at unit scale,
        // start = (x << 10) + (((2 * mv) >> ss) << 6) + 32, clamped to the
        // mi-padded plane (the reference's window clamp is the same set).
        // The whole block is predicted before any of it is stored.
        const int pss_x = pl ? F.ssx : 0, pss_y = pl ? F.ssy : 0;
        const int stx = (sx << 10) + ((2 * t.mv[1]) >> pss_x) * 64 + 32;
        const int sty = (sy << 10) + ((2 * t.mv[0]) >> pss_y) * 64 + 32;
        const int r0 = bd == 12 ? 5 : 3, r1 = bd == 12 ? 9 : 11;
        const int hph = (stx >> 6) & 15, vph = (sty >> 6) & 15;
        for (int k = tid; k < W * H; k += G::N) {
            int i = k >> LW, j = k & (W - 1);
            int xi = ((stx >> 10) + j) - 3, yi = ((sty >> 10) + i) - 3;
            int acc = 0;
            for (int tt = 0; tt < 8; tt++) {
                int vc = c_subpel[3][vph][tt];
                if (!vc) continue;
                int yy = min(max(yi + tt, 0), P.h - 1);
                int hsum = 0;
                for (int u = 0; u < 8; u++) {
                    int hc = c_subpel[3][hph][u];
                    if (hc) hsum += hc * rdp(F, c, cache, pl, yy, min(max(xi + u, 0), P.w - 1));
                }
                acc += vc * ((hsum + ((1 << r0) >> 1)) >> r0);
            }
            s.buf[k] = min(max((acc + (1 << (r1 - 1))) >> r1, 0), maxv);
        }
        g.sync();
        for (int k = tid; k < W * H; k += G::N) tp[(k >> LW) * cs + (k & (W - 1))] = (uint16_t)s.buf[k];
        g.sync();
    }
    if ((t.flags & AV1G_INTRA_CFL) && pl > 0) {
        // predict_chroma_from_luma_into_curr_frame (cdf.rs:17256-17340).  The
        // block's luma transforms may run past the mi-grid plane; their
        // samples there stay in the superblock's staged copy (the reference's
        // LumaOverhang side store, cdf.rs:15938, read at cdf.rs:17292-17305),
        // which spans the whole superblock.  Luma neither in the plane nor in
        // that copy reads as 0.
        const PlaneDev& Y = F.planes[0];
        const int ssx = F.ssx, ssy = F.ssy;
        const int cx = max((int)t.max_luma_w - (1 << ssx), 0), cy = max((int)t.max_luma_h - (1 << ssy), 0);
        long long part = 0;
        for (int k = tid; k < W * H; k += G::N) {
            int i = k >> LW, j = k & (W - 1);
            int ly = min((sy + i) << ssy, cy), lx = min((sx + j) << ssx, cx);
            int acc = 0;
            for (int ddy = 0; ddy <= ssy; ddy++)
                for (int ddx = 0; ddx <= ssx; ddx++) {
                    int yy = ly + ddy, xx = lx + ddx;
                    const bool staged = (unsigned)(yy - c.y0[0]) < (unsigned)c.h[0] &&
                                        (unsigned)(xx - c.x0[0]) < (unsigned)c.w[0];
                    acc += (staged || (yy < Y.h && xx < Y.w)) ? rdp(F, c, cache, 0, yy, xx) : 0;
                }
            int v = acc << (3 - ssx - ssy);
            s.buf[k] = v;
            part += v;
        }
        long long sum = gsum(g, s, part);
        long long half = 1LL << (LW + LH - 1);
        long long avg = sum >= 0 ? (sum + half) >> (LW + LH) : -(((-sum) + half) >> (LW + LH));
        for (int k = tid; k < W * H; k += G::N) {
            int i = k >> LW, j = k & (W - 1);
            if (sy + i >= P.h || sx + j >= P.w) continue;
            long long d = (long long)t.cfl_alpha * (s.buf[k] - avg);
            long long sc = d >= 0 ? (d + 32) >> 6 : -(((-d) + 32) >> 6);
            uint16_t& px = tp[i * cs + j];
            px = (uint16_t)min(max((long long)px + sc, 0LL), (long long)maxv);
        }
        g.sync();
    }
    if (has_res) {
        // curr_frame_step3_merge (cdf.rs:17398-17470): Clip1(pred + residual);
        // luma past the plane is merged too, in the staged copy only (the
        // overhang chroma from luma reads)
#pragma unroll
        for (int q = 0; q < (G::N == 32 ? KP : (W * H + G::N - 1) / G::N); q++) {
            const int k = tid + q * G::N;
            if (k >= W * H) break;
            const int i = k >> LW, j = k & (W - 1);
            if (pl != 0 && (sy + i >= P.h || sx + j >= P.w)) continue;
            int v;
            if constexpr (G::N == 32) v = rv[q];
            else v = __ldg(rp + k);
            uint16_t& px = tp[i * cs + j];
            px = (uint16_t)min(max((int)px + v, 0), maxv);
        }
        g.sync();
    }
    // the TU's final samples to HBM: other superblocks read them once this
    // level is published
    for (int k = tid; k < W * H; k += G::N) {
        const int i = k >> LW, j = k & (W - 1);
        if (sy + i < P.h && sx + j < P.w) st_px(P, hbd, sy + i, sx + j, tp[i * cs + j]);
    }
}

__device__ void run_small(const WarpG& g, WScr& s, const IntraFrame& F, const SbCtx& c, uint16_t* cache,
                          const av1g_intra_tu* rec, Pool pool) {
    switch (rec->tx_size) {
        case 0: intra_tu<0>(g, s, F, c, cache, rec, pool); break;
        case 1: intra_tu<1>(g, s, F, c, cache, rec, pool); break;
        case 2: intra_tu<2>(g, s, F, c, cache, rec, pool); break;
        case 5: intra_tu<5>(g, s, F, c, cache, rec, pool); break;
        case 6: intra_tu<6>(g, s, F, c, cache, rec, pool); break;
        case 7: intra_tu<7>(g, s, F, c, cache, rec, pool); break;
        case 8: intra_tu<8>(g, s, F, c, cache, rec, pool); break;
        case 13: intra_tu<13>(g, s, F, c, cache, rec, pool); break;
        case 14: intra_tu<14>(g, s, F, c, cache, rec, pool); break;
        case 15: intra_tu<15>(g, s, F, c, cache, rec, pool); break;
        default: intra_tu<16>(g, s, F, c, cache, rec, pool); break;
    }
}

__device__ void run_large(const CtaG& g, CScr& s, const IntraFrame& F, const SbCtx& c, uint16_t* cache,
                          const av1g_intra_tu* rec, Pool pool) {
    switch (rec->tx_size) {
        case 3: intra_tu<3>(g, s, F, c, cache, rec, pool); break;
        case 4: intra_tu<4>(g, s, F, c, cache, rec, pool); break;
        case 9: intra_tu<9>(g, s, F, c, cache, rec, pool); break;
        case 10: intra_tu<10>(g, s, F, c, cache, rec, pool); break;
        case 11: intra_tu<11>(g, s, F, c, cache, rec, pool); break;
        case 12: intra_tu<12>(g, s, F, c, cache, rec, pool); break;
        case 17: intra_tu<17>(g, s, F, c, cache, rec, pool); break;
        default: intra_tu<18>(g, s, F, c, cache, rec, pool); break;
    }
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ long long gtimer() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The superblock copy <-> HBM, two samples per thread (plane widths are even,
// superblock origins and row pitches keep the pairs aligned).
template <bool LOAD>
__device__ void move_sb(const IntraFrame& F, const SbCtx& c, uint16_t* cache) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int p = 0; p < F.np; p++) {
        const PlaneDev& P = F.planes[p];
        const int rows = min(c.h[p], P.h - c.y0[p]), pairs = min(c.w[p], P.w - c.x0[p]) >> 1;
        uint16_t* cp = cache + c.off[p];
        for (int r = warp; r < rows; r += kNW) {
            uint8_t* row = P.p + (size_t)(c.y0[p] + r) * P.stride;
            uint16_t* crow = cp + r * c.w[p];
            for (int q = lane; q < pairs; q += 32) {
                if (F.hbd) {
                    uint32_t* g = reinterpret_cast<uint32_t*>(row) + (c.x0[p] >> 1) + q;
                    if (LOAD) {
                        const uint32_t v = *g;
                        crow[2 * q] = (uint16_t)v;
                        crow[2 * q + 1] = (uint16_t)(v >> 16);
                    } else {
                        *g = (uint32_t)crow[2 * q] | ((uint32_t)crow[2 * q + 1] << 16);
                    }
                } else {
                    uint16_t* g = reinterpret_cast<uint16_t*>(row + c.x0[p]) + q;
                    if (LOAD) {
                        const uint16_t v = *g;
                        crow[2 * q] = v & 0xff;
                        crow[2 * q + 1] = v >> 8;
                    } else {
                        *g = (uint16_t)(crow[2 * q] | (crow[2 * q + 1] << 8));
                    }
                }
            }
        }
    }
}

// One residual block to compute: the TU, its frame, where its block goes.
struct ResTask {
    av1g_tu tu;
    int32_t frame;
    int32_t out;
};

// Residual blocks of every intra TU of the batch, ahead of the wavefront:
// they depend on the coefficients only.  Blocks [0, small_blocks) run the
// small TUs one per warp; the others run the large TUs with the whole CTA.
__global__ void __launch_bounds__(kT) intra_res_kernel(const IntraFrame* __restrict__ frames,
                                                       const ResTask* __restrict__ small, int n_small,
                                                       const ResTask* __restrict__ large, int n_large,
                                                       int32_t* __restrict__ res, int small_blocks) {
    __shared__ union {
        WScr w[kNW];
        CScr c;
    } u;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if ((int)blockIdx.x < small_blocks) {
        for (int q = blockIdx.x * kNW + warp; q < n_small; q += small_blocks * kNW) {
            const ResTask tk = small[q];
            const IntraFrame& F = frames[tk.frame];
            const WarpG g{lane};
            int32_t* out = res + tk.out;
            switch (tk.tu.tx_size) {
                case 0: residual_task<0>(g, u.w[warp], F, tk.tu, out); break;
                case 1: residual_task<1>(g, u.w[warp], F, tk.tu, out); break;
                case 2: residual_task<2>(g, u.w[warp], F, tk.tu, out); break;
                case 5: residual_task<5>(g, u.w[warp], F, tk.tu, out); break;
                case 6: residual_task<6>(g, u.w[warp], F, tk.tu, out); break;
                case 7: residual_task<7>(g, u.w[warp], F, tk.tu, out); break;
                case 8: residual_task<8>(g, u.w[warp], F, tk.tu, out); break;
                case 13: residual_task<13>(g, u.w[warp], F, tk.tu, out); break;
                case 14: residual_task<14>(g, u.w[warp], F, tk.tu, out); break;
                case 15: residual_task<15>(g, u.w[warp], F, tk.tu, out); break;
                default: residual_task<16>(g, u.w[warp], F, tk.tu, out); break;
            }
        }
    } else {
        for (int q = blockIdx.x - small_blocks; q < n_large; q += gridDim.x - small_blocks) {
            const ResTask tk = large[q];
            const IntraFrame& F = frames[tk.frame];
            const CtaG g{tid};
            int32_t* out = res + tk.out;
            switch (tk.tu.tx_size) {
                case 3: residual_task<3>(g, u.c, F, tk.tu, out); break;
                case 4: residual_task<4>(g, u.c, F, tk.tu, out); break;
                case 9: residual_task<9>(g, u.c, F, tk.tu, out); break;
                case 10: residual_task<10>(g, u.c, F, tk.tu, out); break;
                case 11: residual_task<11>(g, u.c, F, tk.tu, out); break;
                case 12: residual_task<12>(g, u.c, F, tk.tu, out); break;
                case 17: residual_task<17>(g, u.c, F, tk.tu, out); break;
                default: residual_task<18>(g, u.c, F, tk.tu, out); break;
            }
        }
    }
}

// Stages TU records [b, min(b + kTuWin, end)) into the window and returns
// the window's end (all threads call; the bounds live in registers, the same
// in every thread).
__device__ __forceinline__ int stage_tus(av1g_intra_tu* win, const av1g_intra_tu* __restrict__ tus, int b, int end) {
    const int e = min(b + kTuWin, end);
    const uint4* src = reinterpret_cast<const uint4*>(tus + b);
    uint4* dst = reinterpret_cast<uint4*>(win);
    for (int q = threadIdx.x; q < (e - b) * 4; q += kT) dst[q] = __ldg(src + q);
    return e;
}

__global__ void __launch_bounds__(kT) intra_kernel(const IntraFrame* __restrict__ frames,
                                                   const av1g_intra_tu* __restrict__ tus,
                                                   const SbItem* __restrict__ items, const int2* __restrict__ lvs,
                                                   const int4* __restrict__ waits, int* prog, int* ctl, int nitems,
                                                   const int32_t* __restrict__ res) {
    // ctl[0]: the claim counter; ctl[1 + f]: frame f's abort word
    // dynamic shared memory: Shared | TU window | superblock copy
    extern __shared__ __align__(16) uint8_t dsm[];
    Shared& S = *reinterpret_cast<Shared*>(dsm);
    av1g_intra_tu* win = reinterpret_cast<av1g_intra_tu*>(dsm + kSharedBytes);
    uint16_t* cache = reinterpret_cast<uint16_t*>(dsm + kSharedBytes + kTuWin * sizeof(av1g_intra_tu));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const IntraFrame& F = S.fr;
    const Pool pool{res};
    for (;;) {
        __syncthreads();
        if (tid == 0) S.idx = atomicAdd(&ctl[0], 1);
        __syncthreads();
        const int idx = S.idx;
        if (idx >= nitems) return;
        const SbItem it = items[idx];
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(frames + it.frame);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&S.fr);
            for (int q = tid; q < (int)(sizeof(IntraFrame) / 4); q += kT) dst[q] = __ldg(src + q);
        }
        __syncthreads();
        if (tid == 0) {
            int off = 0;
            for (int p = 0; p < 3; p++) {
                const int ssx = p ? F.ssx : 0, ssy = p ? F.ssy : 0;
                S.sb.x0[p] = it.x0 >> ssx;
                S.sb.y0[p] = it.y0 >> ssy;
                S.sb.w[p] = (1 << it.log2sb) >> ssx;
                S.sb.h[p] = (1 << it.log2sb) >> ssy;
                S.sb.off[p] = off;
                off += p < F.np ? S.sb.w[p] * S.sb.h[p] : 0;
            }
            S.abort_seen = 0;
        }
        __syncthreads();
        // the superblock's own area is written only by its own TUs, and its
        // TU records are inputs: stage both before any wait
        move_sb<true>(F, S.sb, cache);
        int tw0 = it.tu_first;
        int tw1 = stage_tus(win, tus, tw0, it.tu_end);
        // the waits, by level (staged when few; the level of the next one in a register)
        const int4* wsrc = waits + it.wait_first;
        if (it.nwait <= kWaitWin) {
            for (int q = tid; q < it.nwait; q += kT) S.wv[q] = __ldg(wsrc + q);
            wsrc = S.wv;
        }
        int wq = 0;
        __syncthreads();
        int next_wait = it.nwait > 0 ? wsrc[0].x : 0x7fffffff;
        for (int L0 = 0; L0 < it.nlv; L0 += kLvChunk) {
            const int n = min(kLvChunk, it.nlv - L0);
            __syncthreads();
            for (int q = tid; q <= n; q += kT) S.lv[q] = lvs[it.lv_first + L0 + q];
            __syncthreads();
            for (int L = 0; L < n; L++) {
                const int lg = L0 + L;
                if (next_wait <= lg) {
                    // the levels of other superblocks this level reads: poll
                    // with volatile loads, then an acquire load orders the
                    // reads after the progress seen
                    const int w0 = wq;
                    while (wq < it.nwait && wsrc[wq].x <= lg) wq++;
                    next_wait = wq < it.nwait ? wsrc[wq].x : 0x7fffffff;
                    int* abort_word = ctl + 1 + it.frame;
                    const long long bound = *(volatile long long*)&g_wait_ns;
                    for (int q = w0 + tid; q < wq; q += kT) {
                        const int4 w = wsrc[q];
                        const volatile int* f = prog + w.y;
                        if (*f < w.z) {
                            const long long t0 = gtimer();
                            while (*f < w.z) {
                                if (*(volatile int*)abort_word) break;
                                if (gtimer() - t0 > bound) {
                                    atomicExch(abort_word, 1);
                                    break;
                                }
                                __nanosleep(64);
                            }
                        }
                        ld_acquire(prog + w.y);
                    }
                    __syncthreads();
                    if (tid == 0 && *(volatile int*)abort_word) S.abort_seen = 1;
                    __syncthreads();
                }
                const bool publish = S.lv[L].y & kLevelPublished;
                if (!S.abort_seen) {
                    const int b = S.lv[L].x, m = S.lv[L].y & ~kLevelPublished, e = S.lv[L + 1].x;
                    if (e > tw1 && b > tw0) {  // slide the window to this level
                        tw0 = b;
                        tw1 = stage_tus(win, tus, b, it.tu_end);
                        __syncthreads();
                    }
                    for (int k = b + warp; k < m; k += kNW) {
                        WScr& ws = S.s.w[warp];
                        const av1g_intra_tu* rec = win + (k - tw0);
                        if (k >= tw1) {  // a level wider than the window
                            if (lane < 16)
                                reinterpret_cast<uint32_t*>(&ws.tu)[lane] =
                                    __ldg(reinterpret_cast<const uint32_t*>(tus + k) + lane);
                            __syncwarp();
                            rec = &ws.tu;
                        }
                        run_small(WarpG{lane}, ws, F, S.sb, cache, rec, pool);
                        __syncwarp();
                    }
                    if (m < e) {
                        __syncthreads();
                        for (int k = m; k < e; k++) {
                            const av1g_intra_tu* rec = win + (k - tw0);
                            if (k >= tw1) {
                                if (tid < 16)
                                    reinterpret_cast<uint32_t*>(&S.s.c.tu)[tid] =
                                        __ldg(reinterpret_cast<const uint32_t*>(tus + k) + tid);
                                __syncthreads();
                                rec = &S.s.c.tu;
                            }
                            run_large(CtaG{tid}, S.s.c, F, S.sb, cache, rec, pool);
                            __syncthreads();
                        }
                    }
                }
                __syncthreads();
                // publish "lg + 1 levels done" when another superblock waits
                // for it, from the last warp (the first warp starts the next level)
                if (publish && tid == kT - 32) {
                    __threadfence();
                    atomicExch(prog + idx, lg + 1);
                }
            }
        }
    }
}

}  // namespace


namespace {
// Test hook state: a never-satisfied wait is planned into the first
// superblock of every job whose frame is this wide (0: none).
std::atomic<int> g_fault_width{0};

// Before its first level, the first superblock of job f waits for its own
// progress to reach a value it never reaches.
void plan_fault_wait(IntraPlan& plan, int f) {
    for (size_t i = 0; i < plan.items.size(); i++) {
        SbItem& it = plan.items[i];
        if (it.frame != f) continue;
        plan.waits.insert(plan.waits.begin() + it.wait_first, int4{0, (int)i, 0x3fffffff, 0});
        it.nwait++;
        for (size_t k = 0; k < plan.items.size(); k++)
            if (k != i && plan.items[k].wait_first >= it.wait_first) plan.items[k].wait_first++;
        return;
    }
}

// The most dynamic shared memory any launch asks for: the fixed part, the TU
// window and the largest superblock copy (128x128, three full planes, u16).
constexpr size_t kMaxDynSmem = kSharedBytes + kTuWin * sizeof(av1g_intra_tu) + 3 * 128 * 128 * sizeof(uint16_t);
static_assert(kMaxDynSmem <= 227 * 1024, "intra_kernel's shared memory exceeds an SM's");

// The kernel's dynamic shared memory limit is a per-device attribute that
// every launch on the device shares, and engine lanes launch concurrently
// with different sizes: it is raised once per device to the largest size,
// so no launch can find it lowered by another thread between its own
// setting and its launch.
cudaError_t ensure_intra_smem_limit(int dev) {
    static std::mutex mu;
    static bool done[256];
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 256 && done[dev]) return cudaSuccess;
    const cudaError_t e =
        cudaFuncSetAttribute(intra_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxDynSmem);
    if (e == cudaSuccess && dev >= 0 && dev < 256) done[dev] = true;
    return e;
}
}  // namespace

// Host side of av1g_run_intra: the plan (intra_plan.cu), its upload, one
// launch.  frame_status (pinned host memory of n words, or null) receives,
// in stream order after the launch, each job's abort word: non-zero when a
// dependency wait of that frame ran out of time.
av1g_status intra_run_status(const av1g_intra_job* jobs, int n, cudaStream_t st, std::string& err,
                             int32_t* frame_status) {
    int dev = 0;
    cudaGetDevice(&dev);
    IntraPlan plan;
    av1g_status rc = intra_plan(jobs, n, plan, err);
    if (rc != AV1G_OK || plan.items.empty()) {
        if (rc == AV1G_OK && frame_status) memset(frame_status, 0, sizeof(int32_t) * n);
        return rc;
    }
    if (int fw = g_fault_width.load(); fw > 0)
        for (int i = 0; i < n; i++)
            if (jobs[i].hdr->frame_width == fw) plan_fault_wait(plan, i);
    const int nitems = (int)plan.items.size();
    // residual tasks; each TU's device record points at its residual block
    std::vector<ResTask> rs, rl;
    long long res_ints = 0;
    for (const SbItem& it : plan.items)
        for (int k = it.tu_first; k < it.tu_end; k++) {
            av1g_intra_tu& t = plan.tus[k];
            if (!(t.flags & AV1G_INTRA_RESIDUAL)) continue;
            const int px = kTxW[t.tx_size] * kTxH[t.tx_size];
            (px > kSmallPx ? rl : rs).push_back(ResTask{t.res, it.frame, (int32_t)res_ints});
            t.res.coeff_offset = (uint32_t)res_ints;
            res_ints += px;
        }
    if (res_ints >= (1LL << 31)) {
        err = "intra batch: more than 2^31 residual samples";
        return AV1G_EINVAL;
    }
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t off_tus = al(sizeof(IntraFrame) * n);
    const size_t off_items = al(off_tus + sizeof(av1g_intra_tu) * plan.tus.size());
    const size_t off_lv = al(off_items + sizeof(SbItem) * plan.items.size());
    const size_t off_waits = al(off_lv + sizeof(int2) * plan.lvtab.size());
    const size_t off_done = al(off_waits + sizeof(int4) * plan.waits.size());
    const size_t off_ctl = al(off_done + sizeof(int) * plan.items.size());
    const size_t off_rs = al(off_ctl + (1 + (size_t)n) * sizeof(int));
    const size_t off_rl = al(off_rs + sizeof(ResTask) * rs.size());
    const size_t off_maps = al(off_rl + sizeof(ResTask) * rl.size());
    const size_t bytes = off_maps + plan.maps.size();  // uploaded
    const size_t off_res = al(bytes);
    const size_t total = off_res + sizeof(int32_t) * (size_t)res_ints;
    uint8_t* dev_buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev_buf, total, st);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    for (int i = 0; i < n; i++) plan.frames[i].maps = dev_buf + off_maps + plan.map_base[i];
    e = upload_with(dev_buf, bytes, st, [&](uint8_t* host) {
        memcpy(host, plan.frames.data(), sizeof(IntraFrame) * n);
        memcpy(host + off_tus, plan.tus.data(), sizeof(av1g_intra_tu) * plan.tus.size());
        memcpy(host + off_items, plan.items.data(), sizeof(SbItem) * plan.items.size());
        memcpy(host + off_lv, plan.lvtab.data(), sizeof(int2) * plan.lvtab.size());
        if (!plan.waits.empty()) memcpy(host + off_waits, plan.waits.data(), sizeof(int4) * plan.waits.size());
        memset(host + off_done, 0, off_rs - off_done);  // progress, claim counter, abort flag
        if (!rs.empty()) memcpy(host + off_rs, rs.data(), sizeof(ResTask) * rs.size());
        if (!rl.empty()) memcpy(host + off_rl, rl.data(), sizeof(ResTask) * rl.size());
        if (!plan.maps.empty()) memcpy(host + off_maps, plan.maps.data(), plan.maps.size());
    });
    const IntraFrame* dframes = (const IntraFrame*)dev_buf;
    int32_t* dres = (int32_t*)(dev_buf + off_res);
    int sms = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess && (!rs.empty() || !rl.empty())) {
        const int sb_blocks = (int)std::min<long long>(((long long)rs.size() + kNW - 1) / kNW, 16LL * sms);
        const int lb_blocks = (int)std::min<long long>((long long)rl.size(), 4LL * sms);
        intra_res_kernel<<<sb_blocks + lb_blocks, kT, 0, st>>>(dframes, (const ResTask*)(dev_buf + off_rs), (int)rs.size(),
                                                               (const ResTask*)(dev_buf + off_rl), (int)rl.size(), dres,
                                                               sb_blocks);
        e = cudaGetLastError();
    }
    const size_t smem = kSharedBytes + kTuWin * sizeof(av1g_intra_tu) + plan.cache_bytes;
    if (e == cudaSuccess && smem > kMaxDynSmem) e = cudaErrorInvalidValue;  // cannot happen: cache_bytes is bounded
    if (e == cudaSuccess) e = ensure_intra_smem_limit(dev);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, intra_kernel, kT, smem);
    if (e == cudaSuccess) {
        // as many CTAs as the wavefront can keep busy (the superblocks of
        // one depth, twice over since level-granular waits let the next depth
        // start early), not the whole GPU: idle CTAs would only poll while
        // other streams' kernels wait for SMs
        const int grid = std::max(1, std::min({nitems, std::max(per_sm, 1) * sms, 2 * plan.width + 2}));
        intra_kernel<<<grid, kT, smem, st>>>(
            dframes, (const av1g_intra_tu*)(dev_buf + off_tus), (const SbItem*)(dev_buf + off_items),
            (const int2*)(dev_buf + off_lv), (const int4*)(dev_buf + off_waits), (int*)(dev_buf + off_done),
            (int*)(dev_buf + off_ctl), nitems, dres);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && frame_status)
        e = cudaMemcpyAsync(frame_status, dev_buf + off_ctl + sizeof(int), sizeof(int32_t) * n,
                            cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(dev_buf, st);
    if (e != cudaSuccess) {
        err = std::string("intra launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

av1g_status intra_run(const av1g_intra_job* jobs, int n, cudaStream_t st, std::string& err) {
    return intra_run_status(jobs, n, st, err, nullptr);
}

}  // namespace av1g

extern "C" av1g_status av1g_intra_plan_stats_get(const av1g_intra_job* jobs, int32_t n,
                                                  av1g_intra_plan_stats* out) {
    if (!out || n < 0 || (n > 0 && !jobs)) return AV1G_EINVAL;
    av1g::IntraPlan plan;
    std::string err;
    av1g_status rc = av1g::intra_plan(jobs, n, plan, err);
    if (rc != AV1G_OK) return rc;
    *out = av1g_intra_plan_stats{(int32_t)plan.items.size(), (int32_t)plan.tus.size(), (int32_t)plan.waits.size(),
                                 plan.depth, plan.width, 0};
    return AV1G_OK;
}

extern "C" av1g_status av1g_test_intra_wait_fault(int64_t wait_ns, int32_t frame_width) {
    long long ns = wait_ns > 0 ? (long long)wait_ns : av1g::kWaitNs;
    cudaError_t e = cudaMemcpyToSymbol(av1g::g_wait_ns, &ns, sizeof ns);
    if (e != cudaSuccess) return AV1G_EDEVICE;
    av1g::g_fault_width.store(frame_width > 0 ? frame_width : 0);
    return AV1G_OK;
}
