// itx.cuh — dequantization, inverse transforms and the reconstruction merge
// shared by the residual kernel (recon.cu) and the intra wavefront (intra.cu).
//
// Restates dequantize_step1 (src/cdf.rs:13655-13703), inverse_transform_2d and
// its 1-D kernels (src/transform.rs:96-847) and curr_frame_step3_merge
// (src/cdf.rs:17398-17470).  Values are held in int32 and every product is
// formed in 64 bits, which is exact: the reference's intermediates after each
// rounding or clamp fit 32 bits for 8-, 10- and 12-bit content (butterfly
// outputs are bounded by sqrt(2) times their clamped inputs; dequantized
// inputs by 2^(7+BitDepth)).
#pragma once

#include <type_traits>

#include "common.cuh"
#include "av1_spec_tables.h"

namespace av1g {
namespace itx {
// internal linkage: every .cu that includes this header gets its own copy
namespace {


constexpr int kCos128[65] = AV1T_COS128_LOOKUP_INIT;
constexpr int kTxW[19] = AV1T_TX_WIDTH_INIT;
constexpr int kTxH[19] = AV1T_TX_HEIGHT_INIT;
constexpr int kRowShift[19] = AV1T_TRANSFORM_ROW_SHIFT_INIT;

__constant__ AV1T_DC_QLOOKUP_TYPE c_dcq AV1T_DC_QLOOKUP_DIMS = AV1T_DC_QLOOKUP_INIT;
__constant__ AV1T_AC_QLOOKUP_TYPE c_acq AV1T_AC_QLOOKUP_DIMS = AV1T_AC_QLOOKUP_INIT;
__constant__ AV1T_QM_OFFSET_TYPE c_qm_off AV1T_QM_OFFSET_DIMS = AV1T_QM_OFFSET_INIT;
__device__ const AV1T_QUANTIZER_MATRIX_TYPE g_qm AV1T_QUANTIZER_MATRIX_DIMS = AV1T_QUANTIZER_MATRIX_INIT;

constexpr int cos128(int angle) {
    int a = angle & 255;
    return a <= 64 ? kCos128[a] : a <= 128 ? -kCos128[128 - a] : a <= 192 ? -kCos128[a - 128] : kCos128[256 - a];
}
constexpr int sin128(int angle) { return cos128(angle - 64); }
constexpr unsigned brev(int nbits, unsigned x) {
    unsigned t = 0;
    for (int i = 0; i < nbits; i++) t |= ((x >> i) & 1) << (nbits - 1 - i);
    return t;
}

struct Clamp {
    int lo, hi;
};

__device__ __forceinline__ int rnd12(long long x) { return (int)((x + 2048) >> 12); }

// butterfly B (transform.rs:196-209); angle is a compile-time constant
template <int A, int Bi, int ANGLE, int FLIP>
__device__ __forceinline__ void bfly(int* t) {
    constexpr long long c = cos128(ANGLE), s = sin128(ANGLE);
    long long x = (long long)t[A] * c - (long long)t[Bi] * s;
    long long y = (long long)t[A] * s + (long long)t[Bi] * c;
    if (FLIP) { t[A] = rnd12(y); t[Bi] = rnd12(x); }
    else { t[A] = rnd12(x); t[Bi] = rnd12(y); }
}
// butterfly H (transform.rs:211-219)
template <int A, int Bi, int FLIP>
__device__ __forceinline__ void hadd(int* t, Clamp c) {
    constexpr int ai = FLIP ? Bi : A, bi = FLIP ? A : Bi;
    int x = t[ai], y = t[bi];
    t[ai] = min(max(x + y, c.lo), c.hi);
    t[bi] = min(max(x - y, c.lo), c.hi);
}

// Compile-time loops.
template <int I, int N, typename F>
__device__ __forceinline__ void unroll(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        unroll<I + 1, N>(f);
    }
}

// inverse_dct (transform.rs:238-460) for length 1 << N.
template <int N>
__device__ __forceinline__ void idct(int* t, Clamp r) {
    constexpr int L = 1 << N;
    int cp[L];
#pragma unroll
    for (int i = 0; i < L; i++) cp[i] = t[i];
    unroll<0, L>([&](auto i) { t[i] = cp[brev(N, i)]; });
    if constexpr (N == 6) unroll<0, 16>([&](auto i) { bfly<32 + i, 63 - i, 63 - 4 * (int)brev(4, i), 0>(t); });
    if constexpr (N >= 5) unroll<0, 8>([&](auto i) { bfly<16 + i, 31 - i, 6 + ((int)brev(3, 7 - i) << 3), 0>(t); });
    if constexpr (N == 6) unroll<0, 16>([&](auto i) { hadd<32 + i * 2, 33 + i * 2, i & 1>(t, r); });
    if constexpr (N >= 4) unroll<0, 4>([&](auto i) { bfly<8 + i, 15 - i, 12 + ((int)brev(2, 3 - i) << 4), 0>(t); });
    if constexpr (N >= 5) unroll<0, 8>([&](auto i) { hadd<16 + 2 * i, 17 + 2 * i, i & 1>(t, r); });
    if constexpr (N == 6)
        unroll<0, 4>([&](auto i) {
            unroll<0, 2>([&](auto j) { bfly<62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * (int)brev(2, i) + 64 * j, 1>(t); });
        });
    if constexpr (N >= 3) unroll<0, 2>([&](auto i) { bfly<4 + i, 7 - i, 56 - 32 * i, 0>(t); });
    if constexpr (N >= 4) unroll<0, 4>([&](auto i) { hadd<8 + 2 * i, 9 + 2 * i, i & 1>(t, r); });
    if constexpr (N >= 5)
        unroll<0, 2>([&](auto i) {
            unroll<0, 2>([&](auto j) { bfly<30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1>(t); });
        });
    if constexpr (N == 6)
        unroll<0, 8>([&](auto i) { unroll<0, 2>([&](auto j) { hadd<32 + i * 4 + j, 35 + i * 4 - j, i & 1>(t, r); }); });
    unroll<0, 2>([&](auto i) { bfly<2 * i, 2 * i + 1, 32 + 16 * i, 1 - i>(t); });
    if constexpr (N >= 3) unroll<0, 2>([&](auto i) { hadd<4 + 2 * i, 5 + 2 * i, i>(t, r); });
    if constexpr (N >= 4) unroll<0, 2>([&](auto i) { bfly<14 - i, 9 + i, 48 + 64 * i, 1>(t); });
    if constexpr (N >= 5)
        unroll<0, 4>([&](auto i) { unroll<0, 2>([&](auto j) { hadd<16 + 4 * i + j, 19 + 4 * i - j, i & 1>(t, r); }); });
    if constexpr (N == 6)
        unroll<0, 2>([&](auto i) {
            unroll<0, 4>([&](auto j) { bfly<61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1>(t); });
        });
    unroll<0, 2>([&](auto i) { hadd<i, 3 - i, 0>(t, r); });
    if constexpr (N >= 3) bfly<6, 5, 32, 1>(t);
    if constexpr (N >= 4)
        unroll<0, 2>([&](auto i) { unroll<0, 2>([&](auto j) { hadd<8 + 4 * i + j, 11 + 4 * i - j, i>(t, r); }); });
    if constexpr (N >= 5) unroll<0, 4>([&](auto i) { bfly<29 - i, 18 + i, 48 + (i >> 1) * 64, 1>(t); });
    if constexpr (N == 6)
        unroll<0, 4>([&](auto i) { unroll<0, 4>([&](auto j) { hadd<32 + 8 * i + j, 39 + 8 * i - j, i & 1>(t, r); }); });
    if constexpr (N >= 3) unroll<0, 4>([&](auto i) { hadd<i, 7 - i, 0>(t, r); });
    if constexpr (N >= 4) unroll<0, 2>([&](auto i) { bfly<13 - i, 10 + i, 32, 1>(t); });
    if constexpr (N >= 5)
        unroll<0, 2>([&](auto i) { unroll<0, 4>([&](auto j) { hadd<16 + i * 8 + j, 23 + i * 8 - j, i>(t, r); }); });
    if constexpr (N == 6) unroll<0, 8>([&](auto i) { bfly<59 - i, 36 + i, (i < 4 ? 48 : 112), 1>(t); });
    if constexpr (N >= 4) unroll<0, 8>([&](auto i) { hadd<i, 15 - i, 0>(t, r); });
    if constexpr (N >= 5) unroll<0, 4>([&](auto i) { bfly<27 - i, 20 + i, 32, 1>(t); });
    if constexpr (N == 6)
        unroll<0, 8>([&](auto i) {
            hadd<32 + i, 47 - i, 0>(t, r);
            hadd<48 + i, 63 - i, 1>(t, r);
        });
    if constexpr (N >= 5) unroll<0, 16>([&](auto i) { hadd<i, 31 - i, 0>(t, r); });
    if constexpr (N == 6) unroll<0, 8>([&](auto i) { bfly<55 - i, 40 + i, 32, 1>(t); });
    if constexpr (N == 6) unroll<0, 32>([&](auto i) { hadd<i, 63 - i, 0>(t, r); });
}

template <int N>
__device__ __forceinline__ void adst_in(int* t) {  // transform.rs:465-474
    constexpr int L = 1 << N;
    int cp[L];
#pragma unroll
    for (int i = 0; i < L; i++) cp[i] = t[i];
#pragma unroll
    for (int i = 0; i < L; i++) t[i] = cp[(i & 1) ? i - 1 : L - i - 1];
}
template <int N>
__device__ __forceinline__ void adst_out(int* t) {  // transform.rs:476-492
    constexpr int L = 1 << N;
    int cp[L];
#pragma unroll
    for (int i = 0; i < L; i++) cp[i] = t[i];
#pragma unroll
    for (int i = 0; i < L; i++) {
        const unsigned a = (i >> 3) & 1, b = ((i >> 2) & 1) ^ ((i >> 3) & 1), c = ((i >> 1) & 1) ^ ((i >> 2) & 1),
                       d = (i & 1) ^ ((i >> 1) & 1);
        const unsigned idx = ((d << 3) | (c << 2) | (b << 1) | a) >> (4 - N);
        t[i] = (i & 1) ? -cp[idx] : cp[idx];
    }
}

__device__ __forceinline__ void iadst4(int* t) {  // transform.rs:494-525
    long long t0 = t[0], t1 = t[1], t2 = t[2], t3 = t[3];
    long long s0 = 1321 * t0, s1 = 2482 * t0, s2 = 3344 * t1, s3 = 3803 * t2, s4 = 1321 * t2, s5 = 2482 * t3,
              s6 = 3803 * t3;
    long long b7 = t0 - t2 + t3;
    s0 += s3;
    s1 -= s4;
    s3 = s2;
    s2 = 3344 * b7;
    s0 += s5;
    s1 -= s6;
    t[0] = rnd12(s0 + s3);
    t[1] = rnd12(s1 + s3);
    t[2] = rnd12(s2);
    t[3] = rnd12(s0 + s1 - s3);
}

__device__ __forceinline__ void iadst8(int* t, Clamp r) {  // transform.rs:527-556
    adst_in<3>(t);
    unroll<0, 4>([&](auto i) { bfly<2 * i, 2 * i + 1, 60 - 16 * i, 1>(t); });
    unroll<0, 4>([&](auto i) { hadd<i, 4 + i, 0>(t, r); });
    unroll<0, 2>([&](auto i) { bfly<4 + 3 * i, 5 + i, 48 - 32 * i, 1>(t); });
    unroll<0, 2>([&](auto j) { unroll<0, 2>([&](auto i) { hadd<4 * j + i, 2 + 4 * j + i, 0>(t, r); }); });
    unroll<0, 2>([&](auto i) { bfly<2 + 4 * i, 3 + 4 * i, 32, 1>(t); });
    adst_out<3>(t);
}

__device__ __forceinline__ void iadst16(int* t, Clamp r) {  // transform.rs:558-616
    adst_in<4>(t);
    unroll<0, 8>([&](auto i) { bfly<2 * i, 2 * i + 1, 62 - 8 * i, 1>(t); });
    unroll<0, 8>([&](auto i) { hadd<i, 8 + i, 0>(t, r); });
    unroll<0, 2>([&](auto i) {
        bfly<8 + 2 * i, 9 + 2 * i, 56 - 32 * i, 1>(t);
        bfly<13 + 2 * i, 12 + 2 * i, 8 + 32 * i, 1>(t);
    });
    unroll<0, 2>([&](auto j) { unroll<0, 4>([&](auto i) { hadd<8 * j + i, 4 + 8 * j + i, 0>(t, r); }); });
    unroll<0, 2>([&](auto j) { unroll<0, 2>([&](auto i) { bfly<4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, 1>(t); }); });
    unroll<0, 4>([&](auto j) { unroll<0, 2>([&](auto i) { hadd<4 * j + i, 2 + 4 * j + i, 0>(t, r); }); });
    unroll<0, 4>([&](auto i) { bfly<2 + 4 * i, 3 + 4 * i, 32, 1>(t); });
    adst_out<4>(t);
}

__device__ __forceinline__ void iwht4(int* t, int shift) {  // transform.rs:622-643
    int a = t[0] >> shift, c = t[1] >> shift, d = t[2] >> shift, b = t[3] >> shift;
    a += c;
    d -= b;
    int e = (a - d) >> 1;
    b = e - b;
    int c2 = e - c;
    a -= b;
    d += c2;
    t[0] = a;
    t[1] = b;
    t[2] = c2;
    t[3] = d;
}

template <int N>
__device__ __forceinline__ void iidentity(int* t) {  // transform.rs:645-682
#pragma unroll
    for (int i = 0; i < (1 << N); i++) {
        if constexpr (N == 2) t[i] = rnd12((long long)t[i] * 5793);
        else if constexpr (N == 3) t[i] *= 2;
        else if constexpr (N == 4) t[i] = rnd12((long long)t[i] * 11586);
        else t[i] *= 4;
    }
}

// kind: 0 DCT, 1 ADST, 2 identity (apply_row_kernel / apply_col_kernel, transform.rs:791-847)
__device__ __forceinline__ int row_kind(int tt) {
    switch (tt) {
        case 0: case 1: case 4: case 11: return 0;
        case 2: case 3: case 5: case 6: case 7: case 8: case 13: case 15: return 1;
        default: return 2;
    }
}
__device__ __forceinline__ int col_kind(int tt) {
    switch (tt) {
        case 0: case 2: case 5: case 10: return 0;
        case 1: case 3: case 4: case 6: case 7: case 8: case 12: case 14: return 1;
        default: return 2;
    }
}

template <int N>
__device__ __forceinline__ void tx1d(int* t, int kind, Clamp r) {
    if (kind == 0) {
        idct<N>(t, r);
    } else if (kind == 1) {
        if constexpr (N == 2) iadst4(t);
        else if constexpr (N == 3) iadst8(t, r);
        else if constexpr (N == 4) iadst16(t, r);
    } else {
        if constexpr (N <= 5) iidentity<N>(t);
    }
}

struct ReconFrame {
    PlaneDev planes[3];
    const int32_t* coeffs;
    av1g_quant_params q;
    int32_t bd, hbd;
};

template <int N>
constexpr int ilog2() { return N <= 1 ? 0 : 1 + ilog2<N / 2>(); }

// Dequantizes, inverse transforms and merges one TU of size TX.  Every
// thread of the CTA calls it (it contains block barriers); the TU's L =
// max(w, h) threads have `live` set and `lane` in [0, L); `buf` is the TU's
// w*h int scratch in shared memory.
template <int TX>
__device__ void recon_core(const ReconFrame& F, const av1g_tu& tu, bool live, int lane, int* buf) {
    constexpr int W = kTxW[TX], H = kTxH[TX], L = W > H ? W : H;
    constexpr int LW = ilog2<W>(), LH = ilog2<H>();
    constexpr int TW = W < 32 ? W : 32, TH = H < 32 ? H : 32;
    constexpr int ABS_D = LW > LH ? LW - LH : LH - LW;
    const int bd = F.bd;
    const int seg = tu.segment_id > 7 ? 7 : tu.segment_id;
    const bool lossless = F.q.lossless[seg] != 0;
    // A slot's threads can span two warps (L = 64): clear the whole slot,
    // then a block barrier, before any thread writes coefficients.
    for (int k = lane; k < W * H; k += L) buf[k] = 0;
    __syncthreads();
    // --- dequantize_step1 (cdf.rs:13655-13703) into buf (dense W x H) ---
    if (live) {
        const av1g_quant_params& q = F.q;
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
        const int32_t* lv = F.coeffs + tu.coeff_offset;
        for (int k = lane; k < TW * TH; k += L) {
            int i = k / TW, j = k % TW;
            long long qq = k == 0 ? dcq : acq;
            if (qm) qq = (qq * g_qm[qml][p > 0][c_qm_off[TX] + k] + 16) >> 5;
            long long dq = (long long)lv[k] * qq;
            long long mag = (dq < 0 ? -dq : dq) & 0xFFFFFF;
            long long v = (dq < 0 ? -mag : mag) / (1 << denom_sh);  // truncating division, as the reference
            buf[i * W + j] = (int)min(max(v, cmin), cmax);
        }
    }
    __syncthreads();
    // --- row transforms (transform.rs:730-752) ---
    const Clamp rr{-(1 << (bd + 7)), (1 << (bd + 7)) - 1};
    const int crb = bd + 6 > 16 ? bd + 6 : 16;
    const Clamp cr{-(1 << (crb - 1)), (1 << (crb - 1)) - 1};
    if (live && lane < H && lane < 32) {
        int t[W];
        int* rowp = buf + lane * W;
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
    __syncthreads();
    // --- column transforms (transform.rs:758-787) + step-3 merge (cdf.rs:17398-17470) ---
    if (live && lane < W) {
        int t[H];
#pragma unroll
        for (int i = 0; i < H; i++) t[i] = buf[i * W + lane];
        if (lossless) {
            if constexpr (H == 4) iwht4(t, 0);
        } else {
            tx1d<LH>(t, col_kind(tu.tx_type), cr);
        }
        const int csh = lossless ? 0 : 4;
        const int tt = tu.tx_type;
        const bool fud = tt == 4 || tt == 8 || tt == 14 || tt == 6;
        const bool flr = tt == 5 || tt == 7 || tt == 15 || tt == 6;
        const PlaneDev& P = F.planes[tu.plane];
        const int x = tu.x + (flr ? W - 1 - lane : lane);
        const int maxv = (1 << bd) - 1;
        if (x < P.w) {
#pragma unroll
            for (int i = 0; i < H; i++) {
                int y = tu.y + (fud ? H - 1 - i : i);
                if (y >= P.h) continue;
                int res = csh ? (t[i] + (1 << (csh - 1))) >> csh : t[i];
                int v = ld_px(P, F.hbd, y, x) + res;
                st_px(P, F.hbd, y, x, min(max(v, 0), maxv));
            }
        }
    }
}


}  // namespace
}  // namespace itx
}  // namespace av1g
