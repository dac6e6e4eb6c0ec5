// lr.cu — §7.17 loop restoration (Wiener and self-guided filters).
//
// Replaces loop_restoration_frame / loop_restore_block / wiener_filter /
// self_guided_filter / box_filter / get_source_sample
// (src/loop_restoration.rs:268-883) as driven by loop_restore_frame_from_grid
// (src/cdf.rs:20624).
//
// The reference filters 4x4 blocks (MI_SIZE walk), each recomputing its
// 7-tap Wiener rows and its (2r+1)^2 box sums over a halo.  Every quantity it
// computes is a function of the sample position, the restoration unit and the
// 64-row stripe only (stripe boundaries fall on 4x4 block boundaries and unit
// boundaries on stripe boundaries), so the kernel computes each quantity once
// per position.  One CTA owns (plane, stripe, 32-row half of the stripe,
// column tile) where the column tile, min(unit size, 64) wide, lies inside a
// single restoration unit.  The CTA stages the source window with a 3-sample
// halo in shared memory — rows inside the stripe from the CDEF frame, up to 2
// rows beyond it from the deblocked frame, clamped to the plane, exactly
// get_source_sample — then:
//  * Wiener: 7-tap horizontal pass into an intermediate array, 7-tap vertical
//    pass to the output (loop_restoration.rs:742-857);
//  * self-guided: per radius, separable box sums (column sums of the samples
//    and their squares, then row sums), the a/b coefficients with the
//    1/(z+1) term from a 256-entry table, the 3x3 weighting, and the
//    projection (loop_restoration.rs:485-736).  For the r0 pass the
//    reference's weights are zero on even rows of the A/B grid, so those rows
//    are not computed.
// Units of type RESTORE_NONE copy the CDEF samples through.
#include <cstddef>

#include "common.cuh"

namespace av1g {

namespace {

constexpr int TW = 64, TH = 32, H3 = 3;
constexpr int kLrThreads = 256;  // lr_kernel's CTA size
constexpr int SW = TW + 2 * H3, SP = SW + 2;  // source window row pitch (u16)
constexpr int SH = TH + 2 * H3;
constexpr int VW = TW + 2 * H3 + 1;           // column-sum row pitch (odd: rows fall on distinct banks)
constexpr int AR = TH + 2, AP = TW + 2 + 1;   // A/B grid rows / pitch

__constant__ int8_t c_sgr_params[16][4] = {
    {2, 12, 1, 4}, {2, 15, 1, 6}, {2, 18, 1, 8}, {2, 21, 1, 9}, {2, 24, 1, 10}, {2, 29, 1, 11},
    {2, 36, 1, 12}, {2, 45, 1, 13}, {2, 56, 1, 14}, {2, 68, 1, 15}, {0, 0, 1, 5}, {0, 0, 1, 8},
    {0, 0, 1, 11}, {0, 0, 1, 14}, {2, 30, 0, 0}, {2, 75, 0, 0}};

struct Smem {
    uint16_t src[SH * SP];
    int v1[AR * VW];      // column sums; the Wiener intermediate reuses v1/v2
    int v2[AR * VW];
    int B[AR * AP];
    uint16_t A[AR * AP];
    uint16_t a2lut[256];
    int F0[TH * TW];
};
// The Wiener intermediate ((TH + 6) x TW ints) spans the adjacent v1 and v2 arrays.
static_assert((TH + 6) * TW <= 2 * AR * VW, "Wiener intermediate does not fit");
static_assert(offsetof(Smem, v2) == offsetof(Smem, v1) + sizeof(int) * AR * VW, "v1/v2 must be adjacent");

__device__ __forceinline__ int r2u(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

__device__ __forceinline__ int tile_w(const av1g_frame_header& h, int p) {
    int us = h.lr_unit_size[p] > 0 ? h.lr_unit_size[p] : 1;
    return us < TW ? us : TW;
}

__device__ __forceinline__ int n_stripes(const av1g_frame_header& h, int p) {
    int ssy = p ? h.subsampling_y : 0;
    int ph = r2u(h.frame_height, ssy);
    return ((((ph - 1) << ssy) + 8) >> 6) + 1;
}

__device__ __forceinline__ int count_units(int us, int sz) {
    int n = (sz + (us >> 1)) / us;
    return n > 1 ? n : 1;
}

// Box sums, a/b coefficients (box_filter, loop_restoration.rs:594-700) for
// radius R over the A/B grid rows i in [-1, th] (stored at i + 1), columns
// j in [-1, tw].  The self-guided sets use R = 2 only for the first pass,
// which needs only the rows whose plane row is odd; their column sums are
// stored compactly (grid row i + 1 at i + 1 >> 1).  Column sums slide down
// the rows and row sums slide along the columns, so each sum costs two loads
// instead of 2R + 1; the runs have fixed lengths so the loops unroll and the
// coefficient arithmetic of neighbouring positions overlaps.
template <int R, bool HBD>
__device__ void box_coeffs(Smem& s, int th, int tw, int bd, int eps, int y0) {
    constexpr bool ODD = R == 2;
    constexpr int n = (2 * R + 1) * (2 * R + 1);
    const long long n2e = (long long)n * n * eps;
    const unsigned sm = (unsigned)(((1LL << 20) + n2e / 2) / n2e);
    constexpr int one_over_n = ((1 << 12) + n / 2) / n;
    // z = (p * sm + 2^19) >> 20 reaches 255 (a2 = 256) once p * sm >= zsat;
    // clamping p to the first such value keeps every product below 2^32
    // (zsat + sm) and leaves a2 unchanged, so z is computed in 32 bits
    constexpr unsigned zsat = (255u << 20) - (1u << 19);
    const unsigned pcap = (zsat + sm - 1) / sm;
    const int sa = 2 * (bd - 8), sb = bd - 8;
    const int vw = tw + 2 * H3;
    const int rows = th + 2;
    // column sums: one thread per (column, run of 12 grid rows): 3 x 71
    // items, one round of the 256 threads
    constexpr int RUN = 12;
    const int runs = (rows + RUN - 1) / RUN;
    for (int k = threadIdx.x; k < runs * VW; k += blockDim.x) {
        const int ru = k / VW, jj = k - ru * VW;
        if (jj >= vw) continue;
        const int ra = ru * RUN;
        const uint16_t* c = s.src + jj + (ra - 1 + H3 - R) * SP;  // first source row of grid row ra's window
        int s1 = 0, s2 = 0;
#pragma unroll
        for (int d = 0; d <= 2 * R; d++) {
            const int v = c[d * SP];
            s1 += v;
            s2 += v * v;
        }
#pragma unroll
        for (int t = 0; t < RUN; t++) {
            const int row = ra + t;
            if (row >= rows) break;
            if (!ODD || ((y0 + row - 1) & 1)) {
                const int cr = ODD ? row >> 1 : row;
                s.v1[cr * VW + jj] = s1;
                s.v2[cr * VW + jj] = s2;
            }
            const int vo = c[t * SP], vn = c[(t + 2 * R + 1) * SP];
            s1 += vn - vo;
            s2 += vn * vn - vo * vo;
        }
    }
    __syncthreads();
    // row sums and coefficients: one thread per (grid row, run of columns),
    // consecutive threads on consecutive rows of one run, so their column-sum
    // loads are an odd pitch apart (distinct banks); with ODD the work list
    // holds only the odd-plane-row grid rows, so no lane of a warp idles on a
    // skipped row.  Runs of 11 columns (34 rows x 6) or, odd rows only, 5
    // columns (17 rows x 14): one round of the 256 threads either way.
    constexpr int CRUN = ODD ? 5 : 11;
    constexpr int SEGS = (TW + 2 + CRUN - 1) / CRUN;
    const int first = ODD ? ((y0 & 1) ? 1 : 0) : 0;  // grid row r holds plane row y0 + r - 1
    constexpr int STEP = ODD ? 2 : 1;
    const int nrows = (rows - first + STEP - 1) / STEP;
    for (int k = threadIdx.x; k < nrows * SEGS; k += blockDim.x) {
        const int sg = k / nrows, rk = k - sg * nrows;
        const int row = first + rk * STEP;
        const int ja = sg * CRUN - 1, jb = min(tw + 1, ja + CRUN);  // j in [ja, jb)
        if (ja >= jb) continue;
        const int cr = ODD ? rk : row;  // rk == row >> 1 for the odd-only rows
        const int* c1 = s.v1 + cr * VW + ja + H3 - R;
        const int* c2 = s.v2 + cr * VW + ja + H3 - R;
        int b = 0, a = 0;
#pragma unroll
        for (int d = 0; d <= 2 * R; d++) {
            b += c1[d];
            a += c2[d];
        }
        uint16_t* ao = s.A + row * AP + ja + 1;
        int* bo = s.B + row * AP + ja + 1;
#pragma unroll
        for (int t = 0; t < CRUN; t++) {
            if (ja + t >= jb) break;
            // 8-bit: both shifts are 0 (the branch is decided at compile time)
            const int ar = HBD ? (a + (1 << (sa - 1))) >> sa : a;
            const int dr = HBD ? (b + (1 << (sb - 1))) >> sb : b;
            int p = ar * n - dr * dr;
            if (p < 0) p = 0;
            const unsigned z = (min((unsigned)p, pcap) * sm + (1u << 19)) >> 20;
            int a2 = z >= 255 ? 256 : s.a2lut[z];
            // b2 uses the raw box sum b, as the reference does
            // (loop_restoration.rs:660-661); (256 - a2) * b * one_over_n
            // stays below 2^32 at every bit depth (b <= 25 * 4095)
            const unsigned b2 = (unsigned)(256 - a2) * (unsigned)b * (unsigned)one_over_n;
            ao[t] = (uint16_t)a2;
            bo[t] = (int)((b2 + (1u << 11)) >> 12);
            b += c1[t + 2 * R + 1] - c1[t];
            a += c2[t + 2 * R + 1] - c2[t];
        }
    }
    __syncthreads();
}

// 3x3 weighting of A/B (loop_restoration.rs:700-736) for the four outputs
// (i, j0 .. j0 + 3), reading each A/B column once.
__device__ __forceinline__ void box_weight4(const Smem& s, int i, int j0, const int u[4], int pass, int y0,
                                            int out[4]) {
    const uint16_t* a = s.A + i * AP + j0;  // top-left of the first 3x3 window
    const int* b = s.B + i * AP + j0;
    int ac[3][6], bc[3][6];
    int shift;
    if (pass == 0) {
        const bool odd = (y0 + i) & 1;
        shift = odd ? 4 : 5;
        if (odd) {  // centre row only, weights 5 6 5
#pragma unroll
            for (int c = 0; c < 6; c++) {
                ac[1][c] = a[AP + c];
                bc[1][c] = b[AP + c];
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int as = 5 * (ac[1][e] + ac[1][e + 2]) + 6 * ac[1][e + 1];
                int bs = 5 * (bc[1][e] + bc[1][e + 2]) + 6 * bc[1][e + 1];
                int v = as * u[e] + bs, sh = 8 + shift - 4;
                out[e] = (v + (1 << (sh - 1))) >> sh;
            }
        } else {    // rows above and below
#pragma unroll
            for (int c = 0; c < 6; c++) {
                ac[0][c] = a[c] + a[2 * AP + c];
                bc[0][c] = b[c] + b[2 * AP + c];
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int as = 5 * (ac[0][e] + ac[0][e + 2]) + 6 * ac[0][e + 1];
                int bs = 5 * (bc[0][e] + bc[0][e + 2]) + 6 * bc[0][e + 1];
                int v = as * u[e] + bs, sh = 8 + shift - 4;
                out[e] = (v + (1 << (sh - 1))) >> sh;
            }
        }
        return;
    }
#pragma unroll
    for (int rr = 0; rr < 3; rr++)
#pragma unroll
        for (int c = 0; c < 6; c++) {
            ac[rr][c] = a[rr * AP + c];
            bc[rr][c] = b[rr * AP + c];
        }
#pragma unroll
    for (int e = 0; e < 4; e++) {
        int ca = ac[0][e + 1] + ac[1][e] + ac[1][e + 1] + ac[1][e + 2] + ac[2][e + 1];
        int cb = bc[0][e + 1] + bc[1][e] + bc[1][e + 1] + bc[1][e + 2] + bc[2][e + 1];
        int as = 3 * (ac[0][e] + ac[0][e + 2] + ac[2][e] + ac[2][e + 2]) + 4 * ca;
        int bs = 3 * (bc[0][e] + bc[0][e + 2] + bc[2][e] + bc[2][e + 2]) + 4 * cb;
        int v = as * u[e] + bs, sh = 8 + 5 - 4;
        out[e] = (v + (1 << (sh - 1))) >> sh;
    }
}

__global__ void __launch_bounds__(kLrThreads) lr_kernel(const FrameDev* __restrict__ frames,
                                                 const int32_t* __restrict__ starts, int n, int total) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    for (int z = threadIdx.x; z < 256; z += blockDim.x)
        s.a2lut[z] = (uint16_t)(z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_frame_header& h = F.h;
        int local = t - starts[f];
        int plane = 0, stripe = 0, half = 0, ct = 0;
        for (int p = 0; p < h.num_planes; p++) {
            if (h.lr_type[p] == 0) continue;
            int pw = r2u(h.upscaled_width, p ? h.subsampling_x : 0);
            int nct = (pw + tile_w(h, p) - 1) / tile_w(h, p);
            int halves = 2 >> (p ? h.subsampling_y : 0);
            int cnt = nct * halves * n_stripes(h, p);
            if (local < cnt) {
                plane = p;
                ct = local % nct;
                half = (local / nct) % halves;
                stripe = local / (nct * halves);
                break;
            }
            local -= cnt;
        }
        const int ssx = plane ? h.subsampling_x : 0, ssy = plane ? h.subsampling_y : 0;
        const int pw = r2u(h.upscaled_width, ssx), ph = r2u(h.frame_height, ssy);
        const int tw_ = tile_w(h, plane);
        const int x0 = ct * tw_, x1 = min(x0 + tw_, pw);
        const int sstart = (-8 + stripe * 64) >> ssy, send = sstart + (64 >> ssy) - 1;
        const int y0 = max(0, sstart + half * TH), y1 = min(min(ph, send + 1), sstart + half * TH + TH);
        const int tw = x1 - x0, th = y1 - y0;
        if (th <= 0) continue;  // uniform across the CTA
        const int hbd = F.hbd, bd = h.bit_depth;
        const PlaneDev& C = F.upcdef[plane];
        const PlaneDev& Dq = F.updeb[plane];
        const PlaneDev& O = F.lr[plane];
        // restoration unit of this tile (derive_block_geometry, loop_restoration.rs:370-428)
        int us = h.lr_unit_size[plane] > 0 ? h.lr_unit_size[plane] : 1;
        int urows = count_units(us, ph), ucols = count_units(us, pw);
        int ur = min(urows - 1, (((max(0, sstart) << ssy) + 8) >> ssy) / us);
        int uc = min(ucols - 1, x0 / us);
        av1g_lr_unit u{};
        if (F.lr_units[plane] && ur < F.lr_unit_rows[plane] && uc < F.lr_unit_cols[plane])
            u = F.lr_units[plane][ur * F.lr_unit_cols[plane] + uc];
        __syncthreads();
        if (u.type != 1 && u.type != 2) {
            // RESTORE_NONE: copied through, four samples per thread (x0 is a
            // multiple of 32 and plane rows start on 16-byte boundaries, so
            // each group of four is one aligned load and store)
            for (int k = threadIdx.x; k < th * (TW / 4); k += blockDim.x) {
                const int i = k >> 4, j0 = (k & 15) * 4;
                if (j0 >= tw) continue;
                const int y = y0 + i, x = x0 + j0;
                if (j0 + 4 <= tw) {
                    const uint8_t* src = C.p + (size_t)y * C.stride;
                    uint8_t* dst = O.p + (size_t)y * O.stride;
                    if (hbd) *reinterpret_cast<uint2*>(dst + 2 * x) = *reinterpret_cast<const uint2*>(src + 2 * x);
                    else *reinterpret_cast<uint32_t*>(dst + x) = *reinterpret_cast<const uint32_t*>(src + x);
                } else {
                    for (int e = 0; e < 4 && j0 + e < tw; e++) st_px(O, hbd, y, x + e, ld_px(C, hbd, y, x + e));
                }
            }
            continue;
        }
        // source window: get_source_sample (loop_restoration.rs:862-883)
        const int sw = tw + 2 * H3;
        if (x0 >= 4 && x0 + tw + 4 <= pw && !(x0 & 3) && !(tw & 3)) {
            // columns [x0 - 4, x0 + tw + 4) lie inside the plane (and inside
            // both source planes, which are at least pw wide): aligned
            // 4-sample loads, the row routed once per load
            // every thread issues its (at most 3) loads before it unpacks
            // any, so their latencies overlap
            const int ng = (tw + 8) >> 2, items = (th + 2 * H3) * ng;
            const unsigned mag = (1u << 16) / ng + 1;  // k / ng for k < 38 * ng
            constexpr int PER = (SH * ((TW + 8) >> 2) + kLrThreads - 1) / kLrThreads;
            uint2 q[PER];
#pragma unroll
            for (int e = 0; e < PER; e++) {
                const int k = threadIdx.x + e * kLrThreads;
                if (k >= items) break;
                const int i = (int)(((unsigned)k * mag) >> 16), g = k - i * ng;
                const int y = clip3(0, ph - 1, y0 - H3 + i);
                const PlaneDev* P;
                int yy;
                if (y < sstart) {
                    P = &Dq;
                    yy = clip3(0, Dq.h - 1, max(y, sstart - 2));
                } else if (y > send) {
                    P = &Dq;
                    yy = clip3(0, Dq.h - 1, min(y, send + 2));
                } else {
                    P = &C;
                    yy = min(y, C.h - 1);
                }
                const uint8_t* row = P->p + (size_t)yy * P->stride;
                const int xs = x0 - 4 + 4 * g;
                if (hbd) q[e] = *reinterpret_cast<const uint2*>(row + 2 * xs);
                else q[e].x = *reinterpret_cast<const uint32_t*>(row + xs);
            }
#pragma unroll
            for (int e = 0; e < PER; e++) {
                const int k = threadIdx.x + e * kLrThreads;
                if (k >= items) break;
                const int i = (int)(((unsigned)k * mag) >> 16), g = k - i * ng;
                int v[4];
                if (hbd) {
                    v[0] = q[e].x & 0xffff;
                    v[1] = q[e].x >> 16;
                    v[2] = q[e].y & 0xffff;
                    v[3] = q[e].y >> 16;
                } else {
                    v[0] = q[e].x & 0xff;
                    v[1] = (q[e].x >> 8) & 0xff;
                    v[2] = (q[e].x >> 16) & 0xff;
                    v[3] = q[e].x >> 24;
                }
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const int j = 4 * g + t - 1;
                    if (j >= 0 && j < sw) s.src[i * SP + j] = (uint16_t)v[t];
                }
            }
        } else {
            for (int k = threadIdx.x; k < (th + 2 * H3) * SW; k += blockDim.x) {
                int i = k / SW, j = k - i * SW;
                if (j >= sw) continue;
                int x = clip3(0, pw - 1, x0 - H3 + j), y = clip3(0, ph - 1, y0 - H3 + i);
                int v;
                if (y < sstart) v = ld_px(Dq, hbd, clip3(0, Dq.h - 1, max(y, sstart - 2)), min(x, Dq.w - 1));
                else if (y > send) v = ld_px(Dq, hbd, clip3(0, Dq.h - 1, min(y, send + 2)), min(x, Dq.w - 1));
                else v = ld_px(C, hbd, min(y, C.h - 1), min(x, C.w - 1));
                s.src[i * SP + j] = (uint16_t)v;
            }
        }
        __syncthreads();
        const int maxv = (1 << bd) - 1;
        if (u.type == 1) {
            int hf[7], vf[7];
            hf[3] = vf[3] = 128;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                vf[i] = vf[6 - i] = u.wiener[0][i];
                vf[3] -= 2 * u.wiener[0][i];
                hf[i] = hf[6 - i] = u.wiener[1][i];
                hf[3] -= 2 * u.wiener[1][i];
            }
            const int rr0 = bd == 12 ? 5 : 3, rr1 = bd == 12 ? 9 : 11;
            const int off = 1 << (bd + 7 - rr0 - 1);
            const int lim = (1 << (bd + 1 + 7 - rr0)) - 1;
            // four adjacent outputs per thread in both passes: the source
            // samples and intermediate rows they share are loaded once, as
            // vectors (source and intermediate rows start on 16-byte
            // boundaries; columns past tw are computed and not stored)
            int* inter = s.v1;  // (th + 6) x TW
            constexpr int Q4 = TW / 4;
            for (int k = threadIdx.x; k < (th + 6) * Q4; k += blockDim.x) {
                const int i = k / Q4, j0 = (k - i * Q4) * 4;
                if (j0 >= tw) continue;
                const uint2* w2 = reinterpret_cast<const uint2*>(s.src + i * SP + j0);
                int w[12];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const uint2 v = w2[q];
                    w[4 * q] = v.x & 0xffff;
                    w[4 * q + 1] = v.x >> 16;
                    w[4 * q + 2] = v.y & 0xffff;
                    w[4 * q + 3] = v.y >> 16;
                }
                int o[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int acc = hf[3] * w[e + 3] + hf[0] * (w[e] + w[e + 6]) + hf[1] * (w[e + 1] + w[e + 5]) +
                                    hf[2] * (w[e + 2] + w[e + 4]);
                    o[e] = clip3(-off, lim - off, (acc + (1 << (rr0 - 1))) >> rr0);
                }
                *reinterpret_cast<int4*>(inter + i * TW + j0) = make_int4(o[0], o[1], o[2], o[3]);
            }
            __syncthreads();
            for (int k = threadIdx.x; k < th * Q4; k += blockDim.x) {
                const int i = k / Q4, j0 = (k - i * Q4) * 4;
                if (j0 >= tw) continue;
                int4 r[7];
#pragma unroll
                for (int d = 0; d < 7; d++) r[d] = *reinterpret_cast<const int4*>(inter + (i + d) * TW + j0);
                int o[4];
#define LR_VTAP(F) (vf[3] * r[3].F + vf[0] * (r[0].F + r[6].F) + vf[1] * (r[1].F + r[5].F) + vf[2] * (r[2].F + r[4].F))
                const int acc[4] = {LR_VTAP(x), LR_VTAP(y), LR_VTAP(z), LR_VTAP(w)};
#undef LR_VTAP
#pragma unroll
                for (int e = 0; e < 4; e++) o[e] = clip3(0, maxv, (acc[e] + (1 << (rr1 - 1))) >> rr1);
                if (j0 + 4 <= tw && !((x0 + j0) & 3)) {  // one aligned vector store
                    uint8_t* row = O.p + (size_t)(y0 + i) * O.stride;
                    if (hbd)
                        *reinterpret_cast<uint2*>(row + 2 * (x0 + j0)) =
                            make_uint2((uint32_t)o[0] | (uint32_t)o[1] << 16, (uint32_t)o[2] | (uint32_t)o[3] << 16);
                    else
                        *reinterpret_cast<uint32_t*>(row + x0 + j0) =
                            (uint32_t)o[0] | (uint32_t)o[1] << 8 | (uint32_t)o[2] << 16 | (uint32_t)o[3] << 24;
                } else {
                    for (int e = 0; e < 4 && j0 + e < tw; e++) st_px(O, hbd, y0 + i, x0 + j0 + e, o[e]);
                }
            }
            continue;
        }
        // self-guided (loop_restoration.rs:485-588)
        const int set = u.sgr_set < 16 ? u.sgr_set : 15;
        const int r0 = c_sgr_params[set][0], e0 = c_sgr_params[set][1];
        const int r1 = c_sgr_params[set][2], e1 = c_sgr_params[set][3];
        const int w0 = u.sgr_xqd[0], w1 = u.sgr_xqd[1], w2 = 128 - w0 - w1;
        // outputs in runs of four along a row
        constexpr int Q = TW / 4;
        if (r0) {
            if (bd > 8) box_coeffs<2, true>(s, th, tw, bd, e0, y0);  // r0 is 2 in every set that has it
            else box_coeffs<2, false>(s, th, tw, bd, e0, y0);
            // rows of one parity run together (the odd-row and even-row
            // weightings differ), so a warp's two rows share a code path
            const int n_odd = (th + ((y0 & 1) ? 1 : 0)) >> 1;      // rows i with (y0 + i) odd
            const int odd0 = (y0 & 1) ? 0 : 1;
            for (int k = threadIdx.x; k < th * Q; k += blockDim.x) {
                const int rk = k / Q, j0 = (k - rk * Q) * 4;
                const int i = rk < n_odd ? odd0 + 2 * rk : (1 - odd0) + 2 * (rk - n_odd);
                if (j0 >= tw) continue;
                int u[4], f[4];
#pragma unroll
                for (int e = 0; e < 4; e++) u[e] = s.src[(i + H3) * SP + j0 + e + H3];
                box_weight4(s, i, j0, u, 0, y0, f);
#pragma unroll
                for (int e = 0; e < 4; e++) s.F0[i * TW + j0 + e] = f[e];
            }
            __syncthreads();
        }
        if (r1) {  // r1 is 1 in every set that has it
            if (bd > 8) box_coeffs<1, true>(s, th, tw, bd, e1, y0);
            else box_coeffs<1, false>(s, th, tw, bd, e1, y0);
        }
        for (int k = threadIdx.x; k < th * Q; k += blockDim.x) {
            int i = k / Q, j0 = (k - i * Q) * 4;
            if (j0 >= tw) continue;
            int u[4], f1[4];
#pragma unroll
            for (int e = 0; e < 4; e++) u[e] = s.src[(i + H3) * SP + j0 + e + H3];
            if (r1) box_weight4(s, i, j0, u, 1, y0, f1);
            int o[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int uu = u[e] << 4;
                int f0 = r0 ? s.F0[i * TW + j0 + e] : uu;
                int v = w1 * uu + w0 * f0 + w2 * (r1 ? f1[e] : uu);
                o[e] = clip3(0, maxv, (v + (1 << 10)) >> 11);
            }
            if (j0 + 4 <= tw && !((x0 + j0) & 3)) {  // one aligned vector store
                uint8_t* row = O.p + (size_t)(y0 + i) * O.stride;
                if (hbd)
                    *reinterpret_cast<uint2*>(row + 2 * (x0 + j0)) =
                        make_uint2((uint32_t)o[0] | (uint32_t)o[1] << 16, (uint32_t)o[2] | (uint32_t)o[3] << 16);
                else
                    *reinterpret_cast<uint32_t*>(row + x0 + j0) =
                        (uint32_t)o[0] | (uint32_t)o[1] << 8 | (uint32_t)o[2] << 16 | (uint32_t)o[3] << 24;
            } else {
                for (int e = 0; e < 4 && j0 + e < tw; e++) st_px(O, hbd, y0 + i, x0 + j0 + e, o[e]);
            }
        }
    }
}

}  // namespace

size_t lr_smem_bytes() { return sizeof(Smem); }

int tiles_lr(const FrameDev& f) {
    const av1g_frame_header& h = f.h;
    int n = 0;
    for (int p = 0; p < h.num_planes; p++) {
        if (h.lr_type[p] == 0) continue;
        int ssx = p ? h.subsampling_x : 0, ssy = p ? h.subsampling_y : 0;
        int pw = ssx ? (h.upscaled_width + 1) >> 1 : h.upscaled_width;
        int ph = ssy ? (h.frame_height + 1) >> 1 : h.frame_height;
        int us = h.lr_unit_size[p] > 0 ? h.lr_unit_size[p] : 1;
        int tw = us < TW ? us : TW;
        int ns = ((((ph - 1) << ssy) + 8) >> 6) + 1;
        n += ((pw + tw - 1) / tw) * ns * (2 >> ssy);
    }
    return n;
}

void launch_lr(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
               cudaStream_t s) {
    if (total <= 0) return;
    size_t bytes = lr_smem_bytes();
    cudaFuncSetAttribute(lr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    lr_kernel<<<shape_grid(sh, total), kLrThreads, bytes, s>>>(frames, starts, n, total);
}

}  // namespace av1g
