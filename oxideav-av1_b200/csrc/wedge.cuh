// wedge.cuh — the §7.11.3.11 wedge masks, shared by the inter kernel
// (compound and inter-intra wedges) and the intra kernel (the intra half of
// inter-intra wedge blocks).
//
// The six 64x64 master masks (build_master_mask, src/inter_pred.rs:2712) are
// built at compile time so host and device share one definition; a block's
// mask is a window of one master, possibly inverted (wedge_mask,
// inter_pred.rs:2844).  The host resolves the window (direction, offsets,
// inversion) once per block; the device reads the master per sample.
#pragma once
#include <cstdint>

#include "av1_spec_tables.h"

namespace av1g {
namespace wedge {

struct Master {
    uint8_t m[6][64][64];
};
constexpr int cclip(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }
constexpr Master make_master() {
    Master M{};
    const uint8_t odd[] = AV1T_WEDGE_MASTER_OBLIQUE_ODD_INIT;
    const uint8_t even[] = AV1T_WEDGE_MASTER_OBLIQUE_EVEN_INIT;
    const uint8_t vert[] = AV1T_WEDGE_MASTER_VERTICAL_INIT;
    for (int j = 0; j < 64; j++) {
        int shift = 16;
        for (int i = 0; i < 64; i += 2) {
            M.m[3][i][j] = even[cclip(0, 63, j - shift)];
            shift -= 1;
            M.m[3][i + 1][j] = odd[cclip(0, 63, j - shift)];
            M.m[1][i][j] = vert[j];
            M.m[1][i + 1][j] = vert[j];
        }
    }
    for (int i = 0; i < 64; i++)
        for (int j = 0; j < 64; j++) {
            uint8_t v = M.m[3][i][j];
            M.m[2][j][i] = v;
            M.m[4][i][63 - j] = (uint8_t)(64 - v);
            M.m[5][63 - j][i] = (uint8_t)(64 - v);
            M.m[0][j][i] = M.m[1][i][j];
        }
    return M;
}
constexpr Master kMaster = make_master();

// A block's window of a master mask.
struct Orient {
    uint8_t dir, xoff, yoff, invert;
};

// wedge_mask's parameter checks and window (inter_pred.rs:2844-2957), plus
// mask_blend's extent check for a plane block of w x h samples read with
// subsampling (ssx, ssy) from the luma-grid mask.  False for a call the
// reference rejects.
inline bool orient(int mi_size, int idx, int sign, int w, int h, int ssx, int ssy, Orient& o) {
    static const AV1T_WEDGE_CODEBOOK_TYPE codebook AV1T_WEDGE_CODEBOOK_DIMS = AV1T_WEDGE_CODEBOOK_INIT;
    static const AV1T_WEDGE_BITS_TYPE bits AV1T_WEDGE_BITS_DIMS = AV1T_WEDGE_BITS_INIT;
    static const AV1T_NUM_4X4_BLOCKS_WIDE_TYPE n4w_t AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE_INIT;
    static const AV1T_NUM_4X4_BLOCKS_HIGH_TYPE n4h_t AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH_INIT;
    if (mi_size < 0 || mi_size >= 22 || bits[mi_size] == 0 || idx < 0 || idx >= 16 || sign < 0 || sign > 1)
        return false;
    const int n4w = n4w_t[mi_size], n4h = n4h_t[mi_size], lw = n4w * 4, lh = n4h * 4;
    const int shape = n4h > n4w ? 0 : (n4h < n4w ? 1 : 2);
    const uint8_t* e = codebook[shape][idx];
    const int dir = e[0], xoff = 32 - ((e[1] * lw) >> 3), yoff = 32 - ((e[2] * lh) >> 3);
    long long sum = 0;
    for (int i = 0; i < lw; i++) sum += kMaster.m[dir][yoff][xoff + i];
    for (int i = 1; i < lh; i++) sum += kMaster.m[dir][yoff + i][xoff];
    const long long avg = (sum + (lw + lh - 1) / 2) / (lw + lh - 1);
    const int flip = avg < 32;
    o = Orient{(uint8_t)dir, (uint8_t)xoff, (uint8_t)yoff, (uint8_t)(sign != flip)};
    const int mw = ssx ? 2 * w : w, mh = ssy ? 2 * h : h;
    return mw <= lw && (long long)lw * (mh - 1) + mw <= (long long)lw * lh;
}

// The mask read of mask_blend (inter_pred.rs:3136) at plane sample (i, j) of
// the block: the luma-grid mask itself, or the rounded average of its 2 or 4
// luma positions.
__device__ __forceinline__ int at(const Master& M, const Orient& o, int yy, int xx) {
    const int raw = __ldg(&M.m[o.dir][o.yoff + yy][o.xoff + xx]);
    return o.invert ? 64 - raw : raw;
}
__device__ __forceinline__ int mask_px(const Master& M, const Orient& o, int ssx, int ssy, int i, int j) {
    if (!ssx && !ssy) return at(M, o, i, j);
    if (ssx && !ssy) return (at(M, o, i, 2 * j) + at(M, o, i, 2 * j + 1) + 1) >> 1;
    if (!ssx) return (at(M, o, 2 * i, j) + at(M, o, 2 * i + 1, j) + 1) >> 1;
    return (at(M, o, 2 * i, 2 * j) + at(M, o, 2 * i, 2 * j + 1) + at(M, o, 2 * i + 1, 2 * j) +
            at(M, o, 2 * i + 1, 2 * j + 1) + 2) >> 2;
}

}  // namespace wedge
}  // namespace av1g
