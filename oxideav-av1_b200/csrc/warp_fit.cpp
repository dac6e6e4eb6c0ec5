// warp_fit.cpp — the §7.11.3.8 local warp least-squares fit of a
// WARPED_CAUSAL block (host code: at most eight samples per block; the tile
// walk calls it for every such block and the result feeds the inter kernel's
// warp context).
#include <cstdint>

#include "av1_spec_tables.h"
#include "av1g.h"

namespace {

const AV1T_DIV_LUT_TYPE k_div_lut AV1T_DIV_LUT_DIMS = AV1T_DIV_LUT_INIT;

long long rnd2s(long long x, int n) {
    if (n == 0) return x;
    return x >= 0 ? (x + (1LL << (n - 1))) >> n : -((-x + (1LL << (n - 1))) >> n);
}
int clip3i(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

// warp_estimation (src/inter_pred.rs:4083-4226).  Products and sums wrap
// like the reference's release build; the saturating multiplies saturate.
extern "C" av1g_status av1g_warp_estimation(const av1g_warp_sample* cands, int32_t n, int32_t mi_row,
                                            int32_t mi_col, int32_t block_w4, int32_t block_h4, int16_t mv_row,
                                            int16_t mv_col, int32_t params[6], uint8_t* valid) {
    if (n < 0 || (n > 0 && !cands) || !params || !valid) return AV1G_EINVAL;
    auto wadd = [](long long a, long long b) { return (long long)((unsigned long long)a + (unsigned long long)b); };
    auto wsub = [](long long a, long long b) { return (long long)((unsigned long long)a - (unsigned long long)b); };
    auto wneg = [](long long a) { return (long long)(0ull - (unsigned long long)a); };
    auto wmul = [](long long a, long long b) { return (long long)((unsigned long long)a * (unsigned long long)b); };
    auto wabs32 = [](int32_t v) { return v == INT32_MIN ? v : (v < 0 ? -v : v); };
    auto smul = [](long long a, long long b) {
        __int128 q = (__int128)a * b;
        if (q > (__int128)INT64_MAX) return (long long)INT64_MAX;
        if (q < (__int128)INT64_MIN) return (long long)INT64_MIN;
        return (long long)q;
    };
    auto wsub32 = [](int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); };
    auto lsp = [](int32_t a, int32_t b) { return (((long long)a * b) >> 2) + a + b; };
    int cnt = n < 8 ? n : 8;
    int32_t mid_y = (int32_t)((uint32_t)mi_row * 4u + (uint32_t)block_h4 * 2u - 1u);
    int32_t mid_x = (int32_t)((uint32_t)mi_col * 4u + (uint32_t)block_w4 * 2u - 1u);
    int32_t suy = (int32_t)((uint32_t)mid_y * 8u), sux = (int32_t)((uint32_t)mid_x * 8u);
    int32_t duy = (int32_t)((uint32_t)suy + (uint32_t)(int32_t)mv_row);
    int32_t dux = (int32_t)((uint32_t)sux + (uint32_t)(int32_t)mv_col);
    long long a00 = 0, a01 = 0, a11 = 0, bx0 = 0, bx1 = 0, by0 = 0, by1 = 0;
    for (int k = 0; k < cnt; k++) {
        int32_t sy = wsub32(cands[k].sy, suy), sx = wsub32(cands[k].sx, sux);
        int32_t dy = wsub32(cands[k].dy, duy), dx = wsub32(cands[k].dx, dux);
        if (wabs32(wsub32(sx, dx)) < 256 && wabs32(wsub32(sy, dy)) < 256) {
            a00 = wadd(a00, lsp(sx, sx) + 8);
            a01 = wadd(a01, lsp(sx, sy) + 4);
            a11 = wadd(a11, lsp(sy, sy) + 8);
            bx0 = wadd(bx0, lsp(sx, dx) + 8);
            bx1 = wadd(bx1, lsp(sy, dx) + 4);
            by0 = wadd(by0, lsp(sx, dy) + 4);
            by1 = wadd(by1, lsp(sy, dy) + 8);
        }
    }
    long long det = wsub(smul(a00, a11), smul(a01, a01));
    if (det == 0) {
        for (int i = 0; i < 6; i++) params[i] = 0;
        *valid = 0;
        return AV1G_OK;
    }
    unsigned long long ad = det < 0 ? 0ull - (unsigned long long)det : (unsigned long long)det;
    int nb = 63 - __builtin_clzll(ad);
    long long e = (long long)(ad - (1ull << nb));
    long long f = nb > 8 ? (e + (1LL << (nb - 9))) >> (nb - 8) : e << (8 - nb);
    if (f > 256) f = 256;
    long long fac = k_div_lut[f];
    if (det < 0) fac = -fac;
    int sh = nb + 14 - 16;
    if (sh < 0) {
        fac = wmul(fac, 1LL << -sh);
        sh = 0;
    }
    const int32_t one = 1 << 16, nd = 1 << 13;
    auto diag = [&](long long v) { return clip3i(one - nd + 1, one + nd - 1, (int32_t)rnd2s(smul(v, fac), sh)); };
    auto nondiag = [&](long long v) { return clip3i(-nd + 1, nd - 1, (int32_t)rnd2s(smul(v, fac), sh)); };
    params[2] = diag(wsub(wmul(a11, bx0), wmul(a01, bx1)));
    params[3] = nondiag(wadd(wmul(wneg(a01), bx0), wmul(a00, bx1)));
    params[4] = nondiag(wsub(wmul(a11, by0), wmul(a01, by1)));
    params[5] = diag(wadd(wmul(wneg(a01), by0), wmul(a00, by1)));
    long long vx = (long long)mv_col * (1LL << 13) -
                   ((long long)mid_x * (params[2] - one) + (long long)mid_y * params[3]);
    long long vy = (long long)mv_row * (1LL << 13) -
                   ((long long)mid_x * params[4] + (long long)mid_y * (params[5] - one));
    const long long tc = 1LL << 23;
    params[0] = (int32_t)(vx < -tc ? -tc : (vx > tc - 1 ? tc - 1 : vx));
    params[1] = (int32_t)(vy < -tc ? -tc : (vy > tc - 1 ? tc - 1 : vy));
    *valid = 1;
    return AV1G_OK;
}
