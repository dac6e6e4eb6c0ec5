// symbol.cpp — the §8.2 arithmetic symbol decoder and the §8.3 CDF update.
//
// Follows SymbolDecoder (src/symbol_decoder.rs): init_symbol, read_symbol
// with renormalisation and the post-renormalisation range / value check,
// read_bool / read_literal / read_ns, the subexponential readers of §5.9.26-
// §5.9.28 over decoded bools, exit_symbol, and update_cdf.  Bits are read MSB
// first from the caller's bytes (src/bitreader.rs f(n)); reading past the end
// is Error::UnexpectedEnd.  Host code: entropy decoding is serial.
#include <cstring>

#include "av1g.h"

namespace av1g {
void set_framing_error(int code, const char* text);
}

namespace {

int floor_log2(uint32_t x) { return x ? 31 - __builtin_clz(x) : 0; }

// f(n) from the decoder's byte span; false past its end.
bool read_bits(av1g_symbol_decoder& d, int n, uint32_t& v) {
    v = 0;
    if (d.pos + (uint64_t)n > d.size * 8) return false;
    for (int i = 0; i < n; i++, d.pos++) v = (v << 1) | ((d.data[d.pos >> 3] >> (7 - (d.pos & 7))) & 1);
    return true;
}

av1g_status err(int code, const char* text) {
    av1g::set_framing_error(code, text);
    return AV1G_EINVAL;
}

av1g_status end() { return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: unexpected end of data"); }

int64_t inverse_recenter(int64_t r, int64_t v) {
    if (v > 2 * r) return v;
    return (v & 1) ? r - ((v + 1) >> 1) : r + (v >> 1);
}

}  // namespace

extern "C" {

void av1g_update_cdf(uint16_t* cdf, uint32_t symbol, int32_t n) {
    if (!cdf || n < 1) return;
    const uint32_t count = cdf[n];
    const int rate = 3 + (count > 15) + (count > 31) + (floor_log2((uint32_t)n) < 2 ? floor_log2((uint32_t)n) : 2);
    uint32_t tmp = 0;
    for (int i = 0; i < n - 1; i++) {
        if ((uint32_t)i == symbol) tmp = 1u << 15;
        const uint32_t c = cdf[i];
        cdf[i] = (uint16_t)(tmp < c ? c - ((c - tmp) >> rate) : c + ((tmp - c) >> rate));
    }
    if (count < 32) cdf[n] = (uint16_t)(count + 1);
}

av1g_status av1g_symbol_init(av1g_symbol_decoder* d, const uint8_t* data, size_t sz, int32_t disable_cdf_update) {
    if (!d || (!data && sz)) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: null argument");
    memset(d, 0, sizeof *d);
    d->data = data;
    d->size = sz;
    d->disable_cdf_update = disable_cdf_update != 0;
    const int num_bits = sz * 8 < 15 ? (int)(sz * 8) : 15;
    uint32_t buf;
    if (!read_bits(*d, num_bits, buf)) return end();
    d->value = ((1u << 15) - 1) ^ (buf << (15 - num_bits));
    d->range = 1u << 15;
    d->max_bits = (int64_t)sz * 8 - 15;
    return AV1G_OK;
}

av1g_status av1g_symbol_read(av1g_symbol_decoder* d, uint16_t* cdf, int32_t n, uint32_t* symbol) {
    if (!d || !cdf || !symbol || n < 2) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: bad argument");
    // §8.2.6: the first symbol whose scaled boundary the value reaches
    // (a well-formed CDF ends at 32768, so the last symbol always matches;
    // a malformed one is reported instead of read past)
    uint32_t cur = d->range, prev = cur;
    int s = 0;
    for (;; s++) {
        if (s == n) return err(AV1G_FE_SYMBOL_STATE_INVARIANT, "symbol decoder: CDF does not end at 32768");
        prev = cur;
        const uint32_t f = (1u << 15) - cdf[s];
        cur = ((d->range >> 8) * (f >> 6)) >> 1;  // EC_PROB_SHIFT = 6
        cur += 4u * (uint32_t)(n - s - 1);       // EC_MIN_PROB = 4
        if (d->value >= cur) break;
    }
    d->range = prev - cur;
    d->value -= cur;
    // renormalisation
    const int bits = 15 - floor_log2(d->range);
    d->range <<= bits;
    const int64_t avail = d->max_bits > 0 ? d->max_bits : 0;
    const int num_bits = bits < avail ? bits : (int)avail;
    uint32_t nd;
    if (!read_bits(*d, num_bits, nd)) return end();
    d->value = (nd << (bits - num_bits)) ^ (((d->value + 1) << bits) - 1);
    d->max_bits -= bits;
    if (d->range < (1u << 15) || d->range > (1u << 16) - 1 || d->value >= d->range)
        return err(AV1G_FE_SYMBOL_STATE_INVARIANT, "symbol decoder: range / value invariant broken");
    if (!d->disable_cdf_update) av1g_update_cdf(cdf, (uint32_t)s, n);
    *symbol = (uint32_t)s;
    return AV1G_OK;
}

av1g_status av1g_symbol_read_bool(av1g_symbol_decoder* d, uint32_t* bit) {
    uint16_t cdf[3] = {1u << 14, 1u << 15, 0};
    return av1g_symbol_read(d, cdf, 2, bit);
}

av1g_status av1g_symbol_read_literal(av1g_symbol_decoder* d, int32_t n, uint32_t* value) {
    if (!value || n < 0 || n > 32) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: bad argument");
    uint32_t x = 0;
    for (int i = 0; i < n; i++) {
        uint32_t b;
        if (av1g_status st = av1g_symbol_read_bool(d, &b)) return st;
        x = 2 * x + b;
    }
    *value = x;
    return AV1G_OK;
}

av1g_status av1g_symbol_read_ns(av1g_symbol_decoder* d, uint32_t n, uint32_t* value) {
    if (!value || n < 1) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: bad argument");
    const int w = floor_log2(n) + 1;
    const uint32_t m = (1u << w) - n;
    uint32_t v;
    if (av1g_status st = av1g_symbol_read_literal(d, w - 1, &v)) return st;
    if (v < m) {
        *value = v;
        return AV1G_OK;
    }
    uint32_t extra;
    if (av1g_status st = av1g_symbol_read_literal(d, 1, &extra)) return st;
    *value = (v << 1) - m + extra;
    return AV1G_OK;
}

av1g_status av1g_symbol_read_signed_subexp(av1g_symbol_decoder* d, int64_t low, int64_t high, uint32_t k, int64_t r,
                                           int64_t* value) {
    if (!value || high <= low || k > 24) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: bad argument");
    const int64_t mx = high - low;
    r -= low;
    // decode_subexp_bool(mx, k)
    uint32_t i = 0, mk = 0, v = 0;
    const uint32_t num_syms = (uint32_t)mx;
    for (;;) {
        const uint32_t b2 = i ? k + i - 1 : k;
        const uint32_t a = 1u << b2;
        if (num_syms <= mk + 3 * a) {
            uint32_t u;
            if (av1g_status st = av1g_symbol_read_ns(d, num_syms - mk, &u)) return st;
            v = u + mk;
            break;
        }
        uint32_t more;
        if (av1g_status st = av1g_symbol_read_literal(d, 1, &more)) return st;
        if (more) {
            i++;
            mk += a;
        } else {
            uint32_t u;
            if (av1g_status st = av1g_symbol_read_literal(d, (int32_t)b2, &u)) return st;
            v = u + mk;
            break;
        }
    }
    const int64_t x = (r << 1) <= mx ? inverse_recenter(r, v) : mx - 1 - inverse_recenter(mx - 1 - r, v);
    *value = x + low;
    return AV1G_OK;
}

av1g_status av1g_symbol_exit(av1g_symbol_decoder* d, uint64_t* trailing_bit_position, uint64_t* padding_end) {
    if (!d || !trailing_bit_position || !padding_end) return err(AV1G_FE_UNEXPECTED_END, "symbol decoder: null argument");
    if (d->max_bits < -14) return err(AV1G_FE_SYMBOL_EXIT_UNDERFLOW, "symbol decoder: SymbolMaxBits below -14");
    const int64_t pos = (int64_t)d->pos;
    const int64_t keep = d->max_bits + 15 < 15 ? d->max_bits + 15 : 15;
    *trailing_bit_position = (uint64_t)(pos - keep);
    const uint64_t advance = d->max_bits > 0 ? (uint64_t)d->max_bits : 0;
    if (d->pos + advance > d->size * 8) return end();
    d->pos += advance;
    *padding_end = d->pos;
    return AV1G_OK;
}

}  // extern "C"
