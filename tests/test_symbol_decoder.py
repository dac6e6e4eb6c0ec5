"""The §8.2 symbol decoder (host parse layer, row f1) through the C ABI.

Pins: the unit tests of src/symbol_decoder.rs restated — init_symbol's full
and partial windows, the boolean-CDF trace, read_bool, read_literal's MSB-first
composition, update_cdf's adaptation and counter cap, CDF adaptation on and
off, read_ns(1) consuming nothing, decode_subexp_bool's uniform branch,
exit_symbol's byte alignment — and a direct pure-Python statement of §8.2 /
§8.3 run side by side with the library on seeded random bytes and CDFs
(symbols, adapted CDFs, decoder state and exit positions must agree).
"""
import random

import pytest

from oxideav_av1_b200 import framing
from oxideav_av1_b200.framing import FramingError, SymbolDecoder, update_cdf


def test_init_symbol_full_window():
    d = SymbolDecoder(bytes([0b1010_1010, 0b1100_1100]), 2, False)
    assert d.s.value == 0x7FFF ^ 21862 and d.s.range == 1 << 15 and d.s.max_bits == 1 and d.position == 15


def test_init_symbol_partial_window():
    d = SymbolDecoder(bytes([0b1011_0001]), 1, False)
    assert d.s.value == 0x7FFF ^ (177 << 7) and d.s.range == 1 << 15 and d.s.max_bits == -7 and d.position == 8


def test_read_symbol_boolean_cdf_trace():
    d = SymbolDecoder(bytes([0x00, 0x02]), 2, True)
    assert d.s.value == 0x7FFE
    cdf = [1 << 14, 1 << 15, 0]
    assert d.read_symbol(cdf) == 0
    assert (d.s.range, d.s.value, d.s.max_bits, d.position) == (65520, 65515, -1, 16)


def test_read_bool_matches_boolean_trace():
    d = SymbolDecoder(bytes([0x00, 0x02]), 2, False)
    assert d.read_bool() == 0
    assert (d.s.range, d.s.value) == (65520, 65515)


def test_read_literal_composes_bits_msb_first():
    data = bytes([0x12, 0x34, 0x56, 0x78])
    a, b = SymbolDecoder(data, 4, True), SymbolDecoder(data, 4, True)
    lit = a.read_literal(3)
    bits = [b.read_bool() for _ in range(3)]
    assert lit == (bits[0] << 2) | (bits[1] << 1) | bits[2]
    assert (a.s.value, a.s.range, a.position) == (b.s.value, b.s.range, b.position)


def test_update_cdf_pins():
    cdf = [10000, 20000, 32768, 0]
    update_cdf(cdf, 1, 3)
    assert cdf == [9375, 20798, 32768, 1]
    cdf = [16384, 32768, 31]
    update_cdf(cdf, 0, 2)
    assert cdf[2] == 32
    cdf = [16384, 32768, 32]
    update_cdf(cdf, 0, 2)
    assert cdf[2] == 32


def test_read_symbol_adapts_cdf_only_when_enabled():
    data = bytes([0x80, 0, 0, 0])
    cdf = [10923, 21845, 32768, 0]
    SymbolDecoder(data, 4, False).read_symbol(cdf)
    assert cdf != [10923, 21845, 32768, 0] and cdf[3] == 1
    cdf = [10923, 21845, 32768, 0]
    SymbolDecoder(data, 4, True).read_symbol(cdf)
    assert cdf == [10923, 21845, 32768, 0]


def test_read_ns_one_consumes_nothing():
    d = SymbolDecoder(bytes([0xFF, 0x00]), 2, True)
    before = d.position
    assert d.read_ns(1) == 0 and d.position == before


def test_subexp_uniform_branch_is_read_ns():
    data = bytes(4)
    a, b = SymbolDecoder(data, 4, True), SymbolDecoder(data, 4, True)
    # decode_signed_subexp_with_ref_bool(0, 2, 0, 0) reads decode_subexp_bool(2, 0) = read_ns(2)
    v = a.decode_signed_subexp_with_ref_bool(0, 2, 0, 0)
    assert v == b.read_ns(2) and a.position == b.position


def test_exit_symbol_advances_to_byte_boundary():
    d = SymbolDecoder(bytes([0x80, 0x01]), 2, True)
    assert d.position == 15
    assert d.exit_symbol() == (0, 16)
    assert d.position == 16


def test_errors():
    with pytest.raises(FramingError):
        SymbolDecoder(b"", 1, False)  # fewer bytes than sz
    d = SymbolDecoder(bytes([0x55]), 1, True)
    with pytest.raises(FramingError) as e:
        d.read_symbol([1000, 2000, 0])  # CDF not ending at 32768 cannot be decoded
    assert e.value.variant in ("SymbolStateInvariantBroken",)


# --- a direct statement of §8.2 / §8.3, pure Python ---

class PySymbol:
    def __init__(self, data, sz, disable):
        self.data, self.sz, self.disable, self.pos = data, sz, disable, 0
        nb = min(sz * 8, 15)
        buf = self.f(nb)
        self.value = ((1 << 15) - 1) ^ (buf << (15 - nb))
        self.range = 1 << 15
        self.max_bits = sz * 8 - 15

    def f(self, n):
        v = 0
        for _ in range(n):
            v = (v << 1) | ((self.data[self.pos >> 3] >> (7 - (self.pos & 7))) & 1)
            self.pos += 1
        return v

    def read_symbol(self, cdf):
        n = len(cdf) - 1
        cur, s = self.range, -1
        while True:
            s += 1
            prev = cur
            cur = ((self.range >> 8) * (((1 << 15) - cdf[s]) >> 6)) >> 1
            cur += 4 * (n - s - 1)
            if self.value >= cur:
                break
        self.range, self.value = prev - cur, self.value - cur
        bits = 15 - (self.range.bit_length() - 1)
        self.range <<= bits
        nb = min(bits, max(self.max_bits, 0))
        self.value = (self.f(nb) << (bits - nb)) ^ (((self.value + 1) << bits) - 1)
        self.max_bits -= bits
        if not self.disable:
            count = cdf[n]
            rate = 3 + (count > 15) + (count > 31) + min((n).bit_length() - 1, 2)
            tmp = 0
            for i in range(n - 1):
                if i == s:
                    tmp = 1 << 15
                c = cdf[i]
                cdf[i] = c - ((c - tmp) >> rate) if tmp < c else c + ((tmp - c) >> rate)
            if count < 32:
                cdf[n] = count + 1
        return s


def _random_cdf(rng, n):
    cuts = sorted(rng.sample(range(1, 32768), n - 1))
    return cuts + [32768, 0]


@pytest.mark.parametrize("seed", range(6))
def test_matches_direct_statement(seed):
    rng = random.Random(seed)
    sz = rng.randint(2, 400)
    data = bytes(rng.randrange(256) for _ in range(sz))
    disable = seed % 3 == 2
    lib, py = SymbolDecoder(data, sz, disable), PySymbol(data, sz, disable)
    cdfs = [_random_cdf(rng, rng.randint(2, 16)) for _ in range(12)]
    twin = [list(c) for c in cdfs]
    steps = 0
    while py.max_bits > -14 and steps < 4000:
        k = rng.randrange(len(cdfs))
        a, b = lib.read_symbol(cdfs[k]), py.read_symbol(twin[k])
        assert a == b and cdfs[k] == twin[k], steps
        assert (lib.s.value, lib.s.range, lib.s.max_bits, lib.position) == (py.value, py.range, py.max_bits, py.pos)
        steps += 1
    assert steps > 10
    if lib.s.max_bits >= -14:
        t, e = lib.exit_symbol()
        assert e % 8 == 0 and t <= e
