"""The multi-GPU stream dispatcher: placement by free HBM budget (CPU, fake engines).

Each fake engine stands for one GPU's serving engine: a budget, the bytes its
open streams reserve (nine slot payloads each, as av1g_stream_open) and a refusal
(AV1G_ENOMEM_BUDGET -> None) when a stream does not fit, as the engine's own
admission does.  The dispatcher must put each new stream on the engine with
the most free budget, skip engines that refuse it, and return None when no
engine has room.
"""
import types

from oxideav_av1_b200.dispatch import Dispatcher, required_slot_bytes

SEQ_1080 = dict(max_width=1920, max_height=1080, bit_depth=8, subsampling_x=1, subsampling_y=1, num_planes=3,
                sb_size=64)
SEQ_4K10 = dict(max_width=3840, max_height=2160, bit_depth=10, subsampling_x=1, subsampling_y=1, num_planes=3,
                sb_size=128)


class FakeEngine:
    def __init__(self, budget, in_flight=0):
        self.budget, self.reserved, self.in_flight = budget, 0, in_flight
        self.streams = []
        self.closed = False

    def stats(self):
        return types.SimpleNamespace(budget=self.budget, bytes_reserved=self.reserved,
                                     bytes_in_flight=self.in_flight)

    def open_stream(self, seq):
        need = required_slot_bytes(seq)
        if self.reserved + self.in_flight + need > self.budget:
            return None
        self.reserved += need
        self.streams.append(seq)
        return object()

    def close(self):
        self.closed = True


def test_slot_bytes():
    # nine payloads; rows padded to 64 bytes, planes to 256 (1920 = 30 x 64,
    # 960 = 15 x 64; every plane here is a multiple of 256 bytes)
    assert required_slot_bytes(SEQ_1080) == 9 * (1920 * 1080 + 2 * 960 * 540)
    assert required_slot_bytes(SEQ_4K10) == 9 * 2 * (3840 * 2160 + 2 * 1920 * 1080)
    odd = dict(SEQ_1080, max_width=130, max_height=70)
    # luma 192 x 70 = 13440 -> 13568; chroma 128 x 35 = 4480 -> 4608 each
    assert required_slot_bytes(odd) == 9 * (13568 + 2 * 4608)


def test_streams_go_to_the_engine_with_most_free_budget():
    one = required_slot_bytes(SEQ_1080)
    a, b = FakeEngine(10 * one), FakeEngine(4 * one)
    d = Dispatcher([a, b])
    placed = [d.open_stream(SEQ_1080)[0] for _ in range(8)]
    # a has more room until both are even at 4 * one free... a takes the first six
    assert placed[:6] == [0] * 6
    # then they alternate, lowest index first on a tie
    assert placed[6:] == [0, 1]
    assert a.reserved == 7 * one and b.reserved == 1 * one


def test_work_in_flight_counts_against_the_budget():
    one = required_slot_bytes(SEQ_1080)
    a, b = FakeEngine(6 * one, in_flight=5 * one), FakeEngine(3 * one)
    d = Dispatcher([a, b])
    assert d.open_stream(SEQ_1080)[0] == 1


def test_refusing_engines_are_skipped_and_a_full_pool_returns_none():
    one4k = required_slot_bytes(SEQ_4K10)
    small = FakeEngine(one4k - 1)           # can never hold a 4K 10-bit stream
    big = FakeEngine(2 * one4k)
    d = Dispatcher([small, big])
    # small has no 4K room although its free budget is compared first after a tie-break
    assert d.open_stream(SEQ_4K10)[0] == 1
    assert d.open_stream(SEQ_4K10)[0] == 1
    assert d.open_stream(SEQ_4K10) is None
    # a smaller stream still fits on the small engine
    assert d.open_stream(SEQ_1080)[0] == 0
    d.close()
    assert small.closed and big.closed


def test_mixed_placement_balances_bytes_not_counts():
    one, one4k = required_slot_bytes(SEQ_1080), required_slot_bytes(SEQ_4K10)
    a, b = FakeEngine(40 * one), FakeEngine(40 * one)
    d = Dispatcher([a, b])
    assert d.open_stream(SEQ_4K10)[0] == 0
    # the next 1080p streams go to b until b's free bytes fall below a's
    k = 0
    while d.open_stream(SEQ_1080)[0] == 1:
        k += 1
    assert k == one4k // one
