"""Stream dispatcher over several GPUs.

The decode path shards by independent streams: a stream's frames are serial,
different streams share nothing.  A multi-GPU server therefore runs one
serving engine per GPU (each with its own reference slots, lanes and HBM
budget) and places every new stream on one of them.  `Dispatcher` does the
placement: the engine with the most free budget (budget minus the slots
reserved by its open streams and the work in flight) that admits the stream;
an engine that answers AV1G_ENOMEM_BUDGET is skipped, and when none admits the
stream `open_stream` returns None so the caller can retry once streams close
(the same contract as one engine's admission).  No data moves between GPUs:
no collective, no peer memory.
"""
import threading

from . import abi


class Dispatcher:
    def __init__(self, engines):
        """engines: one engine.Engine (or an object with the same stats() /
        open_stream(seq) / close()) per GPU."""
        if not engines:
            raise ValueError("a dispatcher needs at least one engine")
        self.engines = list(engines)
        self.placed = [0] * len(self.engines)
        self._mu = threading.Lock()

    @classmethod
    def on_devices(cls, devices, **engine_kw):
        from .engine import Engine
        return cls([Engine(device=d, **engine_kw) for d in devices])

    @staticmethod
    def free_bytes(e):
        s = e.stats()
        return s.budget - s.bytes_reserved - s.bytes_in_flight

    def open_stream(self, seq):
        """(engine index, stream) on the engine with the most free budget that
        admits the stream, or None when no engine has room."""
        with self._mu:
            order = sorted(range(len(self.engines)), key=lambda i: (-self.free_bytes(self.engines[i]), i))
            for i in order:
                st = self.engines[i].open_stream(seq)
                if st is not None:
                    self.placed[i] += 1
                    return i, st
            return None

    def close(self):
        for e in self.engines:
            e.close()


def required_slot_bytes(seq):
    """What an engine reserves for a stream when it opens (the admission
    unit, av1g_stream_open): nine slot payloads of the largest frame — the
    eight reference slots and the one a refresh writes before it replaces an
    older one — each the cropped planes, u8 or u16, rows padded to 64 bytes
    and planes to 256."""
    w, h = seq["max_width"], seq["max_height"]
    bps = 1 if seq["bit_depth"] == 8 else 2
    total = 0
    for p in range(seq["num_planes"]):
        sx = seq["subsampling_x"] if p else 0
        sy = seq["subsampling_y"] if p else 0
        pitch = (((w + sx) >> sx) * bps + 63) // 64 * 64
        total += (pitch * ((h + sy) >> sy) + 255) // 256 * 256
    return 9 * total


__all__ = ["Dispatcher", "required_slot_bytes", "abi"]
