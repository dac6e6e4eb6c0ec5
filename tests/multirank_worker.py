"""One rank of the world-size-2 CPU check of bench.py's replica path (run by
tests/test_multirank_cpu.py under torch.distributed.run with the gloo
backend).  Each rank builds its own shard of synthetic frames, runs the CPU
oracle's post-filter chain on it, times that, and reduces the time with
bench.max_over_ranks; rank 0 prints one JSON line with every rank's shard
digest, its own time, the reduced time and bench.job_rate."""
import datetime
import hashlib
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402  (registers the package and its synthetic generator)
import oracle  # noqa: E402


def main():
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    frames = [bench.synth.make_frame(bench.frame_seed(rank, i), 96, 64) for i in range(2)]
    t0 = time.perf_counter()
    digest = hashlib.sha256()
    for f in frames:
        for plane in oracle.postfilter_frame(f)[1]:
            digest.update(plane.tobytes())
    own_ms = (time.perf_counter() - t0) * 1e3 + 50.0 * rank  # rank 1 reports the slower step
    worst = bench.max_over_ranks(own_ms, world, "cpu")
    shards = [None] * world
    dist.all_gather_object(shards, digest.hexdigest())
    times = [None] * world
    dist.all_gather_object(times, own_ms)
    if rank == 0:
        print(json.dumps({"world": world, "shards": shards, "times": times, "max_ms": worst,
                          "rate": bench.job_rate(world, len(frames), worst)}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
