"""bench.py's replica path on two ranks, on CPU with the gloo backend.

The multi-GPU run is N independent replicas (no data exchange): each rank
decodes its own shard of frames, the step time is the slowest rank's
(all-reduce MAX) and the rate counts every rank's frames.  Here two CPU ranks
under torch.distributed.run check that shards differ by rank, that the
reduced time is the maximum of the ranks' own times, that the job rate is
world x frames / max time, and that the reference arm, launched the same way,
prints one line from rank 0 while rank 1 exits 0 without output.
"""
import json
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _torchrun(args, timeout):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port())] + args
    return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout)


def test_two_replicas_reduce_the_slowest_time():
    r = _torchrun([str(ROOT / "tests" / "multirank_worker.py")], 300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = lines[0]
    assert out["world"] == 2 and out["shards"][0] != out["shards"][1]
    assert out["max_ms"] == max(out["times"]) and out["times"][1] > out["times"][0]
    assert abs(out["rate"] - 2 * 2 / (out["max_ms"] / 1e3)) < 1e-9 * out["rate"]


def test_reference_arm_prints_once_from_rank_zero():
    r = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"], 600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
    assert lines[0]["value"] > 0 and lines[0]["e2e"]["h2d_bytes_per_step"] == 0
