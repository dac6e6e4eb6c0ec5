"""Run inside the sanitizer subprocess of tests/test_sanitizers.py: the parse
layer and the oracle, both built with AddressSanitizer and
UndefinedBehaviorSanitizer, over every conformance stream (digest checked)
and over bit-flipped copies of the streams (each must parse or be rejected
with a typed error).  argv: host library, oracle library, flips per stream."""
import base64
import ctypes as C
import gzip
import hashlib
import json
import random
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

import __graft_entry__  # noqa: E402

__graft_entry__._package()
import numpy as np  # noqa: E402

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, decoder  # noqa: E402

host = C.CDLL(sys.argv[1])
for name, (res, args) in abi._SIGS.items():
    if hasattr(host, name):
        fn = getattr(host, name)
        fn.restype, fn.argtypes = res, args
abi._lib = host
ora = C.CDLL(sys.argv[2])
ora.ora_postfilter_frame.restype = C.c_int
ora.ora_random_next.restype = C.c_uint32
ora.ora_random_next.argtypes = [C.POINTER(C.c_uint16), C.c_int]
oracle._lib = ora
flips = int(sys.argv[3])

streams = json.load(gzip.open(REPO / "tests" / "golden" / "framing_fixtures.json.gz"))["ivf_streams"]
bad = 0
for s in streams:
    ivf = base64.b64decode(s["ivf"])
    seq, frames = decoder.parse_stream(ivf)
    outs = oracle.decode_stream(frames)
    h = hashlib.sha256()
    for fr, planes in zip(frames, outs):
        if planes is None:
            continue
        for p in planes:
            h.update(p.astype(np.uint8).tobytes() if fr.hdr.bit_depth == 8 else p.astype("<u2").tobytes())
    if h.hexdigest() != s["sha256"]:
        print("digest mismatch", s["name"])
        bad += 1
rng = random.Random(5)
rejected = accepted = 0
for s in streams:
    ivf = bytearray(base64.b64decode(s["ivf"]))
    for _ in range(flips):
        b = bytearray(ivf)
        pos = rng.randrange(44, len(b))   # past the IVF file and first record headers
        b[pos] ^= 1 << rng.randrange(8)
        try:
            decoder.parse_stream(bytes(b))
            accepted += 1
        except abi.Av1gError:
            rejected += 1
print(f"corpus ok, digest mismatches {bad}; bit flips: {accepted} parsed, {rejected} rejected with a typed error")
sys.exit(1 if bad else 0)
