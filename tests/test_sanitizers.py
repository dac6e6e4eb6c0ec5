"""AddressSanitizer + UndefinedBehaviorSanitizer over the host parse layer and the oracle.

The reference runs its parser under libFuzzer with ASan (fuzz/Cargo.toml,
fuzz/fuzz_targets/decode.rs): any bytes must decode or give a typed error,
never crash.  Here the host parse layer (IVF / OBU framing, sequence and
frame headers, the symbol decoder, the tile walk, the stream decoder) and
the C oracle are compiled with -fsanitize=address,undefined (no CUDA: the
decoder runs parse-only, tests/sanitize/stubs.cpp supplies the rest) and
driven, in a subprocess with the ASan runtime preloaded, over every
conformance stream (digests checked through the oracle) and over bit-flipped
copies of every stream (each parses or is rejected with AV1G_EINVAL).  Any
sanitizer report fails the test.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = REPO / "oxideav-av1_b200" / "csrc"
HOST_SRCS = ["warp_fit.cpp", "framing.cpp", "frameheader.cpp", "symbol.cpp", "walker_cdf.cpp", "walker.cpp", "decoder.cpp"]
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-fno-omit-frame-pointer", "-g", "-O1"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


@pytest.fixture(scope="module")
def san_libs(tmp_path_factory):
    d = tmp_path_factory.mktemp("san")
    host = d / "libhost_san.so"
    ora = d / "liboracle_san.so"
    inc = ["-I" + str(REPO / "include"), "-I" + str(CSRC), "-I/usr/local/cuda/include"]
    _run(["g++", "-std=c++17", "-shared", "-fPIC", *SAN, *inc, *[str(CSRC / f) for f in HOST_SRCS],
          str(HERE / "sanitize" / "stubs.cpp"), "-o", str(host)])
    _run(["gcc", "-std=gnu11", "-shared", "-fPIC", *SAN, *inc, "-Wno-missing-braces",
          *map(str, sorted((REPO / "oracle").glob("*.c"))), "-o", str(ora), "-lm"])
    return host, ora


def test_parse_layer_and_oracle_under_asan_ubsan(san_libs):
    host, ora = san_libs
    def lib(name):
        return subprocess.run(["gcc", "-print-file-name=" + name], capture_output=True, text=True).stdout.strip()
    # the ASan runtime first, and the C++ runtime before it is needed, so that
    # the exceptions the walk throws on malformed data are intercepted
    env = dict(os.environ, LD_PRELOAD=lib("libasan.so") + " " + lib("libstdc++.so"),
               ASAN_OPTIONS="detect_leaks=0:abort_on_error=1",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    r = subprocess.run([sys.executable, str(HERE / "sanitize" / "run_corpus.py"), str(host), str(ora), "12"],
                       capture_output=True, text=True, env=env, timeout=900)
    report = r.stdout + r.stderr
    assert "AddressSanitizer" not in report and "runtime error" not in report, report[-4000:]
    assert r.returncode == 0, report[-4000:]
    assert "digest mismatches 0" in r.stdout
