"""Extract the reference's framing golden vectors from its test sources.

Run in a checkout that has the reference crate beside it:

    python tests/golden/make_framing_fixtures.py /root/reference

Reads (text only; nothing of the reference is executed):
  tests/fixture_conformance.rs       every IVF stream a test decodes, with the
                                     shown-frame count the test asserts and,
                                     where present, the SHA-256 digest of the
                                     decoded planes
  tests/sequence_header_fixtures.rs  the 16 SEQUENCE_HEADER OBU payloads and
                                     the field values the test expects
  tests/annexb_conformance.rs        the external Annex B stream, its shown-
                                     frame count and digest
and writes framing_fixtures.json.gz next to this script.
"""
import base64
import gzip
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def _consts(src):
    """NAME -> hex string for every `const NAME: &str = concat!(...)` or
    `const NAME: &str = "..."` literal."""
    out = {}
    for m in re.finditer(r'const\s+([A-Z0-9_]+)\s*:\s*&str\s*=\s*(concat!\((.*?)\)|"([^"]*)")\s*;', src, re.S):
        body = m.group(3) if m.group(3) is not None else '"' + m.group(4) + '"'
        out[m.group(1)] = "".join(re.findall(r'"([^"]*)"', body))
    return out


def ivf_streams(ref):
    src = (ref / "tests" / "fixture_conformance.rs").read_text()
    consts = _consts(src)
    streams = {}
    pat = re.compile(r'(assert_decodes_byte_exact_rle|assert_decodes_byte_exact|assert_decodes_to_digest)\(\s*'
                     r'"([^"]+)"\s*,\s*([A-Z0-9_]+)\s*,\s*("([0-9a-f]{64})"|[A-Z0-9_]+)\s*,\s*(\d+)\s*,?\s*\)', re.S)
    for m in pat.finditer(src):
        kind, name, ivf_const, _, digest, frames = m.groups()
        hexs = consts.get(ivf_const)
        if not hexs or not hexs.lower().startswith("444b4946"):
            continue
        streams[name] = {"name": name, "const": ivf_const, "ivf": base64.b64encode(bytes.fromhex(hexs)).decode(),
                         "shown_frames": int(frames), "sha256": digest if kind == "assert_decodes_to_digest" else None}
    return list(streams.values())


def sequence_headers(ref):
    src = (ref / "tests" / "sequence_header_fixtures.rs").read_text()
    out = []
    for m in re.finditer(r'Fixture\s*\{\s*name:\s*"([^"]+)",\s*payload:\s*&\[([^\]]*)\],\s*expected:\s*Expected\s*\{(.*?)\}',
                         src, re.S):
        name, payload, fields = m.groups()
        data = [int(v, 16) for v in re.findall(r'0x([0-9a-fA-F]{2})', payload)]
        exp = {}
        for k, v in re.findall(r'(\w+):\s*(true|false|\d+)', fields):
            exp[k] = v == "true" if v in ("true", "false") else int(v)
        out.append({"name": name, "payload": bytes(data).hex(), "expected": exp})
    return out


def annexb_stream(ref):
    src = (ref / "tests" / "annexb_conformance.rs").read_text()
    consts = _consts(src)
    frames = int(re.search(r'assert_eq!\(frames\.len\(\),\s*(\d+),\s*"shown frame count"\)', src).group(1))
    digest = re.search(r'sha256_hex\(&out\),\s*"([0-9a-f]{64})"', src).group(1)
    return {"name": "EXT_ANNEXB_96X80_OBU", "annexb": base64.b64encode(bytes.fromhex(consts["EXT_ANNEXB_96X80_OBU"])).decode(),
            "shown_frames": frames, "sha256": digest}


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    data = {"source": "reference tests: fixture_conformance.rs, sequence_header_fixtures.rs, annexb_conformance.rs",
            "ivf_streams": ivf_streams(ref), "sequence_headers": sequence_headers(ref),
            "annexb": annexb_stream(ref)}
    out = HERE / "framing_fixtures.json.gz"
    with gzip.open(out, "wt") as f:
        json.dump(data, f, sort_keys=True)
    print(f"{out}: {len(data['ivf_streams'])} IVF streams, {len(data['sequence_headers'])} sequence headers, "
          f"1 Annex B stream")


if __name__ == "__main__":
    main()
