"""Extract the reference's framing golden vectors from its test sources.

Run in a checkout that has the reference crate beside it:

    python tests/golden/make_framing_fixtures.py <reference checkout>

Reads (text only; nothing of the reference is executed):
  tests/fixture_conformance.rs       every IVF stream a test decodes, with the
                                     shown-frame count the test asserts and
                                     the SHA-256 digest of the decoded planes
                                     (the digest the test asserts, or the
                                     digest of the raw / run-length expected
                                     planes it compares byte for byte)
  tests/sequence_header_fixtures.rs  the 16 SEQUENCE_HEADER OBU payloads and
                                     the field values the test expects
  tests/annexb_conformance.rs        the external Annex B stream, its shown-
                                     frame count and digest
  tests/frame_header_fixtures.rs     the 16 first-frame header payloads with
                                     the field values the test expects, and
                                     the inter-frame header it pins
and writes framing_fixtures.json.gz next to this script.
"""
import base64
import gzip
import hashlib
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
        kind, name, ivf_const, expected, digest, frames = m.groups()
        hexs = consts.get(ivf_const)
        if not hexs or not hexs.lower().startswith("444b4946"):
            continue
        if kind == "assert_decodes_to_digest":
            sha = digest or consts.get(expected)
            source = "digest"
        else:
            # the test compares the decoded planes with these bytes: keep their digest
            body = consts[expected]
            raw = _unrle(body) if kind == "assert_decodes_byte_exact_rle" else bytes.fromhex(body)
            sha = hashlib.sha256(raw).hexdigest()
            source = "expected planes"
        streams[name] = {"name": name, "const": ivf_const, "ivf": base64.b64encode(bytes.fromhex(hexs)).decode(),
                         "shown_frames": int(frames), "sha256": sha, "sha256_source": source}
    return list(streams.values())


def _unrle(body):
    """(value u8, count u16) triples, six hex digits each (fixture_conformance.rs unrle)."""
    out = bytearray()
    for i in range(0, len(body), 6):
        out += bytes([int(body[i:i + 2], 16)]) * int(body[i + 2:i + 6], 16)
    return bytes(out)


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


def _bytes_of(text):
    return bytes(int(v, 16) for v in re.findall(r'0x([0-9a-fA-F]{2})', text))


def _fields(text):
    out = {}
    for k, v in re.findall(r'(\w+):\s*(true|false|None|FrameType::\w+|Some\(\d+\)|0x[0-9a-fA-F]+|\d+)', text):
        if v.startswith("0x"):
            out[k] = int(v, 16)
        elif v in ("true", "false"):
            out[k] = v == "true"
        elif v == "None":
            out[k] = None
        elif v.startswith("FrameType::"):
            out[k] = v.split("::")[1]
        elif v.startswith("Some("):
            out[k] = int(v[5:-1])
        else:
            out[k] = int(v)
    return out


def frame_headers(ref):
    """tests/frame_header_fixtures.rs: per fixture the sequence and first
    frame OBU payloads and the expected header fields (film grain ones under
    film_grain when the fixture has them), plus the inter-frame payloads of
    parses_iftp_inter_frame_header."""
    src = (ref / "tests" / "frame_header_fixtures.rs").read_text()
    src = re.sub(r"//[^\n]*", "", src)
    out = []
    for m in re.finditer(r'Fixture\s*\{\s*name:\s*"([^"]+)",\s*seq_payload:\s*&\[([^\]]*)\],\s*'
                         r'frame_payload:\s*&\[([^\]]*)\],\s*expected:\s*Expected\s*\{(.*?)trace_film_grain:\s*'
                         r'(None|Some\(FilmGrainExpected\s*\{(.*?)\}\))', src, re.S):
        name, seq, frame, fields, fg, fg_fields = m.groups()
        exp = _fields(fields)
        exp["film_grain"] = _fields(fg_fields) if fg_fields else None
        out.append({"name": name, "seq_payload": _bytes_of(seq).hex(), "frame_payload": _bytes_of(frame).hex(),
                    "expected": exp})
    iftp = {}
    for const in ("IFTP_SEQ_PAYLOAD", "IFTP_INTER_FRAME_PAYLOAD"):
        mm = re.search(const + r'\s*:\s*&\[u8\]\s*=\s*&\[([^\]]*)\]', src, re.S)
        iftp[const] = _bytes_of(mm.group(1)).hex()
    return out, iftp


def annexb_stream(ref):
    src = (ref / "tests" / "annexb_conformance.rs").read_text()
    consts = _consts(src)
    frames = int(re.search(r'assert_eq!\(frames\.len\(\),\s*(\d+),\s*"shown frame count"\)', src).group(1))
    digest = re.search(r'sha256_hex\(&out\),\s*"([0-9a-f]{64})"', src).group(1)
    return {"name": "EXT_ANNEXB_96X80_OBU", "annexb": base64.b64encode(bytes.fromhex(consts["EXT_ANNEXB_96X80_OBU"])).decode(),
            "shown_frames": frames, "sha256": digest}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_framing_fixtures.py <reference checkout>")
    ref = Path(sys.argv[1])
    data = {"source": "reference tests: fixture_conformance.rs, sequence_header_fixtures.rs, annexb_conformance.rs, "
                      "frame_header_fixtures.rs",
            "ivf_streams": ivf_streams(ref), "sequence_headers": sequence_headers(ref),
            "annexb": annexb_stream(ref)}
    data["frame_headers"], data["iftp"] = frame_headers(ref)
    out = HERE / "framing_fixtures.json.gz"
    with gzip.open(out, "wt") as f:
        json.dump(data, f, sort_keys=True)
    print(f"{out}: {len(data['ivf_streams'])} IVF streams, {len(data['sequence_headers'])} sequence headers, "
          f"1 Annex B stream, {len(data['frame_headers'])} frame headers")


if __name__ == "__main__":
    main()
