#!/usr/bin/env python3
"""Generate ``av1_spec_tables.h`` — the AV1 normative constant tables.

The AV1 specification fixes a set of integer tables that every conforming
decoder must use bit-for-bit (quantizer lookups, quantizer matrices, the
film-grain Gaussian sequence, the super-resolution and sub-pixel filter
kernels, the intra smoothing weights, ...).  They are data, not code, and a
decoder that differs in a single entry is not conformant, so this build
carries exactly the reference crate's values.  Rather than re-typing ~110 k
numbers by hand, this script reads the Rust array literals out of the
reference source tree and re-emits them as C initialiser macros:

    #define AV1T_<NAME>_DIMS  ...
    #define AV1T_<NAME>_INIT  { ... }

Each consumer (CUDA device code, the C oracle) declares its own array with
its own storage qualifier from the ``_INIT`` macro.

Usage (run in a checkout that has the reference tree; the generated header
is committed, so nothing at build or run time needs the reference):

    python gen_tables.py /path/to/oxideav-av1 > av1_spec_tables.h
"""
import re
import sys
from pathlib import Path

# (rust file, rust const name, C element type) — every table the kernels and
# the oracle read.  File paths are relative to the reference crate root.
TABLES = [
    ("src/superres.rs", "UPSCALE_FILTER", "int16_t"),
    ("src/film_grain_tables.rs", "GAUSSIAN_SEQUENCE", "int16_t"),
    ("src/cdf.rs", "DC_QLOOKUP", "int16_t"),
    ("src/cdf.rs", "AC_QLOOKUP", "int16_t"),
    ("src/qmatrix.rs", "QM_OFFSET", "int16_t"),
    ("src/qmatrix.rs", "QUANTIZER_MATRIX", "uint8_t"),
    ("src/inter_pred.rs", "SUBPEL_FILTERS", "int16_t"),
    ("src/inter_pred.rs", "WARPED_FILTERS", "int16_t"),
    ("src/inter_pred.rs", "DIV_LUT", "int16_t"),
    ("src/inter_pred.rs", "WEDGE_CODEBOOK", "uint8_t"),
    ("src/inter_pred.rs", "QUANT_DIST_LOOKUP", "int8_t"),
    ("src/inter_pred.rs", "QUANT_DIST_WEIGHT", "int8_t"),
    ("src/inter_pred.rs", "WEDGE_MASTER_OBLIQUE_ODD", "uint8_t"),
    ("src/inter_pred.rs", "WEDGE_MASTER_OBLIQUE_EVEN", "uint8_t"),
    ("src/inter_pred.rs", "WEDGE_MASTER_VERTICAL", "uint8_t"),
    ("src/inter_pred.rs", "WEDGE_BITS", "uint8_t"),
    ("src/inter_pred.rs", "II_WEIGHTS_1D", "uint8_t"),
    ("src/inter_pred.rs", "OBMC_MASK_2", "uint8_t"),
    ("src/inter_pred.rs", "OBMC_MASK_4", "uint8_t"),
    ("src/inter_pred.rs", "OBMC_MASK_8", "uint8_t"),
    ("src/inter_pred.rs", "OBMC_MASK_16", "uint8_t"),
    ("src/inter_pred.rs", "OBMC_MASK_32", "uint8_t"),
    ("src/cdf.rs", "INTRA_FILTER_TAPS", "int16_t"),
    ("src/cdf.rs", "SM_WEIGHTS_TX_4X4", "uint8_t"),
    ("src/cdf.rs", "SM_WEIGHTS_TX_8X8", "uint8_t"),
    ("src/cdf.rs", "SM_WEIGHTS_TX_16X16", "uint8_t"),
    ("src/cdf.rs", "SM_WEIGHTS_TX_32X32", "uint8_t"),
    ("src/cdf.rs", "SM_WEIGHTS_TX_64X64", "uint8_t"),
    ("src/cdf.rs", "MODE_TO_ANGLE", "int16_t"),
    ("src/cdf.rs", "DR_INTRA_DERIVATIVE", "int16_t"),
    ("src/cdf.rs", "INTRA_EDGE_KERNEL", "int8_t"),
    ("src/cdf.rs", "SUBSAMPLED_SIZE", "uint8_t"),
    ("src/cdf.rs", "MAX_TX_SIZE_RECT", "uint8_t"),
    ("src/cdf.rs", "NUM_4X4_BLOCKS_WIDE", "uint8_t"),
    ("src/cdf.rs", "NUM_4X4_BLOCKS_HIGH", "uint8_t"),
    ("src/cdf.rs", "TX_WIDTH", "uint8_t"),
    ("src/cdf.rs", "TX_HEIGHT", "uint8_t"),
    ("src/transform.rs", "COS128_LOOKUP", "int16_t"),
    ("src/transform.rs", "TRANSFORM_ROW_SHIFT", "uint8_t"),
]

RANGES = {
    "int8_t": (-128, 127), "uint8_t": (0, 255), "int16_t": (-32768, 32767), "uint16_t": (0, 65535),
}

SYMBOL_FILES = [
    "src/cdf.rs", "src/inter_pred.rs", "src/uncompressed_header_tail.rs", "src/superres.rs",
    "src/qmatrix.rs", "src/transform.rs", "src/film_grain.rs", "src/loop_restoration.rs",
]


def strip_comments(text: str) -> str:
    return re.sub(r"//[^\n]*", "", text)


def collect_symbols(root: Path) -> dict:
    """Integer-valued `const NAME: T = <int>;` definitions usable as table entries."""
    raw = {}
    pat = re.compile(r"(?:pub\s+)?const\s+([A-Z_][A-Z0-9_]*)\s*:\s*[a-z0-9]+\s*=\s*([^;\[]+);")
    for rel in SYMBOL_FILES:
        for m in pat.finditer(strip_comments((root / rel).read_text())):
            raw.setdefault(m.group(1), m.group(2).strip())
    sym = {}
    for _ in range(8):  # resolve expressions that name other constants
        for k, v in raw.items():
            if k in sym:
                continue
            try:
                sym[k] = eval_expr(v.replace(" as usize", "").replace(" as u32", ""), sym)
            except SystemExit:
                pass
    return sym


def find_literal(text: str, name: str):
    m = re.search(r"(?:pub\s+)?(?:const|static)\s+" + name + r"\s*:\s*([^=]+)=\s*\[", text)
    if not m:
        raise SystemExit(f"table {name} not found")
    ty = m.group(1).strip()
    start = m.end() - 1
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "[":
            depth += 1
        elif text[i] == "]":
            depth -= 1
            if depth == 0:
                return ty, text[start:i + 1]
    raise SystemExit(f"unterminated literal for {name}")


def parse_dims(ty: str, sym: dict):
    """`[[[u8; 3344]; 2]; 15]` -> [15, 2, 3344]."""
    dims = []
    inner = ty.strip()
    while inner.startswith("["):
        body = inner[1:inner.rindex("]")]
        # split at the last top-level ';'
        depth = 0
        cut = None
        for i, ch in enumerate(body):
            if ch == "[":
                depth += 1
            elif ch == "]":
                depth -= 1
            elif ch == ";" and depth == 0:
                cut = i
        elem, count = body[:cut], body[cut + 1:].strip()
        dims.append(eval_expr(count, sym))
        inner = elem.strip()
    return dims


def eval_expr(expr: str, sym: dict) -> int:
    e = expr.strip()
    for k in sorted(sym, key=len, reverse=True):
        e = re.sub(r"\b" + k + r"\b", str(sym[k]), e)
    if not re.fullmatch(r"[0-9+\-*/() <>]+", e):
        raise SystemExit(f"cannot evaluate dimension {expr!r} -> {e!r}")
    return int(eval(e.replace("/", "//")))


def literal_values(lit: str, sym: dict):
    body = lit.replace("[", " ").replace("]", " ")
    vals = []
    for tok in body.split(","):
        tok = tok.strip()
        if not tok:
            continue
        tok = re.sub(r"_?(i8|u8|i16|u16|i32|u32|i64|usize)$", "", tok)
        if re.fullmatch(r"-?\d+", tok.replace("_", "")):
            vals.append(int(tok.replace("_", "")))
        else:
            vals.append(eval_expr(tok, sym))
    return vals


def main():
    root = Path(sys.argv[1])
    sym = collect_symbols(root)
    out = [
        "/* Generated by gen_tables.py from the AV1 normative tables as carried by the",
        " * reference decoder crate.  Do not edit by hand.  Each table is an",
        " * initialiser macro so that device code and host code can declare their own",
        " * copy with their own storage qualifier. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
    ]
    for rel, name, cty in TABLES:
        text = strip_comments((root / rel).read_text())
        ty, lit = find_literal(text, name)
        dims = parse_dims(ty, sym)
        vals = literal_values(lit, sym)
        total = 1
        for d in dims:
            total *= d
        if total != len(vals):
            raise SystemExit(f"{name}: dims {dims} want {total} values, got {len(vals)}")
        lo, hi = RANGES[cty]
        if min(vals) < lo or max(vals) > hi:
            raise SystemExit(f"{name}: values [{min(vals)}, {max(vals)}] do not fit {cty}")
        out.append(f"/* {name}: {rel} */")
        out.append(f"#define AV1T_{name}_TYPE {cty}")
        out.append(f"#define AV1T_{name}_DIMS " + "".join(f"[{d}]" for d in dims))
        out.append(f"#define AV1T_{name}_COUNT {total}")
        lines = []
        for i in range(0, len(vals), 24):
            lines.append("  " + ",".join(str(v) for v in vals[i:i + 24]) + ",")
        out.append(f"#define AV1T_{name}_INIT {{ \\")
        out.extend(line + " \\" for line in lines)
        out.append("}")
        out.append("")
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
