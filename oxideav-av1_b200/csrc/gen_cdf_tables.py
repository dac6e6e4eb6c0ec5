"""Generate av1_cdf_tables.h: the §9.4 default CDF tables and the §9.2 scan
orders the tile walker reads, extracted from the reference's Rust literals.

    python gen_cdf_tables.py <reference checkout>

Reads (text only) src/cdf.rs (every `DEFAULT_*_CDF` constant, with the array
shape its type declares, and the small block / transform geometry, context
and transform-set tables the syntax reads) and src/scan.rs (the default /
column / row scans),
and writes av1_cdf_tables.h next to this script.  The tables are normative
data: a decoder must hold them entry for entry, so they are copied, not
re-derived.  The header is committed; the reference is not needed to build.
"""
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

# Small §5.11 / §9.3 tables of block and transform geometry, contexts and
# transform-set maps that the syntax reads (src/cdf.rs).
WALKER_TABLES = [
    "INTRA_MODE_CONTEXT", "COMPOUND_MODE_CTX_MAP", "PALETTE_COLOR_CONTEXT", "PALETTE_COLOR_HASH_MULTIPLIERS",
    "SIZE_GROUP", "MI_WIDTH_LOG2", "MI_HEIGHT_LOG2", "WEDGE_BITS", "ADJUSTED_TX_SIZE", "TX_WIDTH_LOG2",
    "TX_SIZE_SQR_UP", "SIG_REF_DIFF_OFFSET", "MAG_REF_OFFSET_WITH_TX_CLASS", "COEFF_BASE_POS_CTX_OFFSET",
    "COEFF_BASE_CTX_OFFSET", "MAX_TX_DEPTH_TABLE", "SPLIT_TX_SIZE", "MODE_TO_TXFM", "TX_TYPE_IN_SET_INTRA",
    "TX_TYPE_IN_SET_INTER", "TX_TYPE_INTRA_INV_SET1", "TX_TYPE_INTRA_INV_SET2", "TX_TYPE_INTER_INV_SET1",
    "TX_TYPE_INTER_INV_SET2", "TX_TYPE_INTER_INV_SET3", "PARTITION_SUBSIZE", "MAX_TX_SIZE_RECT",
    "NUM_4X4_BLOCKS_WIDE", "NUM_4X4_BLOCKS_HIGH", "SUBSAMPLED_SIZE", "TX_WIDTH", "TX_HEIGHT",
]


def _consts(src):
    """Integer `pub const NAME: usize|u32|i32 = <expr>;` values, evaluated in order."""
    env = {}
    for m in re.finditer(r'pub const ([A-Z0-9_]+)\s*:\s*(?:usize|u32|i32|u8|u16)\s*=\s*([^;\[]+);', src):
        name, expr = m.group(1), m.group(2).strip()
        try:
            env[name] = int(eval(expr.replace("as usize", "").replace("as u32", ""), {}, dict(env)))
        except Exception:
            pass
    return env


def _dims(ty, env):
    """`[[u16; N]; M]` -> [M, N] (outermost first)."""
    dims = []
    t = ty.strip()
    while t.startswith("["):
        inner = t[1:t.rindex("]")]
        depth, cut = 0, None
        for i in range(len(inner) - 1, -1, -1):
            c = inner[i]
            if c == "]":
                depth += 1
            elif c == "[":
                depth -= 1
            elif c == ";" and depth == 0:
                cut = i
                break
        elem, count = inner[:cut], inner[cut + 1:]
        dims.append(int(eval(count.strip(), {}, dict(env))))
        t = elem.strip()
    return dims


def _values(body, env):
    body = re.sub(r"//[^\n]*", "", body)
    toks = [t.strip() for t in re.split(r"[\[\],]", body) if t.strip()]
    return [int(eval(t, {}, dict(env))) for t in toks]


def _c_name(rust):
    # DEFAULT_SKIP_CDF -> Default_Skip_Cdf
    return "_".join(w.capitalize() for w in rust.lower().split("_"))


def extract(src, prefix_re, env):
    out = []
    for m in re.finditer(r'pub (?:const|static) (' + prefix_re + r')\s*:\s*([^=]+)=\s*', src):
        name, ty = m.group(1), m.group(2)
        start = m.end()
        depth, i = 0, start
        while True:
            c = src[i]
            if c == "[":
                depth += 1
            elif c == "]":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        dims = _dims(ty, env)
        vals = _values(src[start:i + 1], env)
        n = 1
        for d in dims:
            n *= d
        if n != len(vals):
            raise SystemExit(f"{name}: {len(vals)} values for shape {dims}")
        out.append((name, dims, vals))
    return out


def emit(tables, ctype):
    lines = []
    for name, dims, vals in tables:
        shape = "".join(f"[{d}]" for d in dims)
        lines.append(f"static const {ctype} {_c_name(name)}{shape} = {{")
        row = dims[-1]
        for k in range(0, len(vals), row):
            lines.append("    " + ", ".join(str(v) for v in vals[k:k + row]) + ",")
        lines.append("};")
    return lines


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_cdf_tables.py <reference checkout>")
    ref = Path(sys.argv[1])
    cdf = (ref / "src" / "cdf.rs").read_text()
    scan = (ref / "src" / "scan.rs").read_text()
    env = _consts(cdf)
    cdfs = extract(cdf, r"DEFAULT_[A-Z0-9_]+_CDF", env)
    scans = extract(scan, r"(?:DEFAULT|MCOL|MROW)_SCAN_[0-9X]+", env)
    small = extract(cdf, "(?:" + "|".join(WALKER_TABLES) + ")", env)
    for name, _, vals in cdfs:
        if max(vals) > 32768 or min(vals) < 0:
            raise SystemExit(f"{name}: value outside 0..32768")
    lines = ["/* av1_cdf_tables.h: AV1 §9.4 default CDFs, §9.2 scan orders and the",
             " * block / transform tables of the §5.11 syntax.",
             " * Generated by gen_cdf_tables.py from the reference's src/cdf.rs and",
             " * src/scan.rs literals; do not edit.  Each CDF row holds the cumulative",
             " * values (the last 32768) followed by the adaptation counter (0). */",
             "#pragma once", "#include <stdint.h>", ""]
    lines += emit(cdfs, "uint16_t")
    lines += emit(scans, "uint16_t")
    lines += emit(small, "int16_t")
    (HERE / "av1_cdf_tables.h").write_text("\n".join(lines) + "\n")
    print(f"{len(cdfs)} CDF tables, {len(scans)} scans")


if __name__ == "__main__":
    main()
