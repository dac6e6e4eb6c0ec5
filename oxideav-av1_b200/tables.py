"""The AV1 normative tables of ``csrc/av1_spec_tables.h`` as numpy arrays.

Parsed from the generated header so host code and tests see exactly the
values compiled into the kernels.
"""
import re
from pathlib import Path

import numpy as np

_HDR = Path(__file__).resolve().parent / "csrc" / "av1_spec_tables.h"
_DT = {"int8_t": np.int8, "uint8_t": np.uint8, "int16_t": np.int16, "uint16_t": np.uint16}


def _load():
    text = _HDR.read_text()
    out = {}
    for m in re.finditer(r"#define AV1T_(\w+)_TYPE (\w+)\n#define AV1T_\1_DIMS ((?:\[\d+\])+)\n"
                         r"#define AV1T_\1_COUNT (\d+)\n#define AV1T_\1_INIT \{ \\\n(.*?)\n\}", text, re.S):
        name, ty, dims, count, body = m.groups()
        vals = [int(v) for v in re.findall(r"-?\d+", body)]
        shape = tuple(int(d) for d in re.findall(r"\d+", dims))
        assert len(vals) == int(count)
        out[name] = np.array(vals, dtype=_DT[ty]).reshape(shape)
    return out


globals().update(_load())
