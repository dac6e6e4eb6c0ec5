"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU calls)."""
import ctypes as C
import re
from pathlib import Path

from oxideav_av1_b200 import abi

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(av1g_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "av1g_run_postfilter" in names and "av1g_run_cdef" in names


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared_functions()) <= set(abi.exported_symbols())


def test_struct_layouts_match_library():
    lib = abi.load()
    for cname, cls in abi._STRUCTS.items():
        assert lib.av1g_struct_size(cname.encode()) == C.sizeof(cls), cname
    assert lib.av1g_struct_size(b"nope") == -1


def test_host_only_entry_points():
    lib = abi.load()
    assert lib.av1g_abi_version() == 1
    # count_units_in_frame (loop_restoration.rs:888)
    assert lib.av1g_lr_units_in_frame(64, 1080) == 17
    assert lib.av1g_lr_units_in_frame(64, 1920) == 30
    assert lib.av1g_lr_units_in_frame(256, 100) == 1
    assert lib.av1g_lr_units_in_frame(64, 96) == 2


def test_empty_batch_is_ok_without_device():
    lib = abi.load()
    assert lib.av1g_run_postfilter(None, 0, 0, None, None) == abi.AV1G_OK
    assert lib.av1g_run_postfilter(None, -1, 0, None, None) == abi.AV1G_EINVAL


def test_noalloc_limits_match_the_header():
    text = (ROOT / "include" / "av1g.h").read_text()
    defs = dict(re.findall(r"#define\s+(AV1G_NOALLOC_[A-Z_]+)\s+(.+)", text))
    assert eval(defs["AV1G_NOALLOC_MAX_FRAMES"], {}) == abi.NOALLOC_MAX_FRAMES
    assert eval(defs["AV1G_NOALLOC_SCRATCH_BYTES"], {}) == abi.NOALLOC_SCRATCH_BYTES
