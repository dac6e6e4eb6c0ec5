"""§5.9 uncompressed header parsing (host parse layer, row f1) through the C ABI.

Pins:
  * tests/frame_header_fixtures.rs — the first frame header of each of the 16
    fixture clips against every field the reference test expects (frame type
    and flags, frame / upscaled size and superres, intrabc, tile layout,
    quantizer, segmentation, delta q / lf, loop filter, CDEF, loop
    restoration, tx mode, reduced tx set, film grain), and the inter-frame
    header of parses_iftp_inter_frame_header including its 134-bit length;
  * tests/fixture_conformance.rs — every frame of all 110 embedded streams:
    the header parses against the reference state carried from frame to
    frame, each frame's tile groups lay out to its last tile, and the shown
    frames add up to the count each reference test asserts.
The post-filter header (av1g_frame_header) each parse fills is checked for
the derived values the kernels rely on.
"""
import base64
import gzip
import json
from pathlib import Path

import pytest

from oxideav_av1_b200 import framing
from oxideav_av1_b200.framing import FramingError

GOLDEN = json.load(gzip.open(Path(__file__).parent / "golden" / "framing_fixtures.json.gz", "rt"))
FRAME_TYPES = {"Key": 0, "Inter": 1, "IntraOnly": 2, "Switch": 3}
REMAP_LR = [0, 3, 1, 2]  # raw lr_type -> FrameRestorationType (none, wiener, sgrproj, switchable numbering)


def _sec(raw):
    return 4 if raw == 3 else raw


@pytest.mark.parametrize("fx", GOLDEN["frame_headers"], ids=lambda f: f["name"])
def test_first_frame_header_fixture(fx):
    seq = framing.parse_sequence_header(bytes.fromhex(fx["seq_payload"]))
    fh = framing.parse_frame_header(bytes.fromhex(fx["frame_payload"]), seq, framing.new_ref_state())
    e, pf = fx["expected"], fh.pf
    got = {
        "show_existing_frame": bool(fh.show_existing_frame),
        "frame_to_show_map_idx": None if fh.frame_to_show_map_idx < 0 else fh.frame_to_show_map_idx,
        "frame_type": fh.frame_type, "show_frame": bool(fh.show_frame), "showable_frame": bool(fh.showable_frame),
        "error_resilient_mode": bool(fh.error_resilient_mode), "disable_cdf_update": bool(fh.disable_cdf_update),
        "allow_screen_content_tools": bool(fh.allow_screen_content_tools),
        "force_integer_mv": bool(fh.force_integer_mv), "order_hint": fh.order_hint,
        "primary_ref_frame": fh.primary_ref_frame, "refresh_frame_flags": fh.refresh_frame_flags,
        "trace_w": pf.upscaled_width, "trace_h": pf.frame_height, "use_superres": bool(pf.use_superres),
        "allow_intrabc": bool(pf.allow_intrabc), "tile_cols": fh.tile_cols, "tile_rows": fh.tile_rows,
        "context_update_tile_id": fh.context_update_tile_id, "trace_base_q_idx": fh.base_q_idx,
        "trace_seg_enabled": bool(fh.segmentation_enabled), "trace_delta_q_present": bool(fh.delta_q_present),
        "trace_delta_lf_present": bool(fh.delta_lf_present), "trace_lf_y": pf.lf_level[0],
        "trace_lf_uv0": pf.lf_level[2], "trace_lf_uv1": pf.lf_level[3], "trace_lf_sharp": pf.lf_sharpness,
        "trace_lf_delta_enabled": bool(pf.lf_delta_enabled), "trace_cdef_damping": pf.cdef_damping,
        "trace_cdef_bits": pf.cdef_bits, "trace_cdef_y_pri0": pf.cdef_y_pri[0], "trace_cdef_uv_pri0": pf.cdef_uv_pri[0],
        "trace_lr_unit_shift": fh.lr_unit_shift, "trace_lr_uv_shift": fh.lr_uv_shift, "trace_tx_mode": fh.tx_mode,
        "trace_reduced_tx_set": bool(fh.reduced_tx_set),
    }
    want = {k: (FRAME_TYPES[v] if k == "frame_type" else v) for k, v in e.items() if k in got}
    diff = {k: (got[k], v) for k, v in want.items() if got[k] != v}
    assert not diff, diff
    assert fh.superres_denom == (e["coded_denom"] + 9 if e["use_superres"] else 8)
    assert (pf.cdef_y_sec[0], pf.cdef_uv_sec[0]) == (_sec(e["trace_cdef_y_sec0_raw"]), _sec(e["trace_cdef_uv_sec0_raw"]))
    assert [pf.lr_type[i] for i in range(3)] == [REMAP_LR[e[f"trace_lr_{c}_type"]] for c in "yuv"]
    g, fg = pf.film_grain, e["film_grain"]
    if fg is None:
        assert not g.apply_grain
    else:
        assert g.apply_grain and (g.grain_seed, bool(fh.update_grain), g.num_y_points, bool(g.chroma_scaling_from_luma),
                                  g.num_cb_points, g.num_cr_points, g.ar_coeff_lag, g.ar_coeff_shift,
                                  g.grain_scale_shift, g.grain_scaling, bool(g.overlap_flag),
                                  bool(g.clip_to_restricted_range)) == \
            (fg["seed"], fg["update_grain"], fg["num_y_points"], fg["chroma_from_luma"], fg["num_cb_points"],
             fg["num_cr_points"], fg["ar_coeff_lag"], fg["ar_coeff_shift"], fg["grain_scale_shift"],
             fg["grain_scaling"], fg["overlap"], fg["clip_restricted"])
    # derived values of the post-filter header
    assert pf.mi_cols == 2 * ((pf.frame_width + 7) >> 3) and pf.mi_rows == 2 * ((pf.frame_height + 7) >> 3)
    assert (pf.bit_depth, pf.num_planes) == (seq.bit_depth, seq.num_planes)
    assert pf.cdef_short_circuited == int(bool(pf.coded_lossless or pf.allow_intrabc or not seq.enable_cdef))


def test_inter_frame_header_pin():
    seq = framing.parse_sequence_header(bytes.fromhex(GOLDEN["iftp"]["IFTP_SEQ_PAYLOAD"]))
    fh = framing.parse_frame_header(bytes.fromhex(GOLDEN["iftp"]["IFTP_INTER_FRAME_PAYLOAD"]), seq,
                                    framing.new_ref_state())
    pf = fh.pf
    assert (fh.show_existing_frame, fh.frame_type, fh.show_frame, fh.showable_frame, fh.error_resilient_mode,
            fh.disable_cdf_update, fh.allow_screen_content_tools, fh.force_integer_mv) == (0, 1, 1, 1, 0, 0, 1, 0)
    assert (fh.order_hint, fh.primary_ref_frame, fh.refresh_frame_flags, pf.allow_intrabc,
            fh.disable_frame_end_update_cdf) == (1, 7, 0x02, 0, 0)
    assert (pf.upscaled_width, pf.frame_height, pf.frame_width, pf.use_superres, pf.mi_cols, pf.mi_rows) == \
        (64, 64, 64, 0, 16, 16)
    assert fh.frame_refs_short_signaling == 0 and list(fh.ref_frame_idx) == [0] * 7
    assert (fh.allow_high_precision_mv, fh.interpolation_filter, fh.is_motion_mode_switchable,
            fh.use_ref_frame_mvs) == (1, 0, 1, 1)
    assert (fh.base_q_idx, fh.segmentation_enabled, fh.delta_q_present) == (120, 0, 0)
    assert (pf.lf_level[0], pf.lf_level[2], pf.lf_level[3], pf.lf_sharpness, pf.lf_delta_enabled) == (0, 10, 4, 0, 1)
    assert (fh.tx_mode, fh.reference_select, fh.skip_mode_present, fh.allow_warped_motion, fh.reduced_tx_set) == \
        (1, 0, 0, 1, 0)
    assert not pf.film_grain.apply_grain
    assert fh.header_bits == 134


@pytest.mark.parametrize("st", GOLDEN["ivf_streams"], ids=lambda s: s["name"])
def test_every_frame_of_the_fixture_streams(st):
    tus = [f.payload for f in framing.IvfReader(base64.b64decode(st["ivf"])).read_all()]
    frames = framing.stream_frame_headers(tus)
    assert sum(1 for fh, _ in frames if fh.show_existing_frame or fh.show_frame) == st["shown_frames"]
    for fh, spans in frames:
        if fh.show_existing_frame:
            continue
        pf = fh.pf
        assert len(spans) == fh.tile_cols * fh.tile_rows and all(sz > 0 for _, _, sz in spans)
        assert fh.mi_col_starts[fh.tile_cols] == pf.mi_cols and fh.mi_row_starts[fh.tile_rows] == pf.mi_rows
        assert pf.upscaled_width >= pf.frame_width and pf.mi_cols == 2 * ((pf.frame_width + 7) >> 3)
        assert pf.uses_lr == int(any(pf.lr_type[i] for i in range(pf.num_planes)))


def test_truncated_headers_are_rejected():
    fx = GOLDEN["frame_headers"][0]
    seq = framing.parse_sequence_header(bytes.fromhex(fx["seq_payload"]))
    payload = bytes.fromhex(fx["frame_payload"])
    full = framing.parse_frame_header(payload, seq, framing.new_ref_state())
    cut = (full.header_bits - 1) // 8
    with pytest.raises(FramingError) as e:
        framing.parse_frame_header(payload[:cut], seq, framing.new_ref_state())
    assert e.value.variant == "UnexpectedEnd"


def test_corrupted_headers_error_cleanly():
    """The reference's decoder never panics on malformed input (its fuzz
    contract): every single-bit corruption of the first bytes of real frame
    headers of the first temporal units, parsed against an empty reference
    state (slots that never held a frame), either parses or raises a framing
    error.  Among them are headers that take their size from an empty slot,
    which must be rejected rather than divide by a zero tile width."""
    for st in GOLDEN["ivf_streams"][:12]:
        tus = [f.payload for f in framing.IvfReader(base64.b64decode(st["ivf"])).read_all()]
        walker = framing.TemporalUnitWalker()
        state = framing.new_ref_state()
        for tu in tus[:3]:
            for d in walker.walk(tu):
                if d.obu_type not in (3, 6):
                    continue
                for bit in range(min(48, 8 * len(d.payload))):
                    p = bytearray(d.payload)
                    p[bit >> 3] ^= 0x80 >> (bit & 7)
                    try:
                        framing.parse_frame_header(bytes(p), walker.seq, state)
                    except FramingError:
                        pass
        framing.stream_frame_headers(tus)  # the uncorrupted stream still parses end to end
