"""Motion-field motion vectors on the device: §7.19 storage and §7.9 projection.

``motion_vector_storage`` mirrors the §7.19 loop at the end of the reference's
frame decode (src/decoder/frame_driver.rs:1119-1160) and
``motion_field_estimation`` mirrors ``motion_field_estimation_core``
(src/inter_pred.rs:7592): same arguments, same meaning, one slot view per
§7.20 reference slot (``None`` = empty).  Arrays are torch CUDA tensors; the
batched forms run any number of frames in one call of the C ABI
(av1g_run_mf_store / av1g_run_mf_project).  No CPU path exists: a missing
library raises.
"""
import ctypes as C

import torch

from . import abi

MFMV_INVALID = abi.MFMV_INVALID


def _stream_ptr(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev(t, dtype, n):
    assert t.is_cuda and t.dtype == dtype and t.is_contiguous() and t.numel() == n, (t.dtype, t.shape)
    return t.data_ptr()


def store_job(mi_rows, mi_cols, is_inter_frame, order_hint, hint_bits, ref_order_hint, ref_frames, mvs,
              mf_ref_frames=None, mf_mvs=None):
    """An av1g_mf_store_job over device tensors (outputs allocated when None).
    Returns (job, mf_ref_frames, mf_mvs).  The job holds raw device pointers:
    keep every tensor alive until the call that runs the job has been made."""
    cells = mi_rows * mi_cols
    dev = ref_frames.device
    if mf_ref_frames is None:
        mf_ref_frames = torch.empty(cells, dtype=torch.int8, device=dev)
    if mf_mvs is None:
        mf_mvs = torch.empty((cells, 2), dtype=torch.int16, device=dev)
    j = abi.MfStoreJob(mi_rows, mi_cols, int(bool(is_inter_frame)), order_hint, hint_bits,
                       (C.c_int32 * 7)(*ref_order_hint), _dev(ref_frames, torch.int8, 2 * cells),
                       _dev(mvs, torch.int16, 4 * cells), _dev(mf_ref_frames, torch.int8, cells),
                       _dev(mf_mvs, torch.int16, 2 * cells))
    return j, mf_ref_frames, mf_mvs


def run_store(jobs, stream=None):
    lib = abi.load()
    arr = (abi.MfStoreJob * len(jobs))(*jobs)
    abi.check(lib.av1g_run_mf_store(arr, len(jobs), _stream_ptr(stream)))


def motion_vector_storage(mi_rows, mi_cols, is_inter_frame, order_hint, hint_bits, ref_order_hint, ref_frames, mvs,
                          stream=None):
    """§7.19 for one frame: ref_frames int8 [cells, 2], mvs int16 [cells, 2, 2]
    (device) -> (mf_ref_frames int8 [cells], mf_mvs int16 [cells, 2])."""
    j, r, m = store_job(mi_rows, mi_cols, is_inter_frame, order_hint, hint_bits, ref_order_hint, ref_frames, mvs)
    run_store([j], stream)
    return r, m


def project_job(slots, ref_frame_idx, order_hints, order_hint, hint_bits, mi_rows, mi_cols, out=None,
                device="cuda"):
    """An av1g_mf_project_job; slots: 8 entries, None or dict(mf_mvs,
    mf_ref_frames (device tensors), saved_order_hints, mi_rows, mi_cols,
    frame_is_intra).  Returns (job, out) with out int16 [7, h8, w8, 2]."""
    h8, w8 = mi_rows >> 1, mi_cols >> 1
    if out is None:
        out = torch.empty((7, h8, w8, 2), dtype=torch.int16, device=device)
    j = abi.MfProjectJob()
    for i, sl in enumerate(slots):
        if sl is None:
            continue
        cells = sl["mi_rows"] * sl["mi_cols"]
        j.slots[i] = abi.MfSlot(_dev(sl["mf_mvs"], torch.int16, 2 * cells),
                                _dev(sl["mf_ref_frames"], torch.int8, cells),
                                (C.c_int32 * 8)(*sl["saved_order_hints"]), sl["mi_rows"], sl["mi_cols"],
                                int(bool(sl["frame_is_intra"])), 0)
    for k in range(7):
        j.ref_frame_idx[k] = ref_frame_idx[k]
    for k in range(8):
        j.order_hints[k] = order_hints[k]
    j.order_hint, j.hint_bits, j.mi_rows, j.mi_cols = order_hint, hint_bits, mi_rows, mi_cols
    j.out = _dev(out, torch.int16, 14 * h8 * w8) if h8 * w8 else None
    return j, out


def run_project(jobs, stream=None):
    lib = abi.load()
    arr = (abi.MfProjectJob * len(jobs))(*jobs)
    abi.check(lib.av1g_run_mf_project(arr, len(jobs), _stream_ptr(stream)))


def motion_field_estimation(slots, ref_frame_idx, order_hints, order_hint, hint_bits, mi_rows, mi_cols,
                            stream=None, device="cuda"):
    """§7.9 for one frame; returns the MotionFieldMvs grid int16 [7, h8, w8, 2]."""
    j, out = project_job(slots, ref_frame_idx, order_hints, order_hint, hint_bits, mi_rows, mi_cols,
                         device=device)
    run_project([j], stream)
    return out
